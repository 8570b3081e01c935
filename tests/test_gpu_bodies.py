"""Colliders on rigid bodies (b3Body of every type) on the GPU against the
oracle.

The world that moves the bodies is the caller's.  Here the test plays that
world on the host: each frame it takes the bodies as the cloth step left them,
advances them by one step (gravity on the dynamic body, constant velocity on
the kinematic one, nothing on the static one), computes their transforms,
world inverse inertias and proxies, and gives the same states, proxies and
report order to the GPU cloth and to the oracle.  The GPU's particle state is
also given to the oracle each frame, so that every step starts from identical
inputs.  Tolerances:
* positions within 1e-5 relative, CG iterations within +-1 (the CG's grid
  reductions sum in another order than the oracle's sequential dots);
* active body contacts within 1% (a contact whose separation lies within
  rounding of zero may differ);
* body velocities after the contact solve within 1e-5 of the largest body
  velocity, centres and orientations within 1e-6: the ordered contact solve
  itself is the oracle's arithmetic in the oracle's order, so what differs
  is the CG's rounding carried through the impulses (measured on a B200:
  1.2e-7 on x, 8.9e-7 on body velocities, 6e-8 on centres over 90 frames).
"""
import math

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


# ---- the host world ---------------------------------------------------------

def _qmat(q):
    x, y, z, w = [np.float32(u) for u in q]
    x2, y2, z2 = x + x, y + y, z + z
    xx, xy, xz = x * x2, x * y2, x * z2
    yy, yz, zz = y * y2, y * z2, z * z2
    wx, wy, wz = w * x2, w * y2, w * z2
    one = np.float32(1.0)
    # columns
    return np.array([[one - (yy + zz), xy + wz, xz - wy], [xy - wz, one - (xx + zz), yz + wx],
                     [xz + wy, yz - wx, one - (xx + yy)]], np.float32).T


def _quat_y(a):
    return (0.0, math.sin(a / 2), 0.0, math.cos(a / 2))


def _state(ty, c, q, v, w, inv_mass, inv_inertia):
    """55 floats: type, R (column-major), p, local centre (0), c0, c, q0, q,
    v, w, 1/m, 1/I (body frame, column-major), world 1/I."""
    R = _qmat(q)
    ii = np.asarray(inv_inertia, np.float32)
    wii = (R @ ii @ R.T).astype(np.float32)
    c = np.asarray(c, np.float32)
    out = [float(ty)] + list(R.T.reshape(-1)) + list(c) + [0.0, 0.0, 0.0] + list(c) + list(c) + list(q) + list(q) + \
        list(v) + list(w) + [inv_mass] + list(ii.T.reshape(-1)) + list(wii.T.reshape(-1))
    return np.asarray(out, np.float32)


def _advance(s, dt, g):
    """One world step of a body: integrate velocity (dynamic: gravity),
    then the sweep (c0 = c, c += dt v, q += dt dq/dt, normalised)."""
    ty = int(s[0])
    if ty == 0:
        return s.copy()
    v = s[30:33].astype(np.float64)
    w = s[33:36].astype(np.float64)
    if ty == 2:
        v = v + dt * np.asarray(g, np.float64)
    c = s[19:22].astype(np.float64) + dt * v
    q = s[26:30].astype(np.float64)
    qx, qy, qz, qw = q
    wx, wy, wz = 0.5 * w
    dq = np.array([wx * qw + wy * qz - wz * qy, wy * qw + wz * qx - wx * qz, wz * qw + wx * qy - wy * qx,
                   -wx * qx - wy * qy - wz * qz])
    q = q + dt * dq
    q = q / np.linalg.norm(q)
    ii = s[37:46].reshape(3, 3).T
    out = _state(ty, c, q, v, w, float(s[36]), ii)
    out[16:19] = s[19:22]        # world centre 0 = the previous centre
    out[22:26] = s[26:30]        # orientation 0 = the previous orientation
    return out


def _aabb(kind, geom, R, p, radius):
    if kind == 0:
        ctr = R @ np.asarray(geom, np.float32) + p
        return ctr - radius, ctr + radius
    if kind == 1:
        a = R @ np.asarray(geom[:3], np.float32) + p
        b = R @ np.asarray(geom[3:], np.float32) + p
        return np.minimum(a, b) - radius, np.maximum(a, b) + radius
    pts = (R @ np.asarray(geom, np.float32).reshape(-1, 3).T).T + p
    return pts.min(0) - radius, pts.max(0) + radius


def _move_proxy(fat, lo, hi, disp):
    """A world broadphase keeping its fat proxies: re-fattened when the
    shape's box leaves them."""
    flo, fhi = fat
    if np.all(flo <= lo) and np.all(hi <= fhi):
        return fat
    d = 2.0 * disp
    nlo, nhi = lo - 0.2 + np.minimum(d, 0.0), hi + 0.2 + np.maximum(d, 0.0)
    return nlo.astype(np.float32), nhi.astype(np.float32)


def _box():
    hx, hy, hz = 0.12, 0.08, 0.12
    verts = np.array([(x, y, z) for x in (-hx, hx) for y in (-hy, hy) for z in (-hz, hz)], np.float32)
    planes = np.array([(1, 0, 0, hx), (-1, 0, 0, hx), (0, 1, 0, hy), (0, -1, 0, hy), (0, 0, 1, hz), (0, 0, -1, hz)],
                      np.float32)
    return verts, planes, (hx, hy, hz)


def _scene(b3g, port, side=16):
    scene = b3g.plain_scene(side)
    gpu = b3g.Cloth(scene.mesh, scene.cdef).setup(scene)
    ora = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for v in (side * (side - 1), side * side - 1):
        gpu.particle(v).set_type(0)
        ora.set_type(v, 0)
    verts, planes, (hx, hy, hz) = _box()
    m = 2.0 * (2 * hx) * (2 * hy) * (2 * hz)
    I = np.diag([m * ((2 * hy) ** 2 + (2 * hz) ** 2) / 12, m * ((2 * hx) ** 2 + (2 * hz) ** 2) / 12,
                 m * ((2 * hx) ** 2 + (2 * hy) ** 2) / 12])
    bodies = [
        _state(2, (0.05, 0.25, 0.0), _quat_y(0.3), (0, 0, 0), (0, 0, 0), 1.0 / m, np.linalg.inv(I)),
        _state(1, (-0.3, -0.45, 0.25), (0, 0, 0, 1), (0.1, 0.45, 0.0), (0, 0, 0), 0.0, np.zeros((3, 3))),
        _state(0, (0.3, -0.3, -0.25), _quat_y(0.5), (0, 0, 0), (0, 0, 0), 0.0, np.zeros((3, 3))),
    ]
    shapes = [(0, 2, np.concatenate([verts.reshape(-1), planes.reshape(-1)]), 0.0, 0.4, verts),
              (1, 0, np.zeros(3, np.float32), 0.1, 0.3, np.zeros(3, np.float32)),
              (2, 1, np.array([-0.15, 0, 0, 0.15, 0, 0], np.float32), 0.05, 0.5,
               np.array([-0.15, 0, 0, 0.15, 0, 0], np.float32))]
    for b in bodies:
        assert gpu.add_body(b) == ora.add_body(b)
    for (b, kind, geom, radius, mu, g) in shapes:
        if kind == 2:
            sg = gpu.add_body_hull(b, verts, planes, mu)
            so = ora.add_body_shape(b, 2, geom, 0.0, mu, len(verts), len(planes))
        elif kind == 0:
            sg = gpu.add_body_sphere(b, g, radius, mu)
            so = ora.add_body_shape(b, 0, g, radius, mu)
        else:
            sg = gpu.add_body_capsule(b, g[:3], g[3:], radius, mu)
            so = ora.add_body_shape(b, 1, g, radius, mu)
        assert sg == so
    return scene, gpu, ora, shapes


def test_body_colliders_per_step(b3g, port):
    """A dynamic box falling onto a cloth pinned at its four corners, a
    kinematic sphere rising into it from below, a static capsule at a rotated
    pose: each frame from identical inputs the GPU's cloth, contacts and
    bodies match the oracle's."""
    scene, gpu, ora, shapes = _scene(b3g, port)
    # the initial proxies agree (ComputeAABB(m_xf) fattened)
    for s in range(3):
        for u, w in zip(gpu.shape_proxy(s), ora.shape_proxy(s)):
            np.testing.assert_allclose(u, w, rtol=0, atol=1e-6)
    g = np.asarray(scene.gravity, np.float32)
    seen = [0, 0, 0]
    worst = {"x": 0.0, "bv": 0.0, "bc": 0.0}
    for step in range(90):
        # the world's step, from the bodies as the last cloth step left them
        for b in range(3):
            s0 = gpu.body(b)
            s1 = _advance(s0, scene.dt, g)
            gpu.set_body(b, s1)
            ora.set_body(b, s1)
        for sid, (b, kind, geom, radius, mu, gg) in enumerate(shapes):
            s1 = gpu.body(b)
            R = s1[1:10].reshape(3, 3).T
            p = s1[10:13]
            s0p = s1[16:19]
            lo, hi = _aabb(kind, gg, R, p, radius)
            fat = _move_proxy(gpu.shape_proxy(sid), lo, hi, p - s0p)
            gpu.set_shape_proxy(sid, *fat)
            ora.set_shape_proxy(sid, *fat)
        gpu.set_report_order([0, 1, 2])
        ora.set_report_order([0, 1, 2])
        st = gpu.state()
        ora.set_state(x=st["x"], v=st["v"], dv=st["dv"])
        a = gpu.step(scene.dt)
        o = ora.step(scene.dt)
        assert abs(a["iterations"] - o["iterations"]) <= 1, step
        assert abs(int(a["active_contacts"]) - int(o["active_contacts"])) <= max(2, o["active_contacts"] // 100), \
            (step, a["active_contacts"], o["active_contacts"])
        ex = rel_err(gpu.state()["x"], ora.state()["x"])
        worst["x"] = max(worst["x"], ex)
        assert ex <= 1e-5, (step, ex)
        vmax = max(1.0, max(float(np.abs(ora.body(b)[30:36]).max()) for b in range(3)))
        for b in range(3):
            gb, ob = gpu.body(b), ora.body(b)
            dv = float(np.abs(gb[30:36] - ob[30:36]).max()) / vmax
            dc = float(np.abs(gb[19:22] - ob[19:22]).max())
            dq = float(np.abs(gb[26:30] - ob[26:30]).max())
            worst["bv"] = max(worst["bv"], dv)
            worst["bc"] = max(worst["bc"], dc, dq)
            assert dv <= 1e-5, (step, b, dv)
            assert dc <= 1e-6 and dq <= 1e-6, (step, b, dc, dq)
            assert np.array_equal(gb[0:1], ob[0:1])
        oc = ora.contact_list()
        for s in range(3):
            seen[s] = max(seen[s], int(oc["active"][oc["shape"] == s].sum()))
    print("worst", worst, "seen", seen)
    # every collider touched the cloth
    assert min(seen) > 0, seen


def test_body_colliders_push_the_box(b3g, port):
    """The cloth catches the dynamic box and throws it back up (free fall
    alone only ever moves it down), and after each step the box's transform
    is its sweep's (SynchronizeTransform) and its proxy holds the box."""
    scene, gpu, ora, shapes = _scene(b3g, port)
    g = np.asarray(scene.gravity, np.float32)
    up = 0.0
    for step in range(60):
        for b in range(3):
            gpu.set_body(b, _advance(gpu.body(b), scene.dt, g))
        for sid, (b, kind, geom, radius, mu, gg) in enumerate(shapes):
            s1 = gpu.body(b)
            R = s1[1:10].reshape(3, 3).T
            lo, hi = _aabb(kind, gg, R, s1[10:13], radius)
            gpu.set_shape_proxy(sid, *_move_proxy(gpu.shape_proxy(sid), lo, hi, s1[10:13] - s1[16:19]))
        gpu.step(scene.dt)
        box = gpu.body(0)
        up = max(up, float(box[31]))
        R = box[1:10].reshape(3, 3).T
        np.testing.assert_allclose(R, _qmat(box[26:30]), atol=1e-6)
        np.testing.assert_allclose(box[10:13], box[19:22] - R @ box[13:16], atol=1e-6)
        lo, hi = _aabb(2, shapes[0][5], R, box[10:13], 0.0)
        flo, fhi = gpu.shape_proxy(0)
        assert np.all(flo <= lo + 1e-6) and np.all(hi <= fhi + 1e-6), step
    assert up > 0.5, up


def test_body_api_errors(b3g):
    scene = b3g.plain_scene(8)
    cloth = b3g.Cloth(scene.mesh, scene.cdef).setup(scene)
    bad = _state(2, (0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (0, 0, 0), 1.0, np.eye(3))
    bad[0] = 5.0
    with pytest.raises(b3g.B3gError):
        cloth.add_body(bad)
    nan = _state(2, (0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (0, 0, 0), 1.0, np.eye(3))
    nan[20] = np.nan
    with pytest.raises(b3g.B3gError):
        cloth.add_body(nan)
    with pytest.raises(b3g.B3gError):
        cloth.add_body_sphere(0, (0, 0, 0), 0.1, 0.3)     # no such body
    b = cloth.add_body(_state(1, (0, -1, 0), (0, 0, 0, 1), (0, 0, 0), (0, 0, 0), 0.0, np.zeros((3, 3))))
    s = cloth.add_body_sphere(b, (0, 0, 0), 0.1, 0.3)
    with pytest.raises(b3g.B3gError):
        cloth.set_shape_proxy(s, (1, 1, 1), (0, 0, 0))   # lo above hi
    with pytest.raises(b3g.B3gError):
        cloth.set_report_order([0, 0])
    for _ in range(3):
        cloth.add_body_sphere(b, (0, 0, 0), 0.1, 0.3)
    with pytest.raises(b3g.B3gError) as e:
        cloth.add_body_sphere(b, (0, 0, 0), 0.1, 0.3)
    assert e.value.status == 8   # B3G_ERR_CAPACITY
    # stepping works with a kinematic body far below
    cloth.step(scene.dt)
