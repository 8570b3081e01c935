"""Soft body on the GPU (b3g_softbody_*) against the CPU oracle.

Tolerances:
* masses and, from identical state, the assembled system A, b and S:
  bit-exact (the element and assembly arithmetic is the reference's; the
  rotation extraction's sin and cos are CUDA's double functions rounded to
  float, equal to the C library's there);
* one step from identical state: CG iterations within +-1 (the GPU sums the
  dot products in another order), positions and velocities within 1e-4
  relative;
* free trajectories: bounded drift, and the bulk motion agrees.
"""
import os

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "softbody_block_ref.npz")


def _pair(b3g, port, scene, opts=None):
    s = scene.sdef
    gpu = b3g.SoftBody(scene.vertices, scene.tets, s).setup(scene, opts)
    ora = port.PortSoftBody(scene.vertices, scene.tets, s.density, s.E, s.nu, s.c_yield, s.c_creep,
                            s.c_max).setup(scene)
    if opts is not None:
        ora.set_solver(opts.stop_rule, opts.tolerance, opts.max_iterations, opts.dot)
    return gpu, ora


def _sync(gpu, ora):
    st, el = gpu.state(), gpu.elements()
    ora.set_state(x=st["x"], v=st["v"])
    ora.set_elements(q=el["q"], eps=el["eps"])


def test_softbody_system_bit_exact(b3g, port):
    scene = b3g.pinned_block_scene(4, 3, 3, spacing=0.5)
    gpu, ora = _pair(b3g, port, scene)
    assert np.array_equal(gpu.masses(), ora.masses())
    for step in range(25):
        if step % 6 == 0:
            gpu.apply_force(7, [3.0, 40.0, -2.0])
            ora.apply_force(7, [3.0, 40.0, -2.0])
        if step in (0, 5, 24):
            _sync(gpu, ora)
            gs, os_ = gpu.system(scene.dt), ora.system(scene.dt)
            for k in ("rowptr", "cols", "vals", "b", "S"):
                assert np.array_equal(gs[k], os_[k]), (step, k)
        gpu.step(scene.dt)
        ora.step(scene.dt)


@pytest.mark.parametrize("form", ["persistent", "fused", "launches"])
@pytest.mark.parametrize("dot", [0, 2])
def test_softbody_step_matches_oracle(b3g, port, dot, form):
    """Each step starts the oracle from the GPU's state (positions,
    velocities, element rotations and plastic strains); the MPCG as one
    persistent launch (two grid reductions per iteration, or one) and as
    three launches per iteration."""
    scene = b3g.pinned_block_scene(5, 4, 3, spacing=0.5)
    opts = b3g.SolverOptions.reference() if dot == 0 else b3g.SolverOptions.relative(1e-5, 200, dot)
    gpu, ora = _pair(b3g, port, scene, opts)
    gpu.set_cg_strategy(form != "launches", fused=form == "fused")
    gpu.set_node_type(3, 1)
    ora.set_type(3, 1)
    gpu.set_velocity(3, [0.2, 0.0, 0.0])
    ora.set_velocity(3, [0.2, 0.0, 0.0])
    for step in range(40):
        _sync(gpu, ora)
        if step % 9 == 0:
            gpu.apply_force(11, [0.0, 60.0, 5.0])
            ora.apply_force(11, [0.0, 60.0, 5.0])
        g = gpu.step(scene.dt)
        o = ora.step(scene.dt)
        assert abs(g["iterations"] - o["iterations"]) <= 1, (step, g["iterations"], o["iterations"])
        gs, os_ = gpu.state(), ora.state()
        assert rel_err(gs["x"], os_["x"]) <= 1e-4, step
        assert rel_err(gs["v"], os_["v"]) <= 1e-4, step
        ge, oe = gpu.elements(), ora.elements()
        assert np.abs(ge["q"] - oe["q"]).max() <= 1e-5, step
        assert np.abs(ge["eps"] - oe["eps"]).max() <= 1e-5, step
    assert np.abs(gpu.elements()["eps"]).max() > 1e-3  # plastic flow happened


def test_softbody_against_reference_golden(b3g, port):
    """The reference's own trajectory (golden file, 120 steps with a
    kinematic node and force pulses): the GPU trajectory stays within a
    bounded drift of it, and the oracle reproduces it exactly."""
    d = np.load(GOLDEN)
    sdef = b3g.SoftBodyDef(*[float(x) for x in d["def"]])
    scene = b3g.SoftBodyScene(d["vertices"], d["tets"], sdef, d["mass_damping"], d["static"],
                              gravity=tuple(float(g) for g in d["gravity"]), dt=float(d["dt"]))
    gpu = b3g.SoftBody(scene.vertices, scene.tets, sdef).setup(scene)
    assert np.array_equal(gpu.masses(), d["mass"])
    gpu.set_node_type(int(d["kinematic"]), 1)
    gpu.set_velocity(int(d["kinematic"]), d["kinematic_v"])
    per = int(d["force_period"])
    drift = []
    for k in range(1, len(d["iterations"]) + 1):
        if (k - 1) % per == 0:
            gpu.apply_force(int(d["force_node"]), d["force"])
        g = gpu.step(scene.dt)
        assert abs(g["iterations"] - int(d["iterations"][k - 1])) <= 1
        if f"x_{k}" in d:
            drift.append(float(np.abs(gpu.state()["x"] - d[f"x_{k}"]).max()))
    print("soft body drift against the reference (m) at the kept steps:", drift)
    assert drift[0] <= 1e-5
    assert max(drift) <= 1e-2


def test_softbody_persistent_cg_large_block(b3g, port):
    """The persistent MPCG on a block with more rows than the GPU has
    threads in one pass of one-row CTAs (several rows per thread), at a
    relative stop: one step from identical state against the oracle and
    against the three-launch form."""
    scene = b3g.pinned_block_scene(48, 48, 48, spacing=1.0 / 48)
    opts = b3g.SolverOptions.relative(1e-5, 400, 2)
    gpu, ora = _pair(b3g, port, scene, opts)
    other = b3g.SoftBody(scene.vertices, scene.tets, scene.sdef).setup(scene, opts)
    other.set_cg_strategy(False)
    for _ in range(3):
        gpu.step(scene.dt)
    st, el = gpu.state(), gpu.elements()
    _sync(gpu, ora)
    other.write_state(st["x"], st["v"])
    other.write_elements(el["q"], el["eps"])
    g = gpu.step(scene.dt)
    o = ora.step(scene.dt)
    h = other.step(scene.dt)
    assert abs(g["iterations"] - o["iterations"]) <= 1, (g["iterations"], o["iterations"])
    assert abs(g["iterations"] - h["iterations"]) <= 1, (g["iterations"], h["iterations"])
    assert rel_err(gpu.state()["x"], ora.state()["x"]) <= 1e-4
    assert rel_err(gpu.state()["v"], ora.state()["v"]) <= 1e-3
    assert rel_err(gpu.state()["x"], other.state()["x"]) <= 1e-4


def test_softbody_free_fall_matches_oracle_bulk(b3g, port):
    scene = b3g.pinned_block_scene(4, 4, 4)
    gpu, ora = _pair(b3g, port, scene)
    d = []
    for step in range(100):
        gpu.step(scene.dt)
        ora.step(scene.dt)
        d.append(float(np.abs(gpu.state()["x"] - ora.state()["x"]).max()))
    print("soft body drift GPU-oracle (m) at 1/10/50/100:", d[0], d[9], d[49], d[99])
    assert d[0] <= 1e-5
    assert max(d) <= 1e-2
    assert abs(gpu.energy() - ora.energy()) <= 1e-2 * max(ora.energy(), 1e-6)


def test_softbody_rejects_degenerate_mesh(b3g):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], np.float32)  # flat: zero volume
    t = np.array([[0, 1, 2, 3]], np.uint32)
    with pytest.raises(b3g.B3gError):
        b3g.SoftBody(v, t, b3g.SoftBodyDef())


def _hull_pair(b3g, port):
    from test_softbody_oracle import softbody_hull_golden

    d, scene = softbody_hull_golden()
    s = scene.sdef
    bodies = (b3g.SoftBody(scene.vertices, scene.tets, s).setup(scene),
              port.PortSoftBody(scene.vertices, scene.tets, s.density, s.E, s.nu, s.c_yield, s.c_creep,
                                s.c_max).setup(scene))
    for b in bodies:
        b.add_hull(d["hull_vertices"], d["hull_planes"], float(d["hull_friction"]))
        for i in range(len(scene.vertices)):
            b.set_node_radius(i, float(d["node_radius"]))
            b.set_node_friction(i, float(d["node_friction"]))
    return d, scene, bodies[0], bodies[1]


def test_softbody_hull_contacts_per_step(b3g, port):
    """Node contacts with a static hull (softbody_contact_manager.cpp,
    softbody_contact_solver.cpp): each step starts the oracle from the GPU's
    positions, velocities and element state; x within 1e-4 relative, the
    contact sets within 2 nodes.  Once the block rests its velocities are
    near zero, so v is held to 1e-4 of the larger of its own size and the
    velocity one step of gravity adds."""
    d, scene, gpu, ora = _hull_pair(b3g, port)
    vscale = float(np.linalg.norm(scene.gravity)) * scene.dt
    seen, worst = 0, 0.0
    for step in range(150):
        _sync(gpu, ora)
        g = gpu.step(scene.dt)
        o = ora.step(scene.dt)
        gc, oc = gpu.contacts(), ora.contacts()
        seen = max(seen, int(oc["active"].sum()))
        assert abs(g["iterations"] - o["iterations"]) <= 1, step
        assert int(np.sum(gc["exists"] != oc["exists"])) <= 2, step
        assert int(np.sum(gc["active"] != oc["active"])) <= 2, step
        gs, os_ = gpu.state(), ora.state()
        assert rel_err(gs["x"], os_["x"]) <= 1e-4, step
        ev = float(np.abs(gs["v"] - os_["v"]).max()) / max(float(np.abs(os_["v"]).max()), vscale)
        worst = max(worst, ev)
        assert ev <= 1e-4, step
    print("softbody hull per step: worst v error", worst, "of scale; most active", seen)
    assert seen > 10  # the block came to rest on the hull


def test_softbody_hull_against_reference_golden(b3g, port):
    """Free run from the reference's start: after one step the same contacts
    and x within 1e-4 m; at steps 25, 75 and 150 the block rests on the hull
    with x within 5e-4 m and the active contacts within 2."""
    d, scene, gpu, _ = _hull_pair(b3g, port)
    for k in range(1, len(d["iterations"]) + 1):
        gpu.step(scene.dt)
        if f"x_{k}" in d:
            x, c = gpu.state()["x"], gpu.contacts()
            dx = float(np.abs(x - d[f"x_{k}"]).max())
            ga, ra = int(c["active"].sum()), int(d[f"contact_active_{k}"].sum())
            print("softbody hull golden: step", k, "max |dx|", dx, "active", ga, ra)
            if k == 1:
                assert dx <= 1e-4
                assert np.array_equal(c["exists"], d["contact_exists_1"])
                assert np.array_equal(c["active"], d["contact_active_1"])
            else:
                assert dx <= 5e-4, k
                assert abs(ga - ra) <= 2, k


def _box(c, h):
    """A box hull (vertices, face planes) with centre c and half extents h."""
    c, h = np.asarray(c, np.float32), np.asarray(h, np.float32)
    v = np.array([c + h * (2 * np.array(s, np.float32) - 1) for s in np.ndindex(2, 2, 2)], np.float32)
    planes = []
    for k in range(3):
        n = np.zeros(3, np.float32)
        n[k] = 1.0
        planes.append((*n, c[k] + h[k]))
        planes.append((*(-n), -(c[k] - h[k])))
    return v, np.array(planes, np.float32)


def test_softbody_two_hulls_per_step(b3g, port):
    """A free block falling onto a ground hull beside a wall hull that its
    side already touches: contacts with both hulls, per step from the GPU's
    state as above; the oracle's contact count equals the GPU's."""
    import dataclasses

    scene = dataclasses.replace(b3g.pinned_block_scene(6, 6, 6, spacing=1.0 / 6),
                                static_nodes=np.zeros(0, np.uint32))
    s = scene.sdef
    gpu = b3g.SoftBody(scene.vertices, scene.tets, s).setup(scene)
    ora = port.PortSoftBody(scene.vertices, scene.tets, s.density, s.E, s.nu, s.c_yield, s.c_creep,
                            s.c_max).setup(scene)
    hulls = [_box((0.0, -0.81, 0.0), (3.0, 0.25, 3.0)), _box((0.78, 0.0, 0.0), (0.25, 2.0, 2.0))]
    for b in (gpu, ora):
        for hv, hp in hulls:
            b.add_hull(hv, hp, 0.6)
        for i in range(len(scene.vertices)):
            b.set_node_radius(i, 0.05)
            b.set_node_friction(i, 0.2)
    vscale = float(np.linalg.norm(scene.gravity)) * scene.dt
    per_hull = np.zeros(2, int)
    for step in range(40):
        _sync(gpu, ora)
        gpu.step(scene.dt)
        ora.step(scene.dt)
        gc, oc = gpu.contacts(), ora.contacts()
        assert abs(int(gc["exists"].sum()) - oc["count"]) <= 2, step
        per_hull = np.maximum(per_hull, gc["active"].reshape(2, -1).sum(axis=1))
        gs, os_ = gpu.state(), ora.state()
        assert rel_err(gs["x"], os_["x"]) <= 1e-4, step
        assert float(np.abs(gs["v"] - os_["v"]).max()) <= 1e-4 * max(float(np.abs(os_["v"]).max()), vscale), step
    assert per_hull.min() > 0, per_hull  # both hulls pushed nodes


def test_softbody_hull_arguments(b3g):
    """Argument and capacity errors of the hull and node-property calls."""
    scene = b3g.pinned_block_scene(3, 3, 3, spacing=0.5)
    body = b3g.SoftBody(scene.vertices, scene.tets, scene.sdef).setup(scene)
    assert body.contacts()["exists"].size == 0  # no hull, no contact slots
    body.step(scene.dt)
    n = len(scene.vertices)
    for call in (lambda: body.set_node_radius(n, 0.1), lambda: body.set_node_radius(0, -1.0),
                 lambda: body.set_node_friction(0, float("nan")),
                 lambda: body.add_hull(np.zeros((0, 3)), np.zeros((0, 4)), 0.5)):
        with pytest.raises(b3g.B3gError) as e:
            call()
        assert e.value.status == 1
    hv, hp = _box((0.0, -3.0, 0.0), (1.0, 0.5, 1.0))
    for _ in range(4):
        body.add_hull(hv, hp, 0.5)
    with pytest.raises(b3g.B3gError) as e:
        body.add_hull(hv, hp, 0.5)
    assert e.value.status == 8
    body.step(scene.dt)
    assert body.contacts()["exists"].size == 4 * n


def test_softbody_coplanar_hulls_contact_order(b3g, port):
    """A block landing on three overlapping hulls whose tops lie in one plane,
    so that nodes over the overlaps rest on two or three hulls at once.  A
    node's contacts are solved in the list order Bounce gives them, which the
    world query's tree decides; per step from the GPU's state, positions,
    velocities and each (hull, node) contact's impulses match the oracle,
    which matches the reference's own list bit for bit
    (test_softbody_overlapping_hulls_match_live_reference)."""
    from bounce_b200.meshes import SoftBodyDef, SoftBodyScene, block_softbody_mesh

    verts, tets = block_softbody_mesh(4, 3, 3, 0.5)
    sdef = SoftBodyDef(density=0.2, E=1000.0, nu=0.33, c_yield=0.1, c_creep=0.5, c_max=1.0)
    scene = SoftBodyScene(verts, tets, sdef, np.full(len(verts), 0.2, np.float32), np.zeros(0, np.uint32))
    boxes = [((-3.0, -1.5, -3.0), (3.0, -0.9, 3.0)), ((-1.2, -1.4, -1.0), (0.3, -0.9, 1.0)),
             ((-0.3, -1.3, -1.0), (1.2, -0.9, 1.0))]
    gpu = b3g.SoftBody(verts, tets, sdef).setup(scene)
    ora = port.PortSoftBody(verts, tets, sdef.density, sdef.E, sdef.nu, sdef.c_yield, sdef.c_creep,
                            sdef.c_max).setup(scene)
    for lo, hi in boxes:
        c, h = (np.add(lo, hi) / 2.0), (np.subtract(hi, lo) / 2.0)
        hv, hp = _box(tuple(c), tuple(h))
        for b in (gpu, ora):
            b.add_hull(hv, hp, 0.4)
    for b in (gpu, ora):
        for i in range(len(verts)):
            b.set_node_radius(i, 0.05)
            b.set_node_friction(i, 0.3)
    n = len(verts)
    vscale = float(np.linalg.norm(scene.gravity)) * scene.dt
    multi = 0
    for step in range(60):
        _sync(gpu, ora)
        gpu.step(scene.dt)
        ora.step(scene.dt)
        gs, os_ = gpu.state(), ora.state()
        assert rel_err(gs["x"], os_["x"]) <= 1e-4, step
        assert float(np.abs(gs["v"] - os_["v"]).max()) <= 1e-4 * max(float(np.abs(os_["v"]).max()), vscale), step
        gc, ol = gpu.contacts(), ora.contact_list()
        oimp = np.zeros((3 * n, 3), np.float32)
        oact = np.zeros(3 * n, np.uint8)
        slot = ol["shape"].astype(np.int64) * n + ol["node"].astype(np.int64)
        oimp[slot] = ol["impulses"]
        oact[slot] = ol["active"]
        both = (gc["active"] != 0) & (oact != 0)
        scale = max(float(np.abs(oimp).max()), 1e-6)
        assert float(np.abs(gc["impulses"][both] - oimp[both]).max(initial=0.0)) <= 1e-3 * scale, step
        nodes = np.nonzero(oact)[0] % n
        multi = max(multi, int((np.bincount(nodes, minlength=n) >= 2).sum()) if nodes.size else 0)
    assert multi > 0
