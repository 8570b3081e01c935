"""The C restatement (oracle/) against the reference's own outputs.

The golden files under tests/golden/ were produced by the reference library
compiled from the Bounce sources (tests/golden/gen_golden.py).  The
restatement reproduces them bit for bit: same element arithmetic, same force
and sparse-row summation order, same sequential FP32 dot products.
"""
import os

import numpy as np
import pytest

from bounce_b200.meshes import ClothDef, Mesh, Scene

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _scene(d):
    mesh = Mesh(d["vertices"], d["triangles"])
    a = d["def"]
    cdef = ClothDef(*[float(x) for x in a])
    sph = []
    if "sphere" in d:
        s = d["sphere"]
        sph = [((float(s[0]), float(s[1]), float(s[2])), float(s[3]), float(s[4]))]
    return Scene("golden", mesh, cdef, d["pinned"], spheres=sph, dt=float(d["dt"]))


@pytest.mark.parametrize("name", ["plain32_ref.npz", "sphere32_ref.npz"])
def test_oracle_trajectory_bit_exact(port, name):
    d = np.load(os.path.join(GOLDEN, name))
    scene = _scene(d)
    c = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    assert np.array_equal(c.state()["mass"], d["mass"])
    steps = len(d["iterations"])
    for k in range(1, steps + 1):
        it = c.step(scene.dt)["iterations"]
        assert it == d["iterations"][k - 1], (k, it)
        if f"x_{k}" in d:
            s = c.state()
            for q in ("x", "v", "dv"):
                assert np.array_equal(s[q], d[f"{q}_{k}"]), (name, k, q, np.abs(s[q] - d[f"{q}_{k}"]).max())
            if f"contact_exists_{k}" in d:
                cts = c.contacts()
                assert np.array_equal(cts["exists"], d[f"contact_exists_{k}"])
                assert np.array_equal(cts["active"], d[f"contact_active_{k}"])
                assert np.array_equal(cts["impulses"], d[f"contact_impulses_{k}"])


def test_oracle_system_bit_exact(port):
    d = np.load(os.path.join(GOLDEN, "system16_bend_ref.npz"))
    scene = _scene(d)
    c = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    c.set_state(x=d["x_1"], v=d["v_1"], dv=d["dv_1"])
    s = c.system(scene.dt)
    for k in ("rowptr", "cols", "vals", "b", "S", "x0", "vertex_of_row"):
        assert np.array_equal(s[k], d[f"sys_{k}"]), k


def test_oracle_mpcg_on_reference_system(port):
    """The restated MPCG on the reference's exported system reproduces the
    reference's own solution m_x (cloth_force_solver.cpp:61-136)."""
    d = np.load(os.path.join(GOLDEN, "system16_bend_ref.npz"))
    sysd = {k[4:]: d[k] for k in d.files if k.startswith("sys_")}
    x, it, stats = port.mpcg(sysd, port.STOP_REFERENCE, 0.0, 20, port.DOT_F32)
    assert 1 <= it <= 20
    assert stats["delta"] <= stats["delta0"]
    # FP64 solve of the same system: the FP32 MPCG answer is close to it
    x64, it64 = port.solve_f64(sysd, 1e-12, 100000)
    S = sysd["S"].astype(bool)
    err = np.abs(x[S] - x64[S]).max() / max(np.abs(x64[S]).max(), 1e-30)
    assert err < 1e-2, err


@pytest.mark.parametrize("dot", [0, 1, 2])
def test_oracle_relative_mode_converges(port, dot):
    from bounce_b200.meshes import plain_scene

    scene = plain_scene(24)
    c = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    c.set_solver(port.STOP_RELATIVE, 1e-4, 50, dot)
    for _ in range(5):
        info = c.step(scene.dt)
        assert info["iterations"] == 50 or info["delta"] <= 1e-8 * info["b_delta"] * (1 + 1e-6)


def self_collision_golden_scene(d):
    """The scene of self_collision11_ref.npz (a cloth folding over a capsule
    with thickness 0.2)."""
    mesh = Mesh(d["vertices"], d["triangles"])
    cdef = ClothDef(*[float(x) for x in d["def"]])
    c = [float(x) for x in d["capsule"]]
    return Scene("golden_self", mesh, cdef, np.zeros(0, np.uint32), capsules=[(c[0:3], c[3:6], c[6], c[7])],
                 dt=float(d["dt"]))


def test_oracle_self_collision_bit_exact(port):
    """Particle-triangle contacts: the restatement reproduces the reference's
    trajectory and its contact list (order, active flags, weights of active
    contacts, impulses) at the kept steps."""
    d = np.load(os.path.join(GOLDEN, "self_collision11_ref.npz"))
    scene = self_collision_golden_scene(d)
    c = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for k in range(1, len(d["iterations"]) + 1):
        assert c.step(scene.dt)["iterations"] == d["iterations"][k - 1], k
        if f"x_{k}" in d:
            s = c.state()
            for q in ("x", "v", "dv"):
                assert np.array_equal(s[q], d[f"{q}_{k}"]), (k, q)
            t = c.tri_contacts()
            w = t["w"].copy()
            w[t["active"] == 0] = 0.0
            assert np.array_equal(t["pt"], d[f"tc_pt_{k}"]), k
            assert np.array_equal(t["active"], d[f"tc_active_{k}"]), k
            assert np.array_equal(w, d[f"tc_w_{k}"]), k
            assert np.array_equal(t["impulses"], d[f"tc_impulses_{k}"]), k
    assert int(d["tc_active_100"].sum()) > 10


def hull_golden_scene(d):
    """The scene of hull16_ref.npz: a 16 x 16 cloth falling onto a static
    hull (the reference's quickhull output, stored in the file)."""
    mesh = Mesh(d["vertices"], d["triangles"])
    cdef = ClothDef(*[float(x) for x in d["def"]])
    return Scene("golden_hull", mesh, cdef, np.zeros(0, np.uint32),
                 hulls=[(d["hull_vertices"], d["hull_planes"], float(d["hull_friction"]))], dt=float(d["dt"]))


def test_oracle_hull_bit_exact(port):
    """Hull colliders (b3HullShape::TestSphere with b3GJK): the restatement
    reproduces the reference's trajectory and body contacts exactly."""
    d = np.load(os.path.join(GOLDEN, "hull16_ref.npz"))
    scene = hull_golden_scene(d)
    c = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for k in range(1, len(d["iterations"]) + 1):
        assert c.step(scene.dt)["iterations"] == d["iterations"][k - 1], k
        if f"x_{k}" in d:
            s = c.state()
            for q in ("x", "v", "dv"):
                assert np.array_equal(s[q], d[f"{q}_{k}"]), (k, q)
            cts = c.contacts()
            assert np.array_equal(cts["exists"], d[f"contact_exists_{k}"]), k
            assert np.array_equal(cts["active"], d[f"contact_active_{k}"]), k
            assert np.array_equal(cts["impulses"], d[f"contact_impulses_{k}"]), k
    assert int(d["contact_active_60"].sum()) > 100
