"""The soft body restatement (oracle/softbody_oracle.c) against the reference.

Against the golden fixture the reference produced (tests/golden/gen_golden.py,
needs no reference tree) and, where the reference library is built here,
against the live b3SoftBody: masses, element matrices, states, element
rotations and plastic strains bit for bit, CG iterations equal.
"""
import os

import numpy as np
import pytest

import oracle
from bounce_b200.meshes import SoftBodyDef, SoftBodyScene, pinned_block_scene

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "softbody_block_ref.npz")


def _golden_scene(d):
    a = [float(x) for x in d["def"]]
    sdef = SoftBodyDef(*a)
    return SoftBodyScene(d["vertices"], d["tets"], sdef, d["mass_damping"], d["static"],
                         gravity=tuple(float(g) for g in d["gravity"]), dt=float(d["dt"]))


def _make(cls, scene):
    s = scene.sdef
    return cls(scene.vertices, scene.tets, s.density, s.E, s.nu, s.c_yield, s.c_creep, s.c_max).setup(scene)


def test_softbody_oracle_matches_golden(port):
    d = np.load(GOLDEN)
    scene = _golden_scene(d)
    b = _make(port.PortSoftBody, scene)
    assert np.array_equal(b.masses(), d["mass"])
    for key in d.files:
        if key.startswith("el") and key.endswith("_K"):
            e = int(key[2:-2])
            ed = b.element_data(e)
            for k in ("K", "invE", "B", "P"):
                assert np.array_equal(ed[k], d[f"el{e}_{k}"]), (e, k)
    b.set_type(int(d["kinematic"]), 1)
    b.set_velocity(int(d["kinematic"]), d["kinematic_v"])
    per = int(d["force_period"])
    for k in range(1, len(d["iterations"]) + 1):
        if (k - 1) % per == 0:
            b.apply_force(int(d["force_node"]), d["force"])
        it = b.step(scene.dt)["iterations"]
        assert it == d["iterations"][k - 1], (k, it)
        if f"x_{k}" in d:
            st, el = b.state(), b.elements()
            assert np.array_equal(st["x"], d[f"x_{k}"]), k
            assert np.array_equal(st["v"], d[f"v_{k}"]), k
            assert np.array_equal(el["q"], d[f"q_{k}"]), k
            assert np.array_equal(el["eps"], d[f"eps_{k}"]), k
    # the plastic flow and the rotations were exercised
    assert np.abs(d["eps_120"]).max() > 1e-2
    assert d["q_120"][:, 3].min() < 0.999


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("dims", [(2, 2, 2), (3, 4, 2)])
def test_softbody_oracle_matches_live_reference(dims):
    scene = pinned_block_scene(*dims, spacing=0.75)
    port = _make(oracle.PortSoftBody, scene)
    ref = _make(oracle.RefSoftBody, scene)
    for e in range(port.t):
        a, b = port.element_data(e), ref.element_data(e)
        for k in a:
            assert np.array_equal(a[k], b[k]), (e, k)
    for k in range(40):
        if k % 5 == 0:
            for o in (port, ref):
                o.apply_force(1, [2.0, 30.0, -1.0])
        a = port.step(scene.dt)
        b = ref.step(scene.dt)
        assert a["iterations"] == b["iterations"]
        sa, sb = port.state(), ref.state()
        assert np.array_equal(sa["x"], sb["x"]) and np.array_equal(sa["v"], sb["v"]), k
        ea, eb = port.elements(), ref.elements()
        assert np.array_equal(ea["q"], eb["q"]) and np.array_equal(ea["eps"], eb["eps"]), k
    assert port.energy() == ref.energy()


def softbody_hull_golden():
    """The scene of softbody_hull_ref.npz: a block falling onto a ground
    hull (the reference's quickhull output, stored in the file)."""
    import os

    from bounce_b200.meshes import SoftBodyDef, SoftBodyScene

    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "softbody_hull_ref.npz"))
    sdef = SoftBodyDef(*[float(x) for x in d["def"]])
    scene = SoftBodyScene(d["vertices"], d["tets"], sdef, d["mass_damping"], np.zeros(0, np.uint32),
                          gravity=tuple(float(g) for g in d["gravity"]), dt=float(d["dt"]))
    return d, scene


def test_softbody_hull_contacts_match_golden(port):
    """Node contacts with a static hull (b3SoftBody with a world,
    softbody_contact_manager.cpp, softbody_contact_solver.cpp): the
    restatement reproduces the reference's trajectory and contacts."""
    d, scene = softbody_hull_golden()
    s = scene.sdef
    b = port.PortSoftBody(scene.vertices, scene.tets, s.density, s.E, s.nu, s.c_yield, s.c_creep,
                          s.c_max).setup(scene)
    b.add_hull(d["hull_vertices"], d["hull_planes"], float(d["hull_friction"]))
    for i in range(len(scene.vertices)):
        b.set_node_radius(i, float(d["node_radius"]))
        b.set_node_friction(i, float(d["node_friction"]))
    for k in range(1, len(d["iterations"]) + 1):
        assert b.step(scene.dt)["iterations"] == d["iterations"][k - 1], k
        if f"x_{k}" in d:
            st, c = b.state(), b.contacts()
            assert np.array_equal(st["x"], d[f"x_{k}"]) and np.array_equal(st["v"], d[f"v_{k}"]), k
            for q in ("exists", "active", "impulses"):
                assert np.array_equal(c[q], d[f"contact_{q}_{k}"]), (k, q)
    assert int(d["contact_active_150"].sum()) > 10


def _box_points(lo, hi):
    return np.array([(x, y, z) for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])], np.float32)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_softbody_overlapping_hulls_match_live_reference():
    """A block landing on three overlapping hulls (a ground slab and two
    boxes whose tops lie in the slab's top plane, overlapping each other).  A node
    touching several hulls has its contacts in the world query's report
    order, which the restatement derives from the broadphase tree; positions,
    velocities and every contact's state and impulses match the reference
    bit for bit."""
    from bounce_b200.meshes import SoftBodyDef, SoftBodyScene, block_softbody_mesh

    verts, tets = block_softbody_mesh(4, 3, 3, 0.5)
    sdef = SoftBodyDef(density=0.2, E=1000.0, nu=0.33, c_yield=0.1, c_creep=0.5, c_max=1.0)
    scene = SoftBodyScene(verts, tets, sdef, np.full(len(verts), 0.2, np.float32), np.zeros(0, np.uint32))
    # the three tops lie in one plane: nodes over the overlaps rest on two or
    # three hulls at once
    boxes = [((-3.0, -1.5, -3.0), (3.0, -0.9, 3.0)), ((-1.2, -1.4, -1.0), (0.3, -0.9, 1.0)),
             ((-0.3, -1.3, -1.0), (1.2, -0.9, 1.0))]
    port = _make(oracle.PortSoftBody, scene)
    ref = _make(oracle.RefSoftBody, scene)
    for lo, hi in boxes:
        hv, hp = ref.add_hull_from_points(_box_points(lo, hi), 0.4)
        port.add_hull(hv, hp, 0.4)
    for b in (port, ref):
        for i in range(len(verts)):
            b.set_node_radius(i, 0.05)
            b.set_node_friction(i, 0.3)
    multi = 0
    for k in range(60):
        a, b = port.step(scene.dt), ref.step(scene.dt)
        assert a["iterations"] == b["iterations"], k
        sa, sb = port.state(), ref.state()
        assert np.array_equal(sa["x"], sb["x"]) and np.array_equal(sa["v"], sb["v"]), k
        la, lb = port.contact_list(), ref.contact_list()
        for q in ("node", "shape", "active", "impulses"):
            assert np.array_equal(la[q], lb[q]), (k, q)
        nodes = lb["node"][lb["active"] != 0]
        multi = max(multi, int((np.bincount(nodes, minlength=len(verts)) >= 2).sum()) if nodes.size else 0)
    assert multi > 0  # some node had two or more active hull contacts at once
