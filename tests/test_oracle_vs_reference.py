"""The restatement against the live reference library (when it is built here).

Skipped when oracle/_ref/libbounce_ref.so is absent (it is compiled from the
reference sources, which only exist where the reference tree is mounted).
"""
import numpy as np
import pytest

import oracle
from bounce_b200.meshes import plain_scene, sewn_scene, sphere_scene

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")


@pytest.mark.parametrize("side", [8, 16])
def test_restated_constructor_matches_reference(side):
    scene = sphere_scene(side)
    real = oracle.RefCloth(scene.mesh, scene.cdef, restated=False)
    rest = oracle.RefCloth(scene.mesh, scene.cdef, restated=True)
    port = oracle.PortCloth(scene.mesh, scene.cdef)
    a, b, c = real.describe(), rest.describe(), port.describe()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
        assert np.array_equal(a[k], c[k]), k
    assert np.array_equal(real.state()["mass"], port.state()["mass"])


def test_sewing_springs_match_reference_constructor():
    """Two panels sewn along their side edges: the same force list (triangles
    and the sewing springs of cloth.cpp:248-262) in the same order."""
    scene = sewn_scene(12)
    real = oracle.RefCloth(scene.mesh, scene.cdef, restated=False)
    port = oracle.PortCloth(scene.mesh, scene.cdef)
    a, c = real.describe(), port.describe()
    assert a["forces"].shape[0] == 2 * scene.mesh.triangle_count + scene.mesh.sewing.shape[0]
    for k in a:
        assert np.array_equal(a[k], c[k]), k


def test_skipping_self_collision_is_exact():
    """At thickness 0 the reference's own b3Cloth::Step (with its cloth
    self-collision pass) and the harness step without it agree bit for bit."""
    scene = sphere_scene(8)
    a = oracle.RefCloth(scene.mesh, scene.cdef, restated=False).setup(scene)
    b = oracle.RefCloth(scene.mesh, scene.cdef, restated=False).setup(scene)
    for _ in range(40):
        a.step(scene.dt, full=True)
        b.step(scene.dt)
        sa, sb = a.state(), b.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sa[q], sb[q])


@pytest.mark.parametrize("maker,steps", [(lambda: plain_scene(20), 25), (lambda: sphere_scene(24), 45),
                                         (lambda: sewn_scene(12), 40)])
def test_port_tracks_reference_bit_exact(maker, steps):
    scene = maker()
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for k in range(steps):
        ri = ref.step(scene.dt)["iterations"]
        pi = port.step(scene.dt)["iterations"]
        assert ri == pi
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sr[q], sp[q]), (k, q)
        cr, cp = ref.contacts(), port.contacts()
        assert cr["count"] == cp["count"]
        assert np.array_equal(cr["impulses"], cp["impulses"])


def test_port_mpcg_reproduces_reference_solution():
    scene = sphere_scene(16)
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    for _ in range(3):
        ref.step(scene.dt)
    sysd = ref.system(scene.dt)
    ref.step(scene.dt)
    x, it, _ = oracle.mpcg(sysd)
    assert it == ref.L.ref_last_iterations()
    # rows are in solver order; m_x is reported by vertex
    dv = ref.state()["dv"]
    assert np.array_equal(x, dv[sysd["vertex_of_row"]])


@pytest.mark.parametrize("maker", [lambda: plain_scene(12), lambda: sphere_scene(12)])
def test_mouse_drag_matches_reference(maker):
    """Created particle + mouse force (cloth.cpp:307-364, mouse_force.cpp:63-227),
    as the testbed's cloth dragger uses them: a static particle at a point of
    a triangle, a mouse force to it, the particle moved every step, then both
    destroyed.  The restatement follows the reference bit for bit through the
    drag, the release and the steps after it."""
    scene = maker()
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for _ in range(5):
        ref.step(scene.dt)
        port.step(scene.dt)
    tri = 60
    xs = ref.state()["x"][scene.mesh.triangles[tri]]
    p0 = (0.2 * xs[0] + 0.3 * xs[1] + 0.5 * xs[2]).astype(np.float32)
    ids = []
    for cl in (ref, port):
        i = cl.create_particle(p0)
        ids.append((i, cl.create_mouse_force(i, tri, 0.2, 0.3, 0.5, 1000.0, 5.0)))
    assert ids[0][0] == ids[1][0] == scene.mesh.vertex_count

    def same():
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sr[q], sp[q]), q

    for k in range(25):
        p = p0 + np.array([0.0, 0.01 * k, 0.005 * k], np.float32)
        for cl, (i, _) in zip((ref, port), ids):
            cl.set_position(i, p)
        assert ref.step(scene.dt)["iterations"] == port.step(scene.dt)["iterations"]
        same()
    for cl, (i, f) in zip((ref, port), ids):
        cl.destroy_force(f)
        cl.destroy_particle(i)
    assert ref.n == port.n == scene.mesh.vertex_count
    for _ in range(8):
        assert ref.step(scene.dt)["iterations"] == port.step(scene.dt)["iterations"]
        same()


def test_capsule_collider_matches_reference():
    """A static capsule collider (b3CapsuleShape::TestSphere, ComputeAABB):
    contacts, positions and velocities bit for bit over the drape and slide."""
    from bounce_b200.meshes import capsule_scene

    scene = capsule_scene(16)
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    active = 0
    for _ in range(120):
        assert ref.step(scene.dt)["iterations"] == port.step(scene.dt)["iterations"]
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sr[q], sp[q]), q
        cr, cp = ref.contacts(), port.contacts()
        assert cr["count"] == cp["count"]
        assert np.array_equal(cr["active"], cp["active"])
        assert np.array_equal(cr["impulses"], cp["impulses"])
        active = max(active, int(cr["active"].sum()))
    assert active > 10


def test_particle_edits_match_reference():
    """Forces, translations, velocities, positions and type changes between
    steps (particle.cpp, particle.h:205-271), on the sphere scene so that type
    changes also drop contacts: the restatement follows the reference bit for
    bit."""
    import edit_script

    scene = sphere_scene(16)
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for step in range(40):
        x = ref.state()["x"]
        edit_script.apply(ref, step, x, gpu=False)
        edit_script.apply(port, step, x, gpu=False)
        assert ref.step(scene.dt)["iterations"] == port.step(scene.dt)["iterations"]
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv", "type"):
            assert np.array_equal(sr[q], sp[q]), (step, q)
        assert ref.contacts()["count"] == port.contacts()["count"]


def _same_tri_contacts(a, b):
    ca, cb = a.tri_contacts(), b.tri_contacts()
    assert ca["count"] == cb["count"]
    for k in ("pt", "active", "impulses"):
        assert np.array_equal(ca[k], cb[k]), k
    # an inactive contact's weights are stale (never set for a new contact)
    on = ca["active"] != 0
    assert np.array_equal(ca["w"][on], cb["w"][on])
    return ca


@pytest.mark.parametrize("edit_from", [None, 84])
def test_self_collision_matches_reference(edit_from):
    """Thickness 0.2: the reference's full b3Cloth::Step with its
    particle-triangle contacts (cloth_contact_manager.cpp, broad_phase.h
    FindPairs, cloth_particle_triangle_contact.cpp, cloth_contact_solver.cpp)
    against the restatement, bit for bit: positions, velocities, and the
    contact list in list order with active flags, barycentric weights and
    impulses.  With edit_from set, the particle edit script runs while the
    cloth is folding (type changes drop a particle's contacts and touch its
    proxy; position edits move its triangles' proxies)."""
    import edit_script
    from bounce_b200.meshes import self_collision_scene

    scene = self_collision_scene(11)
    ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=False).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    most_active, most = 0, 0
    for step in range(130):
        if edit_from is not None:
            x = ref.state()["x"]
            edit_script.apply(ref, step - edit_from, x, gpu=False)
            edit_script.apply(port, step - edit_from, x, gpu=False)
        assert ref.step(scene.dt, full=True)["iterations"] == port.step(scene.dt)["iterations"]
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv", "type"):
            assert np.array_equal(sr[q], sp[q]), (step, q)
        c = _same_tri_contacts(ref, port)
        most = max(most, c["count"])
        most_active = max(most_active, int(c["active"].sum()))
    assert most > 500 and most_active > 50


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_hull_collider_matches_reference(seed):
    """Static hulls from the reference's quickhull over random point clouds:
    b3HullShape::TestSphere runs b3GJK (every simplex case) and, inside the
    hull, its face search; contacts, positions and velocities bit for bit."""
    from bounce_b200.meshes import capsule_scene

    rng = np.random.default_rng(seed)
    pts = (rng.normal(0.0, 0.2, (30, 3)) + np.array([0.0, -0.45, 0.0])).astype(np.float32)
    scene = capsule_scene(16)
    scene.capsules = []
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    hv, hp = ref.add_hull_from_points(pts, 0.3)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    port.add_hull(hv, hp, 0.3)
    active = 0
    for _ in range(150):
        assert ref.step(scene.dt)["iterations"] == port.step(scene.dt)["iterations"]
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sr[q], sp[q]), q
        cr, cp = ref.contacts(), port.contacts()
        assert cr["count"] == cp["count"]
        assert np.array_equal(cr["active"], cp["active"])
        assert np.array_equal(cr["impulses"], cp["impulses"])
        active = max(active, int(cr["active"].sum()))
    assert active > 100


def test_ray_cast_single_matches_reference():
    """b3Cloth::RayCastSingle (the dragger's pick): the restatement finds
    the same triangle, fraction and normal as the reference for vertical
    segments through a falling cloth (the reference's full Step keeps its
    triangle proxies up to date)."""
    scene = sphere_scene(16)
    ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=False).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    rng = np.random.default_rng(3)
    hits = 0
    for _ in range(30):
        ref.step(scene.dt, full=True)
        port.step(scene.dt)
        for _ in range(10):
            p1 = rng.uniform(-0.6, 0.6, 3).astype(np.float32)
            p1[1] = 1.0
            p2 = p1.copy()
            p2[1] = -1.5
            p2[0] += rng.normal(0.0, 0.2)
            p2[2] += rng.normal(0.0, 0.2)
            a, b = ref.ray_cast_single(p1, p2), port.ray_cast_single(p1, p2)
            assert (a is None) == (b is None)
            if a is not None:
                assert a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2])
                hits += 1
    assert hits > 100


def _mixed_radii(cloth, n, seed, frac=1.0):
    """Per-particle radius (0..2 cm) and friction (0..1) for a random subset."""
    rng = np.random.default_rng(seed)
    for i in range(n):
        if rng.uniform() < frac:
            cloth.set_radius(i, float(rng.uniform(0.0, 0.02)))
            cloth.set_friction(i, float(rng.uniform(0.0, 1.0)))


def test_particle_radius_and_friction_match_reference():
    """b3Particle::SetRadius / SetFriction (particle.h:240-255) on the sphere
    scene: radii of 0-2 cm and frictions of 0-1 before the first step, and a
    second set at step 25 while the cloth lies on the sphere (SetRadius moves
    the proxy).  They enter the contact test, the position solve and the
    friction mix; the restatement follows the reference bit for bit.  Both
    step without the self-collision pass, as the GPU does for a cloth created
    with thickness 0; the reference's full Step would turn some
    particle-triangle contacts active here from step 12 on."""
    scene = sphere_scene(16)
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    n = scene.mesh.vertex_count
    _mixed_radii(ref, n, 11)
    _mixed_radii(port, n, 11)
    active = 0
    for step in range(60):
        if step == 25:
            _mixed_radii(ref, n, 12, 0.3)
            _mixed_radii(port, n, 12, 0.3)
        assert ref.step(scene.dt)["iterations"] == port.step(scene.dt)["iterations"], step
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sr[q], sp[q]), (step, q)
        cr, cp = ref.contacts(), port.contacts()
        assert cr["count"] == cp["count"], step
        assert np.array_equal(cr["active"], cp["active"]), step
        assert np.array_equal(cr["impulses"], cp["impulses"]), step
        active = max(active, int(cr["active"].sum()))
    assert active > 20
    assert np.array_equal(ref.describe()["fat_aabb"], port.describe()["fat_aabb"])


def test_overlapping_colliders_match_reference():
    """A cloth draping over a sphere, a capsule lying across its top and a box
    hull whose top is level with both, so that particles touch two or three
    shapes at once.  A particle's contacts are in the list order the world
    query's tree gives; the restatement derives that order from the
    broadphase tree, and its whole contact list (particle, shape, active,
    impulses, in order) matches the reference bit for bit."""
    scene = sphere_scene(16)
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for o in (ref, port):
        o.add_capsule((-0.6, -0.25, 0.0), (0.6, -0.25, 0.0), 0.05, 0.5)
    box = np.array([(x, y, z) for x in (-0.7, -0.15) for y in (-0.6, -0.2) for z in (-0.4, 0.4)], np.float32)
    hv, hp = ref.add_hull_from_points(box, 0.2)
    port.add_hull(hv, hp, 0.2)
    multi = 0
    for step in range(60):
        assert ref.step(scene.dt)["iterations"] == port.step(scene.dt)["iterations"], step
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sr[q], sp[q]), (step, q)
        lr, lp = ref.contact_list(), port.contact_list()
        for q in ("particle", "shape", "active", "impulses"):
            assert np.array_equal(lr[q], lp[q]), (step, q)
        act = lr["particle"][lr["active"] != 0]
        multi = max(multi, int((np.bincount(act, minlength=scene.mesh.vertex_count) >= 2).sum()) if act.size else 0)
    assert multi > 0


def _quat_y(angle):
    import math

    return (0.0, math.sin(0.5 * angle), 0.0, math.cos(0.5 * angle))


def test_body_colliders_match_reference():
    """Colliders on bodies of every type (b3Body, include/bounce/dynamics/
    body.h): a dynamic box (a quickhull hull of density 2) falling onto a
    cloth pinned at its four corners, a kinematic sphere rising into the
    cloth from below, and a static capsule at a rotated pose.  Each frame the
    reference steps its world (b3World::Step moves the bodies); the
    restatement is then given every body's state and every shape's
    broadphase proxy from the reference, and both step the cloth.  The cloth,
    its contact list and the bodies after the cloth step -- velocities and
    sweep changed by the contact solver (cloth_contact_solver.cpp:264-307,
    388-472, 620-718), transform, world inverse inertia and proxies
    synchronised (cloth_solver.cpp:165-181) -- match bit for bit."""
    scene = plain_scene(16)
    side = 16
    ref = oracle.RefCloth(scene.mesh, scene.cdef).setup(scene)
    port = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for o in (ref, port):
        for v in (side * (side - 1), side * side - 1):
            o.set_type(v, 0)
    # bodies and shapes, created in the same order on both sides
    box = np.array([(x, y, z) for x in (-0.12, 0.12) for y in (-0.08, 0.08) for z in (-0.12, 0.12)], np.float32)
    b_box = ref.add_body(2, (0.05, 0.25, 0.0), _quat_y(0.3))
    hv, hp = ref.add_body_hull(b_box, box, 2.0, 0.4)
    b_sph = ref.add_body(1, (-0.3, -0.45, 0.25), velocity=(0.1, 0.45, 0.0))
    ref.add_body_shape(b_sph, 0, (0.0, 0.0, 0.0), 0.1, 1.0, 0.3)
    b_cap = ref.add_body(0, (0.3, -0.3, -0.25), _quat_y(0.5))
    ref.add_body_shape(b_cap, 1, (-0.15, 0.0, 0.0, 0.15, 0.0, 0.0), 0.05, 1.0, 0.5)
    for b in (b_box, b_sph, b_cap):
        port.add_body(ref.body(b))
    port.add_body_shape(b_box, 2, np.concatenate([hv.reshape(-1), hp.reshape(-1)]), 0.0, 0.4, len(hv), len(hp))
    port.add_body_shape(b_sph, 0, (0.0, 0.0, 0.0), 0.1, 0.3)
    port.add_body_shape(b_cap, 1, (-0.15, 0.0, 0.0, 0.15, 0.0, 0.0), 0.05, 0.5)
    seen = {0: 0, 1: 0, 2: 0}
    moved = 0.0
    for step in range(90):
        ref.world_step(scene.dt)
        for b in (b_box, b_sph, b_cap):
            port.set_body(b, ref.body(b))
        for s in range(3):
            port.set_shape_proxy(s, *ref.shape_proxy(s))
        a = ref.step(scene.dt)
        # moving proxies are re-inserted into the world's tree, so its report
        # order (which decides the list order of one particle's new contacts
        # with several shapes) comes from the reference's world
        port.set_report_order(ref.report_order())
        b = port.step(scene.dt)
        assert a["iterations"] == b["iterations"], step
        sr, sp = ref.state(), port.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sr[q], sp[q]), (step, q)
        lr, lp = ref.contact_list(), port.contact_list()
        for q in ("particle", "shape", "active", "impulses"):
            assert np.array_equal(lr[q], lp[q]), (step, q)
        for bb in (b_box, b_sph, b_cap):
            assert np.array_equal(ref.body(bb), port.body(bb)), (step, bb)
        for s in range(3):
            for u, w in zip(ref.shape_proxy(s), port.shape_proxy(s)):
                assert np.array_equal(u, w), (step, s)
        for s in range(3):
            seen[s] = max(seen[s], int(lr["active"][lr["shape"] == s].sum()))
        moved = max(moved, float(np.abs(ref.body(b_box)[30:33]).max()))
    # every body touched the cloth, and the cloth pushed the dynamic box
    assert min(seen.values()) > 0, seen
    assert moved > 0.0
