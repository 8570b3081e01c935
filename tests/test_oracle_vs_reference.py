"""The restatement against the live reference library (when it is built here).

Skipped when oracle/_ref/libbounce_ref.so is absent (it is compiled from the
reference sources, which only exist where the reference tree is mounted).
"""
import numpy as np
import pytest

import oracle
from bounce_b200.meshes import plain_scene, sphere_scene

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


@pytest.mark.parametrize("maker,steps", [(lambda: plain_scene(20), 25), (lambda: sphere_scene(24), 45)])
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
