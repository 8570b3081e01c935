"""The two assembly forms give the same floats.

* ``records``: every element evaluated once a step into a record, each
  block of A summed from its own term list in the reference's order;
* ``rows``: each row recomputes its incident elements, in two passes.

A and b are compared bit for bit (as unsigned words, so signed zeros count)
on single cloths with every element kind, from stretched and from partly
compressed states (so that some stretch and spring stiffness terms are off);
batched steps with either form give bit-identical trajectories.  The records
form itself is checked against the oracle by the parity tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _system(cloth, dt, form):
    cloth.set_assembly(form)
    assert cloth.assembly() == form
    cloth.assemble(dt)
    return cloth.system()


def _scene(b3g, maker):
    if maker == "plain":
        return b3g.plain_scene(24)
    if maker == "sewn":
        return b3g.sewn_scene(16)
    return b3g.sphere_scene(24)


@pytest.mark.parametrize("maker", ["plain", "sphere", "sewn", "mouse"])
@pytest.mark.parametrize("squeeze", [1.0, 0.996])
def test_assembly_forms_bit_identical(b3g, maker, squeeze):
    scene = _scene(b3g, maker)
    gpu = b3g.Cloth(scene.mesh, scene.cdef).setup(scene)
    x0 = scene.mesh.vertices
    if maker == "mouse":
        tri = 300
        p0 = (x0[scene.mesh.triangles[tri]].mean(axis=0) + [0.0, 0.05, 0.0]).astype(np.float32)
        gpu.create_particle(p0)
        gpu.create_mouse_force(scene.mesh.vertex_count, tri, 0.2, 0.3, 0.5, 800.0, 4.0)
        x0 = np.concatenate([x0, p0[None]])
    rng = np.random.default_rng(17)
    centre = x0.mean(axis=0)
    x = (centre + squeeze * (x0 - centre) + rng.normal(0, 2e-3, x0.shape)).astype(np.float32)
    v = rng.normal(0, 0.1, x0.shape).astype(np.float32)
    gpu.write_state(x=x, v=v)
    rows = _system(gpu, scene.dt, "rows")
    recs = _system(gpu, scene.dt, "records")
    assert np.array_equal(rows["rowptr"], recs["rowptr"])
    assert np.array_equal(rows["cols"], recs["cols"])
    assert np.array_equal(_bits(rows["vals"]), _bits(recs["vals"]))
    assert np.array_equal(_bits(rows["b"]), _bits(recs["b"]))
    assert np.any(recs["vals"]) and np.any(recs["b"])
    gpu.close()


def test_batched_steps_identical_across_forms(b3g):
    scenes = [b3g.plain_scene(16, seed=21), b3g.sphere_scene(24, seed=22), b3g.plain_scene(40, seed=23),
              b3g.sewn_scene(16, seed=24)]
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    runs = {}
    for form in ("rows", "records"):
        cloths = [b3g.Cloth(s.mesh, s.cdef).setup(s, opts) for s in scenes]
        for c in cloths:
            c.set_assembly(form)
        batch = b3g.Batch(8)
        batch.set_schedule(4, (11, 12))
        for _ in range(10):
            batch.step(cloths, scenes[0].dt)
        runs[form] = [c.state() for c in cloths]
        for c in cloths:
            c.close()
    for a, r in zip(runs["rows"], runs["records"]):
        for q in ("x", "v", "dv"):
            assert np.array_equal(_bits(a[q]), _bits(r[q])), q


def test_records_are_the_default(b3g):
    scene = b3g.sphere_scene(16)
    gpu = b3g.Cloth(scene.mesh, scene.cdef).setup(scene)
    assert gpu.assembly() == "records"
    gpu.set_assembly("rows")
    assert gpu.assembly() == "rows"
    with pytest.raises(Exception):
        gpu.set_assembly("columns")
    gpu.close()
