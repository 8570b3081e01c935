"""Batched stepping (b3g_batch_step) against stepping alone and the oracle."""
import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


def _mix(b3g):
    scenes = [b3g.plain_scene(16, seed=11), b3g.sphere_scene(24, seed=12), b3g.plain_scene(40, seed=13),
              b3g.sphere_scene(48, seed=14), b3g.plain_scene(70, seed=15), b3g.plain_scene(20, seed=16)]
    scenes[2].cdef.streching = 5e4
    scenes[4].cdef.shearing = 5e3
    return scenes


def _cloths(b3g, scenes, opts):
    return [b3g.Cloth(s.mesh, s.cdef).setup(s, opts) for s in scenes]


@pytest.mark.parametrize("cluster,split", [(1, ()), (4, (11, 12)), (8, (11, 12))])
def test_batch_alone_equals_mixed(b3g, cluster, split):
    """Each cloth's trajectory is bit-identical whether it is stepped alone or
    together with the others (fixed per-cloth reduction trees)."""
    scenes = _mix(b3g)
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    mixed = _cloths(b3g, scenes, opts)
    alone = _cloths(b3g, scenes, opts)
    bm = b3g.Batch(16)
    ba = b3g.Batch(16)
    bm.set_schedule(cluster, split)
    ba.set_schedule(cluster, split)
    dt = scenes[0].dt
    for step in range(12):
        bm.step(mixed, dt)
        for c in alone:
            ba.step([c], dt)
    for a, m in zip(alone, mixed):
        sa, sm = a.state(), m.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sa[q], sm[q]), q


def test_batch_matches_oracle_per_step(b3g, port):
    scenes = _mix(b3g)
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    cloths = _cloths(b3g, scenes, opts)
    oras = [port.PortCloth(s.mesh, s.cdef).setup(s) for s in scenes]
    for o in oras:
        o.set_solver(1, 1e-4, 200, 2)
    batch = b3g.Batch(16)
    batch.set_schedule(4, (12,))
    dt = scenes[0].dt
    for step in range(20):
        states = [c.state() for c in cloths]
        for o, st in zip(oras, states):
            o.set_state(x=st["x"], v=st["v"], dv=st["dv"])
        out = batch.step(cloths, dt, per_cloth=True)
        for k, (c, o) in enumerate(zip(cloths, oras)):
            oi = o.step(dt)
            assert abs(out["per_cloth"][k]["iterations"] - oi["iterations"]) <= 1, (step, k)
            e = rel_err(c.state()["x"], o.state()["x"])
            assert e <= 1e-4, (step, k, e)


def test_batch_matches_plain_path(b3g):
    scenes = _mix(b3g)[:3]
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    plain = _cloths(b3g, scenes, opts)
    batched = _cloths(b3g, scenes, opts)
    batch = b3g.Batch(8)
    dt = scenes[0].dt
    for step in range(10):
        for c in plain:
            c.step(dt)
        batch.step(batched, dt)
        for p, q in zip(plain, batched):
            assert np.abs(p.state()["x"] - q.state()["x"]).max() <= 1e-4


def test_autotune_picks_a_valid_schedule(b3g):
    scenes = _mix(b3g)
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    cloths = _cloths(b3g, scenes, opts)
    batch = b3g.Batch(16)
    batch.step(cloths, scenes[0].dt)
    before = [c.state()["x"].copy() for c in cloths]
    sched = batch.autotune(cloths, scenes[0].dt)
    assert sched["cluster"] in (1, 2, 4, 8)
    assert sched["tuned_cg_ms"] > 0
    for c, x in zip(cloths, before):  # autotuning leaves the cloths unchanged
        assert np.array_equal(c.state()["x"], x)
    batch.step(cloths, scenes[0].dt)


@pytest.mark.parametrize("cluster,split", [(1, ()), (8, (11, 12))])
def test_batch_mixed_dot_precisions_equal_alone(b3g, cluster, split):
    """A batch whose cloths use different dot precisions (FP32, compensated,
    FP64) runs the kernel that reads each cloth's precision on the device;
    every cloth's trajectory is bit-identical to stepping it in a batch of
    its own, which runs the kernel specialised for its precision."""
    scenes = _mix(b3g)
    dots = [b3g.DOT_F32, b3g.DOT_COMPENSATED, b3g.DOT_F64, b3g.DOT_F32, b3g.DOT_F64, b3g.DOT_COMPENSATED]
    mixed = [b3g.Cloth(s.mesh, s.cdef).setup(s, b3g.SolverOptions.relative(1e-4, 200, d))
             for s, d in zip(scenes, dots)]
    alone = [b3g.Cloth(s.mesh, s.cdef).setup(s, b3g.SolverOptions.relative(1e-4, 200, d))
             for s, d in zip(scenes, dots)]
    bm, ba = b3g.Batch(16), b3g.Batch(16)
    bm.set_schedule(cluster, split)
    ba.set_schedule(cluster, split)
    dt = scenes[0].dt
    for step in range(8):
        bm.step(mixed, dt)
        for c in alone:
            ba.step([c], dt)
    for a, m in zip(alone, mixed):
        sa, sm = a.state(), m.state()
        for q in ("x", "v", "dv"):
            assert np.array_equal(sa[q], sm[q]), q
