"""Parity at the benchmark sizes, through checks that do not need a long
oracle run: the 256x256 headline cloth (bending springs and the sphere) and
the 512-cloth batch."""
import os
import sys

import numpy as np
import pytest

from helpers import oracle_floor_step, rel_err, system_blocks

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def test_headline_assembly_bit_exact_and_one_step(b3g, port):
    """256x256 with bending and the sphere, a few steps into the fall: the
    assembled system matches the oracle bit for bit; the system is symmetric
    up to the rounding of the stretch element's second-derivative factor; the
    GPU's CG solution meets the stop rule in the FP64-recomputed residual; and
    one step from identical inputs matches the oracle."""
    from precision_study import true_residual

    scene = b3g.sphere_scene(256)
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    gpu = b3g.Cloth(scene.mesh, scene.cdef).setup(scene, opts)
    gpu.set_cg_strategy(True)
    # 8 steps: about 9 cm of fall, above the sphere (no active contact, which
    # the oracle, started from the GPU's state without contacts, could not see)
    for _ in range(8):
        gpu.step(scene.dt)
    st = gpu.state()
    ora = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    ora.set_solver(opts.stop_rule, opts.tolerance, opts.max_iterations, opts.dot)
    ora.set_state(x=st["x"], v=st["v"], dv=st["dv"])

    gpu.assemble(scene.dt)
    gs = gpu.system()
    os_ = ora.system(scene.dt)
    rowptr, cols = gs["rowptr"].astype(np.int64), gs["cols"].astype(np.int64)
    vals = gs["vals"].reshape(-1, 3, 3)
    # bit-exact against the oracle, block by block
    gb, gbv = system_blocks(gs)
    ob, obv = system_blocks(os_, os_["vertex_of_row"])
    assert len(ob) > 800000
    for key, val in ob.items():
        assert np.array_equal(gb[key], val), key
    assert np.array_equal(gbv, obv)
    # symmetry: A_ij = A_ji^T
    rows = np.repeat(np.arange(rowptr.size - 1), np.diff(rowptr))
    index = {(int(r), int(c)): k for k, (r, c) in enumerate(zip(rows, cols))}
    worst = 0.0
    for k in range(0, len(rows), 97):
        r, c = int(rows[k]), int(cols[k])
        a = vals[k].astype(np.float64)
        b = vals[index[(c, r)]].astype(np.float64).T
        worst = max(worst, float(np.abs(a - b).max() / max(np.abs(a).max(), 1e-30)))
    assert worst <= 1e-5, worst

    # one step from identical inputs.  At this size two correct solvers whose
    # dots round differently part by more than the 1e-4 stop tolerance in v,
    # so both solve to 1e-5 here, which isolates the step's own parity.
    tight = b3g.SolverOptions.relative(1e-5, 400, b3g.DOT_F64)
    gpu.set_solver(tight)
    ora.set_solver(tight.stop_rule, tight.tolerance, tight.max_iterations, tight.dot)
    g = gpu.step(scene.dt)
    o = ora.step(scene.dt)
    assert abs(g["iterations"] - o["iterations"]) <= 2, (g["iterations"], o["iterations"])
    assert rel_err(gpu.state()["x"], ora.state()["x"]) <= 1e-4
    assert rel_err(gpu.state()["v"], ora.state()["v"]) <= 1e-4
    # the GPU's solution of the step's system
    assert true_residual(gs, gpu.state()["dv"].astype(np.float64)) <= 1.2e-5


def test_batch512_sample_matches_oracle(b3g, port):
    """The 512-cloth batch (sides 16..128, the autotuned schedule): a sample
    of cloths, each started on the oracle from the GPU's state, matches the
    oracle per step."""
    scenes = b3g.batch_scenes(512, seed=3)
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    cloths = [b3g.Cloth(s.mesh, s.cdef).setup(s, opts) for s in scenes]
    batch = b3g.Batch(1024)
    dt = scenes[0].dt
    batch.step(cloths, dt)
    batch.autotune(cloths, dt)
    sample = [0, 37, 101, 200, 311, 402, 477, 511]
    oras = []
    for k in sample:
        o = port.PortCloth(scenes[k].mesh, scenes[k].cdef).setup(scenes[k])
        o.set_solver(opts.stop_rule, opts.tolerance, opts.max_iterations, opts.dot)
        oras.append(o)
    for step in range(4):
        for k, o in zip(sample, oras):
            st = cloths[k].state()
            o.set_state(x=st["x"], v=st["v"], dv=st["dv"])
        out = batch.step(cloths, dt, per_cloth=True)
        for k, o in zip(sample, oras):
            oi = o.step(dt)
            assert abs(out["per_cloth"][k]["iterations"] - oi["iterations"]) <= 1, (step, k)
            assert rel_err(cloths[k].state()["x"], o.state()["x"]) <= 1e-4, (step, k)


def test_headline_in_contact_one_step(b3g, port):
    """The headline cloth draped on the sphere, at the benchmark's own setting
    (CG to relative residual 1e-4, FP64 dots, the persistent CG).  After 20
    steps of fall, within the benchmark's timed steps, over 10,000 particles
    touch the sphere.  The oracle is
    given the GPU's whole state: positions, velocities, the CG warm start,
    the body-contact list with its impulses and the particles' fat AABBs.
    Then both take one step.
     - The contact update at the step start is the same arithmetic on the
       same positions, so the active contacts handed to the solver agree
       exactly.
     - CG iterations agree within +-1, positions within 1e-4 relative.
     - Velocities: at a 1e-4 stop two correct solvers whose dots round
       differently part by about 2e-4 of the largest velocity.  The bound is
       twice the oracle's own spread, measured by stepping clones of its whole
       state with compensated and with FP64 dots, or 1e-4 where that is
       larger.
     - The contacts alive after the step agree within 0.1%: a particle whose
       new fat AABB lies within rounding of the sphere's proxy may differ."""
    scene = b3g.sphere_scene(256)
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    gpu = b3g.Cloth(scene.mesh, scene.cdef).setup(scene, opts)
    gpu.set_cg_strategy(True)
    for _ in range(20):
        gpu.step(scene.dt)
    st = gpu.state()
    gc = gpu.contacts()
    lo, hi = gpu.proxies()
    ora = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    ora.set_solver(opts.stop_rule, opts.tolerance, opts.max_iterations, opts.dot)
    ora.set_state(x=st["x"], v=st["v"], dv=st["dv"])
    live = np.nonzero(gc["exists"])[0]
    ora.set_contacts(live, np.zeros(live.size, np.uint32), gc["impulses"][live])
    ora.set_proxies(lo, hi)
    assert ora.contacts()["count"] == live.size

    clones = oracle_floor_step(port, scene, ora, scene.dt, opts.stop_rule, opts.tolerance, opts.max_iterations)
    g = gpu.step(scene.dt)
    o = ora.step(scene.dt)
    assert o["active_contacts"] > 10000, o["active_contacts"]
    assert g["active_contacts"] == o["active_contacts"], (g["active_contacts"], o["active_contacts"])
    assert abs(g["iterations"] - o["iterations"]) <= 1, (g["iterations"], o["iterations"])
    gs, os_ = gpu.state(), ora.state()
    ex = rel_err(gs["x"], os_["x"])
    ev = rel_err(gs["v"], os_["v"])
    floor_v = max(rel_err(c["v"], os_["v"]) for c in clones)
    print(f"in contact: {o['active_contacts']} active, iterations {g['iterations']}/{o['iterations']}, "
          f"x rel {ex:.2e}, v rel {ev:.2e}, oracle's own v spread {floor_v:.2e}")
    assert ex <= 1e-4, ex
    assert ev <= max(1e-4, 2.0 * floor_v), (ev, floor_v)
    ge = gpu.contacts()["exists"].astype(bool)
    oe = ora.contacts()["exists"].astype(bool)
    assert np.count_nonzero(ge != oe) <= max(2, oe.sum() // 1000), np.count_nonzero(ge != oe)
