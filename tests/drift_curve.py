"""Trajectory drift of the CUDA path against the oracle, step by step.

Both sides start from the same cloth and step freely, each from its own
state; the curve is max |x_gpu - x_oracle| (metres) after every step.  Beside
it, the floor: the oracle against itself with the other CG dot precision
(the same algorithm rounded differently).  Where the motion is chaotic (a
cloth folding, a particle on the contact boundary) two correct solvers part
ways, and the GPU curve is compared with that floor, not with zero.
Bulk quantities are reported too: the difference of the mean height and the
relative difference of the energy (b3Cloth::GetEnergy, cloth.cpp:366-374).

Workloads (100 steps each, the CG to relative residual 1e-4 as the
benchmark configurations state it):
* plain: 32x32 grid, stretch 1e4, shear 1e3, damping 0.05, corners of row 0
  pinned, at most 50 CG iterations, FP32 dots;
* sphere: 256x256 grid with bending springs 1e2 falling on a static sphere
  (r = 0.3 m, friction 0.3), at most 200 CG iterations, FP64 dots (the
  headline benchmark's setting).
The floor's solver differs from the oracle's only in the dot precision
(FP64 against FP32 and the other way round).

The reference's own rule (at most 20 iterations, stop at delta <=
FLT_EPSILON^2 b_delta) does not converge on the 256x256 cloth: the oracle
itself turns non-finite within about 40 steps there, and the GPU reports
B3G_ERR_NUMERICAL too, so that rule is not a drift workload.

The oracle is only the checker here.  Run on a machine with a GPU:

    python tests/drift_curve.py --json drift.json
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)


def run(b3g, oracle, name, scene, steps, opts):
    gpu = b3g.Cloth(scene.mesh, scene.cdef).setup(scene, opts)
    gpu.set_cg_strategy(True, fused=True)
    ora = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    ora.set_solver(opts.stop_rule, opts.tolerance, opts.max_iterations, opts.dot)
    floor = oracle.PortCloth(scene.mesh, scene.cdef).setup(scene)
    other = b3g.DOT_F32 if opts.dot == b3g.DOT_F64 else b3g.DOT_F64
    floor.set_solver(opts.stop_rule, opts.tolerance, opts.max_iterations, other)
    rows = []
    for step in range(1, steps + 1):
        g = gpu.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
        o = ora.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
        floor.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
        xg, xo, xf = gpu.state()["x"], ora.state()["x"], floor.state()["x"]
        eo = ora.energy()
        rows.append({
            "step": step,
            "drift_m": float(np.abs(xg - xo).max()),
            "floor_m": float(np.abs(xf - xo).max()),
            "mean_y_diff_m": float(abs(xg[:, 1].mean() - xo[:, 1].mean())),
            "energy_rel_diff": float(abs(gpu.energy() - eo) / max(abs(eo), 1e-12)),
            "iterations": [int(g["iterations"]), int(o["iterations"])],
            "contacts": [int(g.get("active_contacts", 0)), int(o.get("active_contacts", 0))],
        })
    print(f"{name}: step | drift GPU-oracle (m) | floor f32 vs f64 dots (m) | mean y diff (m) | energy rel diff")
    marks = sorted({1, 2, 5, 10, 20, 50, 100, 150, steps} & set(range(1, steps + 1)))
    for r in rows:
        if r["step"] in marks:
            print(f"  {r['step']:4d} | {r['drift_m']:.3e} | {r['floor_m']:.3e} | "
                  f"{r['mean_y_diff_m']:.3e} | {r['energy_rel_diff']:.3e}")
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--plain-side", type=int, default=32)
    ap.add_argument("--plain-steps", type=int, default=100)
    ap.add_argument("--sphere-side", type=int, default=256)
    ap.add_argument("--sphere-steps", type=int, default=100)
    ap.add_argument("--json", default="")
    args = ap.parse_args()

    import oracle

    oracle.build(port=True, ref=False)
    import bounce_b200 as b3g

    out = {
        "plain": run(b3g, oracle, f"plain {args.plain_side}^2", b3g.plain_scene(args.plain_side),
                     args.plain_steps, b3g.SolverOptions.relative(1e-4, 50, b3g.DOT_F32)),
        "sphere": run(b3g, oracle, f"sphere {args.sphere_side}^2", b3g.sphere_scene(args.sphere_side),
                      args.sphere_steps, b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)),
    }
    if args.json:
        with open(args.json, "w") as f:
            json.dump(out, f)


if __name__ == "__main__":
    main()
