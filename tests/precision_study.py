"""Precision study of the CG inner products on a large, stiff cloth.

Workload: a 1024x1024 grid (1,048,576 vertices, 2,093,058 triangles),
stretch 1e5, shear 1e3, damping 0.1, the two corners of row 0 pinned, 50
steps at dt = 1/60 s.  The force evaluation, assembly and SpMV stay FP32
(as in the reference); the CG dot products (alpha, beta, the residual norm)
accumulate in (a) FP32, (b) compensated FP32 or (c) FP64.  CG stops at
relative residual 1e-4 (cap 2000 iterations).

Two measurements:

1. Trajectories.  One GPU cloth per dot precision is stepped 50 times
   (persistent CG).  Reported per step: CG iterations and the residual the
   CG reached.  At the check steps the step's linear system is exported
   before the step, and the CG solution of the step is compared with an
   FP64 CPU solve of the same system (the oracle's FP64 Jacobi-PCG to
   relative residual 1e-10): relative error of dv, the position error it
   causes (h * max |dv - dv_64|), and the residual of the GPU solution
   recomputed in FP64 in the stop rule's norm (the CG's own figure is a
   recurrence, which can drift from the true residual).

2. Same system.  At the check steps of the FP64-dot trajectory, that one
   system is solved on the GPU by the standalone MPCG entry point in each
   dot precision, and on the CPU by the oracle's MPCG with the reference's
   own sequential FP32 dots; all against one FP64 CPU solve.  This isolates
   the dot precision from trajectory divergence.

The oracle is only the checker here.  Run on a machine with a GPU:

    python tests/precision_study.py --side 1024 --steps 50 --check 1,10,25,50 \
        --json precision.json
"""
import argparse
import json
import multiprocessing as mp
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

NAMES = {0: "fp32", 1: "compensated", 2: "fp64"}


def spmv64(sysd, x):
    """y = A x in FP64 over the exported block-CSR system (x: (n, 3))."""
    rowptr = sysd["rowptr"].astype(np.int64)
    cols = sysd["cols"].astype(np.int64)
    # vals hold 9 floats per block, column-major b3Mat33: a[c][r] at 3 c + r
    a = sysd["vals"].reshape(-1, 3, 3).astype(np.float64)
    xc = x[cols]
    prod = np.einsum("kcr,kc->kr", a, xc)
    rows = np.repeat(np.arange(rowptr.size - 1), np.diff(rowptr))
    y = np.zeros_like(x)
    for d in range(3):
        y[:, d] = np.bincount(rows, weights=prod[:, d], minlength=rowptr.size - 1)
    return y


def true_residual(sysd, x):
    """The stop rule's norm, recomputed in FP64 from the solution:
    sqrt(r.P^-1 r / b.P^-1 b) with r = S (b - A x), b filtered by S and P the
    diagonal of A (cloth_force_solver.cpp:70-100)."""
    rowptr = sysd["rowptr"].astype(np.int64)
    cols = sysd["cols"].astype(np.int64)
    rows = np.repeat(np.arange(rowptr.size - 1), np.diff(rowptr))
    a = sysd["vals"].reshape(-1, 3, 3).astype(np.float64)
    d = np.zeros((rowptr.size - 1, 3))
    on = cols == rows
    d[rows[on]] = np.stack([a[on, 0, 0], a[on, 1, 1], a[on, 2, 2]], axis=1)
    pinv = 1.0 / d
    S = sysd["S"].astype(np.float64)[:, None]
    b = S * sysd["b"].reshape(-1, 3).astype(np.float64)
    r = S * (b - spmv64(sysd, np.asarray(x, np.float64)))
    return float(np.sqrt(np.sum(r * r * pinv) / max(np.sum(b * b * pinv), 1e-300)))


def _solve_job(args):
    path, tol = args
    import oracle

    d = np.load(path)
    sysd = {k: d[k] for k in d.files}
    t0 = time.perf_counter()
    x, it = oracle.solve_f64(sysd, tol=tol, max_iterations=1000000)
    return path, x, it, time.perf_counter() - t0


def _seq_f32_job(args):
    """The oracle's MPCG with the reference's sequential FP32 dots on one system."""
    path, tol, cap = args
    import oracle

    d = np.load(path)
    sysd = {k: d[k] for k in d.files}
    n = sysd["rowptr"].size - 1
    t0 = time.perf_counter()
    x, it, stats = oracle.mpcg(sysd, stop_rule=1, tol=tol, max_iterations=cap, dot=0)
    return path, np.asarray(x).reshape(n, 3), it, time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--side", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--check", default="1,10,25,50")
    ap.add_argument("--cap", type=int, default=2000)
    ap.add_argument("--workers", type=int, default=min(8, os.cpu_count() or 1))
    ap.add_argument("--json", default="")
    ap.add_argument("--cg", choices=["persistent", "fused"], default="persistent",
                    help="the persistent CG with two grid reductions per iteration, or one (fused)")
    args = ap.parse_args()
    checks = sorted({int(s) for s in args.check.split(",") if s})

    # the CPU workers start by spawn, before anything touches the GPU
    pool = mp.get_context("spawn").Pool(args.workers)
    tmp = tempfile.mkdtemp(prefix="precision_")

    import bounce_b200 as b3g
    from helpers import call_mpcg, device_system

    scene = b3g.stiff_scene(args.side, steps=args.steps)
    dt = scene.dt
    t0 = time.perf_counter()
    cloths = {}
    for dot in (0, 1, 2):
        c = b3g.Cloth(scene.mesh, scene.cdef).setup(scene, b3g.SolverOptions.relative(1e-4, args.cap, dot))
        c.set_cg_strategy(True, fused=args.cg == "fused")
        cloths[dot] = c
    build_s = time.perf_counter() - t0
    n = cloths[2].n

    traj = {NAMES[d]: [] for d in cloths}
    pending = []  # (variant, step, system path, gpu dv, true residual, the CG's own residual)
    same = {}     # step -> system path of the FP64-dot trajectory
    for step in range(1, args.steps + 1):
        for dot, c in cloths.items():
            sysd = None
            if step in checks:
                c.assemble(dt)
                sysd = c.system()
            out = c.step(dt)
            rec = {"step": step, "iterations": out["iterations"], "status": out.get("status", 0),
                   "cg_residual": float(np.sqrt(out["delta"] / out["b_delta"])) if out["b_delta"] > 0 else 0.0}
            traj[NAMES[dot]].append(rec)
            if sysd is not None:
                path = os.path.join(tmp, f"sys_{NAMES[dot]}_{step}.npz")
                np.savez(path, **sysd)
                dv = c.state()["dv"].astype(np.float64)
                pending.append((NAMES[dot], step, path, dv, true_residual(sysd, dv), rec["cg_residual"]))
                if dot == 2:
                    same[step] = (path, sysd)
        print(f"step {step}: " + ", ".join(f"{NAMES[d]} {traj[NAMES[d]][-1]['iterations']} it" for d in cloths),
              flush=True)

    # same system, every dot precision on the GPU (standalone MPCG entry point)
    same_gpu = {}
    for step, (path, sysd) in same.items():
        dsys = device_system(sysd)
        for dot in (0, 1, 2):
            st, x, it, stats = call_mpcg(b3g, "b3g_mpcg_solve", dsys, b3g.SolverOptions.relative(1e-4, args.cap, dot))
            same_gpu[(step, NAMES[dot])] = (x.astype(np.float64), it, st, true_residual(sysd, x.astype(np.float64)))

    # FP64 CPU solves (and the reference's sequential FP32 dots) in parallel
    paths = sorted({p for _, _, p, _, _, _ in pending})
    f64 = {p: (x, it, s) for p, x, it, s in pool.map(_solve_job, [(p, 1e-10) for p in paths])}
    seq = {p: (x, it, s) for p, x, it, s in
           pool.map(_seq_f32_job, [(same[s][0], 1e-4, args.cap) for s in sorted(same)])}
    pool.close()

    h = dt
    checks_out = []
    for name, step, path, dv, tres, cres in pending:
        x64 = f64[path][0]
        err = np.abs(dv - x64)
        checks_out.append({"variant": name, "step": step, "dv_rel_err": float(np.linalg.norm(dv - x64) /
                                                                              max(np.linalg.norm(x64), 1e-300)),
                           "position_err_m": float(h * err.max()), "true_residual": tres,
                           "cg_residual": cres, "cg_over_true": cres / tres if tres > 0 else None,
                           "f64_iterations": f64[path][1], "f64_solve_s": f64[path][2]})
    same_out = []
    for step, (path, sysd) in same.items():
        x64 = f64[path][0]
        for name in ("fp32", "compensated", "fp64"):
            x, it, st, tres = same_gpu[(step, name)]
            same_out.append({"step": step, "solver": f"gpu {name} dots", "iterations": it, "status": st,
                             "dv_rel_err": float(np.linalg.norm(x - x64) / max(np.linalg.norm(x64), 1e-300)),
                             "position_err_m": float(h * np.abs(x - x64).max()), "true_residual": tres})
        xs, its, secs = seq[path]
        xs = xs.astype(np.float64)
        same_out.append({"step": step, "solver": "cpu oracle, sequential fp32 dots (the reference's order)",
                         "iterations": its, "status": 0,
                         "dv_rel_err": float(np.linalg.norm(xs - x64) / max(np.linalg.norm(x64), 1e-300)),
                         "position_err_m": float(h * np.abs(xs - x64).max()), "true_residual": true_residual(sysd, xs),
                         "cpu_s": secs})

    final = {NAMES[d]: c.state()["x"].astype(np.float64) for d, c in cloths.items()}
    drift = {name: float(np.abs(final[name] - final["fp64"]).max()) for name in ("fp32", "compensated")}
    summary = {}
    for name, recs in traj.items():
        it = np.array([r["iterations"] for r in recs])
        summary[name] = {"iterations_mean": float(it.mean()), "iterations_max": int(it.max()),
                         "steps_at_cap": int((it >= args.cap).sum()),
                         "cg_residual_max": float(max(r["cg_residual"] for r in recs)),
                         "final_position_diff_vs_fp64_dots_m": drift.get(name, 0.0)}
    result = {"workload": f"grid{args.side}_stiff", "cg": args.cg, "vertices": n, "steps": args.steps, "checks": checks,
              "cap": args.cap, "build_s": build_s, "summary": summary, "trajectory_checks": checks_out,
              "same_system": same_out, "per_step": traj}
    print(json.dumps({k: result[k] for k in ("workload", "vertices", "summary")}, indent=1))
    for r in checks_out:
        print("traj", r)
    for r in same_out:
        print("same", r)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(result, f, indent=1)
    for c in cloths.values():
        c.close()


if __name__ == "__main__":
    main()
