"""Benchmark of the implicit cloth step on B200.

Workload (default): one 256 x 256 cloth (65,536 vertices, 130,050 triangles,
194,565 bending springs) with a static sphere collider, dt = 1/60 s, 8
velocity / 2 position contact iterations, CG to relative residual 1e-4 (at
most 200 iterations -- this cloth needs about 70 to 110 -- FP64 inner
products).  Metric: cloth vertex-steps per
second, whole job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent cloth per rank (replicas: a single cloth's step
has no exchange to shard), launched by torch.distributed.run; the reported
value is all ranks' vertex-steps over the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from bounce_b200 import replicas  # noqa: E402  (rank partition and max-over-ranks timing)

METRIC = "cloth vertex-steps/s"
UNIT = "vertex-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--side", type=int, default=256)
    ap.add_argument("--cg", choices=["fused", "persistent"], default="persistent",
                    help="the headline cloth's CG: one persistent launch with one grid reduction per "
                         "iteration (fused) or two")
    ap.add_argument("--assembly", choices=["records", "rows"], default="records",
                    help="how every cloth's system is assembled: each element evaluated once into a record "
                         "(records) or recomputed by each of its rows in two passes (rows); same floats")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--serve-seconds", type=float, default=30.0)
    ap.add_argument("--skip-batch", action="store_true")
    ap.add_argument("--skip-serve", action="store_true")
    # profiling aids: leave out the single-cloth headline, or the one-cloth-at-a-time
    # comparison inside the batched section
    ap.add_argument("--skip-single", action="store_true")
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-softbody", action="store_true")
    ap.add_argument("--skip-self", action="store_true")
    ap.add_argument("--skip-colliders", action="store_true")
    ap.add_argument("--collider-side", type=int, default=128)
    ap.add_argument("--self-side", type=int, default=24)
    ap.add_argument("--softbody-side", type=int, default=40)
    ap.add_argument("--softbody-steps", type=int, default=10)
    ap.add_argument("--skip-stiff", action="store_true")
    ap.add_argument("--stiff-side", type=int, default=1024)
    ap.add_argument("--skip-fp64", action="store_true")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (read + write) of one persistent-CG launch, by (cloth side, CG
# form): (bytes of one captured launch, that launch's CG iterations), from
# one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum).
# * 256 x 256: the whole system stays in L2 after its first touch, so the
#   figure holds for any iteration count (None).
# * 1024 x 1024: the 293 MB system streams from HBM once at the start (A x0)
#   and once per iteration, so the traffic scales with 1 + iterations (the
#   captured launch, the third step from rest, ran 10 iterations).
# Sizes and forms without a capture report null.
GRID_CG_TRAFFIC = {
    (256, "persistent"): (36536320 + 8448000, None),
    (1024, "persistent"): (4107670528 + 631533568, 10),
    (1024, "fused"): (3919580160 + 676790272, 10),
}
# DRAM bytes over algorithmic bytes of the batched CG launch (512 cloths):
# 19.46 GB of DRAM traffic against 20.48 GB algorithmic (the average of the
# run's two timed launches; the captured launch is the second).
BATCH_CG_TRAFFIC_RATIO = (16734817024 + 2720797440) / 20483036026.0


def grid_cg_traffic(side: int, form: str, iterations: float):
    """DRAM bytes of one persistent-CG launch of `iterations` CG iterations,
    from the captured launch of the same size and form (null without one)."""
    cap = GRID_CG_TRAFFIC.get((side, form))
    if cap is None:
        return None
    bytes_, its = cap
    return bytes_ if its is None else bytes_ * (1.0 + iterations) / (1.0 + its)


def algorithmic_bytes(info: dict, kernel: str) -> float:
    """Bytes one launch of a kernel must move at least (FP32, full block pattern)."""
    n, blocks, t, s = info["vertices"], info["blocks"], info["triangles"], info["springs"]
    if kernel == "cg_spmv":
        # A values + column ids, p gathered once, s written, filter and degree bytes
        return 40.0 * blocks + 12 * n + 12 * n + 2 * n
    if kernel == "cg_update":
        return (5 * 12 + 2 * 12) * n
    if kernel == "cg_direction":
        return (3 * 12 + 12 + 1) * n
    if kernel == "cg_init":
        return 40.0 * blocks + (12 * 3 + 1 + 3 * 12) * n
    if kernel.startswith("grid_cg"):
        # the whole persistent solve: the start (A x0: A once, m_x, b, P^-1
        # read, r and z written, filter byte), then per iteration the MPCG's
        # minimum, whatever the form: A values and columns once (40 B per
        # block), the row pointer (4 B per row), the direction read and the
        # product written (24 B per row), one fused vector pass reading p, s,
        # x, r, P^-1 and the filter and writing x, r, p (100 B per row)
        iters = float(kernel.split(":")[1])
        return 40.0 * blocks + 73.0 * n + iters * (40.0 * blocks + 128.0 * n)
    if kernel == "assemble":
        inc = 3 * t + 2 * s
        return 36.0 * blocks + (24 + 24 + 4 + 1 + 24) * n + 40.0 * t + 24.0 * s + 8.0 * inc
    return 0.0


def fp64_error(system: dict, dv: np.ndarray, tol: float = 1e-11) -> dict:
    """One step's CG solution against an FP64 solve of the same system on the
    host (scipy, Jacobi-preconditioned CG to relative residual `tol`, started
    from the GPU's solution).  The system is the step's A and b with the
    filter S applied (static rows identity, right-hand side zero).  Returns the
    relative 2-norm error of dv and the relative residual of the GPU's dv
    recomputed in FP64 in the P^-1 norm, the norm of the CG stop rule."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    t0 = time.perf_counter()
    rowptr, cols = system["rowptr"].astype(np.int64), system["cols"].astype(np.int64)
    n = rowptr.size - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rowptr))
    blk = system["vals"].reshape(-1, 3, 3).astype(np.float64)  # [block][column][row]
    three = np.arange(3, dtype=np.int64)
    ri = np.broadcast_to(3 * rows[:, None, None] + three[None, None, :], blk.shape).ravel()
    ci = np.broadcast_to(3 * cols[:, None, None] + three[None, :, None], blk.shape).ravel()
    A = sp.csr_matrix((blk.ravel(), (ri, ci)), shape=(3 * n, 3 * n))
    s3 = np.repeat(system["S"].astype(np.float64), 3)
    Sd = sp.diags(s3)
    Af = (Sd @ A @ Sd + sp.diags(1.0 - s3)).tocsr()
    bf = s3 * system["b"].astype(np.float64)
    pinv = 1.0 / Af.diagonal()
    M = sp.diags(pinv)
    x0 = s3 * dv.reshape(-1).astype(np.float64)
    its = [0]

    def count(_):
        its[0] += 1

    x64, info = spl.cg(Af, bf, x0=x0, rtol=tol, atol=0.0, maxiter=20000, M=M, callback=count)
    r = bf - Af @ x0
    res = float(np.sqrt((r @ (pinv * r)) / (bf @ (pinv * bf))))
    err = float(np.linalg.norm(x0 - x64) / np.linalg.norm(x64))
    return {"rel_dv_error": err, "true_residual_fp64": res, "fp64_cg_iterations": its[0],
            "fp64_converged": info == 0, "seconds": time.perf_counter() - t0}


def run_ours(args, rank, world):
    import bounce_b200 as b3g
    import torch

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    scene = b3g.sphere_scene(args.side, seed=2 + rank)
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    cloth = b3g.Cloth(scene.mesh, scene.cdef, device=dev).setup(scene, opts)
    # the whole solve in one persistent cooperative launch
    cloth.set_cg_strategy(True, fused=args.cg == "fused")
    cloth.set_assembly(args.assembly)
    info = cloth.info()
    n = info["vertices"]
    # L2 flush buffer (> 126 MB L2), written between timed steps
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")

    for _ in range(args.warmup):
        cloth.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = b3g.kernel_launch_count()
    step_ms, iters, contacts = [], [], []
    with ClockSampler(dev) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            st = cloth.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
            step_ms.append(st["step_ms"])
            iters.append(st["iterations"])
            contacts.append(st["active_contacts"])
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    launches = b3g.kernel_launch_count() - launches0
    # every rank steps its own replica; the job takes as long as the slowest rank
    dev_s = sum(step_ms) / 1000.0
    value = replicas.aggregate_rate(n * args.steps, dev_s)
    dev_s = replicas.max_over_ranks(dev_s)
    if world > 1:
        torch.distributed.barrier()

    # end to end through the public API with host buffers: per step the
    # external forces go host->device, the positions come back device->host,
    # both through page-locked host buffers
    forces = torch.zeros((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    pos = torch.zeros((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cloth.apply_forces(forces)
        cloth.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
        cloth.positions(pos)
    e2e_s = time.perf_counter() - t0
    e2e = replicas.aggregate_rate(n * args.steps, e2e_s)

    # accuracy of one step: its system, then the GPU's CG solution, against
    # an FP64 solve of that system on the host
    fp64 = None
    if not args.skip_fp64:
        cloth.assemble(scene.dt)
        system = cloth.system()
        cloth.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
        fp64 = fp64_error(system, cloth.state()["dv"])

    # per-kernel device times for the roofline
    prof = []
    for _ in range(args.profile_steps):
        flush.zero_()
        torch.cuda.synchronize()
        prof.append(cloth.step_profiled(scene.dt, scene.velocity_iterations, scene.position_iterations))
    if not prof:
        prof.append(cloth.step_profiled(scene.dt, scene.velocity_iterations, scene.position_iterations))
    it_total = sum(p["cg_iterations"] for p in prof)
    persistent = all(p["cg_update_ms"] == 0.0 for p in prof)
    kern = {
        "assemble": (sum(p["assemble_ms"] for p in prof), len(prof)),
        "cg_init": (sum(p["cg_init_ms"] for p in prof), len(prof)),
        "cg_spmv": (sum(p["cg_spmv_ms"] for p in prof), max(it_total, 1)),
        "cg_update": (sum(p["cg_update_ms"] for p in prof), max(it_total, 1)),
        "cg_direction": (sum(p["cg_direction_ms"] for p in prof), max(it_total, 1)),
        "finalize": (sum(p["finalize_ms"] for p in prof), len(prof)),
        "post": (sum(p["post_ms"] for p in prof), len(prof)),
        "contacts_update": (sum(p["contacts_update_ms"] for p in prof), len(prof)),
    }
    if persistent:
        # one persistent launch per step holds the whole CG
        kern.pop("cg_update")
        kern.pop("cg_direction")
        kern["grid_cg"] = kern.pop("cg_spmv")
        kern["grid_cg"] = (kern["grid_cg"][0], len(prof))
    total = sum(v[0] for v in kern.values())
    dom = max(kern, key=lambda k: kern[k][0])
    avg_ms = kern[dom][0] / kern[dom][1]
    alg = algorithmic_bytes(info, dom if dom != "grid_cg" else f"grid_cg:{it_total / len(prof)}")
    peak, peak_kind = peaks()
    achieved = alg / (avg_ms / 1000.0) / 1e9
    # the assembly (both of its launches) against the same roofline
    asm_ms = kern["assemble"][0] / kern["assemble"][1]
    asm_alg = algorithmic_bytes(info, "assemble")
    assembly = {"form": cloth.assembly(), "ms": asm_ms, "algorithmic_bytes": asm_alg,
                "achieved": asm_alg / (asm_ms / 1000.0) / 1e9,
                "frac": asm_alg / (asm_ms / 1000.0) / 1e9 / peak, "unit": "GB/s"}
    cloth.close()
    return {
        "value": value, "ms_per_step": 1000.0 * dev_s / args.steps, "wall_s": wall, "e2e": e2e, "fp64": fp64,
        "iterations_mean": float(np.mean(iters)), "active_contacts_mean": float(np.mean(contacts)),
        "launches": launches, "clocks": clocks.summary(), "info": info,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (grid_cg_traffic(args.side, args.cg, it_total / len(prof))
                                 if dom == "grid_cg" else None),
                     "traffic_source": "ncu capture of one launch at this size",
                     "algorithmic_bytes_per_launch": alg, "avg_launch_ms": avg_ms,
                     "share": kern[dom][0] / total if total else None},
        "kernel_ms": {k: v[0] / v[1] for k, v in kern.items()},
        "assembly": assembly,
    }


def run_stiff(args, dev: int):
    """The 1024 x 1024 study cloth (1,048,576 vertices, 2,093,058 triangles,
    no bending): stretch 1e5, damping 0.1, shear 1e3, the two corners of row
    0 pinned, no jitter, CG to relative residual 1e-4 (at most 2000
    iterations) with FP64 dots.  Of its 50 steps from rest, steps 3-49 are
    timed with CUDA events (the first three build the step graph and load
    the modules), once with each persistent CG form.  Its system, 7.3 M
    blocks or 293 MB of values and columns, is larger than L2, so every CG
    iteration streams it from HBM.  Each form's roofline is of its CG launch,
    from three more steps launched kernel by kernel; the section reports the
    faster form at its top level."""
    import bounce_b200 as b3g

    side = args.stiff_side
    scene = b3g.stiff_scene(side)
    opts = b3g.SolverOptions.relative(1e-4, 2000, b3g.DOT_F64)
    peak, peak_kind = peaks()
    forms = {}
    for form in ("persistent", "fused"):
        cloth = b3g.Cloth(scene.mesh, scene.cdef, device=dev).setup(scene, opts)
        cloth.set_cg_strategy(True, fused=form == "fused")
        cloth.set_assembly(args.assembly)
        info = cloth.info()
        warm = 3
        warm_its = [int(cloth.step(scene.dt)["iterations"]) for _ in range(warm)]
        ms, its = [], []
        for _ in range(warm, scene.steps):
            st = cloth.step(scene.dt)
            ms.append(st["step_ms"])
            its.append(st["iterations"])
        prof = [cloth.step_profiled(scene.dt) for _ in range(3)]
        cloth.close()
        cg_ms = sum(p["cg_spmv_ms"] for p in prof) / len(prof)
        cg_it = sum(p["cg_iterations"] for p in prof) / len(prof)
        alg = algorithmic_bytes(info, f"grid_cg:{cg_it}")
        achieved = alg / (cg_ms / 1e3) / 1e9
        n = info["vertices"]
        forms[form] = {
            "ms_per_step": sum(ms) / len(ms), "vertex_steps_per_s": n * len(ms) / (sum(ms) / 1e3),
            "cg_iterations_mean": float(np.mean(its)), "cg_iterations_max": int(max(its)),
            "warmup_cg_iterations": warm_its,
            "us_per_cg_iteration": 1e3 * cg_ms / max(cg_it, 1.0),
            "roofline": {"bound": "hbm", "kernel": "grid_cg" if form == "persistent" else "grid_cg_fused",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": grid_cg_traffic(side, form, cg_it),
                         "dram_frac": (grid_cg_traffic(side, form, cg_it) / (cg_ms / 1e3) / 1e9 / peak
                                       if grid_cg_traffic(side, form, cg_it) else None),
                         "algorithmic_bytes_per_launch": alg, "avg_launch_ms": cg_ms,
                         "cg_iterations_per_launch": cg_it}}
    best = max(forms, key=lambda f: forms[f]["vertex_steps_per_s"])
    out = {"workload": f"grid{side}x{side}_stiff", "vertices": info["vertices"], "blocks": info["blocks"],
           "steps": f"3-{scene.steps - 1}", "cg": "relative residual 1e-4, max 2000, fp64 dots",
           "cg_strategy": best}
    out.update(forms[best])
    out["by_strategy"] = forms
    return out


def run_batched(args, dev: int, cpu_sample: bool = False):
    """Many cloths of uneven sizes per launch: 512 cloths, side U{16..128},
    stretch log-U[1e3, 1e5], shear log-U[1e2, 1e4], row 0 pinned, 100 steps
    (`--batch-steps`), each step one launch of the batch's CUDA graph; against
    the plain one-cloth-at-a-time GPU path on the same cloths and steps."""
    import bounce_b200 as b3g

    # weak scaling over ranks: the job holds batch_count cloths per rank, and
    # each rank takes its share of whole cloths (no collective in the step)
    env = replicas.rank_env()
    every = b3g.batch_scenes(args.batch_count * env.world, seed=3)
    shards = replicas.plan_shards([s.mesh.vertex_count for s in every], env.world)
    scenes = [every[k] for k in shards[env.rank]]
    opts = b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64)
    cloths = [b3g.Cloth(sc.mesh, sc.cdef, device=dev).setup(sc, opts) for sc in scenes]
    for c in cloths:
        c.set_assembly(args.assembly)
    rows = sum(c.n for c in cloths)
    dt = scenes[0].dt
    batch = b3g.Batch(max(1024, len(cloths)), device=dev)
    for _ in range(args.warmup):
        batch.step(cloths, dt)
    sched = batch.autotune(cloths, dt)
    blocks = np.array([c.info()["blocks"] for c in cloths], dtype=np.float64)
    nrows = np.array([c.n for c in cloths], dtype=np.float64)
    ms, cg_ms, iters, cg_bytes = [], [], [], []
    launches0 = b3g.kernel_launch_count()
    for _ in range(args.batch_steps):
        out = batch.step(cloths, dt, per_cloth=True)
        ms.append(out["step_ms"])
        cg_ms.append(out["cg_ms"])
        iters.append(out["cg_iterations_total"] / out["count"])
        it = np.array([pc["iterations"] for pc in out["per_cloth"]], dtype=np.float64)
        # the same per-cloth count as the persistent single-cloth solve
        cg_bytes.append(float(np.sum(40.0 * blocks + 73.0 * nrows + it * (40.0 * blocks + 146.0 * nrows))))
    launches = b3g.kernel_launch_count() - launches0
    batched = replicas.aggregate_rate(rows * len(ms), sum(ms) / 1000.0)
    for c in cloths:
        c.close()
    batch.close()
    # the plain single-instance path on the same cloths, the same steps from
    # rest: each cloth alone with each CG form (per-iteration launches in a
    # graph loop, the persistent CG, the fused persistent CG); each cloth
    # counts at its fastest
    plain_v, plain_by = None, {}
    if not args.skip_plain:
        per = []
        for strategy in ("launches", "persistent", "fused"):
            plain = [b3g.Cloth(sc.mesh, sc.cdef, device=dev).setup(sc, opts) for sc in scenes]
            t = np.zeros(len(plain))
            for k, c in enumerate(plain):
                c.set_assembly(args.assembly)
                if strategy != "launches":
                    c.set_cg_strategy(True, fused=strategy == "fused")
                for _ in range(args.warmup):
                    c.step(dt)
                for _ in range(args.batch_steps):
                    t[k] += c.step(dt)["step_ms"]
                c.close()
            per.append(t)
            plain_by[strategy] = replicas.aggregate_rate(rows * args.batch_steps, float(t.sum()) / 1000.0)
        best = np.minimum(np.minimum(per[0], per[1]), per[2])
        plain_v = replicas.aggregate_rate(rows * args.batch_steps, float(best.sum()) / 1000.0)
    return {"cloths": int(replicas.sum_over_ranks(len(scenes))), "vertices": int(replicas.sum_over_ranks(rows)),
            "vertex_steps_per_s": batched,
            "ms_per_step": sum(ms) / len(ms), "plain_vertex_steps_per_s": plain_v,
            "plain_by_strategy": plain_by,
            "plain": "each cloth alone, at the fastest of its three CG forms",
            "speedup_vs_plain": batched / plain_v if plain_v else None, "cg_iterations_mean": float(np.mean(iters)),
            "schedule": {"cluster": sched["cluster"],
                         "split_size_classes": [k for k, v in enumerate(sched["split_class"]) if v]},
            "gpu_launches": launches, "steps": len(ms),
            "roofline": {"bound": "hbm", "kernel": "batch_cg", "achieved": sum(cg_bytes) / (sum(cg_ms) / 1e3) / 1e9,
                         "peak": peaks()[0], "peak_kind": peaks()[1], "unit": "GB/s",
                         "frac": sum(cg_bytes) / (sum(cg_ms) / 1e3) / 1e9 / peaks()[0],
                         "algorithmic_bytes_per_launch": sum(cg_bytes) / len(cg_bytes),
                         "traffic": BATCH_CG_TRAFFIC_RATIO * sum(cg_bytes) / len(cg_bytes),
                         "traffic_source": "DRAM/algorithmic ratio of one captured 512-cloth launch",
                         "dram_frac": (BATCH_CG_TRAFFIC_RATIO * sum(cg_bytes) / (sum(cg_ms) / 1e3) / 1e9
                                       / peaks()[0]),
                         "avg_launch_ms": sum(cg_ms) / len(cg_ms), "share": sum(cg_ms) / sum(ms)},
            "l2": "inputs larger than L2 (about 1 GB of resident cloth state)",
            "cpu_baseline": cpu_batch_sample(args.batch_count) if cpu_sample else None}


def run_softbody(args, dev: int, cpu_sample: bool):
    """The soft body step (b3SoftBody::Step) on a side^3 tetrahedral block of
    1 m edge, hanging from one node, with the reference's pinned soft body
    material and its own MPCG rule (20 iterations).  At side 40: 68,921 nodes
    and 320,000 tetrahedra, whose per-element stiffness matrices alone
    (12 x 12 floats each) are 184 MB, above L2.  The CPU figure is the oracle
    (the C restatement, one core) on the same block for two steps."""
    import bounce_b200 as b3g

    side = args.softbody_side
    scene = b3g.pinned_block_scene(side, side, side, spacing=1.0 / side)
    n, t = len(scene.vertices), len(scene.tets)
    by = {}
    for form in ("launches", "persistent", "fused"):
        body = b3g.SoftBody(scene.vertices, scene.tets, scene.sdef, device=dev).setup(scene)
        body.set_cg_strategy(form != "launches", fused=form == "fused")
        for _ in range(args.warmup):
            body.step(scene.dt)
        launches0 = b3g.kernel_launch_count()
        ms, iters = [], []
        for _ in range(args.softbody_steps):
            s = body.step(scene.dt)
            ms.append(s["step_ms"])
            iters.append(s["iterations"])
        launches = b3g.kernel_launch_count() - launches0
        nnz = body.block_count()
        body.close()
        by[form] = {"ms_per_step": sum(ms) / len(ms), "node_steps_per_s": n * len(ms) / (sum(ms) / 1e3),
                    "cg_iterations_mean": float(np.mean(iters)), "gpu_launches": launches, "steps": len(ms)}
    # algorithmic bytes of one step (FP32): the element kernel reads an
    # element's vertices, rest frame, Ke, B, P and state and writes R, q, eps,
    # f0, f_plastic (1,512 B); the assembly reads R, Ke, f0, f_plastic and the
    # incidences per element (708 B), per node its state (41 B) and per block
    # the column, the gathered x and the value written (52 B); each CG
    # iteration moves 40 B per block and 164 B per row, the CG start 40 B per
    # block and 100 B per row; the integration 48 B per node.
    for form, f in by.items():
        it = f["cg_iterations_mean"]
        step_bytes = 1512.0 * t + 708.0 * t + 41.0 * n + 52.0 * nnz + (40.0 * nnz + 100.0 * n) + \
            it * (40.0 * nnz + 164.0 * n) + 48.0 * n
        achieved = step_bytes / (f["ms_per_step"] / 1e3) / 1e9
        f["roofline"] = {"bound": "hbm", "kernel": "whole step", "achieved": achieved, "peak": peaks()[0],
                         "peak_kind": peaks()[1], "unit": "GB/s", "frac": achieved / peaks()[0],
                         "algorithmic_bytes_per_step": step_bytes}
    out = {"workload": f"block{side}x{side}x{side}_pinned", "nodes": n, "tetrahedra": t, "blocks": nnz,
           "cg": "reference rule (20 iterations, f32 dots)",
           "cg_strategy": "persistent cooperative launch (the default)"}
    out.update(by["persistent"])
    out["by_strategy"] = by
    if cpu_sample:
        import oracle

        ora = oracle.PortSoftBody(scene.vertices, scene.tets, scene.sdef.density, scene.sdef.E, scene.sdef.nu,
                                  scene.sdef.c_yield, scene.sdef.c_creep, scene.sdef.c_max).setup(scene)
        t0 = time.perf_counter()
        for _ in range(2):
            ora.step(scene.dt)
        sec = time.perf_counter() - t0
        ora.close()
        out["cpu_baseline"] = {"value": n * 2 / sec, "unit": "node-steps/s", "cores": 1, "kind": "port",
                               "sample": f"the oracle's soft body step, 2 steps of the same block, {sec / 2:.2f} s/step"}
    out["hull"] = run_softbody_hull(args, dev, cpu_sample)
    return out


def run_softbody_hull(args, dev: int, cpu_sample: bool):
    """The same block, free, resting on a static ground hull (a 6 x 0.5 x 6 m
    box whose top is 0.06 m below the block; node radius 0.05, friction 0.2,
    hull friction 0.6): node contacts (GJK TestSphere, velocity and position
    iterations) inside the step.  12 steps to land, then 10 timed with CUDA
    events.  The CPU figure is the oracle on the same scene, 2 steps after
    the same 12."""
    import dataclasses

    import bounce_b200 as b3g

    side = args.softbody_side
    scene = dataclasses.replace(b3g.pinned_block_scene(side, side, side, spacing=1.0 / side),
                                static_nodes=np.zeros(0, np.uint32))
    hv, hp = box_hull(3.0, 0.25, 3.0, -0.81)
    land, timed = 12, 10

    def dress(b):
        b.add_hull(hv, hp, 0.6)
        for i in range(len(scene.vertices)):
            b.set_node_radius(i, 0.05)
            b.set_node_friction(i, 0.2)
        return b

    body = dress(b3g.SoftBody(scene.vertices, scene.tets, scene.sdef, device=dev).setup(scene))
    for _ in range(land):
        body.step(scene.dt)
    ms = [body.step(scene.dt)["step_ms"] for _ in range(timed)]
    active = int(body.contacts()["active"].sum())
    body.close()
    n = len(scene.vertices)
    out = {"workload": f"block{side}x{side}x{side}_on_hull", "nodes": n, "steps": f"{land}-{land + timed - 1}",
           "ms_per_step": sum(ms) / len(ms), "node_steps_per_s": n * len(ms) / (sum(ms) / 1e3),
           "active_contacts": active}
    if cpu_sample:
        import oracle

        s = scene.sdef
        ora = dress(oracle.PortSoftBody(scene.vertices, scene.tets, s.density, s.E, s.nu, s.c_yield, s.c_creep,
                                        s.c_max).setup(scene))
        for _ in range(land):
            ora.step(scene.dt)
        t0 = time.perf_counter()
        for _ in range(2):
            ora.step(scene.dt)
        sec = time.perf_counter() - t0
        ora.close()
        out["cpu_baseline"] = {"value": n * 2 / sec, "unit": "node-steps/s", "cores": 1, "kind": "port",
                               "sample": f"the oracle on the same scene, steps {land}-{land + 1}, {sec / 2:.2f} s/step"}
    return out


def run_self_collision(args, dev: int, cpu_sample: bool):
    """Self-collision (thickness 0.2): the reference's self-collision scene
    scaled to a side x side grid of 1 m spacing over a capsule as long as the
    cloth, CG at the reference's 20-iteration rule.  Steps 0-59 fall (contacts
    exist, none active); steps 60-119, the fold, are timed on the GPU with
    CUDA events.  The CPU figure is the
    reference's own full b3Cloth::Step on the same cloth over the same 60
    steps, one core.  A first cloth runs the 120 steps untimed as warm-up."""
    import bounce_b200 as b3g

    scene = b3g.self_collision_scene(args.self_side)
    lo, hi = 60, 120
    # warm-up: one untimed pass of the same 120 steps on another cloth, so
    # that first-use costs (module loading, the contact list's first growth
    # to this scene's size) stay out of the timed steps
    warm = b3g.Cloth(scene.mesh, scene.cdef, device=dev).setup(scene)
    warm.set_cg_strategy(True)
    for _ in range(hi):
        warm.step(scene.dt)
    warm.close()
    cloth = b3g.Cloth(scene.mesh, scene.cdef, device=dev).setup(scene)
    cloth.set_cg_strategy(True)  # the whole CG in one persistent launch
    for _ in range(lo):
        cloth.step(scene.dt)
    launches0 = b3g.kernel_launch_count()
    ms, contacts, active, levels = [], [], [], []
    for _ in range(lo, hi):
        ms.append(cloth.step(scene.dt)["step_ms"])
        st = cloth.self_stats()
        contacts.append(st["contacts"])
        active.append(st["active"])
        levels.append(st["levels"])
    launches = b3g.kernel_launch_count() - launches0
    cloth.close()
    n = scene.mesh.vertex_count
    out = {"workload": f"grid{args.self_side}_self_collision_capsule", "vertices": n,
           "triangles": scene.mesh.triangle_count, "steps": f"{lo}-{hi - 1}",
           "ms_per_step": sum(ms) / len(ms), "ms_median": float(np.median(ms)), "ms_max": float(max(ms)),
           "vertex_steps_per_s": n * len(ms) / (sum(ms) / 1e3),
           "tri_contacts_mean": float(np.mean(contacts)), "active_mean": float(np.mean(active)),
           "active_max": int(max(active)), "levels_mean": float(np.mean(levels)), "gpu_launches": launches}
    if cpu_sample:
        import oracle

        if oracle.ref_available():
            ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=True).setup(scene)
            for _ in range(lo):
                ref.step(scene.dt, full=True)
            t0 = time.perf_counter()
            for _ in range(lo, hi):
                ref.step(scene.dt, full=True)
            sec = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": n * (hi - lo) / sec, "unit": "vertex-steps/s", "cores": 1,
                                   "kind": "reference",
                                   "sample": f"the reference's full b3Cloth::Step, steps {lo}-{hi - 1} of the same "
                                             f"cloth, {1e3 * sec / (hi - lo):.1f} ms/step"}
    return out


def box_hull(hx: float, hy: float, hz: float, cy: float):
    """A box as a hull (vertices and face planes, world frame) centred at
    (0, cy, 0)."""
    v = np.array([(sx * hx, cy + sy * hy, sz * hz) for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)], np.float32)
    planes = np.array([(1, 0, 0, hx), (-1, 0, 0, hx), (0, 1, 0, cy + hy), (0, -1, 0, -(cy - hy)), (0, 0, 1, hz),
                       (0, 0, -1, hz)], np.float32)
    return v, planes


def run_colliders(args, dev: int, cpu_sample: bool):
    """Static capsule and hull colliders: a side x side cloth (bending on)
    falling onto a capsule (a rod along z) and onto a box hull (a 0.7 m
    table top), 10 steps timed with CUDA events after it lands.  The CPU
    figure is the reference's b3Cloth::Step on the same cloth and shape (its
    quickhull builds the box from the same eight corners), two steps."""
    import bounce_b200 as b3g

    side = args.collider_side
    out = {}
    for kind in ("capsule", "hull"):
        scene = b3g.capsule_scene(side)
        if kind == "hull":
            hv, hp = box_hull(0.35, 0.05, 0.35, -0.4)
            scene.capsules = []
            scene.hulls = [(hv, hp, 0.3)]
        cloth = b3g.Cloth(scene.mesh, scene.cdef, device=dev).setup(scene)
        cloth.set_cg_strategy(True)
        for _ in range(40):  # fall onto the shape
            cloth.step(scene.dt)
        ms, active = [], []
        for _ in range(10):
            st = cloth.step(scene.dt)
            ms.append(st["step_ms"])
            active.append(st["active_contacts"])
        cloth.close()
        n = scene.mesh.vertex_count
        r = {"workload": f"grid{side}_{kind}", "vertices": n, "steps": "40-49", "ms_per_step": sum(ms) / len(ms),
             "vertex_steps_per_s": n * len(ms) / (sum(ms) / 1e3), "active_contacts_mean": float(np.mean(active))}
        if cpu_sample:
            import oracle

            if oracle.ref_available():
                ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=True)
                ref.set_gravity(scene.gravity)
                if kind == "capsule":
                    for (a, b, rad, mu) in scene.capsules:
                        ref.add_capsule(a, b, rad, mu)
                else:
                    ref.add_hull_from_points(hv, 0.3)
                t0 = time.perf_counter()
                for _ in range(2):
                    ref.step(scene.dt)
                sec = time.perf_counter() - t0
                r["cpu_baseline"] = {"value": n * 2 / sec, "unit": "vertex-steps/s", "cores": 1, "kind": "reference",
                                     "sample": f"the reference's b3Cloth::Step, the first 2 steps of the same cloth "
                                               f"and shape, {sec / 2:.2f} s/step"}
        out[kind] = r
    return out


def run_serving(args, dev: int):
    from bounce_b200 import serving

    # the offered load exceeds one GPU's capacity: the stream is served for its
    # 30 s and a 5 s drain, and requests still queued then are reported
    return serving.run_poisson(rate=2000.0, seconds=args.serve_seconds, budget_bytes=150 * 10**9, device=dev,
                               drain_limit_s=5.0)


def _reference_worker(job):
    """One host process: the reference (compiled from its sources) building and
    stepping one cloth on one core."""
    side, steps, warm = job
    import oracle

    import bounce_b200 as b3g

    scene = b3g.sphere_scene(side, seed=2)
    t0 = time.perf_counter()
    ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=True).setup(scene)
    build_s = time.perf_counter() - t0
    for _ in range(warm):
        ref.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
    oracle.ref_profile_reset()
    t0 = time.perf_counter()
    for _ in range(steps):
        ref.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
    dt = time.perf_counter() - t0
    solve = oracle.ref_profile().get("Cloth Solve", (0.0, 0))[0]
    return {"n": scene.mesh.vertex_count, "steps": steps, "seconds": dt, "solve_s": solve, "build_s": build_s}


def cpu_reference_sample(side: int, steps: int, warm: int, procs: int = 0):
    """The reference stepping the headline cloth on the host cores: one
    independent replica per core (the reference is single-threaded), the
    rate being the vertex-steps of all replicas over the slowest one's time.
    The workers start by spawn."""
    import multiprocessing as mp

    procs = procs or int(os.environ.get("B3G_REFERENCE_PROCS", "0")) or (os.cpu_count() or 1)
    if procs == 1:
        outs = [_reference_worker((side, steps, warm))]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            outs = pool.map(_reference_worker, [(side, steps, warm)] * procs)
    n = outs[0]["n"]
    slowest = max(o["seconds"] for o in outs)
    per = outs[0]
    value = sum(o["n"] * o["steps"] for o in outs) / slowest
    return {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": (f"{procs} independent replicas, one per host core, each {steps} steps (after {warm} "
                       f"warm-up) of the same {side}x{side} cloth with the reference b3Cloth::Step minus the inert "
                       f"self-collision pass, CG at the reference's own 20-iteration rule; per replica "
                       f"{per['seconds'] / steps:.2f} s/step, of which 'Cloth Solve' {per['solve_s'] / steps:.2f} "
                       f"s/step; slowest replica {slowest / steps:.2f} s/step; constructor {per['build_s']:.1f} s; "
                       f"one core alone: {n * steps / per['seconds']:.3g} vertex-steps/s"),
            "seconds": slowest}


def _reference_batch_worker(job):
    """One host process: the reference stepping its share of the batched
    cloths (same seeded scenes), `steps` steps each, one after another."""
    count, indices, steps = job
    import oracle

    import bounce_b200 as b3g

    scenes = b3g.batch_scenes(count, seed=3)
    vs, sec = 0, 0.0
    for k in indices:
        sc = scenes[k]
        ref = oracle.RefCloth(sc.mesh, sc.cdef, restated=True).setup(sc)
        t0 = time.perf_counter()
        for _ in range(steps):
            ref.step(sc.dt, sc.velocity_iterations, sc.position_iterations)
        sec += time.perf_counter() - t0
        vs += sc.mesh.vertex_count * steps
        del ref
    return {"vertex_steps": vs, "seconds": sec}


def cpu_batch_sample(count: int, every: int = 8, steps: int = 2, procs: int = 0):
    """The reference on the batched workload: every `every`-th of the
    `count` cloths, dealt round-robin to one process per host core; the rate is
    all vertex-steps over the slowest process's stepping time."""
    import multiprocessing as mp

    procs = procs or int(os.environ.get("B3G_REFERENCE_PROCS", "0")) or (os.cpu_count() or 1)
    picked = list(range(0, count, every))
    jobs = [(count, picked[w::procs], steps) for w in range(procs) if picked[w::procs]]
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        outs = pool.map(_reference_batch_worker, jobs)
    slowest = max(o["seconds"] for o in outs)
    vs = sum(o["vertex_steps"] for o in outs)
    return {"value": vs / slowest, "unit": UNIT, "cores": len(jobs), "kind": "reference",
            "sample": f"{len(picked)} of the {count} batched cloths (every {every}th), {steps} steps each with the "
                      f"reference b3Cloth::Step at its own 20-iteration CG rule, spread over {len(jobs)} processes "
                      f"(one per host core); slowest process {slowest:.2f} s"}


def summary(line: dict) -> dict:
    """The section headlines, repeated compactly at the end of the line."""
    def g(d, *keys):
        for k in keys:
            if not isinstance(d, dict):
                return None
            d = d.get(k)
        return round(d, 4) if isinstance(d, float) else d

    b, s, st = line.get("batched"), line.get("serving"), line.get("stiff1024")
    return {
        "headline_vertex_steps_per_s": g(line, "value"), "headline_e2e": g(line, "e2e", "value"),
        "headline_frac": g(line, "roofline", "frac"), "headline_fp64_rel_dv_error": g(line, "fp64", "rel_dv_error"),
        "assembly_ms": g(line, "assembly", "ms"), "assembly_frac": g(line, "assembly", "frac"),
        "batched_vertex_steps_per_s": g(b, "vertex_steps_per_s"), "batched_speedup_vs_plain": g(b, "speedup_vs_plain"),
        "batched_frac": g(b, "roofline", "frac"),
        "serving_vertex_steps_per_s": g(s, "vertex_steps_per_s"), "serving_tick_p50_ms": g(s, "p50_step_ms"),
        "serving_tick_p99_ms": g(s, "p99_step_ms"), "serving_busy": g(s, "device_busy_fraction"),
        "serving_seconds_offered": g(s, "seconds_offered"),
        "stiff1024_vertex_steps_per_s": g(st, "vertex_steps_per_s"), "stiff1024_frac": g(st, "roofline", "frac"),
        "stiff1024_dram_frac": g(st, "roofline", "dram_frac"), "batched_dram_frac": g(b, "roofline", "dram_frac"),
        "softbody_node_steps_per_s": g(line.get("softbody"), "node_steps_per_s"),
        "softbody_frac": g(line.get("softbody"), "roofline", "frac"),
    }


def host_cpu():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def main():
    args = parse()
    world, rank, local = dist_env()
    if args.impl == "reference":
        if rank != 0:
            return
        steps = max(1, min(args.steps, 3))
        warm = min(args.warmup, 1)
        base = cpu_reference_sample(args.side, steps, warm)
        line = {"metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
                "warmup": warm, "ms_per_step": 1000.0 * base["seconds"] / steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                "config": {"workload": f"grid{args.side}x{args.side}_bending_sphere", "vertices": args.side ** 2,
                           "host_cpu": host_cpu()},
                "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    if args.skip_single:
        batched = None if args.skip_batch else run_batched(args, local)
        served = None if args.skip_serve else run_serving(args, local)
        soft = None if args.skip_softbody else run_softbody(args, local, False)
        selfc = None if args.skip_self else run_self_collision(args, local, False)
        colliders = None if args.skip_colliders else run_colliders(args, local, False)
        stiff = None if args.skip_stiff else run_stiff(args, local)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": None, "unit": UNIT, "note": "headline skipped (--skip-single)",
                              "batched": batched, "serving": served, "softbody": soft, "self_collision": selfc,
                              "colliders": colliders, "stiff1024": stiff}))
        if world > 1:
            import torch

            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    r = run_ours(args, rank, world)
    batched = None if args.skip_batch else run_batched(args, local, rank == 0 and world == 1
                                                         and not args.no_cpu_baseline)
    served = None if args.skip_serve else run_serving(args, local)
    stiff = None if args.skip_stiff else run_stiff(args, local)
    soft = None if args.skip_softbody else run_softbody(args, local, rank == 0 and world == 1
                                                         and not args.no_cpu_baseline)
    selfc = None if args.skip_self else run_self_collision(args, local, rank == 0 and world == 1
                                                            and not args.no_cpu_baseline)
    colliders = None if args.skip_colliders else run_colliders(args, local, rank == 0 and world == 1
                                                                and not args.no_cpu_baseline)
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            base = cpu_reference_sample(args.side, 2, 0)
            base = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as e:  # the reference library was not built here
            base = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    n = r["info"]["vertices"]
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"grid{args.side}x{args.side}_bending_sphere", "vertices": n,
                   "triangles": r["info"]["triangles"], "springs": r["info"]["springs"],
                   "blocks": r["info"]["blocks"], "cg": "relative residual 1e-4, max 200, fp64 dots",
                   "cg_strategy": ("persistent cooperative launch, one grid reduction per iteration"
                                   if args.cg == "fused" else "persistent cooperative launch, two grid "
                                                              "reductions per iteration"),
                   "contact_iterations": [8, 2], "parallelism": f"replicas{world}",
                   "l2": "flushed (256 MB write) before every timed step",
                   "cg_iterations_mean": r["iterations_mean"], "active_contacts_mean": r["active_contacts_mean"]},
        "clocks": r["clocks"],
        "e2e": {"value": r["e2e"], "unit": UNIT, "h2d_bytes_per_step": 12 * n, "d2h_bytes_per_step": 12 * n},
        "gpu_launches": r["launches"],
        "roofline": r["roofline"],
        "kernel_ms": r["kernel_ms"],
        "assembly": r["assembly"],
        "cpu_baseline": base,
        "fp64": r["fp64"],
        "batched": batched,
        "serving": served,
        "stiff1024": stiff,
        "softbody": soft,
        "self_collision": selfc,
        "colliders": colliders,
    }
    line["summary"] = summary(line)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
