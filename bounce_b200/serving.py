"""Request loop for the cloth-step server: Poisson arrivals of cloths of
log-uniform size, each to be advanced a uniform number of steps, 25% of them
over a static sphere, admitted under an HBM budget (b3g_server)."""
from __future__ import annotations

import time

import numpy as np

from . import STATIC, Server, SolverOptions, DOT_F64
from .meshes import ClothDef, grid_mesh


def run_poisson(rate: float = 2000.0, seconds: float = 30.0, side_lo: int = 8, side_hi: int = 256,
                steps_lo: int = 1, steps_hi: int = 60, sphere_fraction: float = 0.25,
                budget_bytes: int = 150 * 10**9, max_active: int = 16384, seed: int = 7, device: int = 0,
                drain_limit_s: float = 120.0, cluster: int = 4, split_classes=tuple(range(9, 20))) -> dict:
    """Run the stream in real time; returns throughput and latency figures."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=int(rate * seconds * 1.5) + 16)
    arrivals = np.cumsum(gaps)
    arrivals = arrivals[arrivals < seconds]
    nreq = len(arrivals)
    sides = np.exp(rng.uniform(np.log(side_lo), np.log(side_hi), size=nreq)).astype(int).clip(side_lo, side_hi)
    steps = rng.integers(steps_lo, steps_hi + 1, size=nreq)
    sphere = rng.uniform(size=nreq) < sphere_fraction
    meshes = {}
    for s in np.unique(sides):  # one jittered grid per size, built before the clock starts
        meshes[int(s)] = grid_mesh(int(s), 1.0, 1e-3, seed + int(s))
    cdef = ClothDef(density=1.0, streching=1e4, shearing=1e3, damping=0.05, friction=0.3)
    # split-instance over clusters of 4 CTAs for cloths of 512 vertices and
    # more, block-per-instance below (the fastest of the schedules tried on
    # this stream: clusters of 1, 4 and 8, splits from 2^9 or 2^11)
    srv = Server(budget_bytes=budget_bytes, max_active=max_active,
                 solver=SolverOptions.relative(1e-4, 200, DOT_F64), cluster=cluster, split_classes=split_classes,
                 device=device)
    types_cache = {}
    ids = []
    t0 = time.perf_counter()
    i = 0
    ticks = 0
    while True:
        now = time.perf_counter() - t0
        while i < nreq and arrivals[i] <= now:
            side = int(sides[i])
            mesh = meshes[side]
            if side not in types_cache:
                ty = np.full(side * side, 2, np.uint8)
                ty[[0, side - 1]] = STATIC
                types_cache[side] = ty
            sph = [((0.0, -0.5, 0.0), 0.3, 0.3)] if sphere[i] else []
            ids.append(srv.submit(mesh, cdef, types_cache[side], sph, int(steps[i]), float(arrivals[i])))
            i += 1
        st = srv.stats()
        if i >= nreq and st["active"] == 0 and st["queued"] == 0:
            break
        if now > seconds + drain_limit_s:
            break
        if st["active"] == 0 and st["queued"] > 0:
            time.sleep(0.0005)  # waiting for host topology workers
        srv.tick(now)
        ticks += 1
    wall = time.perf_counter() - t0
    st = srv.stats()
    lat = []
    for rid in ids:
        info = srv.poll(rid)
        if info["state"] == 3:
            lat.append(info["finished"] - info["arrival"])
    lat = np.asarray(lat) if lat else np.zeros(1)
    srv.close()
    return {
        "requests": nreq, "completed": int(st["completed"]), "rejected": int(st["rejected"]),
        "seconds_offered": seconds, "wall_s": wall, "ticks": int(st["ticks"]),
        "vertex_steps": int(st["vertex_steps"]), "vertex_steps_per_s": st["vertex_steps"] / wall,
        "device_busy_s": st["busy_ms"] / 1000.0, "device_busy_fraction": st["busy_ms"] / 1000.0 / wall,
        "unfinished": nreq - int(st["completed"]) - int(st["rejected"]),
        "p50_step_ms": st["p50_step_ms"], "p99_step_ms": st["p99_step_ms"], "max_step_ms": st["max_step_ms"],
        "p50_request_s": float(np.percentile(lat, 50)), "p99_request_s": float(np.percentile(lat, 99)),
        "peak_active": int(st["peak_active"]), "peak_bytes": int(st["peak_bytes"]),
        "schedule": {"cluster": cluster, "split_size_classes": list(split_classes)},
    }
