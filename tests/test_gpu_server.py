"""Serving with continuous batching (b3g_server)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _wait_prepared(srv, ids, timeout=60.0):
    t0 = time.time()
    while time.time() - t0 < timeout:
        if all(srv.poll(i)["state"] >= 1 for i in ids):
            return
        time.sleep(0.01)
    raise TimeoutError("requests not prepared")


def test_result_same_alone_and_in_the_mix(b3g):
    target = b3g.sphere_scene(24, seed=21)
    # alone
    a = b3g.Server(budget_bytes=2 << 30, max_active=64)
    rid = a.submit_scene(target, steps=12)
    _wait_prepared(a, [rid])
    a.drain()
    alone = a.result(rid)
    # in a mix: other requests before, during and after it, different sizes and step counts
    m = b3g.Server(budget_bytes=2 << 30, max_active=64)
    rng = np.random.default_rng(5)
    others = []
    for k in range(6):
        sc = b3g.plain_scene(int(rng.integers(8, 48)), seed=100 + k)
        others.append(m.submit_scene(sc, steps=int(rng.integers(1, 20))))
    _wait_prepared(m, others)
    m.tick()
    m.tick()
    rid2 = m.submit_scene(target, steps=12)
    for k in range(4):
        sc = b3g.sphere_scene(int(rng.integers(8, 40)), seed=200 + k)
        others.append(m.submit_scene(sc, steps=int(rng.integers(1, 30))))
    _wait_prepared(m, others + [rid2])
    m.drain()
    mixed = m.result(rid2)
    assert np.array_equal(alone, mixed)
    info = m.poll(rid2)
    assert info["state"] == 3 and info["steps_done"] == 12


def test_server_matches_plain_cloth(b3g):
    scene = b3g.sphere_scene(20, seed=31)
    srv = b3g.Server(budget_bytes=1 << 30, max_active=8)
    rid = srv.submit_scene(scene, steps=15)
    _wait_prepared(srv, [rid])
    srv.drain()
    cloth = b3g.Cloth(scene.mesh, scene.cdef).setup(scene, b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64))
    for _ in range(15):
        cloth.step(scene.dt)
    assert np.abs(srv.result(rid) - cloth.positions()).max() <= 1e-4


def test_admission_respects_the_budget(b3g):
    scenes = [b3g.plain_scene(int(s), seed=40 + k) for k, s in enumerate([30, 40, 50, 30, 40, 50, 60, 20])]
    probe = b3g.Server(budget_bytes=1 << 30, max_active=8)
    rid = probe.submit_scene(scenes[6], steps=1)
    _wait_prepared(probe, [rid])
    biggest = probe.poll(rid)["bytes"]
    budget = int(biggest * 2.2)
    srv = b3g.Server(budget_bytes=budget, max_active=8)
    ids = [srv.submit_scene(sc, steps=5) for sc in scenes]
    _wait_prepared(srv, ids)
    srv.drain()
    st = srv.stats()
    assert st["completed"] == len(scenes)
    assert st["peak_bytes"] <= budget
    assert st["peak_active"] < len(scenes)  # the budget held some back
    assert st["p99_step_ms"] >= st["p50_step_ms"] > 0


def test_admission_respects_the_slot_limit(b3g):
    """More prepared requests than slots, all admissible by memory: one tick
    admits at most max_active of them, and every request still completes."""
    scenes = [b3g.plain_scene(16, seed=60 + k) for k in range(12)]
    srv = b3g.Server(budget_bytes=1 << 34, max_active=4)
    ids = [srv.submit_scene(sc, steps=3) for sc in scenes]
    _wait_prepared(srv, ids)
    t = srv.tick(0.0)
    assert t["active"] <= 4 and t["admitted"] <= 4, t
    srv.drain()
    st = srv.stats()
    assert st["completed"] == len(scenes)
    assert st["peak_active"] <= 4


def test_oversized_request_is_rejected(b3g):
    srv = b3g.Server(budget_bytes=1 << 20, max_active=4)
    rid = srv.submit_scene(b3g.plain_scene(64), steps=1)
    t0 = time.time()
    while srv.poll(rid)["state"] < 3 and time.time() - t0 < 30:
        time.sleep(0.01)
    info = srv.poll(rid)
    assert info["state"] == 4 and info["status"] == 8  # failed, capacity
