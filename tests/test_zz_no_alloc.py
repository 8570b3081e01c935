"""b3g_mpcg_solve_noalloc: the block-CSR MPCG for callers that cannot
allocate device memory when they solve (a frame loop that reserved all of
its memory at load time, memory already held by another framework's caching
allocator).  Its scratch is a static device array inside libb3g.so; the
results must equal those of b3g_mpcg_solve, which allocates its scratch per
call, on two calls in a row.  Both run the same kernels on the same grid
with the same reduction order, so they agree bit for bit (stricter than the
relative 1e-4 of the other parity tests).  The larger system is solved
first, so a smaller one after it would read any stale scratch left by the
earlier call.  Collected last so that a run stopping at its first failure
has run every other test already."""
import os

import numpy as np
import pytest

from helpers import call_mpcg, device_system, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "system16_bend_ref.npz")


def _systems(b3g):
    scene = b3g.sphere_scene(64)
    cloth = b3g.Cloth(scene.mesh, scene.cdef).setup(scene)
    for _ in range(3):
        cloth.step(scene.dt)
    cloth.assemble(scene.dt)
    yield cloth.system()
    cloth.close()
    d = np.load(GOLDEN)
    yield {k[4:]: d[k] for k in d.files if k.startswith("sys_")}


def test_noalloc_matches_allocating_solver(b3g):
    for sysd in _systems(b3g):
        dsys = device_system(sysd)
        for opts in (b3g.SolverOptions.reference(), b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_F64),
                     b3g.SolverOptions.relative(1e-4, 200, b3g.DOT_COMPENSATED)):
            for call in range(2):
                s1, x1, it1, st1 = call_mpcg(b3g, "b3g_mpcg_solve", dsys, opts)
                s2, x2, it2, st2 = call_mpcg(b3g, "b3g_mpcg_solve_noalloc", dsys, opts)
                assert s1 == 0 and s2 == 0, (s1, s2)
                assert it1 == it2, (call, it1, it2)
                assert np.array_equal(x2, x1), (call, rel_err(x2, x1))
                assert st1.delta == st2.delta and st1.delta0 == st2.delta0, (call, st1.delta, st2.delta)


def test_noalloc_rejects_systems_above_its_capacity(b3g):
    import torch

    L = b3g.lib()
    n = 65536 + 1
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda:0")
    p = dummy.data_ptr()
    o = b3g.SolverOptions.reference().as_c()
    import ctypes as C

    status = L.b3g_mpcg_solve_noalloc(n, p, p, p, p, p, p, C.byref(o), p, None, None, None)
    assert status == 8  # B3G_ERR_CAPACITY, before any device work
