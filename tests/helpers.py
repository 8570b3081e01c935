"""Shared helpers of the parity tests."""
import numpy as np


def system_blocks(sys, vertex_of_row=None):
    """{(row vertex, col vertex): 9 floats} and b by vertex, from an exported system."""
    rowptr, cols, vals = sys["rowptr"], sys["cols"], sys["vals"].reshape(-1, 9)
    n = rowptr.size - 1
    vor = np.arange(n) if vertex_of_row is None else vertex_of_row
    blocks = {}
    for r in range(n):
        i = int(vor[r])
        for k in range(int(rowptr[r]), int(rowptr[r + 1])):
            blocks[(i, int(vor[int(cols[k])]))] = vals[k]
    b = np.zeros((n, 3), np.float32)
    b[vor] = sys["b"].reshape(-1, 3)
    return blocks, b


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def oracle_floor_step(port, scene, ora, dt, stop_rule, tol, max_iter, dress=None):
    """Positions and velocities after one step of clones of the oracle `ora` -- its whole
    state: positions, velocities, CG warm start, body contacts with their
    impulses and the particles' proxies -- with compensated and with FP64
    dots.  Against `ora`'s own step they measure how far the same algorithm
    moves under different rounding alone; a truncated CG (the reference's
    20-iteration rule) is sensitive at some steps.  `dress(clone)` applies
    per-particle settings; call before `ora` steps."""
    st = ora.state()
    ca = ora.contacts()
    fat = ora.describe()["fat_aabb"]
    live = np.nonzero(ca["exists"])[0]
    out = []
    for dot in (1, 2):
        c = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
        if dress:
            dress(c)
        c.set_solver(stop_rule, tol, max_iter, dot)
        c.set_state(x=st["x"], v=st["v"], dv=st["dv"])
        c.set_contacts(live, np.zeros(live.size, np.uint32), ca["impulses"][live])
        c.set_proxies(fat[:, :3], fat[:, 3:])
        c.step(dt)
        cs = c.state()
        out.append({"x": cs["x"], "v": cs["v"]})
    return out


def device_system(sysd, device="cuda:0"):
    """Copy an exported block-CSR system to device tensors (uint32 as int32 bits)."""
    import torch

    def t(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a).view(dt)).to(device)

    return {"n": int(sysd["rowptr"].size - 1), "rowptr": t(sysd["rowptr"], np.int32), "cols": t(sysd["cols"], np.int32),
            "vals": t(sysd["vals"], np.float32), "b": t(sysd["b"], np.float32), "S": t(sysd["S"], np.float32),
            "x0": t(sysd["x0"], np.float32)}


def call_mpcg(b3g, entry, dsys, opts, x=None):
    """Call a standalone MPCG entry point of libb3g.so on device tensors;
    returns (status, x as numpy (n, 3), iterations, stats)."""
    import ctypes as C

    import torch

    n = dsys["n"]
    if x is None:
        x = torch.zeros(3 * n, dtype=torch.float32, device=dsys["b"].device)
    it = C.c_uint32(0)
    st = b3g.StepStatsC()
    o = opts.as_c()
    fn = getattr(b3g.lib(), entry)
    torch.cuda.synchronize()
    status = fn(n, dsys["rowptr"].data_ptr(), dsys["cols"].data_ptr(), dsys["vals"].data_ptr(), dsys["b"].data_ptr(),
                dsys["S"].data_ptr(), dsys["x0"].data_ptr(), C.byref(o), x.data_ptr(), C.byref(it), C.byref(st), None)
    torch.cuda.synchronize()
    return status, x.cpu().numpy().reshape(-1, 3), it.value, st
