"""The C++ shim (include/b3g_cloth.hpp) compiles against the C ABI and links
with libb3g.so; without a GPU it reports B3G_ERR_NO_DEVICE through b3gError."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = r'''
#include <cstdio>
#include "b3g_cloth.hpp"
int main() {
    float v[9] = {0,0,0, 1,0,0, 0,0,1};
    uint32_t t[3] = {2, 1, 0};
    b3g_mesh_desc m = {3, v, 1, t, 0, nullptr};
    b3g_cloth_def d = {1.0f, 1e4f, 1e3f, 0.0f, 0.0f, 0.05f, 0.0f, 0.3f};
    try {
        b3gCloth c(m, d);
        float g[3] = {0.0f, -9.8f, 0.0f};
        c.SetGravity(g);
        c.GetParticle(0).SetType(B3G_STATIC);
        b3g_step_stats s = c.Step(1.0f / 60.0f, 8, 2);
        // a mouse drag as the testbed's cloth dragger does it
        b3g_particle_def pd = {};
        pd.position[0] = 0.3f; pd.position[1] = 0.1f; pd.position[2] = 0.3f;
        b3gParticle mp = c.CreateParticle(pd);
        b3g_mouse_force_def md = {mp.GetVertex(), 0u, 0.3f, 0.3f, 0.4f, 1000.0f, 5.0f};
        uint32_t f = c.CreateMouseForce(md);
        s = c.Step(1.0f / 60.0f, 8, 2);
        c.DestroyForce(f);
        c.DestroyParticle(mp);
        s = c.Step(1.0f / 60.0f, 8, 2);
        std::printf("stepped %u\n", s.iterations);
        return 0;
    } catch (const b3gError& e) {
        std::printf("status %d\n", (int)e.status);
        return e.status == B3G_ERR_NO_DEVICE ? 3 : 1;
    }
}
'''


def test_shim_compiles_and_runs(b3g, tmp_path):
    src = tmp_path / "shim.cpp"
    src.write_text(PROG)
    exe = tmp_path / "shim"
    libdir = os.path.dirname(b3g.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lb3g", f"-Wl,-rpath,{libdir}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    import torch

    if torch.cuda.is_available():
        assert r.returncode == 0, r.stdout + r.stderr
    else:
        assert r.returncode == 3, r.stdout + r.stderr
