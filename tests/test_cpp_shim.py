"""The C++ shim (include/b3g_cloth.hpp) compiles against the C ABI and links
with libb3g.so.  Without a GPU it reports B3G_ERR_NO_DEVICE through
b3gError; on a GPU it steps a cloth through a mouse drag and onto a
kinematic sphere body, and its final positions equal those of the same
sequence run through the Python front-end (the same library calls, so bit
for bit)."""
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
        // a kinematic sphere body rising under the triangle (SetWorld with a b3Body)
        b3g_body_state b = {};
        b.type = 1;
        b.rotation[0] = b.rotation[4] = b.rotation[8] = 1.0f;
        b.position[0] = b.world_center0[0] = b.world_center[0] = 0.3f;
        b.position[1] = b.world_center0[1] = b.world_center[1] = -0.3f;
        b.position[2] = b.world_center0[2] = b.world_center[2] = 0.3f;
        b.orientation0[3] = b.orientation[3] = 1.0f;
        b.linear_velocity[1] = 1.0f;
        uint32_t body = c.AddBody(b);
        float zero[3] = {0.0f, 0.0f, 0.0f};
        uint32_t shape = c.AddBodySphere(body, zero, 0.25f, 0.3f);
        float lo[3], hi[3];
        c.GetShapeProxy(shape, lo, hi);
        c.SetShapeProxy(shape, lo, hi);
        s = c.Step(1.0f / 60.0f, 8, 2);
        b3g_body_state after = c.GetBody(body);
        std::printf("stepped %u body %.9g\n", s.iterations, after.position[1]);
        for (uint32_t i = 0; i < 3; ++i) {
            float p[3];
            c.GetParticle(i).GetPosition(p);
            std::printf("%.9g %.9g %.9g\n", p[0], p[1], p[2]);
        }
        return 0;
    } catch (const b3gError& e) {
        std::printf("status %d\n", (int)e.status);
        return e.status == B3G_ERR_NO_DEVICE ? 3 : 1;
    }
}
'''


def _run_shim(b3g, tmp_path):
    src = tmp_path / "shim.cpp"
    src.write_text(PROG)
    exe = tmp_path / "shim"
    libdir = os.path.dirname(b3g.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lb3g", f"-Wl,-rpath,{libdir}"], check=True)
    return subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)


def test_shim_compiles_and_reports_no_device(b3g, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present: test_shim_steps_a_cloth_on_the_gpu runs the shim")
    r = _run_shim(b3g, tmp_path)
    assert r.returncode == 3, r.stdout + r.stderr


@pytest.mark.gpu
def test_shim_steps_a_cloth_on_the_gpu(b3g, tmp_path):
    import numpy as np

    r = _run_shim(b3g, tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0].startswith("stepped")
    shim_x = np.array([[float(t) for t in ln.split()] for ln in lines[1:4]], np.float32)
    # the same sequence through the Python front-end
    mesh = b3g.Mesh(np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1]], np.float32), np.array([[2, 1, 0]], np.uint32))
    cloth = b3g.Cloth(mesh, b3g.ClothDef(1.0, 1e4, 1e3, 0.0, 0.0, 0.05, 0.0, 0.3))
    cloth.set_gravity((0.0, -9.8, 0.0))
    cloth.particle(0).set_type(b3g.STATIC)
    cloth.step(1.0 / 60.0, 8, 2)
    mp = cloth.create_particle((0.3, 0.1, 0.3))
    f = cloth.create_mouse_force(mp, 0, 0.3, 0.3, 0.4, 1000.0, 5.0)
    cloth.step(1.0 / 60.0, 8, 2)
    cloth.destroy_force(f)
    cloth.destroy_particle(mp)
    cloth.step(1.0 / 60.0, 8, 2)
    body = np.zeros(55, np.float32)
    body[0] = 1.0
    body[[1, 5, 9]] = 1.0
    for k in (10, 16, 19):
        body[k:k + 3] = (0.3, -0.3, 0.3)
    body[25] = body[29] = 1.0
    body[31] = 1.0
    bid = cloth.add_body(body)
    cloth.add_body_sphere(bid, (0.0, 0.0, 0.0), 0.25, 0.3)
    cloth.step(1.0 / 60.0, 8, 2)
    assert np.float32(lines[0].split()[-1]) == cloth.body(bid)[11]  # %.9g round-trips a float
    x = cloth.positions()
    cloth.close()
    assert np.array_equal(shim_x, x), (shim_x, x)
    assert not np.array_equal(x[1], mesh.vertices[1])  # it moved
