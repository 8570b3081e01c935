"""Generate the golden fixtures from the reference library itself.

Runs the reference (oracle/_ref/libbounce_ref.so, compiled from the Bounce
sources by oracle/Makefile; needs the reference tree on disk) on seeded
synthetic cloths and stores its outputs as compressed .npz files next to this
script.  The parity tests check the C restatement (oracle/) and the CUDA path
against these files, so they need neither the reference tree nor this script.

    python tests/golden/gen_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from bounce_b200.meshes import (capsule_scene, pinned_block_scene, plain_scene, self_collision_scene,  # noqa: E402
                                sphere_scene)


def trajectory(scene, steps, keep):
    ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=False).setup(scene)
    out = {"vertices": scene.mesh.vertices, "triangles": scene.mesh.triangles, "def": scene.cdef.as_array(),
           "pinned": np.asarray(scene.pinned, np.uint32), "dt": np.float32(scene.dt)}
    if scene.spheres:
        c, r, mu = scene.spheres[0]
        out["sphere"] = np.array([c[0], c[1], c[2], r, mu], np.float32)
    iters = []
    for k in range(1, steps + 1):
        iters.append(ref.step(scene.dt, scene.velocity_iterations, scene.position_iterations)["iterations"])
        if k in keep:
            s = ref.state()
            out[f"x_{k}"] = s["x"]
            out[f"v_{k}"] = s["v"]
            out[f"dv_{k}"] = s["dv"]
            if scene.spheres:
                cts = ref.contacts()
                out[f"contact_exists_{k}"] = cts["exists"]
                out[f"contact_active_{k}"] = cts["active"]
                out[f"contact_impulses_{k}"] = cts["impulses"]
    out["iterations"] = np.asarray(iters, np.uint32)
    out["mass"] = ref.state()["mass"]
    return out


def self_collision(scene, steps, keep):
    """The reference's full b3Cloth::Step (self-collision included) on the
    self-collision scene: states and the particle-triangle contact list (list
    order; weights only where active) at the kept steps."""
    ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=False).setup(scene)
    a, b, r, mu = scene.capsules[0]
    out = {"vertices": scene.mesh.vertices, "triangles": scene.mesh.triangles, "def": scene.cdef.as_array(),
           "capsule": np.array([*a, *b, r, mu], np.float32), "dt": np.float32(scene.dt)}
    iters = []
    for k in range(1, steps + 1):
        iters.append(ref.step(scene.dt, scene.velocity_iterations, scene.position_iterations, full=True)["iterations"])
        if k in keep:
            s = ref.state()
            out[f"x_{k}"], out[f"v_{k}"], out[f"dv_{k}"] = s["x"], s["v"], s["dv"]
            c = ref.tri_contacts()
            w = c["w"].copy()
            w[c["active"] == 0] = 0.0
            out[f"tc_pt_{k}"], out[f"tc_active_{k}"] = c["pt"], c["active"]
            out[f"tc_w_{k}"], out[f"tc_impulses_{k}"] = w, c["impulses"]
    out["iterations"] = np.asarray(iters, np.uint32)
    return out


def hull_points():
    """A slab-like hull's point cloud: two 12-gons of radius 0.35 m at heights
    -0.35 and -0.45 m (the reference's quickhull merges it into a box)."""
    ang = np.linspace(0.0, 2.0 * np.pi, 13)[:-1]
    pts = [(0.35 * np.cos(a), y, 0.35 * np.sin(a)) for y in (-0.35, -0.45) for a in ang]
    return np.asarray(pts, np.float32)


def hull_trajectory(side, steps, keep):
    """A cloth falling onto a static hull that the reference's quickhull
    builds: the hull's vertices and planes, states and body contacts at the
    kept steps."""
    scene = capsule_scene(side)
    scene.capsules = []
    ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=False).setup(scene)
    hv, hp = ref.add_hull_from_points(hull_points(), 0.3)
    out = {"vertices": scene.mesh.vertices, "triangles": scene.mesh.triangles, "def": scene.cdef.as_array(),
           "hull_vertices": hv, "hull_planes": hp, "hull_friction": np.float32(0.3), "dt": np.float32(scene.dt)}
    iters = []
    for k in range(1, steps + 1):
        iters.append(ref.step(scene.dt, scene.velocity_iterations, scene.position_iterations)["iterations"])
        if k in keep:
            s = ref.state()
            out[f"x_{k}"], out[f"v_{k}"], out[f"dv_{k}"] = s["x"], s["v"], s["dv"]
            c = ref.contacts()
            out[f"contact_exists_{k}"], out[f"contact_active_{k}"] = c["exists"], c["active"]
            out[f"contact_impulses_{k}"] = c["impulses"]
    out["iterations"] = np.asarray(iters, np.uint32)
    return out


def softbody_ground_points():
    """A ground slab's corners: 6 m x 0.5 m x 6 m, top at y = -1.5 m."""
    return np.array([(x, y, z) for x in (-3.0, 3.0) for y in (-2.0, -1.5) for z in (-3.0, 3.0)], np.float32)


def softbody_hull(steps, keep):
    """A 4 x 3 x 3 block (0.5 m cells, nothing pinned) falling onto a static
    ground hull built by the reference's quickhull; every node with radius
    0.05 and friction 0.2 (as examples/testbed/tests/smash_softbody.h sets
    them).  States and node contacts at the kept steps."""
    scene = pinned_block_scene(4, 3, 3, 0.5)
    sd = scene.sdef
    args = (scene.vertices, scene.tets, sd.density, sd.E, sd.nu, sd.c_yield, sd.c_creep, sd.c_max)
    scene.static_nodes = np.zeros(0, np.uint32)
    ref = oracle.RefSoftBody(*args).setup(scene)
    hv, hp = ref.add_hull_from_points(softbody_ground_points(), 0.6)
    for i in range(len(scene.vertices)):
        ref.set_node_radius(i, 0.05)
        ref.set_node_friction(i, 0.2)
    out = {"vertices": scene.vertices, "tets": scene.tets,
           "def": np.array([sd.density, sd.E, sd.nu, sd.c_yield, sd.c_creep, sd.c_max], np.float32),
           "mass_damping": scene.mass_damping, "dt": np.float32(scene.dt),
           "gravity": np.asarray(scene.gravity, np.float32), "hull_vertices": hv, "hull_planes": hp,
           "hull_friction": np.float32(0.6), "node_radius": np.float32(0.05), "node_friction": np.float32(0.2)}
    iters = []
    for k in range(1, steps + 1):
        iters.append(ref.step(scene.dt)["iterations"])
        if k in keep:
            st, c = ref.state(), ref.contacts()
            out[f"x_{k}"], out[f"v_{k}"] = st["x"], st["v"]
            out[f"contact_exists_{k}"], out[f"contact_active_{k}"] = c["exists"], c["active"]
            out[f"contact_impulses_{k}"] = c["impulses"]
    out["iterations"] = np.asarray(iters, np.uint32)
    return out


def system(scene):
    ref = oracle.RefCloth(scene.mesh, scene.cdef, restated=False).setup(scene)
    ref.step(scene.dt, scene.velocity_iterations, scene.position_iterations)
    sys_ = ref.system(scene.dt)
    out = {"vertices": scene.mesh.vertices, "triangles": scene.mesh.triangles, "def": scene.cdef.as_array(),
           "pinned": np.asarray(scene.pinned, np.uint32), "dt": np.float32(scene.dt)}
    st = ref.state()
    out.update({"x_1": st["x"], "v_1": st["v"], "dv_1": st["dv"]})
    out.update({f"sys_{k}": v for k, v in sys_.items()})
    return out


def softbody(w, h, d, spacing, steps, keep):
    """The pinned block with node 3 kinematic (moving at 0.1 m/s along x) and
    a force pulse on node 10 every 7 steps: states, element rotations and
    plastic strains at the kept steps, and the element data."""
    scene = pinned_block_scene(w, h, d, spacing)
    sd = scene.sdef
    args = (scene.vertices, scene.tets, sd.density, sd.E, sd.nu, sd.c_yield, sd.c_creep, sd.c_max)
    ref = oracle.RefSoftBody(*args).setup(scene)
    kin, kin_v, fnode, fvec, fper = 3, np.array([0.1, 0.0, 0.0], np.float32), 10, np.array([0.0, 50.0, 3.0], np.float32), 7
    ref.set_type(kin, 1)
    ref.set_velocity(kin, kin_v)
    out = {"vertices": scene.vertices, "tets": scene.tets,
           "def": np.array([sd.density, sd.E, sd.nu, sd.c_yield, sd.c_creep, sd.c_max], np.float32),
           "mass_damping": scene.mass_damping, "static": scene.static_nodes, "dt": np.float32(scene.dt),
           "gravity": np.asarray(scene.gravity, np.float32), "kinematic": np.uint32(kin), "kinematic_v": kin_v,
           "force_node": np.uint32(fnode), "force": fvec, "force_period": np.uint32(fper),
           "mass": ref.masses()}
    for e in range(0, ref.t, max(1, ref.t // 8)):
        ed = ref.element_data(e)
        for k, v in ed.items():
            out[f"el{e}_{k}"] = v
    iters = []
    for k in range(1, steps + 1):
        if (k - 1) % fper == 0:
            ref.apply_force(fnode, fvec)
        iters.append(ref.step(scene.dt)["iterations"])
        if k in keep:
            st, el = ref.state(), ref.elements()
            out[f"x_{k}"], out[f"v_{k}"] = st["x"], st["v"]
            out[f"q_{k}"], out[f"eps_{k}"] = el["q"], el["eps"]
    out["iterations"] = np.asarray(iters, np.uint32)
    return out


def main():
    oracle.build(port=True, ref=True)
    files = {
        "softbody_block_ref.npz": softbody(5, 3, 4, 0.5, 120, {1, 40, 80, 120}),
        "plain32_ref.npz": trajectory(plain_scene(32, seed=1), 30, {1, 10, 30}),
        "sphere32_ref.npz": trajectory(sphere_scene(32, seed=2), 40, {1, 20, 30, 40}),
        "system16_bend_ref.npz": system(sphere_scene(16, seed=4)),
        "self_collision11_ref.npz": self_collision(self_collision_scene(11), 130, {1, 60, 90, 100, 115, 130}),
        "hull16_ref.npz": hull_trajectory(16, 120, {1, 30, 60, 120}),
        "softbody_hull_ref.npz": softbody_hull(150, {1, 25, 75, 150}),
    }
    only = set(sys.argv[1:])
    for name, data in files.items():
        if only and name not in only:
            continue
        np.savez_compressed(os.path.join(HERE, name), **data)
        print(name, os.path.getsize(os.path.join(HERE, name)), "bytes")


if __name__ == "__main__":
    main()
