"""B200-native implicit cloth step with Bounce's ``b3Cloth`` semantics.

The compute path is libb3g.so (hand-written CUDA for sm_100a behind the C ABI
in include/b3g.h).  This module is a thin ctypes front-end with the shape of
the reference's C++ classes:

* ``Cloth``       ~ ``b3Cloth``  (include/bounce/cloth/cloth.h:99-158)
* ``Particle``    ~ ``b3Particle`` (include/bounce/cloth/particle.h:63-111)
* ``SolverOptions``  the CG stop rule / iteration cap / dot precision

There is no CPU fallback: if libb3g.so is missing the import of the native
library raises, and without a CUDA device ``Cloth(...)`` raises B3gError.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from .meshes import (DYNAMIC, KINEMATIC, STATIC, ClothDef, Mesh, Scene, batch_scenes, capsule_scene, grid_mesh,  # noqa: F401
                     plain_scene, self_collision_scene, sewn_scene, sphere_scene, stiff_scene, SoftBodyDef,
                     SoftBodyScene,
                     block_softbody_mesh, pinned_block_scene)

HERE = os.path.dirname(os.path.abspath(__file__))
# B3G_LIBRARY: another build of libb3g.so to load instead of the in-tree one
LIB_PATH = os.environ.get("B3G_LIBRARY") or os.path.join(HERE, "_lib", "libb3g.so")

STOP_REFERENCE, STOP_RELATIVE = 0, 1
CG_LAUNCHES, CG_PERSISTENT = 0, 1
DOT_F32, DOT_COMPENSATED, DOT_F64 = 0, 1, 2

STATUS = {0: "ok", 1: "invalid argument", 2: "degenerate mesh", 3: "no CUDA device", 4: "out of memory",
          5: "CUDA error", 6: "numerical breakdown in CG", 7: "device wait timed out", 8: "capacity exceeded",
          9: "unsupported mesh"}


class B3gError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")
        self.status = status


class MeshDesc(C.Structure):
    _fields_ = [("vertex_count", C.c_uint32), ("vertices", C.c_void_p), ("triangle_count", C.c_uint32),
                ("triangles", C.c_void_p), ("sewing_line_count", C.c_uint32), ("sewing_lines", C.c_void_p)]


class ClothDefC(C.Structure):
    _fields_ = [(k, C.c_float) for k in ("density", "streching", "shearing", "bending", "sewing", "damping",
                                          "thickness", "friction")]


class SolverOptsC(C.Structure):
    _fields_ = [("stop_rule", C.c_int), ("tolerance", C.c_float), ("max_iterations", C.c_uint32), ("dot", C.c_int)]


class SoftBodyDefC(C.Structure):
    _fields_ = [("density", C.c_float), ("E", C.c_float), ("nu", C.c_float), ("c_yield", C.c_float),
                ("c_creep", C.c_float), ("c_max", C.c_float)]


class StepStatsC(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("delta0", C.c_double), ("delta", C.c_double), ("b_delta", C.c_double),
                ("active_contacts", C.c_uint32), ("contacts", C.c_uint32), ("step_ms", C.c_float)]


class PhaseTimesC(C.Structure):
    _fields_ = [(k, C.c_float) for k in ("contacts_update_ms", "assemble_ms", "cg_init_ms", "cg_spmv_ms",
                                          "cg_update_ms", "cg_direction_ms", "finalize_ms",
                                          "contact_position_ms", "post_ms")] + \
               [("cg_iterations", C.c_uint32), ("contact_position_launches", C.c_uint32)]


class ParticleDefC(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("velocity", C.c_float * 3), ("force", C.c_float * 3),
                ("mass", C.c_float), ("radius", C.c_float), ("friction", C.c_float)]


class MouseForceDefC(C.Structure):
    _fields_ = [("particle", C.c_uint32), ("triangle", C.c_uint32), ("w2", C.c_float), ("w3", C.c_float),
                ("w4", C.c_float), ("mouse", C.c_float), ("damping", C.c_float)]


class BodyStateC(C.Structure):
    """b3g_body_state: a rigid body's transform, sweep, velocities and mass
    (b3Body, include/bounce/dynamics/body.h)."""
    _fields_ = [("type", C.c_int32), ("rotation", C.c_float * 9), ("position", C.c_float * 3),
                ("local_center", C.c_float * 3), ("world_center0", C.c_float * 3), ("world_center", C.c_float * 3),
                ("orientation0", C.c_float * 4), ("orientation", C.c_float * 4), ("linear_velocity", C.c_float * 3),
                ("angular_velocity", C.c_float * 3), ("inv_mass", C.c_float), ("inv_inertia", C.c_float * 9),
                ("world_inv_inertia", C.c_float * 9)]


def body_state_from_array(a) -> BodyStateC:
    """A body state from its 55 floats: type, rotation (9, column-major),
    position, local centre, world centre 0 and 1, orientation 0 and 1 (x y z
    w), linear and angular velocity, inverse mass, inverse inertia (9) and
    world inverse inertia (9)."""
    a = np.asarray(a, np.float32).reshape(-1)
    if a.size != 55:
        raise ValueError("a body state has 55 floats")
    b = BodyStateC()
    b.type = int(a[0])
    k = 1
    for name, t in BodyStateC._fields_[1:]:
        m = getattr(t, "_length_", 1)
        if m == 1:
            setattr(b, name, float(a[k]))
        else:
            getattr(b, name)[:] = [float(u) for u in a[k:k + m]]
        k += m
    return b


def body_state_to_array(b: BodyStateC) -> np.ndarray:
    out = [float(b.type)]
    for name, t in BodyStateC._fields_[1:]:
        v = getattr(b, name)
        out.extend([v] if getattr(t, "_length_", 1) == 1 else list(v))
    return np.asarray(out, np.float32)


class ClothInfoC(C.Structure):
    _fields_ = [(k, C.c_uint32) for k in ("vertices", "triangles", "springs", "blocks", "sell_entries",
                                           "max_degree")]


class BatchScheduleC(C.Structure):
    _fields_ = [("cluster", C.c_uint32), ("split_class", C.c_uint8 * 32), ("tuned_cg_ms", C.c_float)]


class BatchStatsC(C.Structure):
    _fields_ = [("count", C.c_uint32), ("rows", C.c_uint32), ("tasks", C.c_uint32),
                ("cg_iterations_total", C.c_uint32), ("cg_iterations_max", C.c_uint32), ("step_ms", C.c_float),
                ("cg_ms", C.c_float)]


class ServerConfigC(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_active", C.c_uint32), ("dt", C.c_float),
                ("velocity_iterations", C.c_uint32), ("position_iterations", C.c_uint32),
                ("gravity", C.c_float * 3), ("solver", SolverOptsC), ("schedule", BatchScheduleC),
                ("host_threads", C.c_uint32)]


class ServerTickC(C.Structure):
    _fields_ = [(k, C.c_uint32) for k in ("admitted", "stepped", "completed", "active", "queued", "rows")] + \
               [("bytes_used", C.c_uint64), ("tick_ms", C.c_float)]


class RequestInfoC(C.Structure):
    _fields_ = [("state", C.c_uint32), ("status", C.c_int), ("steps_done", C.c_uint32), ("steps_total", C.c_uint32),
                ("vertex_count", C.c_uint32), ("arrival", C.c_double), ("admitted", C.c_double),
                ("finished", C.c_double), ("bytes", C.c_uint64)]


class ServerStatsC(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("ticks", "steps", "vertex_steps", "admitted", "completed", "rejected")] + \
               [("busy_ms", C.c_double), ("active", C.c_uint32), ("queued", C.c_uint32), ("peak_active", C.c_uint32),
                ("peak_bytes", C.c_uint64), ("p50_step_ms", C.c_float), ("p99_step_ms", C.c_float),
                ("max_step_ms", C.c_float)]


_lib = None


def lib() -> C.CDLL:
    """Load libb3g.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m bounce_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, u32, f32, i32 = C.c_void_p, C.c_uint32, C.c_float, C.c_int
        sig = {
            "b3g_cloth_create": [C.POINTER(MeshDesc), C.POINTER(ClothDefC), i32, C.POINTER(vp)],
            "b3g_cloth_destroy": [vp],
            "b3g_cloth_set_gravity": [vp, vp],
            "b3g_cloth_get_gravity": [vp, vp],
            "b3g_cloth_set_solver": [vp, C.POINTER(SolverOptsC)],
            "b3g_cloth_add_static_sphere": [vp, vp, f32, f32, C.POINTER(u32)],
            "b3g_cloth_clear_colliders": [vp],
            "b3g_cloth_add_static_capsule": [vp, vp, vp, f32, f32, C.POINTER(u32)],
            "b3g_cloth_add_static_hull": [vp, vp, u32, vp, u32, f32, C.POINTER(u32)],
            "b3g_cloth_create_particle": [vp, C.POINTER(ParticleDefC), C.POINTER(u32)],
            "b3g_cloth_destroy_particle": [vp, u32],
            "b3g_cloth_create_mouse_force": [vp, C.POINTER(MouseForceDefC), C.POINTER(u32)],
            "b3g_cloth_destroy_force": [vp, u32],
            "b3g_particle_set_type": [vp, u32, i32],
            "b3g_particle_get_type": [vp, u32, C.POINTER(i32)],
            "b3g_particle_set_position": [vp, u32, vp],
            "b3g_particle_get_position": [vp, u32, vp],
            "b3g_particle_set_velocity": [vp, u32, vp],
            "b3g_particle_get_velocity": [vp, u32, vp],
            "b3g_particle_get_mass": [vp, u32, C.POINTER(f32)],
            "b3g_particle_apply_force": [vp, u32, vp],
            "b3g_particle_apply_translation": [vp, u32, vp],
            "b3g_particle_set_radius": [vp, u32, f32],
            "b3g_particle_get_radius": [vp, u32, C.POINTER(f32)],
            "b3g_particle_set_friction": [vp, u32, f32],
            "b3g_particle_get_friction": [vp, u32, C.POINTER(f32)],
            "b3g_cloth_set_types": [vp, vp],
            "b3g_cloth_apply_forces": [vp, vp],
            "b3g_cloth_apply_translations": [vp, vp],
            "b3g_cloth_step": [vp, f32, u32, u32, C.POINTER(StepStatsC)],
            "b3g_cloth_assemble": [vp, f32],
            "b3g_cloth_read_state": [vp, vp, vp, vp],
            "b3g_cloth_write_state": [vp, vp, vp, vp],
            "b3g_cloth_read_masses": [vp, vp],
            "b3g_cloth_get_energy": [vp, C.POINTER(f32)],
            "b3g_cloth_read_contacts": [vp, vp, vp, vp],
            "b3g_cloth_read_proxies": [vp, vp, vp],
            "b3g_cloth_read_tri_contacts": [vp, C.POINTER(u32), vp, vp, vp, vp],
            "b3g_cloth_ray_cast_single": [vp, vp, vp, C.POINTER(u32), C.POINTER(f32), vp, C.POINTER(i32)],
            "b3g_cloth_ray_cast": [vp, vp, vp, f32, u32, C.POINTER(f32), vp, C.POINTER(i32)],
            "b3g_cloth_get_self_stats": [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)],
            "b3g_cloth_last_stats": [vp, C.POINTER(StepStatsC)],
            "b3g_cloth_add_body": [vp, C.POINTER(BodyStateC), C.POINTER(u32)],
            "b3g_cloth_set_body": [vp, u32, C.POINTER(BodyStateC)],
            "b3g_cloth_get_body": [vp, u32, C.POINTER(BodyStateC)],
            "b3g_cloth_add_body_sphere": [vp, u32, vp, f32, f32, C.POINTER(u32)],
            "b3g_cloth_add_body_capsule": [vp, u32, vp, vp, f32, f32, C.POINTER(u32)],
            "b3g_cloth_add_body_hull": [vp, u32, vp, u32, vp, u32, f32, C.POINTER(u32)],
            "b3g_cloth_set_shape_proxy": [vp, u32, vp, vp],
            "b3g_cloth_get_shape_proxy": [vp, u32, vp, vp],
            "b3g_cloth_set_report_order": [vp, vp, u32],
            "b3g_cloth_read_system": [vp, C.POINTER(u32), vp, vp, vp, vp, vp, vp],
            "b3g_cloth_step_profiled": [vp, f32, u32, u32, C.POINTER(PhaseTimesC), C.POINTER(StepStatsC)],
            "b3g_cloth_get_info": [vp, C.POINTER(ClothInfoC)],
            "b3g_cloth_set_cg_strategy": [vp, i32],
            "b3g_cloth_set_assembly": [vp, i32],
            "b3g_cloth_get_assembly": [vp],
            "b3g_debug_cg_barrier_timeout": [vp, u32, C.POINTER(i32)],
            "b3g_mpcg_solve": [u32, vp, vp, vp, vp, vp, vp, C.POINTER(SolverOptsC), vp, C.POINTER(u32),
                               C.POINTER(StepStatsC), vp],
            "b3g_batch_create": [i32, u32, C.POINTER(vp)],
            "b3g_batch_destroy": [vp],
            "b3g_batch_step": [vp, vp, u32, f32, u32, u32, vp, C.POINTER(BatchStatsC)],
            "b3g_batch_set_schedule": [vp, C.POINTER(BatchScheduleC)],
            "b3g_batch_get_schedule": [vp, C.POINTER(BatchScheduleC)],
            "b3g_batch_autotune": [vp, vp, u32, f32, C.POINTER(BatchScheduleC)],
            "b3g_server_create": [i32, C.POINTER(ServerConfigC), C.POINTER(vp)],
            "b3g_server_destroy": [vp],
            "b3g_server_submit": [vp, C.POINTER(MeshDesc), C.POINTER(ClothDefC), vp, vp, u32, u32, C.c_double,
                                  C.POINTER(C.c_uint64)],
            "b3g_server_tick": [vp, C.c_double, C.POINTER(ServerTickC)],
            "b3g_server_poll": [vp, C.c_uint64, C.POINTER(RequestInfoC)],
            "b3g_server_result": [vp, C.c_uint64, vp],
            "b3g_server_release": [vp, C.c_uint64],
            "b3g_server_stats": [vp, C.POINTER(ServerStatsC)],
            "b3g_mpcg_solve_noalloc": [u32, vp, vp, vp, vp, vp, vp, C.POINTER(SolverOptsC), vp, C.POINTER(u32),
                                       C.POINTER(StepStatsC), vp],
            "b3g_softbody_create": [u32, vp, u32, vp, C.POINTER(SoftBodyDefC), i32, C.POINTER(vp)],
            "b3g_softbody_destroy": [vp],
            "b3g_softbody_set_gravity": [vp, vp],
            "b3g_softbody_set_node_type": [vp, u32, i32],
            "b3g_softbody_set_mass_damping": [vp, u32, f32],
            "b3g_softbody_apply_force": [vp, u32, vp],
            "b3g_softbody_set_velocity": [vp, u32, vp],
            "b3g_softbody_set_position": [vp, u32, vp],
            "b3g_softbody_set_solver": [vp, C.POINTER(SolverOptsC)],
            "b3g_softbody_set_cg_strategy": [vp, i32],
            "b3g_softbody_step": [vp, f32, u32, u32, C.POINTER(StepStatsC)],
            "b3g_softbody_read_state": [vp, vp, vp],
            "b3g_softbody_write_state": [vp, vp, vp],
            "b3g_softbody_read_elements": [vp, vp, vp],
            "b3g_softbody_write_elements": [vp, vp, vp],
            "b3g_softbody_read_masses": [vp, vp],
            "b3g_softbody_energy": [vp, C.POINTER(f32)],
            "b3g_softbody_export_system": [vp, f32, u32, vp, vp, vp, vp, vp, C.POINTER(u32)],
            "b3g_softbody_add_static_hull": [vp, vp, u32, vp, u32, f32, C.POINTER(u32)],
            "b3g_softbody_set_node_radius": [vp, u32, f32],
            "b3g_softbody_set_node_friction": [vp, u32, f32],
            "b3g_softbody_read_contacts": [vp, vp, vp, vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.b3g_cloth_vertex_count.argtypes = [vp]
        L.b3g_cloth_vertex_count.restype = u32
        for name in ("b3g_softbody_node_count", "b3g_softbody_element_count"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = u32
        L.b3g_status_string.argtypes = [C.c_int]
        L.b3g_status_string.restype = C.c_char_p
        L.b3g_kernel_launch_count.argtypes = []
        L.b3g_kernel_launch_count.restype = C.c_uint64
        _lib = L
    return _lib


def check(status: int, what: str) -> None:
    if status != 0:
        raise B3gError(status, what)


def _ptr(a: np.ndarray) -> int:
    """The address of `a`'s data.  The caller keeps `a` alive across the call
    that uses the address: a temporary array may be freed (and its memory
    reused) before the call runs."""
    return a.ctypes.data


def _f3(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(3))


@dataclass
class SolverOptions:
    stop_rule: int = STOP_REFERENCE
    tolerance: float = 0.0
    max_iterations: int = 20
    dot: int = DOT_F32

    @staticmethod
    def reference() -> "SolverOptions":
        """b3SolveMPCG's own rule: 20 iterations, delta <= FLT_EPSILON^2 b_delta."""
        return SolverOptions(STOP_REFERENCE, 0.0, 20, DOT_F32)

    @staticmethod
    def relative(tol: float = 1e-4, max_iterations: int = 50, dot: int = DOT_F64) -> "SolverOptions":
        return SolverOptions(STOP_RELATIVE, tol, max_iterations, dot)

    def as_c(self) -> SolverOptsC:
        return SolverOptsC(self.stop_rule, self.tolerance, self.max_iterations, self.dot)


class Particle:
    """One particle of a Cloth (b3Particle)."""

    def __init__(self, cloth: "Cloth", vertex: int):
        self.cloth = cloth
        self.vertex = vertex

    def set_type(self, t: int) -> None:
        check(lib().b3g_particle_set_type(self.cloth.h, self.vertex, t), "set_type")

    def get_type(self) -> int:
        out = C.c_int(0)
        check(lib().b3g_particle_get_type(self.cloth.h, self.vertex, C.byref(out)), "get_type")
        return out.value

    def set_position(self, x) -> None:
        x3 = _f3(x)
        check(lib().b3g_particle_set_position(self.cloth.h, self.vertex, _ptr(x3)), "set_position")

    def get_position(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        check(lib().b3g_particle_get_position(self.cloth.h, self.vertex, _ptr(out)), "get_position")
        return out

    def set_velocity(self, v) -> None:
        v3 = _f3(v)
        check(lib().b3g_particle_set_velocity(self.cloth.h, self.vertex, _ptr(v3)), "set_velocity")

    def get_velocity(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        check(lib().b3g_particle_get_velocity(self.cloth.h, self.vertex, _ptr(out)), "get_velocity")
        return out

    def get_mass(self) -> float:
        out = C.c_float(0)
        check(lib().b3g_particle_get_mass(self.cloth.h, self.vertex, C.byref(out)), "get_mass")
        return out.value

    def apply_force(self, f) -> None:
        f3 = _f3(f)
        check(lib().b3g_particle_apply_force(self.cloth.h, self.vertex, _ptr(f3)), "apply_force")

    def apply_translation(self, t) -> None:
        t3 = _f3(t)
        check(lib().b3g_particle_apply_translation(self.cloth.h, self.vertex, _ptr(t3)), "apply_translation")

    def set_radius(self, r: float) -> None:
        check(lib().b3g_particle_set_radius(self.cloth.h, self.vertex, r), "set_radius")

    def get_radius(self) -> float:
        out = C.c_float(0.0)
        check(lib().b3g_particle_get_radius(self.cloth.h, self.vertex, C.byref(out)), "get_radius")
        return float(out.value)

    def set_friction(self, f: float) -> None:
        check(lib().b3g_particle_set_friction(self.cloth.h, self.vertex, f), "set_friction")

    def get_friction(self) -> float:
        out = C.c_float(0.0)
        check(lib().b3g_particle_get_friction(self.cloth.h, self.vertex, C.byref(out)), "get_friction")
        return float(out.value)


class Cloth:
    """A cloth on one GPU (b3Cloth)."""

    def __init__(self, mesh: Mesh, cdef: ClothDef, device: int = 0):
        L = lib()
        self._verts = np.ascontiguousarray(mesh.vertices, np.float32)
        self._tris = np.ascontiguousarray(mesh.triangles, np.uint32)
        self._sew = np.ascontiguousarray(mesh.sewing, np.uint32)
        md = MeshDesc(mesh.vertex_count, _ptr(self._verts), mesh.triangle_count, _ptr(self._tris),
                      int(self._sew.shape[0]), _ptr(self._sew) if self._sew.size else None)
        d = ClothDefC(cdef.density, cdef.streching, cdef.shearing, cdef.bending, cdef.sewing, cdef.damping,
                      cdef.thickness, cdef.friction)
        h = C.c_void_p()
        check(L.b3g_cloth_create(C.byref(md), C.byref(d), device, C.byref(h)), "b3g_cloth_create")
        self.h = h
        self.n_mesh = mesh.vertex_count
        self.n = mesh.vertex_count      # particles: the mesh's, then created ones
        self.nsph = 0
        self.stats = StepStatsC()

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().b3g_cloth_destroy(self.h)
            self.h = None

    __del__ = close

    # created particles and mouse forces (b3Cloth::CreateParticle / CreateForce)
    def create_particle(self, position, velocity=(0.0, 0.0, 0.0), force=(0.0, 0.0, 0.0), mass: float = 0.0,
                        radius: float = 0.0, friction: float = 0.0) -> int:
        """A particle outside the mesh (mass 0: static); returns its index."""
        d = ParticleDefC((C.c_float * 3)(*_f3(position)), (C.c_float * 3)(*_f3(velocity)),
                         (C.c_float * 3)(*_f3(force)), mass, radius, friction)
        idx = C.c_uint32(0)
        check(lib().b3g_cloth_create_particle(self.h, C.byref(d), C.byref(idx)), "create_particle")
        self.n = int(lib().b3g_cloth_vertex_count(self.h))
        return int(idx.value)

    def destroy_particle(self, index: int) -> None:
        check(lib().b3g_cloth_destroy_particle(self.h, index), "destroy_particle")
        self.n = int(lib().b3g_cloth_vertex_count(self.h))

    def create_mouse_force(self, particle: int, triangle: int, w2: float, w3: float, w4: float, mouse: float,
                           damping: float) -> int:
        """Ties `particle` to the point w2 x(v1) + w3 x(v2) + w4 x(v3) of `triangle`; returns the force id."""
        d = MouseForceDefC(particle, triangle, w2, w3, w4, mouse, damping)
        fid = C.c_uint32(0)
        check(lib().b3g_cloth_create_mouse_force(self.h, C.byref(d), C.byref(fid)), "create_mouse_force")
        return int(fid.value)

    def destroy_force(self, force_id: int) -> None:
        check(lib().b3g_cloth_destroy_force(self.h, force_id), "destroy_force")

    # b3Cloth API
    def set_gravity(self, g) -> None:
        g3 = _f3(g)
        check(lib().b3g_cloth_set_gravity(self.h, _ptr(g3)), "set_gravity")

    def get_gravity(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        check(lib().b3g_cloth_get_gravity(self.h, _ptr(out)), "get_gravity")
        return out

    def set_solver(self, opts: SolverOptions) -> None:
        o = opts.as_c()
        check(lib().b3g_cloth_set_solver(self.h, C.byref(o)), "set_solver")

    def add_sphere(self, center, radius: float, friction: float) -> int:
        sid = C.c_uint32(0)
        c3 = _f3(center)
        check(lib().b3g_cloth_add_static_sphere(self.h, _ptr(c3), radius, friction, C.byref(sid)),
              "add_static_sphere")
        self.nsph += 1
        return sid.value

    def add_capsule(self, a, b, radius: float, friction: float) -> int:
        """A static capsule collider: segment a-b (world frame), `radius`."""
        sid = C.c_uint32(0)
        a3, b3 = _f3(a), _f3(b)
        check(lib().b3g_cloth_add_static_capsule(self.h, _ptr(a3), _ptr(b3), radius, friction,
                                                 C.byref(sid)), "add_static_capsule")
        self.nsph += 1
        return sid.value

    def add_hull(self, vertices, planes, friction: float) -> int:
        """A static convex hull collider: vertices (n, 3) and face planes
        (f, 4: normal, offset), world frame."""
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        p = np.ascontiguousarray(planes, np.float32).reshape(-1, 4)
        sid = C.c_uint32(0)
        check(lib().b3g_cloth_add_static_hull(self.h, _ptr(v), len(v), _ptr(p), len(p), friction, C.byref(sid)),
              "add_static_hull")
        self.nsph += 1
        return sid.value

    def clear_colliders(self) -> None:
        check(lib().b3g_cloth_clear_colliders(self.h), "clear_colliders")
        self.nsph = 0

    # ---- colliders on bodies (b3Cloth::SetWorld with b3Body) ----

    def add_body(self, state) -> int:
        """A body for body colliders; `state` is a BodyStateC or its 55
        floats (body_state_from_array)."""
        b = state if isinstance(state, BodyStateC) else body_state_from_array(state)
        bid = C.c_uint32(0)
        check(lib().b3g_cloth_add_body(self.h, C.byref(b), C.byref(bid)), "add_body")
        return bid.value

    def set_body(self, body: int, state) -> None:
        b = state if isinstance(state, BodyStateC) else body_state_from_array(state)
        check(lib().b3g_cloth_set_body(self.h, body, C.byref(b)), "set_body")

    def body(self, body: int) -> np.ndarray:
        """The body's state as 55 floats, after the cloth's contact solve and
        synchronisation changed it."""
        b = BodyStateC()
        check(lib().b3g_cloth_get_body(self.h, body, C.byref(b)), "get_body")
        return body_state_to_array(b)

    def add_body_sphere(self, body: int, center, radius: float, friction: float) -> int:
        sid = C.c_uint32(0)
        c3 = _f3(center)
        check(lib().b3g_cloth_add_body_sphere(self.h, body, _ptr(c3), radius, friction, C.byref(sid)),
              "add_body_sphere")
        self.nsph += 1
        return sid.value

    def add_body_capsule(self, body: int, a, b, radius: float, friction: float) -> int:
        sid = C.c_uint32(0)
        a3, b3 = _f3(a), _f3(b)
        check(lib().b3g_cloth_add_body_capsule(self.h, body, _ptr(a3), _ptr(b3), radius, friction, C.byref(sid)),
              "add_body_capsule")
        self.nsph += 1
        return sid.value

    def add_body_hull(self, body: int, vertices, planes, friction: float) -> int:
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        p = np.ascontiguousarray(planes, np.float32).reshape(-1, 4)
        sid = C.c_uint32(0)
        check(lib().b3g_cloth_add_body_hull(self.h, body, _ptr(v), len(v), _ptr(p), len(p), friction,
                                            C.byref(sid)), "add_body_hull")
        self.nsph += 1
        return sid.value

    def set_shape_proxy(self, shape: int, lo, hi) -> None:
        a, b = _f3(lo), _f3(hi)
        check(lib().b3g_cloth_set_shape_proxy(self.h, shape, _ptr(a), _ptr(b)), "set_shape_proxy")

    def shape_proxy(self, shape: int):
        lo, hi = np.zeros(3, np.float32), np.zeros(3, np.float32)
        check(lib().b3g_cloth_get_shape_proxy(self.h, shape, _ptr(lo), _ptr(hi)), "get_shape_proxy")
        return lo, hi

    def set_report_order(self, order) -> None:
        """The world query's report order of the colliders (empty: derived)."""
        o = np.ascontiguousarray(order, np.uint32).reshape(-1)
        check(lib().b3g_cloth_set_report_order(self.h, _ptr(o) if o.size else None, o.size), "set_report_order")

    def particle(self, i: int) -> Particle:
        return Particle(self, i)

    get_particle = particle

    def set_types(self, types) -> None:
        t = np.ascontiguousarray(types, np.uint8)
        check(lib().b3g_cloth_set_types(self.h, _ptr(t)), "set_types")

    def apply_forces(self, f) -> None:
        a = np.ascontiguousarray(f, np.float32)
        check(lib().b3g_cloth_apply_forces(self.h, _ptr(a)), "apply_forces")

    def apply_translations(self, t) -> None:
        a = np.ascontiguousarray(t, np.float32)
        check(lib().b3g_cloth_apply_translations(self.h, _ptr(a)), "apply_translations")

    def step(self, dt: float, velocity_iterations: int = 8, position_iterations: int = 2) -> dict:
        check(lib().b3g_cloth_step(self.h, dt, velocity_iterations, position_iterations, C.byref(self.stats)),
              "step")
        s = self.stats
        return {"iterations": s.iterations, "delta0": s.delta0, "delta": s.delta, "b_delta": s.b_delta,
                "active_contacts": s.active_contacts, "contacts": s.contacts, "step_ms": s.step_ms}

    def step_profiled(self, dt: float, velocity_iterations: int = 8, position_iterations: int = 2) -> dict:
        t = PhaseTimesC()
        check(lib().b3g_cloth_step_profiled(self.h, dt, velocity_iterations, position_iterations, C.byref(t),
                                            C.byref(self.stats)), "step_profiled")
        out = {k: getattr(t, k) for k, _ in PhaseTimesC._fields_}
        out["iterations"] = self.stats.iterations
        return out

    def set_cg_strategy(self, persistent, fused: bool = False) -> None:
        """False: per-iteration launches in a graph loop; True: one persistent
        cooperative launch (fused: one grid reduction per iteration)."""
        code = 0 if not persistent else 2 if fused else 1
        check(lib().b3g_cloth_set_cg_strategy(self.h, code), "set_cg_strategy")

    def set_assembly(self, form: str) -> None:
        """'records': every element evaluated once a step, each block summed
        from its own term list (the default where the layout allows it);
        'rows': each row recomputes its incident elements in two passes.
        Both give the same floats."""
        code = {"records": 0, "rows": 1}[form]
        check(lib().b3g_cloth_set_assembly(self.h, code), "set_assembly")

    def assembly(self) -> str:
        """The assembly form in use ('rows' where the layout does not allow
        the records)."""
        return "records" if lib().b3g_cloth_get_assembly(self.h) == 0 else "rows"

    def info(self) -> dict:
        i = ClothInfoC()
        check(lib().b3g_cloth_get_info(self.h, C.byref(i)), "get_info")
        return {k: getattr(i, k) for k, _ in ClothInfoC._fields_}

    def assemble(self, dt: float) -> None:
        check(lib().b3g_cloth_assemble(self.h, dt), "assemble")

    def state(self) -> dict:
        x = np.zeros((self.n, 3), np.float32)
        v = np.zeros((self.n, 3), np.float32)
        dv = np.zeros((self.n, 3), np.float32)
        check(lib().b3g_cloth_read_state(self.h, _ptr(x), _ptr(v), _ptr(dv)), "read_state")
        return {"x": x, "v": v, "dv": dv}

    def positions(self, out: np.ndarray | None = None) -> np.ndarray:
        x = out if out is not None else np.zeros((self.n, 3), np.float32)
        check(lib().b3g_cloth_read_state(self.h, _ptr(x), None, None), "read_state")
        return x

    def write_state(self, x=None, v=None, dv=None) -> None:
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (x, v, dv)]
        check(lib().b3g_cloth_write_state(self.h, *[None if a is None else _ptr(a) for a in arrs]), "write_state")

    def masses(self) -> np.ndarray:
        m = np.zeros(self.n, np.float32)
        check(lib().b3g_cloth_read_masses(self.h, _ptr(m)), "read_masses")
        return m

    def energy(self) -> float:
        e = C.c_float(0)
        check(lib().b3g_cloth_get_energy(self.h, C.byref(e)), "get_energy")
        return e.value

    def contacts(self) -> dict:
        k = max(self.nsph, 1)
        ex = np.zeros(k * self.n, np.uint8)
        ac = np.zeros(k * self.n, np.uint8)
        imp = np.zeros((k * self.n, 3), np.float32)
        check(lib().b3g_cloth_read_contacts(self.h, _ptr(ex), _ptr(ac), _ptr(imp)), "read_contacts")
        return {"exists": ex[: self.nsph * self.n], "active": ac[: self.nsph * self.n],
                "impulses": imp[: self.nsph * self.n]}

    def proxies(self):
        """The particles' fat AABBs: (lo, hi), n x 3 each."""
        lo = np.zeros((self.n, 3), np.float32)
        hi = np.zeros((self.n, 3), np.float32)
        check(lib().b3g_cloth_read_proxies(self.h, _ptr(lo), _ptr(hi)), "read_proxies")
        return lo, hi

    def ray_cast_single(self, p1, p2):
        """b3Cloth::RayCastSingle: (triangle, fraction, normal) of the first
        triangle the segment p1 -> p2 hits, or None."""
        a, b = _f3(p1), _f3(p2)
        t, f, hit = C.c_uint32(0), C.c_float(0.0), C.c_int(0)
        n = np.zeros(3, np.float32)
        check(lib().b3g_cloth_ray_cast_single(self.h, _ptr(a), _ptr(b), C.byref(t), C.byref(f), _ptr(n),
                                              C.byref(hit)), "ray_cast_single")
        return (int(t.value), float(f.value), n) if hit.value else None

    def ray_cast(self, p1, p2, triangle: int, max_fraction: float = 1.0):
        """b3Cloth::RayCast against one triangle: (fraction, normal) or None."""
        a, b = _f3(p1), _f3(p2)
        f, hit = C.c_float(0.0), C.c_int(0)
        n = np.zeros(3, np.float32)
        check(lib().b3g_cloth_ray_cast(self.h, _ptr(a), _ptr(b), max_fraction, triangle, C.byref(f), _ptr(n),
                                       C.byref(hit)), "ray_cast")
        return (float(f.value), n) if hit.value else None

    def tri_contacts(self) -> dict:
        """Particle-triangle contacts (thickness > 0) in list order, head
        first: (particle, triangle) pairs, active flags, weights w2, w3, w4
        (zero while inactive), impulses (normal, tangent 1, tangent 2)."""
        cnt = C.c_uint32(0)
        L = lib()
        check(L.b3g_cloth_read_tri_contacts(self.h, C.byref(cnt), None, None, None, None), "read_tri_contacts")
        m = cnt.value
        pt = np.zeros((max(m, 1), 2), np.uint32)
        ac = np.zeros(max(m, 1), np.uint8)
        w = np.zeros((max(m, 1), 3), np.float32)
        imp = np.zeros((max(m, 1), 3), np.float32)
        check(L.b3g_cloth_read_tri_contacts(self.h, C.byref(cnt), _ptr(pt), _ptr(ac), _ptr(w), _ptr(imp)),
              "read_tri_contacts")
        return {"count": m, "pt": pt[:m], "active": ac[:m], "w": w[:m], "impulses": imp[:m]}

    def self_stats(self) -> dict:
        a, b, c = C.c_uint32(0), C.c_uint32(0), C.c_uint32(0)
        check(lib().b3g_cloth_get_self_stats(self.h, C.byref(a), C.byref(b), C.byref(c)), "get_self_stats")
        return {"contacts": a.value, "active": b.value, "levels": c.value}

    def system(self) -> dict:
        nnz = C.c_uint32(0)
        L = lib()
        check(L.b3g_cloth_read_system(self.h, C.byref(nnz), None, None, None, None, None, None), "read_system")
        rowptr = np.zeros(self.n + 1, np.uint32)
        cols = np.zeros(nnz.value, np.uint32)
        vals = np.zeros(9 * nnz.value, np.float32)
        b = np.zeros(3 * self.n, np.float32)
        S = np.zeros(self.n, np.float32)
        x0 = np.zeros(3 * self.n, np.float32)
        check(L.b3g_cloth_read_system(self.h, C.byref(nnz), _ptr(rowptr), _ptr(cols), _ptr(vals), _ptr(b), _ptr(S),
                                      _ptr(x0)), "read_system")
        return {"rowptr": rowptr, "cols": cols, "vals": vals, "b": b, "S": S, "x0": x0}

    def setup(self, scene: Scene, opts: SolverOptions | None = None) -> "Cloth":
        """Gravity, pinned vertices and colliders of a Scene."""
        self.set_gravity(scene.gravity)
        types = np.full(self.n, DYNAMIC, np.uint8)
        types[np.asarray(scene.pinned, np.int64)] = STATIC
        self.set_types(types)
        for (c, r, mu) in scene.spheres:
            self.add_sphere(c, r, mu)
        for (a, b, r, mu) in scene.capsules:
            self.add_capsule(a, b, r, mu)
        for (hv, hp, mu) in scene.hulls:
            self.add_hull(hv, hp, mu)
        if opts is not None:
            self.set_solver(opts)
        return self


class Batch:
    """Many cloths stepped together (b3g_batch): fixed launches per step, the
    CG in one persistent launch, one cloth per CTA or per cluster."""

    def __init__(self, capacity: int = 1024, device: int = 0):
        h = C.c_void_p()
        check(lib().b3g_batch_create(device, capacity, C.byref(h)), "b3g_batch_create")
        self.h = h
        self.stats = BatchStatsC()

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().b3g_batch_destroy(self.h)
            self.h = None

    __del__ = close

    @staticmethod
    def _handles(cloths):
        arr = (C.c_void_p * len(cloths))(*[c.h.value for c in cloths])
        return arr

    def step(self, cloths, dt: float, velocity_iterations: int = 8, position_iterations: int = 2,
             per_cloth: bool = False):
        arr = self._handles(cloths)
        stats = (StepStatsC * len(cloths))() if per_cloth else None
        check(lib().b3g_batch_step(self.h, arr, len(cloths), dt, velocity_iterations, position_iterations,
                                   stats, C.byref(self.stats)), "batch_step")
        s = self.stats
        out = {"count": s.count, "rows": s.rows, "tasks": s.tasks, "cg_iterations_total": s.cg_iterations_total,
               "cg_iterations_max": s.cg_iterations_max, "step_ms": s.step_ms, "cg_ms": s.cg_ms}
        if per_cloth:
            out["per_cloth"] = [{"iterations": x.iterations, "delta": x.delta, "b_delta": x.b_delta,
                                 "active_contacts": x.active_contacts, "contacts": x.contacts} for x in stats]
        return out

    def schedule(self) -> dict:
        sc = BatchScheduleC()
        check(lib().b3g_batch_get_schedule(self.h, C.byref(sc)), "get_schedule")
        return {"cluster": sc.cluster, "split_class": list(sc.split_class), "tuned_cg_ms": sc.tuned_cg_ms}

    def set_schedule(self, cluster: int = 1, split_classes=()) -> None:
        sc = BatchScheduleC()
        sc.cluster = cluster
        for k in split_classes:
            sc.split_class[k] = 1
        check(lib().b3g_batch_set_schedule(self.h, C.byref(sc)), "set_schedule")

    def autotune(self, cloths, dt: float) -> dict:
        arr = self._handles(cloths)
        sc = BatchScheduleC()
        check(lib().b3g_batch_autotune(self.h, arr, len(cloths), dt, C.byref(sc)), "autotune")
        return {"cluster": sc.cluster, "split_class": list(sc.split_class), "tuned_cg_ms": sc.tuned_cg_ms}


class Server:
    """Continuous-batching cloth-step server (b3g_server)."""

    def __init__(self, budget_bytes: int, max_active: int = 1024, dt: float = 1.0 / 60.0,
                 velocity_iterations: int = 8, position_iterations: int = 2, gravity=(0.0, -9.8, 0.0),
                 solver: SolverOptions | None = None, cluster: int = 1, split_classes=(), host_threads: int = 0,
                 device: int = 0):
        cfg = ServerConfigC()
        cfg.hbm_budget_bytes = int(budget_bytes)
        cfg.max_active = max_active
        cfg.dt = dt
        cfg.velocity_iterations = velocity_iterations
        cfg.position_iterations = position_iterations
        for k in range(3):
            cfg.gravity[k] = gravity[k]
        cfg.solver = (solver or SolverOptions.relative(1e-4, 200, DOT_F64)).as_c()
        cfg.schedule.cluster = cluster
        for k in split_classes:
            cfg.schedule.split_class[k] = 1
        cfg.host_threads = host_threads
        h = C.c_void_p()
        check(lib().b3g_server_create(device, C.byref(cfg), C.byref(h)), "b3g_server_create")
        self.h = h
        self._keep = []

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().b3g_server_destroy(self.h)
            self.h = None

    __del__ = close

    def submit(self, mesh: Mesh, cdef: ClothDef, types=None, spheres=(), steps: int = 1, arrival: float = 0.0) -> int:
        v = np.ascontiguousarray(mesh.vertices, np.float32)
        t = np.ascontiguousarray(mesh.triangles, np.uint32)
        md = MeshDesc(mesh.vertex_count, _ptr(v), mesh.triangle_count, _ptr(t), 0, None)
        d = ClothDefC(cdef.density, cdef.streching, cdef.shearing, cdef.bending, cdef.sewing, cdef.damping,
                      cdef.thickness, cdef.friction)
        ty = None if types is None else np.ascontiguousarray(types, np.uint8)
        sp = np.ascontiguousarray(np.asarray([[c[0], c[1], c[2], r, mu] for (c, r, mu) in spheres], np.float32)
                                  .reshape(-1))
        rid = C.c_uint64(0)
        check(lib().b3g_server_submit(self.h, C.byref(md), C.byref(d), None if ty is None else _ptr(ty),
                                      _ptr(sp) if sp.size else None, len(spheres), steps, arrival, C.byref(rid)),
              "server_submit")
        return rid.value

    def submit_scene(self, scene: Scene, steps: int, arrival: float = 0.0) -> int:
        types = np.full(scene.mesh.vertex_count, DYNAMIC, np.uint8)
        types[np.asarray(scene.pinned, np.int64)] = STATIC
        return self.submit(scene.mesh, scene.cdef, types, scene.spheres, steps, arrival)

    def tick(self, now: float = 0.0) -> dict:
        t = ServerTickC()
        check(lib().b3g_server_tick(self.h, now, C.byref(t)), "server_tick")
        return {k: getattr(t, k) for k, _ in ServerTickC._fields_}

    def poll(self, rid: int) -> dict:
        i = RequestInfoC()
        check(lib().b3g_server_poll(self.h, rid, C.byref(i)), "server_poll")
        return {k: getattr(i, k) for k, _ in RequestInfoC._fields_}

    def result(self, rid: int) -> np.ndarray:
        n = self.poll(rid)["vertex_count"]
        out = np.zeros((n, 3), np.float32)
        check(lib().b3g_server_result(self.h, rid, _ptr(out)), "server_result")
        return out

    def release(self, rid: int) -> None:
        check(lib().b3g_server_release(self.h, rid), "server_release")

    def stats(self) -> dict:
        s = ServerStatsC()
        check(lib().b3g_server_stats(self.h, C.byref(s)), "server_stats")
        return {k: getattr(s, k) for k, _ in ServerStatsC._fields_}

    def drain(self, now: float = 0.0, max_ticks: int = 100000) -> int:
        """Tick until no request is queued or active; returns the ticks run."""
        n = 0
        while n < max_ticks:
            st = self.stats()
            if st["active"] == 0 and st["queued"] == 0:
                break
            self.tick(now)
            n += 1
        return n


def kernel_launch_count() -> int:
    return int(lib().b3g_kernel_launch_count())


class SoftBody:
    """A b3SoftBody on the GPU (b3g_softbody_*): tetrahedral corotated FEM
    with plasticity and the reference's MPCG, stepped without a world."""

    def __init__(self, vertices, tets, sdef, device: int = 0):
        L = lib()
        self._v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        self._t = np.ascontiguousarray(tets, np.uint32).reshape(-1, 4)
        d = SoftBodyDefC(sdef.density, sdef.E, sdef.nu, sdef.c_yield, sdef.c_creep, sdef.c_max)
        h = C.c_void_p()
        check(L.b3g_softbody_create(len(self._v), _ptr(self._v), len(self._t), _ptr(self._t), C.byref(d), device,
                                    C.byref(h)), "b3g_softbody_create")
        self.h = h.value
        self.n, self.t = len(self._v), len(self._t)
        self.nhull = 0
        self.stats = StepStatsC()

    def close(self) -> None:
        if getattr(self, "h", None):
            L = lib() if _lib is not None else None
            if L is not None:
                L.b3g_softbody_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self, scene, opts: SolverOptions | None = None) -> "SoftBody":
        """Gravity, mass damping and static nodes of a SoftBodyScene."""
        self.set_gravity(scene.gravity)
        for i, dmp in enumerate(scene.mass_damping):
            if dmp != 0.0:
                self.set_mass_damping(i, float(dmp))
        for i in scene.static_nodes:
            self.set_node_type(int(i), 0)
        if opts is not None:
            self.set_solver(opts)
        return self

    def set_gravity(self, g) -> None:
        a = _f3(g)
        check(lib().b3g_softbody_set_gravity(self.h, _ptr(a)), "softbody_set_gravity")

    def set_node_type(self, i: int, type_: int) -> None:
        check(lib().b3g_softbody_set_node_type(self.h, i, type_), "softbody_set_node_type")

    def set_mass_damping(self, i: int, d: float) -> None:
        check(lib().b3g_softbody_set_mass_damping(self.h, i, d), "softbody_set_mass_damping")

    def apply_force(self, i: int, f) -> None:
        a = _f3(f)
        check(lib().b3g_softbody_apply_force(self.h, i, _ptr(a)), "softbody_apply_force")

    def set_velocity(self, i: int, v) -> None:
        a = _f3(v)
        check(lib().b3g_softbody_set_velocity(self.h, i, _ptr(a)), "softbody_set_velocity")

    def set_position(self, i: int, x) -> None:
        a = _f3(x)
        check(lib().b3g_softbody_set_position(self.h, i, _ptr(a)), "softbody_set_position")

    def set_solver(self, o: SolverOptions) -> None:
        c = SolverOptsC(o.stop_rule, o.tolerance, o.max_iterations, o.dot)
        check(lib().b3g_softbody_set_solver(self.h, C.byref(c)), "softbody_set_solver")

    def set_cg_strategy(self, persistent: bool, fused: bool = False) -> None:
        """True (the default): the MPCG as one persistent cooperative launch
        (fused: one grid reduction per iteration); False: three launches per
        CG iteration."""
        code = 0 if not persistent else 2 if fused else 1
        check(lib().b3g_softbody_set_cg_strategy(self.h, code), "softbody_set_cg_strategy")

    def add_hull(self, vertices, planes, friction: float) -> int:
        """A static convex hull the nodes collide with: vertices (n, 3) and
        face planes (f, 4: normal, offset), world frame."""
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        p = np.ascontiguousarray(planes, np.float32).reshape(-1, 4)
        sid = C.c_uint32(0)
        check(lib().b3g_softbody_add_static_hull(self.h, _ptr(v), len(v), _ptr(p), len(p), friction, C.byref(sid)),
              "softbody_add_static_hull")
        self.nhull += 1
        return sid.value

    def set_node_radius(self, i: int, r: float) -> None:
        check(lib().b3g_softbody_set_node_radius(self.h, i, r), "softbody_set_node_radius")

    def set_node_friction(self, i: int, f: float) -> None:
        check(lib().b3g_softbody_set_node_friction(self.h, i, f), "softbody_set_node_friction")

    def contacts(self) -> dict:
        """Node contacts per (hull, node), hull-major: exists, active and the
        (normal, tangent, tangent) impulses."""
        m = self.nhull * self.n
        ex = np.zeros(m, np.uint8)
        ac = np.zeros(m, np.uint8)
        imp = np.zeros(3 * m, np.float32)
        check(lib().b3g_softbody_read_contacts(self.h, _ptr(ex), _ptr(ac), _ptr(imp)), "softbody_read_contacts")
        return {"exists": ex, "active": ac, "impulses": imp.reshape(-1, 3)}

    def step(self, dt: float, velocity_iterations: int = 8, position_iterations: int = 2) -> dict:
        check(lib().b3g_softbody_step(self.h, dt, velocity_iterations, position_iterations, C.byref(self.stats)),
              "softbody_step")
        s = self.stats
        return {"iterations": s.iterations, "delta0": s.delta0, "delta": s.delta, "b_delta": s.b_delta,
                "step_ms": s.step_ms}

    def state(self) -> dict:
        x = np.zeros((self.n, 3), np.float32)
        v = np.zeros((self.n, 3), np.float32)
        check(lib().b3g_softbody_read_state(self.h, _ptr(x), _ptr(v)), "softbody_read_state")
        return {"x": x, "v": v}

    def write_state(self, x=None, v=None) -> None:
        xs = None if x is None else np.ascontiguousarray(x, np.float32)
        vs = None if v is None else np.ascontiguousarray(v, np.float32)
        check(lib().b3g_softbody_write_state(self.h, None if xs is None else _ptr(xs),
                                             None if vs is None else _ptr(vs)), "softbody_write_state")

    def elements(self) -> dict:
        q = np.zeros((self.t, 4), np.float32)
        e = np.zeros((self.t, 6), np.float32)
        check(lib().b3g_softbody_read_elements(self.h, _ptr(q), _ptr(e)), "softbody_read_elements")
        return {"q": q, "eps": e}

    def write_elements(self, q=None, eps=None) -> None:
        qs = None if q is None else np.ascontiguousarray(q, np.float32)
        es = None if eps is None else np.ascontiguousarray(eps, np.float32)
        check(lib().b3g_softbody_write_elements(self.h, None if qs is None else _ptr(qs),
                                                None if es is None else _ptr(es)), "softbody_write_elements")

    def masses(self) -> np.ndarray:
        m = np.zeros(self.n, np.float32)
        check(lib().b3g_softbody_read_masses(self.h, _ptr(m)), "softbody_read_masses")
        return m

    def energy(self) -> float:
        e = C.c_float(0.0)
        check(lib().b3g_softbody_energy(self.h, C.byref(e)), "softbody_energy")
        return float(e.value)

    def block_count(self) -> int:
        """Blocks of the assembled matrix (its nonzero 3x3 blocks)."""
        cnt = C.c_uint32(0)
        check(lib().b3g_softbody_export_system(self.h, 1.0 / 60.0, 0, None, None, None, None, None, C.byref(cnt)),
              "softbody_export_system")
        return int(cnt.value)

    def system(self, dt: float) -> dict:
        """A (rows in the reference's list order), b and S of one force solve
        from the current state; the state is not changed."""
        cnt = C.c_uint32(0)
        L = lib()
        check(L.b3g_softbody_export_system(self.h, dt, 0, None, None, None, None, None, C.byref(cnt)),
              "softbody_export_system")
        m = cnt.value
        rowptr = np.zeros(self.n + 1, np.uint32)
        cols = np.zeros(m, np.uint32)
        vals = np.zeros(9 * m, np.float32)
        b = np.zeros(3 * self.n, np.float32)
        S = np.zeros(self.n, np.float32)
        check(L.b3g_softbody_export_system(self.h, dt, m, _ptr(rowptr), _ptr(cols), _ptr(vals), _ptr(b), _ptr(S),
                                           C.byref(cnt)), "softbody_export_system")
        return {"rowptr": rowptr, "cols": cols, "vals": vals, "b": b, "S": S}
