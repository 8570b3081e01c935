"""ctypes front-ends for the two CPU checkers (test infrastructure only).

* `PortCloth` wraps ``_build/liboracle.so``: the C restatement of the
  reference's cloth step (cloth_oracle.c).
* `RefCloth` wraps ``_ref/libbounce_ref.so``: the reference library itself,
  compiled from its unmodified sources by the Makefile next to this file,
  with ref_harness.cpp.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use
this package; the product (bounce_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libbounce_ref.so")

STOP_REFERENCE, STOP_RELATIVE = 0, 1
DOT_F32, DOT_COMPENSATED, DOT_F64 = 0, 1, 2

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


# Root of the reference's source tree (include/ and src/), read only by the
# build of the reference library below; the environment variable
# B3G_REFERENCE_DIR overrides the default.
REFERENCE_DIR = os.environ.get("B3G_REFERENCE_DIR", "/root/reference")


def build(port: bool = True, ref: bool = True) -> None:
    """Compile the checkers (the reference part needs its sources on disk)."""
    targets = []
    if port:
        targets.append("port")
    if ref and os.path.isdir(os.path.join(REFERENCE_DIR, "src")):
        targets.append("ref")
    if targets:
        subprocess.run(["make", "-s", "-C", HERE, "-j8", f"REF={REFERENCE_DIR}"] + targets, check=True)


class _OcStepInfo(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("delta0", C.c_double), ("delta", C.c_double),
                ("b_delta", C.c_double), ("active_contacts", C.c_uint32), ("contacts", C.c_uint32),
                ("active_tri_contacts", C.c_uint32), ("tri_contacts", C.c_uint32)]


_port = None
_ref = None


def port_lib():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            build(port=True, ref=False)
        L = C.CDLL(PORT_LIB)
        L.oc_create.restype = C.c_void_p
        L.oc_create.argtypes = [_f32p, C.c_uint32, _u32p, C.c_uint32, _u32p, C.c_uint32, _f32p]
        L.oc_destroy.argtypes = [C.c_void_p]
        L.oc_set_gravity.argtypes = [C.c_void_p, _f32p]
        L.oc_set_type.argtypes = [C.c_void_p, C.c_uint32, C.c_int]
        L.oc_set_radius.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.oc_set_friction.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.oc_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_set_contacts.argtypes = [C.c_void_p, C.c_uint32, _u32p, _u32p, _f32p]
        L.oc_add_body.restype = C.c_int
        L.oc_add_body.argtypes = [C.c_void_p, _f32p]
        L.oc_set_body.argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.oc_get_body.argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.oc_add_body_shape.restype = C.c_int
        L.oc_add_body_shape.argtypes = [C.c_void_p, C.c_uint32, C.c_int, _f32p, C.c_uint32, C.c_uint32, C.c_float,
                                        C.c_float]
        L.oc_set_shape_proxy.argtypes = [C.c_void_p, C.c_uint32, _f32p, _f32p]
        L.oc_set_report_order.argtypes = [C.c_void_p, _u32p, C.c_uint32]
        L.oc_get_shape_proxy.argtypes = [C.c_void_p, C.c_uint32, _f32p, _f32p]
        L.oc_set_proxies.argtypes = [C.c_void_p, _f32p, _f32p]
        for name in ("oc_apply_force", "oc_apply_translation", "oc_set_position", "oc_set_velocity"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.oc_add_sphere.argtypes = [C.c_void_p, _f32p, C.c_float, C.c_float]
        L.oc_add_capsule.argtypes = [C.c_void_p, _f32p, _f32p, C.c_float, C.c_float]
        L.oc_add_hull.argtypes = [C.c_void_p, _f32p, C.c_uint32, _f32p, C.c_uint32, C.c_float]
        L.oc_set_solver.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_uint32, C.c_int]
        L.oc_step.argtypes = [C.c_void_p, C.c_float, C.c_uint32, C.c_uint32, C.POINTER(_OcStepInfo)]
        L.oc_get_state.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _u8p]
        L.oc_energy.restype = C.c_float
        L.oc_energy.argtypes = [C.c_void_p]
        L.oc_describe.restype = C.c_uint32
        L.oc_describe.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_get_contacts.restype = C.c_uint32
        L.oc_get_contacts.argtypes = [C.c_void_p, _u8p, _u8p, _f32p]
        L.oc_get_contact_list.restype = C.c_uint32
        L.oc_get_contact_list.argtypes = [C.c_void_p, C.c_uint32] + [C.c_void_p] * 4
        L.oc_ray_cast_single.restype = C.c_int
        L.oc_ray_cast_single.argtypes = [C.c_void_p, _f32p, _f32p, C.POINTER(C.c_uint32), C.POINTER(C.c_float), _f32p]
        L.oc_get_tri_contacts.restype = C.c_uint32
        L.oc_get_tri_contacts.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_force_count.restype = C.c_uint32
        L.oc_force_count.argtypes = [C.c_void_p]
        L.oc_spring_count.restype = C.c_uint32
        L.oc_spring_count.argtypes = [C.c_void_p]
        L.oc_get_springs.argtypes = [C.c_void_p, _u32p, _f32p, _f32p]
        L.oc_build_system.restype = C.c_uint32
        L.oc_build_system.argtypes = [C.c_void_p, C.c_float]
        L.oc_get_system.argtypes = [C.c_void_p, _u32p, _u32p, _f32p, _f32p, _f32p, _f32p, _u32p]
        L.oc_mpcg.restype = C.c_uint32
        L.oc_mpcg.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, _f32p, _f32p, _f32p, C.c_int, C.c_float,
                              C.c_uint32, C.c_int, _f32p, _f64p]
        L.oc_create_particle.restype = C.c_uint32
        L.oc_create_particle.argtypes = [C.c_void_p, _f32p, C.c_void_p, C.c_float, C.c_float, C.c_float]
        L.oc_destroy_particle.restype = C.c_int
        L.oc_destroy_particle.argtypes = [C.c_void_p, C.c_uint32]
        L.oc_create_mouse_force.restype = C.c_uint32
        L.oc_create_mouse_force.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32] + [C.c_float] * 5
        L.oc_destroy_force.restype = C.c_int
        L.oc_destroy_force.argtypes = [C.c_void_p, C.c_uint32]
        L.oc_particle_count.restype = C.c_uint32
        L.oc_particle_count.argtypes = [C.c_void_p]
        L.oc_solve_f64.restype = C.c_uint32
        L.oc_solve_f64.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, _f32p, _f32p, _f32p, C.c_double,
                                   C.c_uint32, _f64p]
        _port = L
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(f"{REF_LIB} is not built (make -C oracle ref)")
        L = C.CDLL(REF_LIB)
        L.ref_cloth_create.restype = C.c_void_p
        L.ref_cloth_create.argtypes = [_f32p, C.c_uint32, _u32p, C.c_uint32, _u32p, C.c_uint32, _f32p, C.c_int]
        L.ref_cloth_destroy.argtypes = [C.c_void_p]
        L.ref_cloth_set_gravity.argtypes = [C.c_void_p, _f32p]
        L.ref_cloth_set_type.argtypes = [C.c_void_p, C.c_uint32, C.c_int]
        L.ref_cloth_set_radius.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.ref_cloth_add_body.restype = C.c_uint32
        L.ref_cloth_add_body.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, _f32p, _f32p]
        L.ref_cloth_add_body_shape.restype = C.c_uint32
        L.ref_cloth_add_body_shape.argtypes = [C.c_void_p, C.c_uint32, C.c_int, _f32p, C.c_float, C.c_float, C.c_float]
        L.ref_cloth_add_body_hull.restype = C.c_uint32
        L.ref_cloth_add_body_hull.argtypes = [C.c_void_p, C.c_uint32, _f32p, C.c_uint32, C.c_float, C.c_float, _f32p,
                                              _f32p, C.POINTER(C.c_uint32)]
        L.ref_cloth_get_body.argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.ref_cloth_get_shape_proxy.argtypes = [C.c_void_p, C.c_uint32, _f32p, _f32p]
        L.ref_world_step.argtypes = [C.c_void_p, C.c_float, C.c_uint32, C.c_uint32]
        L.ref_world_report_order.restype = C.c_uint32
        L.ref_world_report_order.argtypes = [C.c_void_p, _u32p]
        L.ref_world_set_gravity.argtypes = [C.c_void_p, _f32p]
        L.ref_cloth_set_friction.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        for name in ("ref_cloth_apply_force", "ref_cloth_apply_translation", "ref_cloth_set_position",
                     "ref_cloth_set_velocity"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.ref_cloth_add_sphere.argtypes = [C.c_void_p, _f32p, C.c_float, C.c_float]
        L.ref_cloth_add_capsule.argtypes = [C.c_void_p, _f32p, _f32p, C.c_float, C.c_float]
        L.ref_cloth_add_hull.restype = C.c_uint32
        L.ref_cloth_add_hull.argtypes = [C.c_void_p, _f32p, C.c_uint32, C.c_float, _f32p, _f32p,
                                         C.POINTER(C.c_uint32)]
        L.ref_cloth_step.argtypes = [C.c_void_p, C.c_float, C.c_uint32, C.c_uint32, C.c_int]
        L.ref_last_iterations.restype = C.c_uint32
        L.ref_cloth_get_state.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _u8p]
        L.ref_cloth_energy.restype = C.c_float
        L.ref_cloth_energy.argtypes = [C.c_void_p]
        L.ref_cloth_describe.restype = C.c_uint32
        L.ref_cloth_describe.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_cloth_get_contacts.restype = C.c_uint32
        L.ref_cloth_get_contacts.argtypes = [C.c_void_p, _u8p, _u8p, _f32p]
        L.ref_cloth_get_contact_list.restype = C.c_uint32
        L.ref_cloth_get_contact_list.argtypes = [C.c_void_p, C.c_uint32] + [C.c_void_p] * 4
        L.ref_cloth_ray_cast_single.restype = C.c_int
        L.ref_cloth_ray_cast_single.argtypes = [C.c_void_p, _f32p, _f32p, C.POINTER(C.c_uint32), C.POINTER(C.c_float),
                                                _f32p]
        L.ref_cloth_get_tri_contacts.restype = C.c_uint32
        L.ref_cloth_get_tri_contacts.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_cloth_build_system.restype = C.c_uint32
        L.ref_cloth_build_system.argtypes = [C.c_void_p, C.c_float]
        L.ref_cloth_get_system.argtypes = [C.c_void_p, _u32p, _u32p, _f32p, _f32p, _f32p, _f32p, _u32p]
        L.ref_cloth_create_particle.restype = C.c_uint32
        L.ref_cloth_create_particle.argtypes = [C.c_void_p, _f32p, C.c_void_p, C.c_float, C.c_float, C.c_float]
        L.ref_cloth_destroy_particle.restype = C.c_int
        L.ref_cloth_destroy_particle.argtypes = [C.c_void_p, C.c_uint32]
        L.ref_cloth_create_mouse_force.restype = C.c_uint32
        L.ref_cloth_create_mouse_force.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32] + [C.c_float] * 5
        L.ref_cloth_destroy_force.restype = C.c_int
        L.ref_cloth_destroy_force.argtypes = [C.c_void_p, C.c_uint32]
        L.ref_cloth_particle_count.restype = C.c_uint32
        L.ref_cloth_particle_count.argtypes = [C.c_void_p]
        L.ref_profile_read.restype = C.c_uint32
        L.ref_profile_read.argtypes = [C.c_char_p, C.c_uint32, _f64p, np.ctypeslib.ndpointer(np.uint64)]
        L.ref_profile_reset.argtypes = []
        _ref = L
    return _ref


class _Base:
    """Shared state accessors; subclasses bind the library calls."""

    def __init__(self, mesh, cdef):
        self.n_mesh = mesh.vertex_count
        self.t = mesh.triangle_count
        self._verts = np.ascontiguousarray(mesh.vertices, np.float32).reshape(-1)
        self._tris = np.ascontiguousarray(mesh.triangles, np.uint32).reshape(-1)
        sew = np.ascontiguousarray(mesh.sewing, np.uint32).reshape(-1)
        self._sew = sew if sew.size else np.zeros(4, np.uint32)
        self._nsew = int(mesh.sewing.shape[0])
        self._def = cdef.as_array()

    @property
    def n(self) -> int:
        """Particles: the mesh's, then created ones."""
        return int(self._particle_count()) if getattr(self, "h", None) else self.n_mesh

    def create_particle(self, position, velocity=None, mass=0.0, radius=0.0, friction=0.0) -> int:
        """b3Cloth::CreateParticle: returns the particle's index (after every existing one)."""
        vel = None if velocity is None else np.asarray(velocity, np.float32)
        return int(self._create_particle(np.asarray(position, np.float32), None if vel is None else vel.ctypes.data,
                                         mass, radius, friction))

    def destroy_particle(self, index: int) -> None:
        if self._destroy_particle(index) != 0:
            raise ValueError(f"particle {index} is not a created particle")

    def create_mouse_force(self, particle: int, triangle: int, w2: float, w3: float, w4: float, mouse: float,
                           damping: float) -> int:
        """b3Cloth::CreateForce of a b3MouseForceDef: returns its id."""
        return int(self._create_mouse_force(particle, triangle, w2, w3, w4, mouse, damping))

    def destroy_force(self, force_id: int) -> None:
        if self._destroy_force(force_id) != 0:
            raise ValueError(f"no force {force_id}")

    def state(self):
        x = np.zeros(3 * self.n, np.float32)
        v = np.zeros(3 * self.n, np.float32)
        dv = np.zeros(3 * self.n, np.float32)
        m = np.zeros(self.n, np.float32)
        ty = np.zeros(self.n, np.uint8)
        self._get_state(x, v, dv, m, ty)
        return {"x": x.reshape(-1, 3), "v": v.reshape(-1, 3), "dv": dv.reshape(-1, 3), "mass": m, "type": ty}

    def describe(self):
        nf = self._describe(None, None, None)
        tri = np.zeros(6 * self.t, np.float32)
        fat = np.zeros(6 * self.n, np.float32)
        forces = np.zeros(8 * max(nf, 1), np.float32)
        self._describe(tri.ctypes.data, fat.ctypes.data, forces.ctypes.data)
        return {"tri_rest": tri.reshape(-1, 6), "fat_aabb": fat.reshape(-1, 6),
                "forces": forces.reshape(-1, 8)[:nf]}

    def contacts(self):
        ex = np.zeros(self.n, np.uint8)
        ac = np.zeros(self.n, np.uint8)
        imp = np.zeros(3 * self.n, np.float32)
        cnt = self._get_contacts(ex, ac, imp)
        return {"count": int(cnt), "exists": ex, "active": ac, "impulses": imp.reshape(-1, 3)}

    def contact_list(self):
        """Every body contact from the list's head: particle, shape, active,
        impulses (normal, tangent x, tangent y)."""
        fn = self._get_contact_list
        m = int(fn(0, None, None, None, None))
        part = np.zeros(max(m, 1), np.uint32)
        shape = np.zeros(max(m, 1), np.uint32)
        act = np.zeros(max(m, 1), np.uint8)
        imp = np.zeros(3 * max(m, 1), np.float32)
        fn(m, part.ctypes.data, shape.ctypes.data, act.ctypes.data, imp.ctypes.data)
        return {"particle": part[:m], "shape": shape[:m], "active": act[:m], "impulses": imp.reshape(-1, 3)[:m]}

    def ray_cast_single(self, p1, p2):
        """b3Cloth::RayCastSingle: (triangle, fraction, normal) or None."""
        t, f = C.c_uint32(0), C.c_float(0.0)
        n = np.zeros(3, np.float32)
        hit = self._ray_cast_single(np.asarray(p1, np.float32), np.asarray(p2, np.float32), C.byref(t), C.byref(f), n)
        return (int(t.value), float(f.value), n) if hit else None

    def tri_contacts(self):
        """Particle-triangle contacts in list order (head first)."""
        m = int(self._get_tri_contacts(None, None, None, None))
        pt = np.zeros(2 * max(m, 1), np.uint32)
        ac = np.zeros(max(m, 1), np.uint8)
        w = np.zeros(3 * max(m, 1), np.float32)
        imp = np.zeros(3 * max(m, 1), np.float32)
        self._get_tri_contacts(pt.ctypes.data, ac.ctypes.data, w.ctypes.data, imp.ctypes.data)
        return {"count": m, "pt": pt.reshape(-1, 2)[:m], "active": ac[:m], "w": w.reshape(-1, 3)[:m],
                "impulses": imp.reshape(-1, 3)[:m]}

    def system(self, dt: float):
        nnz = self._build_system(dt)
        rowptr = np.zeros(self.n + 1, np.uint32)
        cols = np.zeros(max(nnz, 1), np.uint32)
        vals = np.zeros(9 * max(nnz, 1), np.float32)
        b = np.zeros(3 * self.n, np.float32)
        S = np.zeros(self.n, np.float32)
        x0 = np.zeros(3 * self.n, np.float32)
        vor = np.zeros(self.n, np.uint32)
        self._get_system(rowptr, cols, vals, b, S, x0, vor)
        return {"rowptr": rowptr, "cols": cols[:nnz], "vals": vals[:9 * nnz], "b": b, "S": S, "x0": x0,
                "vertex_of_row": vor}

    # scene helpers
    def setup(self, scene):
        self.set_gravity(scene.gravity)
        for p in scene.pinned:
            self.set_type(int(p), 0)
        for (c, r, mu) in scene.spheres:
            self.add_sphere(c, r, mu)
        for (a, b, r, mu) in getattr(scene, "capsules", ()):
            self.add_capsule(a, b, r, mu)
        for (hv, hp, mu) in getattr(scene, "hulls", ()):
            self.add_hull(hv, hp, mu)
        return self


class PortCloth(_Base):
    """The C restatement."""

    def __init__(self, mesh, cdef):
        super().__init__(mesh, cdef)
        self.L = port_lib()
        self.h = self.L.oc_create(self._verts, self.n_mesh, self._tris, self.t, self._sew, self._nsew, self._def)
        self.last = _OcStepInfo()

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oc_destroy(self.h)
            self.h = None

    def set_gravity(self, g):
        self.L.oc_set_gravity(self.h, np.asarray(g, np.float32))

    def set_type(self, vertex, ty):
        self.L.oc_set_type(self.h, vertex, ty)

    def set_radius(self, vertex, radius):
        self.L.oc_set_radius(self.h, vertex, radius)

    def set_friction(self, vertex, friction):
        self.L.oc_set_friction(self.h, vertex, friction)

    def set_state(self, x=None, v=None, dv=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1) for a in (x, v, dv)]
        self.L.oc_set_state(self.h, *[None if a is None else a.ctypes.data for a in arrs])

    def set_contacts(self, particles, shapes, impulses):
        """Replace the body-contact list: contacts from the list's tail (the
        oldest) to its head, each (particle, shape, 3 impulses)."""
        p = np.ascontiguousarray(particles, np.uint32).reshape(-1)
        s = np.ascontiguousarray(shapes, np.uint32).reshape(-1)
        imp = np.ascontiguousarray(impulses, np.float32).reshape(-1)
        assert p.size == s.size and imp.size == 3 * p.size
        self.L.oc_set_contacts(self.h, p.size, p if p.size else np.zeros(1, np.uint32),
                               s if s.size else np.zeros(1, np.uint32), imp if imp.size else np.zeros(3, np.float32))

    def add_body(self, desc):
        """A body (55-float state, as RefCloth.body() returns) for body shapes."""
        return int(self.L.oc_add_body(self.h, np.ascontiguousarray(desc, np.float32)))

    def set_body(self, body, desc):
        self.L.oc_set_body(self.h, body, np.ascontiguousarray(desc, np.float32))

    def body(self, body):
        d = np.zeros(55, np.float32)
        self.L.oc_get_body(self.h, body, d)
        return d

    def add_body_shape(self, body, kind, geom, radius, friction, nv=0, nf=0):
        """kind 0 sphere (centre), 1 capsule (ends), 2 hull (vertices then
        planes); geometry in the body's frame."""
        g = np.ascontiguousarray(geom, np.float32).reshape(-1)
        return int(self.L.oc_add_body_shape(self.h, body, kind, g, nv, nf, radius, friction))

    def set_report_order(self, order):
        o = np.ascontiguousarray(order, np.uint32)
        self.L.oc_set_report_order(self.h, o if o.size else np.zeros(1, np.uint32), o.size)

    def set_shape_proxy(self, shape, lo, hi):
        self.L.oc_set_shape_proxy(self.h, shape, np.asarray(lo, np.float32), np.asarray(hi, np.float32))

    def shape_proxy(self, shape):
        lo, hi = np.zeros(3, np.float32), np.zeros(3, np.float32)
        self.L.oc_get_shape_proxy(self.h, shape, lo, hi)
        return lo, hi

    def set_proxies(self, lo, hi):
        """Overwrite the particles' fat AABBs (n x 3 each)."""
        self.L.oc_set_proxies(self.h, np.ascontiguousarray(lo, np.float32).reshape(-1),
                              np.ascontiguousarray(hi, np.float32).reshape(-1))

    def apply_force(self, vertex, f):
        self.L.oc_apply_force(self.h, vertex, np.asarray(f, np.float32))

    def apply_translation(self, vertex, t):
        self.L.oc_apply_translation(self.h, vertex, np.asarray(t, np.float32))

    def set_position(self, vertex, x):
        self.L.oc_set_position(self.h, vertex, np.asarray(x, np.float32))

    def set_velocity(self, vertex, v):
        self.L.oc_set_velocity(self.h, vertex, np.asarray(v, np.float32))

    def add_sphere(self, center, radius, friction):
        return self.L.oc_add_sphere(self.h, np.asarray(center, np.float32), radius, friction)

    def add_capsule(self, a, b, radius, friction):
        return self.L.oc_add_capsule(self.h, np.asarray(a, np.float32), np.asarray(b, np.float32), radius, friction)

    def add_hull(self, vertices, planes, friction):
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
        p = np.ascontiguousarray(planes, np.float32).reshape(-1)
        return self.L.oc_add_hull(self.h, v, v.size // 3, p, p.size // 4, friction)

    def set_solver(self, stop_rule=STOP_REFERENCE, tol=0.0, max_iterations=20, dot=DOT_F32):
        self.L.oc_set_solver(self.h, stop_rule, tol, max_iterations, dot)

    def step(self, dt, vel_iters=8, pos_iters=2):
        self.L.oc_step(self.h, dt, vel_iters, pos_iters, C.byref(self.last))
        return {"iterations": self.last.iterations, "delta0": self.last.delta0, "delta": self.last.delta,
                "b_delta": self.last.b_delta, "active_contacts": self.last.active_contacts,
                "contacts": self.last.contacts, "active_tri_contacts": self.last.active_tri_contacts,
                "tri_contacts": self.last.tri_contacts}

    def energy(self):
        return float(self.L.oc_energy(self.h))

    def springs(self):
        ns = self.L.oc_spring_count(self.h)
        pairs = np.zeros(2 * max(ns, 1), np.uint32)
        rest = np.zeros(max(ns, 1), np.float32)
        ks = np.zeros(max(ns, 1), np.float32)
        self.L.oc_get_springs(self.h, pairs, rest, ks)
        return pairs[:2 * ns].reshape(-1, 2), rest[:ns], ks[:ns]

    def _get_state(self, *a):
        self.L.oc_get_state(self.h, *a)

    def _particle_count(self):
        return self.L.oc_particle_count(self.h)

    def _create_particle(self, *a):
        return self.L.oc_create_particle(self.h, *a)

    def _destroy_particle(self, i):
        return self.L.oc_destroy_particle(self.h, i)

    def _create_mouse_force(self, *a):
        return self.L.oc_create_mouse_force(self.h, *a)

    def _destroy_force(self, i):
        return self.L.oc_destroy_force(self.h, i)

    def _describe(self, a, b, c):
        return self.L.oc_describe(self.h, a, b, c)

    def _get_contacts(self, *a):
        return self.L.oc_get_contacts(self.h, *a)

    def _get_contact_list(self, *a):
        return self.L.oc_get_contact_list(self.h, *a)

    def _get_tri_contacts(self, *a):
        return self.L.oc_get_tri_contacts(self.h, *a)

    def _ray_cast_single(self, *a):
        return self.L.oc_ray_cast_single(self.h, *a)

    def _build_system(self, dt):
        return self.L.oc_build_system(self.h, dt)

    def _get_system(self, *a):
        self.L.oc_get_system(self.h, *a)


class RefCloth(_Base):
    """The reference library (compiled from its sources)."""

    def __init__(self, mesh, cdef, restated: bool = True):
        super().__init__(mesh, cdef)
        self.L = ref_lib()
        self.h = self.L.ref_cloth_create(self._verts, self.n_mesh, self._tris, self.t, self._sew, self._nsew,
                                         self._def, 1 if restated else 0)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_cloth_destroy(self.h)
            self.h = None

    def set_gravity(self, g):
        self.L.ref_cloth_set_gravity(self.h, np.asarray(g, np.float32))

    def set_type(self, vertex, ty):
        self.L.ref_cloth_set_type(self.h, vertex, ty)

    def set_radius(self, vertex, radius):
        self.L.ref_cloth_set_radius(self.h, vertex, radius)

    def set_friction(self, vertex, friction):
        self.L.ref_cloth_set_friction(self.h, vertex, friction)

    def add_body(self, type_, position, orientation=(0.0, 0.0, 0.0, 1.0), velocity=(0.0, 0.0, 0.0),
                 angular_velocity=(0.0, 0.0, 0.0)):
        f = lambda a: np.asarray(a, np.float32)
        return int(self.L.ref_cloth_add_body(self.h, type_, f(position), f(orientation), f(velocity),
                                             f(angular_velocity)))

    def add_body_shape(self, body, kind, geom, radius, density, friction):
        return int(self.L.ref_cloth_add_body_shape(self.h, body, kind, np.asarray(geom, np.float32), radius, density,
                                                   friction))

    def add_body_hull(self, body, points, density, friction):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1)
        verts = np.zeros(3 * 256, np.float32)
        planes = np.zeros(4 * 256, np.float32)
        nf = C.c_uint32(0)
        nv = self.L.ref_cloth_add_body_hull(self.h, body, pts, pts.size // 3, density, friction, verts, planes,
                                            C.byref(nf))
        return verts[:3 * nv].reshape(-1, 3).copy(), planes[:4 * nf.value].reshape(-1, 4).copy()

    def body(self, body):
        d = np.zeros(55, np.float32)
        self.L.ref_cloth_get_body(self.h, body, d)
        return d

    def shape_proxy(self, shape):
        lo, hi = np.zeros(3, np.float32), np.zeros(3, np.float32)
        self.L.ref_cloth_get_shape_proxy(self.h, shape, lo, hi)
        return lo, hi

    def report_order(self):
        """The world's shapes in its query's report order."""
        o = np.zeros(64, np.uint32)
        m = self.L.ref_world_report_order(self.h, o)
        return o[:m].copy()

    def world_step(self, dt, velocity_iterations=8, position_iterations=2):
        self.L.ref_world_step(self.h, dt, velocity_iterations, position_iterations)

    def set_world_gravity(self, g):
        self.L.ref_world_set_gravity(self.h, np.asarray(g, np.float32))

    def apply_force(self, vertex, f):
        self.L.ref_cloth_apply_force(self.h, vertex, np.asarray(f, np.float32))

    def apply_translation(self, vertex, t):
        self.L.ref_cloth_apply_translation(self.h, vertex, np.asarray(t, np.float32))

    def set_position(self, vertex, x):
        self.L.ref_cloth_set_position(self.h, vertex, np.asarray(x, np.float32))

    def set_velocity(self, vertex, v):
        self.L.ref_cloth_set_velocity(self.h, vertex, np.asarray(v, np.float32))

    def add_sphere(self, center, radius, friction):
        self.L.ref_cloth_add_sphere(self.h, np.asarray(center, np.float32), radius, friction)

    def add_capsule(self, a, b, radius, friction):
        self.L.ref_cloth_add_capsule(self.h, np.asarray(a, np.float32), np.asarray(b, np.float32), radius, friction)

    def add_hull_from_points(self, points, friction):
        """A static hull that the reference's quickhull builds from `points`;
        returns its vertices (n, 3) and face planes (f, 4)."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1)
        verts = np.zeros(3 * 256, np.float32)
        planes = np.zeros(4 * 256, np.float32)
        nf = C.c_uint32(0)
        nv = self.L.ref_cloth_add_hull(self.h, pts, pts.size // 3, friction, verts, planes, C.byref(nf))
        return verts[:3 * nv].reshape(-1, 3).copy(), planes[:4 * nf.value].reshape(-1, 4).copy()

    def step(self, dt, vel_iters=8, pos_iters=2, full=False):
        self.L.ref_cloth_step(self.h, dt, vel_iters, pos_iters, 1 if full else 0)
        return {"iterations": int(self.L.ref_last_iterations())}

    def energy(self):
        return float(self.L.ref_cloth_energy(self.h))

    def _get_state(self, *a):
        self.L.ref_cloth_get_state(self.h, *a)

    def _particle_count(self):
        return self.L.ref_cloth_particle_count(self.h)

    def _create_particle(self, *a):
        return self.L.ref_cloth_create_particle(self.h, *a)

    def _destroy_particle(self, i):
        return self.L.ref_cloth_destroy_particle(self.h, i)

    def _create_mouse_force(self, *a):
        return self.L.ref_cloth_create_mouse_force(self.h, *a)

    def _destroy_force(self, i):
        return self.L.ref_cloth_destroy_force(self.h, i)

    def _describe(self, a, b, c):
        return self.L.ref_cloth_describe(self.h, a, b, c)

    def _get_contacts(self, *a):
        return self.L.ref_cloth_get_contacts(self.h, *a)

    def _get_contact_list(self, *a):
        return self.L.ref_cloth_get_contact_list(self.h, *a)

    def _get_tri_contacts(self, *a):
        return self.L.ref_cloth_get_tri_contacts(self.h, *a)

    def _ray_cast_single(self, *a):
        return self.L.ref_cloth_ray_cast_single(self.h, *a)

    def _build_system(self, dt):
        return self.L.ref_cloth_build_system(self.h, dt)

    def _get_system(self, *a):
        self.L.ref_cloth_get_system(self.h, *a)


def ref_profile():
    """Accumulated reference profile scopes: {name: (seconds, calls)}."""
    L = ref_lib()
    k = L.ref_profile_read(None, 0, np.zeros(64, np.float64), np.zeros(64, np.uint64))
    buf = C.create_string_buffer(4096)
    secs = np.zeros(max(k, 1), np.float64)
    calls = np.zeros(max(k, 1), np.uint64)
    L.ref_profile_read(buf, 4096, secs, calls)
    names = buf.value.decode().split("\n")[:k]
    return {nm: (float(secs[i]), int(calls[i])) for i, nm in enumerate(names)}


def ref_profile_reset():
    ref_lib().ref_profile_reset()


def mpcg(system, stop_rule=STOP_REFERENCE, tol=0.0, max_iterations=20, dot=DOT_F32):
    """The oracle's MPCG on an exported system; returns (x (n,3), iterations, stats)."""
    L = port_lib()
    n = system["rowptr"].size - 1
    x = np.zeros(3 * n, np.float32)
    stats = np.zeros(3, np.float64)
    it = L.oc_mpcg(n, system["rowptr"], system["cols"], system["vals"], system["b"], system["S"],
                   system["x0"], stop_rule, tol, max_iterations, dot, x, stats)
    return x.reshape(-1, 3), int(it), {"delta0": stats[0], "b_delta": stats[1], "delta": stats[2]}


def solve_f64(system, tol=1e-12, max_iterations=100000):
    """FP64 filtered Jacobi-PCG of the same system; returns x (n,3) float64."""
    L = port_lib()
    n = system["rowptr"].size - 1
    x = np.zeros(3 * n, np.float64)
    it = L.oc_solve_f64(n, system["rowptr"], system["cols"], system["vals"], system["b"], system["S"],
                        system["x0"], tol, max_iterations, x)
    return x.reshape(-1, 3), int(it)


# ---------------------------------------------------------------------------
# Soft body: softbody_oracle.c (PortSoftBody) and the reference's b3SoftBody
# through ref_softbody.cpp (RefSoftBody), with one interface.

class _OsStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("delta0", C.c_double), ("delta", C.c_double),
                ("b_delta", C.c_double)]


_sb_port_ready = False
_sb_ref_ready = False


def _sb_port():
    global _sb_port_ready
    L = port_lib()
    if not _sb_port_ready:
        L.os_create.restype = C.c_void_p
        L.os_create.argtypes = [C.c_uint32, _f32p, C.c_uint32, _u32p] + [C.c_float] * 6
        L.os_destroy.argtypes = [C.c_void_p]
        L.os_node_count.restype = C.c_uint32
        L.os_node_count.argtypes = [C.c_void_p]
        L.os_set_type.argtypes = [C.c_void_p, C.c_uint32, C.c_int]
        L.os_set_mass_damping.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.os_set_gravity.argtypes = [C.c_void_p, _f32p]
        L.os_apply_force.argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.os_set_velocity.argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.os_set_solver.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_uint32, C.c_int]
        L.os_step.argtypes = [C.c_void_p, C.c_float, C.c_uint32, C.c_uint32, C.POINTER(_OsStats)]
        L.os_get_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.os_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.os_get_masses.argtypes = [C.c_void_p, _f32p]
        L.os_get_elements.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.os_set_elements.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.os_get_element_data.argtypes = [C.c_void_p, C.c_uint32, _f32p, _f32p, _f32p, _f32p]
        L.os_energy.restype = C.c_float
        L.os_energy.argtypes = [C.c_void_p]
        L.os_system.restype = C.c_uint32
        L.os_system.argtypes = [C.c_void_p, C.c_float, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p]
        L.os_set_node_radius.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.os_set_node_friction.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.os_add_hull.restype = C.c_int
        L.os_add_hull.argtypes = [C.c_void_p, _f32p, C.c_uint32, _f32p, C.c_uint32, C.c_float]
        L.os_get_contacts.restype = C.c_uint32
        L.os_get_contacts.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.os_get_contact_list.restype = C.c_uint32
        L.os_get_contact_list.argtypes = [C.c_void_p, C.c_uint32] + [C.c_void_p] * 4
        _sb_port_ready = True
    return L


def _sb_ref():
    global _sb_ref_ready
    L = ref_lib()
    if not _sb_ref_ready:
        L.ref_softbody_create.restype = C.c_void_p
        L.ref_softbody_create.argtypes = [_f32p, C.c_uint32, _u32p, C.c_uint32, _f32p]
        L.ref_softbody_destroy.argtypes = [C.c_void_p]
        L.ref_softbody_set_type.argtypes = [C.c_void_p, C.c_uint32, C.c_int]
        L.ref_softbody_set_mass_damping.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.ref_softbody_set_gravity.argtypes = [C.c_void_p, _f32p]
        L.ref_softbody_apply_force.argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.ref_softbody_set_velocity.argtypes = [C.c_void_p, C.c_uint32, _f32p]
        L.ref_softbody_step.argtypes = [C.c_void_p, C.c_float, C.c_uint32, C.c_uint32]
        L.ref_softbody_last_iterations.restype = C.c_uint32
        L.ref_softbody_get_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_softbody_get_masses.argtypes = [C.c_void_p, _f32p]
        L.ref_softbody_get_elements.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_softbody_get_element_data.argtypes = [C.c_void_p, C.c_uint32, _f32p, _f32p, _f32p, _f32p]
        L.ref_softbody_energy.restype = C.c_float
        L.ref_softbody_energy.argtypes = [C.c_void_p]
        L.ref_softbody_add_hull.restype = C.c_uint32
        L.ref_softbody_add_hull.argtypes = [C.c_void_p, _f32p, C.c_uint32, C.c_float, _f32p, _f32p,
                                            C.POINTER(C.c_uint32)]
        L.ref_softbody_set_node_radius.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.ref_softbody_set_node_friction.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.ref_softbody_get_contacts.restype = C.c_uint32
        L.ref_softbody_get_contacts.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_softbody_get_contact_list.restype = C.c_uint32
        L.ref_softbody_get_contact_list.argtypes = [C.c_void_p, C.c_uint32] + [C.c_void_p] * 4
        _sb_ref_ready = True
    return L


def _addr(a):
    return None if a is None else a.ctypes.data


class _SoftBase:
    """Common soft-body front-end; `scene` is a bounce_b200.SoftBodyScene-like
    object (vertices (n,3) float32, tets (t,4) uint32, def fields, node types,
    mass damping, gravity)."""

    def setup(self, scene):
        self.set_gravity(scene.gravity)
        for i, d in enumerate(scene.mass_damping):
            if d != 0.0:
                self.set_mass_damping(i, float(d))
        for i in scene.static_nodes:
            self.set_type(int(i), 0)
        return self

    def state(self):
        x = np.zeros((self.n, 3), np.float32)
        v = np.zeros((self.n, 3), np.float32)
        self._get_state(x, v)
        return {"x": x, "v": v}

    def elements(self):
        q = np.zeros((self.t, 4), np.float32)
        e = np.zeros((self.t, 6), np.float32)
        self._get_elements(q, e)
        return {"q": q, "eps": e}

    def contacts(self):
        """Node contacts with the (single) hull: per node exists, active,
        impulses (normal, tangent x, tangent y)."""
        ex = np.zeros(self.n, np.uint8)
        ac = np.zeros(self.n, np.uint8)
        imp = np.zeros(3 * self.n, np.float32)
        cnt = self._get_contacts(ex.ctypes.data, ac.ctypes.data, imp.ctypes.data)
        return {"count": int(cnt), "exists": ex, "active": ac, "impulses": imp.reshape(-1, 3)}

    def contact_list(self):
        """Every node-body contact from the list's head: node, hull, active,
        impulses (normal, tangent x, tangent y)."""
        fn = self._get_contact_list
        m = int(fn(0, None, None, None, None))
        node = np.zeros(max(m, 1), np.uint32)
        shape = np.zeros(max(m, 1), np.uint32)
        act = np.zeros(max(m, 1), np.uint8)
        imp = np.zeros(3 * max(m, 1), np.float32)
        fn(m, node.ctypes.data, shape.ctypes.data, act.ctypes.data, imp.ctypes.data)
        return {"node": node[:m], "shape": shape[:m], "active": act[:m], "impulses": imp.reshape(-1, 3)[:m]}

    def element_data(self, e):
        K = np.zeros(144, np.float32)
        invE = np.zeros(9, np.float32)
        B = np.zeros(72, np.float32)
        P = np.zeros(72, np.float32)
        self._get_element_data(e, K, invE, B, P)
        return {"K": K.reshape(16, 3, 3), "invE": invE.reshape(3, 3), "B": B, "P": P}


class PortSoftBody(_SoftBase):
    def add_hull(self, vertices, planes, friction):
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
        p = np.ascontiguousarray(planes, np.float32).reshape(-1)
        return self.L.os_add_hull(self.h, v, v.size // 3, p, p.size // 4, friction)

    def set_node_radius(self, i, r):
        self.L.os_set_node_radius(self.h, i, r)

    def set_node_friction(self, i, f):
        self.L.os_set_node_friction(self.h, i, f)

    def _get_contacts(self, *a):
        return self.L.os_get_contacts(self.h, *a)

    def _get_contact_list(self, *a):
        return self.L.os_get_contact_list(self.h, *a)

    def __init__(self, vertices, tets, density, E, nu, c_yield, c_creep, c_max):
        self.L = _sb_port()
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
        t = np.ascontiguousarray(tets, np.uint32).reshape(-1)
        self.n, self.t = v.size // 3, t.size // 4
        self.h = self.L.os_create(self.n, v, self.t, t, density, E, nu, c_yield, c_creep, c_max)
        self.last = _OsStats()

    def close(self):
        if getattr(self, "h", None):
            self.L.os_destroy(self.h)
            self.h = None

    __del__ = close

    def set_type(self, i, type_):
        self.L.os_set_type(self.h, i, type_)

    def set_mass_damping(self, i, d):
        self.L.os_set_mass_damping(self.h, i, d)

    def set_gravity(self, g):
        self.L.os_set_gravity(self.h, np.asarray(g, np.float32))

    def apply_force(self, i, f):
        self.L.os_apply_force(self.h, i, np.asarray(f, np.float32))

    def set_velocity(self, i, v):
        self.L.os_set_velocity(self.h, i, np.asarray(v, np.float32))

    def set_solver(self, stop_rule=STOP_REFERENCE, tol=0.0, max_iterations=20, dot=DOT_F32):
        self.L.os_set_solver(self.h, stop_rule, tol, max_iterations, dot)

    def step(self, dt, vel_iters=8, pos_iters=2):
        self.L.os_step(self.h, dt, vel_iters, pos_iters, C.byref(self.last))
        s = self.last
        return {"iterations": s.iterations, "delta0": s.delta0, "delta": s.delta, "b_delta": s.b_delta}

    def _get_state(self, x, v):
        self.L.os_get_state(self.h, _addr(x), _addr(v))

    def set_state(self, x=None, v=None):
        xs = None if x is None else np.ascontiguousarray(x, np.float32)
        vs = None if v is None else np.ascontiguousarray(v, np.float32)
        self.L.os_set_state(self.h, _addr(xs), _addr(vs))

    def _get_elements(self, q, e):
        self.L.os_get_elements(self.h, _addr(q), _addr(e))

    def set_elements(self, q=None, eps=None):
        qs = None if q is None else np.ascontiguousarray(q, np.float32)
        es = None if eps is None else np.ascontiguousarray(eps, np.float32)
        self.L.os_set_elements(self.h, _addr(qs), _addr(es))

    def _get_element_data(self, e, K, invE, B, P):
        self.L.os_get_element_data(self.h, e, K, invE, B, P)

    def masses(self):
        m = np.zeros(self.n, np.float32)
        self.L.os_get_masses(self.h, m)
        return m

    def energy(self):
        return float(self.L.os_energy(self.h))

    def system(self, dt):
        """A (rows in the reference's list order), b and S of one force solve
        from the current state; the state is left unchanged."""
        need = self.L.os_system(self.h, dt, 0, None, None, None, None, None)
        rowptr = np.zeros(self.n + 1, np.uint32)
        cols = np.zeros(need, np.uint32)
        vals = np.zeros(9 * need, np.float32)
        b = np.zeros(3 * self.n, np.float32)
        S = np.zeros(self.n, np.float32)
        self.L.os_system(self.h, dt, need, _addr(rowptr), _addr(cols), _addr(vals), _addr(b), _addr(S))
        return {"rowptr": rowptr, "cols": cols, "vals": vals, "b": b, "S": S}


class RefSoftBody(_SoftBase):
    def add_hull_from_points(self, points, friction):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1)
        verts = np.zeros(3 * 256, np.float32)
        planes = np.zeros(4 * 256, np.float32)
        nf = C.c_uint32(0)
        nv = self.L.ref_softbody_add_hull(self.h, pts, pts.size // 3, friction, verts, planes, C.byref(nf))
        return verts[:3 * nv].reshape(-1, 3).copy(), planes[:4 * nf.value].reshape(-1, 4).copy()

    def set_node_radius(self, i, r):
        self.L.ref_softbody_set_node_radius(self.h, i, r)

    def set_node_friction(self, i, f):
        self.L.ref_softbody_set_node_friction(self.h, i, f)

    def _get_contacts(self, *a):
        return self.L.ref_softbody_get_contacts(self.h, *a)

    def _get_contact_list(self, *a):
        return self.L.ref_softbody_get_contact_list(self.h, *a)

    def __init__(self, vertices, tets, density, E, nu, c_yield, c_creep, c_max):
        self.L = _sb_ref()
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
        t = np.ascontiguousarray(tets, np.uint32).reshape(-1)
        self.n, self.t = v.size // 3, t.size // 4
        d = np.array([density, E, nu, c_yield, c_creep, c_max], np.float32)
        self.h = self.L.ref_softbody_create(v, self.n, t, self.t, d)

    def close(self):
        if getattr(self, "h", None):
            self.L.ref_softbody_destroy(self.h)
            self.h = None

    __del__ = close

    def set_type(self, i, type_):
        self.L.ref_softbody_set_type(self.h, i, type_)

    def set_mass_damping(self, i, d):
        self.L.ref_softbody_set_mass_damping(self.h, i, d)

    def set_gravity(self, g):
        self.L.ref_softbody_set_gravity(self.h, np.asarray(g, np.float32))

    def apply_force(self, i, f):
        self.L.ref_softbody_apply_force(self.h, i, np.asarray(f, np.float32))

    def set_velocity(self, i, v):
        self.L.ref_softbody_set_velocity(self.h, i, np.asarray(v, np.float32))

    def step(self, dt, vel_iters=8, pos_iters=2):
        self.L.ref_softbody_step(self.h, dt, vel_iters, pos_iters)
        return {"iterations": int(self.L.ref_softbody_last_iterations())}

    def _get_state(self, x, v):
        self.L.ref_softbody_get_state(self.h, _addr(x), _addr(v))

    def _get_elements(self, q, e):
        self.L.ref_softbody_get_elements(self.h, _addr(q), _addr(e))

    def _get_element_data(self, e, K, invE, B, P):
        self.L.ref_softbody_get_element_data(self.h, e, K, invE, B, P)

    def masses(self):
        m = np.zeros(self.n, np.float32)
        self.L.ref_softbody_get_masses(self.h, m)
        return m

    def energy(self):
        return float(self.L.ref_softbody_energy(self.h))
