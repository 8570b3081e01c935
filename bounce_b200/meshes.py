"""Cloth meshes and the synthetic workloads used by the tests and the benchmark.

`grid_mesh` builds the same topology as Bounce's ``b3GridClothMesh``
(include/bounce/cloth/grid_cloth_mesh.h:26-94): vertices stored row-major,
``v(i, j) = i * (W + 1) + j``, in the x-z plane centred at the origin, and two
triangles per cell, ``(v3, v2, v1)`` and ``(v1, v4, v3)``.  The reference
template has unit spacing; here the grid is scaled to ``size`` metres and can
carry a seeded Gaussian jitter, applied before the cloth is built so that the
rest state includes it.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# b3ParticleType (include/bounce/cloth/particle.h:27-32)
STATIC, KINEMATIC, DYNAMIC = 0, 1, 2


@dataclass
class ClothDef:
    """b3ClothDef (include/bounce/cloth/cloth.h:56-95)."""

    density: float = 0.0
    streching: float = 0.0
    shearing: float = 0.0
    bending: float = 0.0
    sewing: float = 0.0
    damping: float = 0.0
    thickness: float = 0.0
    friction: float = 0.2

    def as_array(self) -> np.ndarray:
        return np.array([self.density, self.streching, self.shearing, self.bending, self.sewing,
                         self.damping, self.thickness, self.friction], dtype=np.float32)


@dataclass
class Mesh:
    vertices: np.ndarray            # float32 (N, 3)
    triangles: np.ndarray           # uint32 (T, 3)
    sewing: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.uint32))  # (s1, s2, v1, v2)

    @property
    def vertex_count(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def triangle_count(self) -> int:
        return int(self.triangles.shape[0])


def grid_mesh(side: int, size: float = 1.0, jitter: float = 0.0, seed: int = 0) -> Mesh:
    """A side x side vertex grid, (side-1)^2 cells, 2 (side-1)^2 triangles."""
    if side < 2:
        raise ValueError("a grid needs at least 2 vertices per side")
    w = side - 1
    j, i = np.meshgrid(np.arange(side), np.arange(side))
    verts = np.zeros((side * side, 3), dtype=np.float64)
    verts[:, 0] = (j.reshape(-1) / w - 0.5) * size
    verts[:, 2] = (i.reshape(-1) / w - 0.5) * size
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        verts += rng.normal(0.0, jitter, size=verts.shape)
    ci, cj = np.meshgrid(np.arange(w), np.arange(w), indexing="ij")
    ci = ci.reshape(-1)
    cj = cj.reshape(-1)
    v1 = ci * side + cj
    v2 = (ci + 1) * side + cj
    v3 = (ci + 1) * side + cj + 1
    v4 = ci * side + cj + 1
    tris = np.empty((2 * w * w, 3), dtype=np.uint32)
    tris[0::2] = np.stack([v3, v2, v1], axis=1)
    tris[1::2] = np.stack([v1, v4, v3], axis=1)
    return Mesh(verts.astype(np.float32), tris)


@dataclass
class Scene:
    """One cloth with everything a step sequence needs."""

    name: str
    mesh: Mesh
    cdef: ClothDef
    pinned: np.ndarray                      # vertex ids made static
    gravity: tuple = (0.0, -9.8, 0.0)
    spheres: list = field(default_factory=list)   # (center (3,), radius, friction)
    capsules: list = field(default_factory=list)  # (a (3,), b (3,), radius, friction): static, world frame
    hulls: list = field(default_factory=list)     # (vertices (n, 3), planes (f, 4), friction): static, world frame
    dt: float = 1.0 / 60.0
    steps: int = 100
    velocity_iterations: int = 8
    position_iterations: int = 2
    tol: float = 1e-4
    max_iterations: int = 50


def plain_scene(side: int = 32, seed: int = 1, steps: int = 100) -> Scene:
    """Single cloth, no contacts: 1 m x 1 m, 1 kg/m^2, stretch 1e4, shear 1e3,
    damping 0.05, gravity (0, -9.8, 0), the two corners of row 0 pinned,
    jitter N(0, 1e-3 m)."""
    mesh = grid_mesh(side, 1.0, 1e-3, seed)
    cdef = ClothDef(density=1.0, streching=1e4, shearing=1e3, damping=0.05, friction=0.3)
    pins = np.array([0, side - 1], dtype=np.uint32)
    return Scene(f"grid{side}_plain", mesh, cdef, pins, steps=steps)


def sphere_scene(side: int = 256, seed: int = 2, steps: int = 200) -> Scene:
    """Single large cloth: stretch + shear + bending springs (1e2) on every
    edge-adjacent triangle pair, a static sphere of radius 0.3 m 0.5 m below
    the cloth centre, friction 0.3, jitter N(0, 1e-3 m)."""
    mesh = grid_mesh(side, 1.0, 1e-3, seed)
    cdef = ClothDef(density=1.0, streching=1e4, shearing=1e3, bending=1e2, damping=0.05, friction=0.3)
    pins = np.array([0, side - 1], dtype=np.uint32)
    sph = [((0.0, -0.5, 0.0), 0.3, 0.3)]
    return Scene(f"grid{side}_bend_sphere", mesh, cdef, pins, spheres=sph, steps=steps)


def capsule_scene(side: int = 32, seed: int = 5, steps: int = 120) -> Scene:
    """A cloth falling over a static capsule (a rod along z, radius 0.1 m,
    0.4 m below the cloth), stretch 1e4, shear 1e3, bending 1e2, damping
    0.05, friction 0.3, jitter N(0, 1e-3 m), nothing pinned."""
    mesh = grid_mesh(side, 1.0, 1e-3, seed)
    cdef = ClothDef(density=1.0, streching=1e4, shearing=1e3, bending=1e2, damping=0.05, friction=0.3)
    caps = [((0.1, -0.4, -0.6), (-0.1, -0.4, 0.6), 0.1, 0.3)]
    return Scene(f"grid{side}_capsule", mesh, cdef, np.zeros(0, np.uint32), capsules=caps, steps=steps)


def self_collision_scene(side: int = 11, seed: int = 6, steps: int = 150) -> Scene:
    """The reference's self-collision scene (examples/testbed/tests/
    cloth_self_collision.h:24-60): a side x side vertex grid of 1 m spacing,
    5 m up, density 1, stretch 1e5, no shear or damping, thickness 0.2,
    friction 0.3, falling onto a static capsule from (0, 0, -5) to (0, 0, 5)
    (larger cloths: as long as the cloth), radius 1, friction 1.  Jitter
    N(0, 1e-3 m); nothing pinned."""
    mesh = grid_mesh(side, float(side - 1), 1e-3, seed)
    mesh.vertices[:, 1] += np.float32(5.0)
    cdef = ClothDef(density=1.0, streching=1e5, thickness=0.2, friction=0.3)
    half = max(5.0, 0.5 * (side - 1))  # larger cloths: the capsule spans the cloth
    caps = [((0.0, 0.0, -half), (0.0, 0.0, half), 1.0, 1.0)]
    return Scene(f"grid{side}_self_collision", mesh, cdef, np.zeros(0, np.uint32), capsules=caps, steps=steps)


def stiff_scene(side: int = 1024, steps: int = 50) -> Scene:
    """Ill-conditioned large cloth: stretch 1e5, damping 0.1, shear 1e3, no jitter."""
    mesh = grid_mesh(side, 1.0, 0.0, 0)
    cdef = ClothDef(density=1.0, streching=1e5, shearing=1e3, damping=0.1, friction=0.3)
    pins = np.array([0, side - 1], dtype=np.uint32)
    return Scene(f"grid{side}_stiff", mesh, cdef, pins, steps=steps)


def sewn_scene(side: int = 16, seed: int = 4, gap: float = 0.05, sewing: float = 1e3, steps: int = 60) -> Scene:
    """Two grid panels, one `gap` below the other, sewn along both side edges
    (column 0 and column side-1 of every row) like a sleeve: sewing springs
    of rest length 0 (b3ClothDef::sewing, cloth.cpp:248-262).  Stretch 1e4,
    shear 1e3, damping 0.05, jitter N(0, 1e-3 m), the two top corners of
    both panels pinned."""
    a = grid_mesh(side, 1.0, 1e-3, seed)
    b = grid_mesh(side, 1.0, 1e-3, seed + 1)
    nb = a.vertex_count
    verts = np.concatenate([a.vertices, b.vertices + np.array([0.0, -gap, 0.0], np.float32)]).astype(np.float32)
    tris = np.concatenate([a.triangles, b.triangles + np.uint32(nb)]).astype(np.uint32)
    rows = np.arange(side, dtype=np.uint32)
    left, right = rows * side, rows * side + (side - 1)
    edge = np.concatenate([left, right])
    sew = np.stack([np.zeros_like(edge), np.ones_like(edge), edge, edge + np.uint32(nb)], axis=1).astype(np.uint32)
    mesh = Mesh(verts, tris, sew)
    cdef = ClothDef(density=1.0, streching=1e4, shearing=1e3, sewing=sewing, damping=0.05, friction=0.3)
    pins = np.array([0, side - 1, nb, nb + side - 1], dtype=np.uint32)
    return Scene(f"sewn{side}", mesh, cdef, pins, steps=steps)


def batch_scenes(count: int = 512, seed: int = 3, side_lo: int = 16, side_hi: int = 128,
                 steps: int = 100) -> list:
    """Many independent cloths: side ~ U{side_lo..side_hi}, stretch log-U[1e3, 1e5],
    shear log-U[1e2, 1e4], the whole row 0 pinned."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        side = int(rng.integers(side_lo, side_hi + 1))
        ks = float(10.0 ** rng.uniform(3.0, 5.0))
        kh = float(10.0 ** rng.uniform(2.0, 4.0))
        mesh = grid_mesh(side, 1.0, 1e-3, seed * 100003 + k)
        cdef = ClothDef(density=1.0, streching=ks, shearing=kh, damping=0.05, friction=0.3)
        pins = np.arange(side, dtype=np.uint32)
        out.append(Scene(f"batch{k}_{side}", mesh, cdef, pins, steps=steps))
    return out


# ---------------------------------------------------------------------------
# Soft bodies

@dataclass
class SoftBodyDef:
    """b3SoftBodyDef (include/bounce/softbody/softbody.h:64-99); its
    defaults are the reference's."""

    density: float = 0.1
    E: float = 100.0
    nu: float = 0.3
    c_yield: float = float(np.finfo(np.float32).max)
    c_creep: float = 0.0
    c_max: float = 0.0


@dataclass
class SoftBodyScene:
    vertices: np.ndarray            # (n, 3) float32
    tets: np.ndarray                # (t, 4) uint32
    sdef: SoftBodyDef
    mass_damping: np.ndarray        # (n,) float32, b3SoftBodyNode::SetMassDamping
    static_nodes: np.ndarray        # node ids set to e_staticSoftBodyNode
    gravity: tuple = (0.0, -9.8, 0.0)
    dt: float = 1.0 / 60.0
    velocity_iterations: int = 8
    position_iterations: int = 2
    steps: int = 100


def block_softbody_mesh(w: int, h: int, d: int, spacing: float = 1.0) -> tuple:
    """The tetrahedral block of b3BlockSoftBodyMesh<W, H, D>
    (include/bounce/softbody/block_softbody_mesh.h:24-120): (W+1)(H+1)(D+1)
    vertices on a grid of the given spacing centred at the origin, vertex
    (x, y, z) at index (x (H+1) + y)(D+1) + z, and 5 tetrahedra per cell in
    the two mirrored splits the template alternates by the cell parity."""
    xs, ys, zs = np.meshgrid(np.arange(w + 1), np.arange(h + 1), np.arange(d + 1), indexing="ij")
    verts = np.stack([xs, ys, zs], axis=-1).reshape(-1, 3).astype(np.float32)
    verts = (verts + np.array([-0.5 * w, -0.5 * h, -0.5 * d], np.float32)) * np.float32(spacing)

    def vid(x, y, z):
        return (x * (h + 1) + y) * (d + 1) + z

    tets = []
    for x in range(w):
        for y in range(h):
            for z in range(d):
                c0 = vid(x, y, z)
                c1 = c0 + 1
                c3 = vid(x + 1, y, z)
                c2 = c3 + 1
                c7 = vid(x + 1, y + 1, z)
                c6 = c7 + 1
                c4 = vid(x, y + 1, z)
                c5 = c4 + 1
                if (x + y + z) % 2 == 1:
                    tets += [(c2, c1, c6, c3), (c6, c3, c4, c7), (c4, c1, c6, c5), (c3, c1, c4, c0), (c6, c1, c4, c3)]
                else:
                    tets += [(c0, c2, c5, c1), (c7, c2, c0, c3), (c5, c2, c7, c6), (c7, c0, c5, c4), (c0, c2, c7, c5)]
    return verts, np.asarray(tets, np.uint32)


def pinned_block_scene(w: int = 4, h: int = 4, d: int = 4, spacing: float = 1.0, steps: int = 100) -> SoftBodyScene:
    """A block hanging from one node, with the material of the reference's
    pinned soft body (examples/testbed/tests/pinned_softbody.h:27-59):
    density 0.2, E 1000, nu 0.33, yield 0.1, creep 0.5, max plastic strain 1,
    mass damping 0.2 on every node, the first node of largest height static,
    gravity (0, -9.8, 0).  The block stands in for that scene's quickhull
    sphere mesh."""
    verts, tets = block_softbody_mesh(w, h, d, spacing)
    sdef = SoftBodyDef(density=0.2, E=1000.0, nu=0.33, c_yield=0.1, c_creep=0.5, c_max=1.0)
    pin = int(np.argmax(verts[:, 1]))  # the first index of the largest y
    return SoftBodyScene(verts, tets, sdef, np.full(len(verts), 0.2, np.float32), np.array([pin], np.uint32),
                         steps=steps)
