// Device-side layout of one cloth and the kernels of one implicit step.
//
// Layout (all in HBM, owned by the cloth handle):
//  * per-vertex state as SoA planes of length n: x, v, f_ext, y (translation),
//    mx (last CG solution, the warm start), b, dv, r, p, s, pinv, z, p2 (3
//    planes each), mass (1 plane), type (u8);
//  * the block matrix A in sliced ELL (SELL-32): rows in slices of 32, one
//    slice padded to its widest row; entry (row 32 q + lane, slot k) sits at
//    slice_off[q] + 32 k + lane, so a warp reading slot k of its 32 rows reads
//    32 consecutive words per plane.  Values are 9 planes of E floats
//    (column-major b3Mat33 order), columns one u32 plane.  Slot 0 of every row
//    is its diagonal block; padding slots point at the row itself with zero
//    values;
//  * per-vertex incidence lists (CSR) of the elements touching the vertex, in
//    the order Bounce applies its forces (force list = reverse creation order,
//    src/bounce/cloth/cloth.cpp:353-358), each with the SELL slots of the
//    element's vertices inside the vertex's row.  Assembly is row-owned:
//    one thread owns one row and accumulates only its own row -- no atomics,
//    no colouring, deterministic.  By default every element is evaluated
//    once a step into a record and each block of the row is summed from its
//    own term list; the other form recomputes each incident element per row.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/b3g.h"

namespace b3g {

constexpr int kMaxSpheres = 4;
constexpr int kSlice = 32;
constexpr int kMaxPosIters = 16;  // B3G_MAX_POSITION_ITERATIONS

// Device scalars of one cloth's step (CG state, reductions, contact flags).
struct StepScalars {
    // CG
    double delta;       // current r.P^-1 r
    double delta0;
    double b_delta;
    double pAp;
    float alpha, beta;
    uint32_t iter;
    uint32_t cont;      // 1 while the CG loop should run another iteration
    uint32_t status;    // 0 ok, else b3g_status
    // last-block counters of the grid reductions
    uint32_t ticket[4];
    // contacts: smallest separation of each position iteration, as
    // order-preserving ints (0 = nothing below zero)
    int min_sep[kMaxPosIters];
    uint32_t active_contacts;
    uint32_t contacts;
    // step parameters (written by the host before each step)
    float dt;
    uint32_t vel_iters, pos_iters;
    uint32_t step_index;
    uint32_t max_iter;
    int stop_rule;
    float tol;
    int dot;
    float gx, gy, gz;
};

struct GridBarrier;

// A static collider: a sphere (kind 0), a capsule (kind 1, segment a-b in
// the world frame, its body at the origin) or a convex hull (kind 2, world
// frame, its body at the origin).
struct SphereDev {
    float cx, cy, cz, radius, friction;
    float lo[3], hi[3];   // fat AABB of the shape proxy
    uint32_t kind;        // 0 sphere, 1 capsule, 2 hull
    float ax, ay, az, bx, by, bz;
    const float* hull;    // hull: nhv vertices (3 floats), then nhf planes (normal, offset)
    uint32_t nhv, nhf;
    uint32_t rank;        // position among the shapes a world query reports (new contacts of one
                          // step are listed in that order)
    uint32_t body1;       // 0: a static shape in the world frame (as above); else 1 + the index of
                          // the body it sits on, its geometry (centre, segment, hull) in that
                          // body's frame and its proxy in ClothDev::shape_fat
};

// Ranks the colliders sph[0..count) by the world broadphase's report order
// (cloth_api.cu).
void rank_colliders(SphereDev* sph, uint32_t count);

struct ClothDev {
    uint32_t n, t, ns, nsph;
    uint32_t nslices, max_deg, E;
    const uint32_t* slice_off;  // nslices + 1
    const uint8_t* row_deg;     // n
    const uint32_t* cols;       // E
    float* vals;                // 9 E

    const uint32_t* inc_ptr;    // n + 1
    const uint32_t* inc_elem;   // triangle id; bit 31: spring id; bits 31 and 30: mouse force id
    const uint32_t* inc_meta;   // corner/end (bits 0-1), slots of element vertices (8 bits each from bit 8)

    const uint4* tri;           // v1, v2, v3, 0
    const float4* tri_rest;     // du1, dv1, du2, dv2
    const float2* tri_rest2;    // inv_det, alpha
    const uint2* spr;           // p1, p2 (vertex ids)
    const float4* spr_par;      // L0, ks, kd, 0
    const uint4* mouse_v;       // mouse forces: particle, triangle's v1, v2, v3
    const float4* mouse_par;    // 2 per mouse force: (w2, w3, w4, mouse), (damping, 0, 0, 0)
    uint32_t nmouse;

    float k_stretch, k_shear, k_damp;
    float thickness, friction;  // the triangles' radius and friction (b3ClothDef, cloth.cpp:136-137)
    float *p_radius, *p_friction;  // per particle (b3Particle::m_radius, m_friction), n each

    float *x, *v, *fext, *y, *mx;
    const float* mass;
    uint8_t* type;
    float *b, *dv, *r, *p, *s, *pinv;
    float *z, *p2;              // S P^-1 r and the second direction buffer (persistent CG)
    float *fat_lo, *fat_hi;

    // the assembly's first pass hands the second each row's dfdx first-touch
    // order (slot ids at the row's SELL positions) and its length
    uint8_t *asm_touch, *asm_ntouch;
    // slot-major assembly (slot_asm != 0, the default where the layout
    // allows it): per-element records written once a step by
    // k_elem_records (planes of float4: 15 a triangle, 3 a spring, 5 a
    // mouse force), the per-block term lists (topology.h) read by
    // k_assemble_blocks, and each block's dfdx products with its column's v
    // and y (6 planes of E floats) that k_assemble_rhs sums into b
    uint32_t slot_asm;
    const uint32_t *term_qk, *term_slot, *terms;
    float4 *tri_rec, *spr_rec, *mouse_rec;
    float* asm_kv;

    // contacts, [sphere][vertex]
    uint8_t* c_exists;
    uint8_t* c_active;
    uint32_t* c_key;            // creation key: step index * kMaxSpheres + sphere
    float* c_normal;            // 3 planes of nsph * n
    float* c_t1;
    float* c_t2;
    float* c_imp;               // normal, tangent x, tangent y
    float* c_point;             // capsules: the shape point of the contact (3 planes of nsph * n)
    SphereDev sph[kMaxSpheres];
    b3g_body_state* bodies;     // the bodies of body colliders (device copies), nbody of them
    float* shape_fat;           // per collider its world-broadphase proxy (lo xyz, hi xyz); body shapes only
    uint32_t nbody;
    // the soft body's MPCG mode of the persistent CG (a soft body's system
    // viewed as a ClothDev): x0 unfiltered, b_delta with diag(A), which
    // cg_diag holds (3 planes); 0 for cloths
    uint32_t cg_soft;
    const float* cg_diag;

    StepScalars* sc;
    GridBarrier* bar;           // persistent-CG grid barrier
    void* partials;             // reduction partials, >= max(grid, persistent CG blocks) * 32 bytes
    uint32_t grid;              // blocks of the row kernels
    uint32_t block;             // threads of the row kernels

    // self-collision (thickness > 0, single cloths only; null otherwise):
    // triangle fat AABBs (3 planes of t each) and the broadphase move buffer
    // as flags, and the particles whose particle-triangle contacts a type
    // change dropped (removed at the next contact update)
    float *tri_lo, *tri_hi;
    uint8_t *t_moved, *p_moved, *p_purge;
};

// A launch over several cloths: global thread g works on row
// g - prefix[k] of descs[k], where prefix[k] <= g < prefix[k + 1].
struct RowSpan {
    const ClothDev* descs;      // device array of count cloth descriptors
    const uint32_t* prefix;     // device array of count + 1 row offsets
    uint32_t count, total, max_deg;
    uint32_t hulls;             // nonzero when some cloth has a hull collider
    uint32_t slot_asm;          // nonzero when every cloth has the slot-major assembly
    const uint32_t* eprefix;    // device array of count + 1 element offsets (triangles, springs, mouse forces)
    uint32_t etotal;
};

cudaError_t launch_span_contacts_update(const RowSpan& sp, cudaStream_t st);
cudaError_t launch_span_assemble(const RowSpan& sp, int block, cudaStream_t st);
cudaError_t launch_span_finalize(const RowSpan& sp, cudaStream_t st);
cudaError_t launch_span_contact_position(const RowSpan& sp, uint32_t it, cudaStream_t st);
cudaError_t launch_span_post(const RowSpan& sp, cudaStream_t st);

// A ray p1 -> p2 against the cloth's triangles (b3Cloth::RayCast /
// RayCastSingle): `best` is device scratch for the winning (fraction,
// triangle) key, `out` receives the result.
struct RayHit {
    uint32_t hit, triangle;
    float fraction;
    float normal[3];
};
struct RayQuery {
    float p1[3], p2[3], max_fraction;
    unsigned long long* best;
    RayHit* out;
};
cudaError_t launch_ray_cast(const ClothDev& c, const RayQuery& q, cudaStream_t st);
// The result kernel alone, for a key already in q.best (one triangle).
cudaError_t launch_ray_result(const ClothDev& c, const RayQuery& q, cudaStream_t st);

// Host launchers (cloth_kernels.cu).  The assembly's two kernels need
// assemble_smem_bytes() of dynamic shared memory; a block size <= 0 asks for
// assemble_block_for() of the rows' widest degree.
size_t assemble_smem_bytes(uint32_t max_deg, int block);
int assemble_block_for(uint32_t max_deg, bool multi);
cudaError_t launch_contacts_update(const ClothDev& c, cudaStream_t st);
cudaError_t launch_assemble(const ClothDev& c, int block, cudaStream_t st);
// CG kernels: when use_graph is set, the reduction tail of init/update sets
// the while-node condition `cond`; otherwise every iteration kernel returns
// early once the device flag StepScalars::cont is 0.
cudaError_t launch_cg_init(const ClothDev& c, int dot, cudaGraphConditionalHandle cond, int use_graph,
                           cudaStream_t st);
cudaError_t launch_cg_iteration(const ClothDev& c, int dot, cudaGraphConditionalHandle cond, int use_graph,
                                cudaStream_t st);
// The three kernels of one CG iteration, one at a time (profiling).
cudaError_t launch_cg_part(const ClothDev& c, int dot, int part, cudaStream_t st);
cudaError_t launch_finalize(const ClothDev& c, cudaStream_t st);
// xyz per particle <-> three planes (host transfers go through the staging buffer)
cudaError_t launch_planes_to_xyz(const float* planes, float* xyz, uint32_t n, cudaStream_t st);
cudaError_t launch_xyz_to_planes(const float* xyz, float* planes, uint32_t n, cudaStream_t st);
cudaError_t launch_contact_position(const ClothDev& c, uint32_t it, cudaStream_t st);
cudaError_t launch_post(const ClothDev& c, cudaStream_t st);

// Sequential particle edits (set type / position / velocity, apply force /
// translation) in call order, and whole-cloth array forms.
struct ParticleOp {
    uint32_t vertex, kind;
    float a[3];
};
enum {
    OP_SET_TYPE = 0,
    OP_SET_POSITION = 1,
    OP_SET_VELOCITY = 2,
    OP_APPLY_FORCE = 3,
    OP_APPLY_TRANSLATION = 4,
    OP_SET_RADIUS = 5,
    OP_SET_FRICTION = 6
};
cudaError_t launch_particle_ops(const ClothDev& c, const ParticleOp* ops, uint32_t count, cudaStream_t st);
cudaError_t launch_set_types(const ClothDev& c, const uint8_t* types, cudaStream_t st);
cudaError_t launch_add_vectors(const ClothDev& c, float* dst_planes, const float* src_xyz, int only_dynamic,
                               cudaStream_t st);
cudaError_t launch_clear_contacts(const ClothDev& c, cudaStream_t st);

uint64_t kernel_launches();
void count_launches(uint64_t k);

}  // namespace b3g
