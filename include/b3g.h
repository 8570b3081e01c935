/*
 * b3g -- B200-native implicit cloth step with Bounce's b3Cloth semantics.
 *
 * C ABI of libb3g.so.  Every call returns a b3g_status; nothing aborts.  A
 * cloth handle owns its device buffers and one CUDA stream; host pointers are
 * borrowed for the duration of a call.  Distinct handles may be used from
 * distinct host threads; one handle is not re-entrant.  There is no CPU
 * fallback: without a usable CUDA device, b3g_cloth_create returns
 * B3G_ERR_NO_DEVICE.
 *
 * Reference interfaces each entry point replaces are cited as path:line
 * within the Bounce source tree (Kazade/bounce).
 */
#ifndef B3G_H
#define B3G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    B3G_OK = 0,
    B3G_ERR_INVALID_ARGUMENT = 1, /* null pointer, index out of range, bad option */
    B3G_ERR_DEGENERATE_MESH = 2,  /* zero-area triangle, zero-length edge, vertex index out of range */
    B3G_ERR_NO_DEVICE = 3,        /* no CUDA device / driver */
    B3G_ERR_OUT_OF_MEMORY = 4,    /* device or host allocation failed */
    B3G_ERR_CUDA = 5,             /* any other CUDA runtime error */
    B3G_ERR_NUMERICAL = 6,        /* NaN/Inf in the CG scalars (breakdown) */
    B3G_ERR_TIMEOUT = 7,          /* a bounded device-side wait gave up */
    B3G_ERR_CAPACITY = 8,         /* request above a fixed capacity (spheres, batch slots, budget) */
    B3G_ERR_UNSUPPORTED = 9       /* mesh feature outside what the kernels handle (vertex degree) */
} b3g_status;

/* b3ParticleType (include/bounce/cloth/particle.h:27-32) */
typedef enum { B3G_STATIC = 0, B3G_KINEMATIC = 1, B3G_DYNAMIC = 2 } b3g_particle_type;

/* b3ClothMesh (include/bounce/cloth/cloth_mesh.h:43-53): vertices as xyz
 * triples, triangles as vertex triples, sewing lines as (s1, s2, v1, v2). */
typedef struct {
    uint32_t vertex_count;
    const float* vertices;
    uint32_t triangle_count;
    const uint32_t* triangles;
    uint32_t sewing_line_count;
    const uint32_t* sewing_lines;
} b3g_mesh_desc;

/* b3ClothDef (include/bounce/cloth/cloth.h:56-95) */
typedef struct {
    float density;
    float streching;
    float shearing;
    float bending;
    float sewing;
    float damping;
    float thickness;
    float friction;
} b3g_cloth_def;

/* CG stop rule.  REFERENCE is b3SolveMPCG's own rule
 * (src/bounce/cloth/cloth_force_solver.cpp:105-113): at most max_iterations
 * (the reference fixes 20) and delta <= FLT_EPSILON^2 * b_delta.  RELATIVE
 * stops at sqrt(delta / b_delta) <= tolerance. */
typedef enum { B3G_STOP_REFERENCE = 0, B3G_STOP_RELATIVE = 1 } b3g_stop_rule;

/* Accumulation of the CG inner products (alpha, beta, residual). */
typedef enum { B3G_DOT_F32 = 0, B3G_DOT_COMPENSATED = 1, B3G_DOT_F64 = 2 } b3g_dot_mode;

typedef struct {
    b3g_stop_rule stop_rule;
    float tolerance;          /* RELATIVE only */
    uint32_t max_iterations;  /* >= 1 */
    b3g_dot_mode dot;
} b3g_solver_opts;

typedef struct {
    uint32_t iterations;      /* CG iterations of the last step */
    double delta0;            /* r^T P^-1 r at CG start */
    double delta;             /* r^T P^-1 r at CG exit */
    double b_delta;           /* filtered b^T P^-1 b */
    uint32_t active_contacts; /* body contacts handed to the contact solver */
    uint32_t contacts;        /* body contacts alive after the step */
    float step_ms;            /* device time of the step (CUDA events) */
} b3g_step_stats;

typedef struct b3g_cloth b3g_cloth;

/* ---- cloth lifetime ---------------------------------------------------- */

/* b3Cloth::b3Cloth (src/bounce/cloth/cloth.cpp:96-266): lumped masses,
 * rest-state triangle frames, one stretch and one shear element per triangle,
 * a bending spring per edge-adjacent triangle pair, a spring per sewing line.
 * The mesh is copied; it need not outlive the call. */
b3g_status b3g_cloth_create(const b3g_mesh_desc* mesh, const b3g_cloth_def* def, int device,
                            b3g_cloth** out);
/* b3Cloth::~b3Cloth (cloth.cpp:268-288) */
b3g_status b3g_cloth_destroy(b3g_cloth* cloth);

/* ---- configuration ----------------------------------------------------- */

/* b3Cloth::SetGravity / GetGravity (include/bounce/cloth/cloth.h:106-110) */
b3g_status b3g_cloth_set_gravity(b3g_cloth* cloth, const float gravity[3]);
b3g_status b3g_cloth_get_gravity(const b3g_cloth* cloth, float gravity[3]);
b3g_status b3g_cloth_set_solver(b3g_cloth* cloth, const b3g_solver_opts* opts);
/* A static sphere collider: b3Cloth::SetWorld (cloth.cpp:290) with a static
 * b3Body carrying a b3SphereShape (src/bounce/dynamics/shapes/sphere_shape.cpp).
 * At most B3G_MAX_SPHERES per cloth. */
#define B3G_MAX_SPHERES 4
b3g_status b3g_cloth_add_static_sphere(b3g_cloth* cloth, const float center[3], float radius,
                                       float friction, uint32_t* shape_id);
/* b3Cloth::SetWorld(nullptr): drop every collider and its contacts. */
/* A static capsule collider (b3CapsuleShape, include/bounce/dynamics/shapes/
 * capsule_shape.h) on a static body at the origin: segment a-b in world
 * coordinates, `radius`; contacts as b3CapsuleShape::TestSphere
 * (src/bounce/dynamics/shapes/capsule_shape.cpp:186-284).  Shares the
 * collider capacity with spheres. */
b3g_status b3g_cloth_add_static_capsule(b3g_cloth* cloth, const float a[3], const float b[3], float radius,
                                        float friction, uint32_t* shape_id);
/* A static convex hull collider (b3HullShape, include/bounce/dynamics/shapes/
 * hull_shape.h) on a static body at the origin: `vertices` (3 floats each)
 * and face planes (`planes`: normal xyz and offset, 4 floats each) in world
 * coordinates, hull radius 0 (B3_HULL_RADIUS); contacts as
 * b3HullShape::TestSphere (src/bounce/dynamics/shapes/hull_shape.cpp:187-254,
 * GJK from src/bounce/collision/gjk/gjk.cpp:579-740).  At most 4096 vertices
 * and faces.  Shares the collider capacity with spheres and capsules. */
b3g_status b3g_cloth_add_static_hull(b3g_cloth* cloth, const float* vertices, uint32_t vertex_count,
                                     const float* planes, uint32_t face_count, float friction, uint32_t* shape_id);
b3g_status b3g_cloth_clear_colliders(b3g_cloth* cloth);

/* ---- colliders on bodies -------------------------------------------------- */

/* Colliders on rigid bodies of any type, for a cloth in a world whose bodies
 * move (b3Cloth::SetWorld with b3Body, include/bounce/dynamics/body.h).  The
 * caller's world keeps stepping the bodies; before each cloth step the caller
 * gives the cloth every body's state and every body shape's broadphase proxy
 * as its world has them, and after the step reads them back: the cloth's
 * contact solver changes dynamic bodies' velocities and sweeps
 * (cloth_contact_solver.cpp:264-307, 388-472, 620-718) and synchronises the
 * transform, world inverse inertia and proxies of every non-static body it
 * touched (cloth_solver.cpp:165-181).  A cloth with any body collider solves
 * its body contacts in one ordered pass over its contact list on the GPU,
 * as the reference does: correct for any body type, and serial.  Not with
 * self-collision (thickness > 0), in a batch or in a server. */
typedef struct {
    int32_t type;                 /* b3BodyType: 0 static, 1 kinematic, 2 dynamic */
    float rotation[9];            /* m_xf.rotation, column-major */
    float position[3];            /* m_xf.position */
    float local_center[3];        /* m_sweep.localCenter */
    float world_center0[3];       /* m_sweep.worldCenter0 */
    float world_center[3];        /* m_sweep.worldCenter */
    float orientation0[4];        /* m_sweep.orientation0, x y z w */
    float orientation[4];         /* m_sweep.orientation */
    float linear_velocity[3];
    float angular_velocity[3];
    float inv_mass;               /* m_invMass */
    float inv_inertia[9];         /* m_invI, body frame, column-major */
    float world_inv_inertia[9];   /* m_worldInvI */
} b3g_body_state;

b3g_status b3g_cloth_add_body(b3g_cloth* cloth, const b3g_body_state* state, uint32_t* body_id);
b3g_status b3g_cloth_set_body(b3g_cloth* cloth, uint32_t body_id, const b3g_body_state* state);
b3g_status b3g_cloth_get_body(const b3g_cloth* cloth, uint32_t body_id, b3g_body_state* state);
/* Shapes on a body, geometry in the body's frame (b3SphereShape,
 * b3CapsuleShape, b3HullShape); each takes a collider slot (shape_id, shared
 * with the static colliders) and starts with the proxy
 * ComputeAABB(m_xf) fattened by B3_AABB_EXTENSION. */
b3g_status b3g_cloth_add_body_sphere(b3g_cloth* cloth, uint32_t body_id, const float center[3], float radius,
                                     float friction, uint32_t* shape_id);
b3g_status b3g_cloth_add_body_capsule(b3g_cloth* cloth, uint32_t body_id, const float a[3], const float b[3],
                                      float radius, float friction, uint32_t* shape_id);
b3g_status b3g_cloth_add_body_hull(b3g_cloth* cloth, uint32_t body_id, const float* vertices, uint32_t vertex_count,
                                   const float* planes, uint32_t face_count, float friction, uint32_t* shape_id);
/* A body shape's proxy in the caller's world broadphase (b3Shape::GetAABB). */
b3g_status b3g_cloth_set_shape_proxy(b3g_cloth* cloth, uint32_t shape_id, const float lo[3], const float hi[3]);
b3g_status b3g_cloth_get_shape_proxy(const b3g_cloth* cloth, uint32_t shape_id, float lo[3], float hi[3]);
/* The order in which the caller's world query reports the colliders
 * (b3World::QueryAABB walks its dynamic tree): a particle's new contacts with
 * several colliders in one step enter the contact list in that order.  By
 * default the order is derived from the colliders' proxies inserted into a
 * tree in creation order, which is the world's own while its proxies have
 * not moved; with moving bodies give the world's order before each step.
 * count 0 returns to the derived order. */
b3g_status b3g_cloth_set_report_order(b3g_cloth* cloth, const uint32_t* order, uint32_t count);

/* ---- created particles and mouse forces ------------------------------------ */

/* b3ParticleDef (include/bounce/cloth/particle.h:38-60).  mass 0 makes a
 * static particle (of mass 1, particle.cpp:34-39).  radius and friction are
 * the particle's own (b3g_particle_set_radius). */
typedef struct {
    float position[3];
    float velocity[3];
    float force[3];
    float mass;
    float radius;
    float friction;
} b3g_particle_def;

/* b3Cloth::CreateParticle (src/bounce/cloth/cloth.cpp:307-322): the new
 * particle's index follows every existing particle; use it with the
 * b3g_particle_* calls.  The cloth's layout is rebuilt around its state. */
b3g_status b3g_cloth_create_particle(b3g_cloth* cloth, const b3g_particle_def* def, uint32_t* index);
/* b3Cloth::DestroyParticle (cloth.cpp:324-351), created particles only: its
 * mouse forces and contacts go with it; particles created after it move
 * down one index. */
b3g_status b3g_cloth_destroy_particle(b3g_cloth* cloth, uint32_t index);

/* b3MouseForceDef (include/bounce/cloth/forces/mouse_force.h:26-40): particle
 * `particle` tied by a spring of stiffness `mouse` and damping `damping` to
 * the point w2 x(v1) + w3 x(v2) + w4 x(v3) of `triangle`. */
typedef struct {
    uint32_t particle, triangle;
    float w2, w3, w4;
    float mouse, damping;
} b3g_mouse_force_def;

/* b3Cloth::CreateForce (cloth.cpp:353-358) of a mouse force, applied before
 * every earlier force (mouse_force.cpp:63-227); returns an id for
 * b3g_cloth_destroy_force.  b3Cloth::DestroyForce (cloth.cpp:360-364).
 * Cloths that a server owns cannot take created particles or forces. */
b3g_status b3g_cloth_create_mouse_force(b3g_cloth* cloth, const b3g_mouse_force_def* def, uint32_t* force_id);
b3g_status b3g_cloth_destroy_force(b3g_cloth* cloth, uint32_t force_id);

/* ---- particles (include/bounce/cloth/particle.h:63-111) ------------------ */

b3g_status b3g_particle_set_type(b3g_cloth* cloth, uint32_t vertex, b3g_particle_type type);
b3g_status b3g_particle_get_type(const b3g_cloth* cloth, uint32_t vertex, b3g_particle_type* type);
b3g_status b3g_particle_set_position(b3g_cloth* cloth, uint32_t vertex, const float position[3]);
b3g_status b3g_particle_get_position(const b3g_cloth* cloth, uint32_t vertex, float position[3]);
b3g_status b3g_particle_set_velocity(b3g_cloth* cloth, uint32_t vertex, const float velocity[3]);
b3g_status b3g_particle_get_velocity(const b3g_cloth* cloth, uint32_t vertex, float velocity[3]);
b3g_status b3g_particle_get_mass(const b3g_cloth* cloth, uint32_t vertex, float* mass);
b3g_status b3g_particle_apply_force(b3g_cloth* cloth, uint32_t vertex, const float force[3]);
b3g_status b3g_particle_apply_translation(b3g_cloth* cloth, uint32_t vertex, const float translation[3]);
/* b3Particle::SetRadius / GetRadius, SetFriction / GetFriction (particle.h:
 * 93-102, 240-260).  A particle starts with the cloth's thickness and
 * friction.  The radius enters its body contacts (b3ParticleBodyContact::
 * Update, cloth_particle_body_contact.cpp:24-47, and the position solve) and
 * its proxy, which SetRadius moves (Synchronize(0)); the friction enters
 * b3MixFriction with the shape's.  On a cloth created with thickness > 0 both
 * also enter its particle-triangle contacts.  A cloth created with thickness
 * 0 runs no particle-triangle contacts at all, even when a particle's radius
 * is set above 0 (the reference would then test them).  Radius and friction
 * must be finite and >= 0. */
b3g_status b3g_particle_set_radius(b3g_cloth* cloth, uint32_t vertex, float radius);
b3g_status b3g_particle_get_radius(const b3g_cloth* cloth, uint32_t vertex, float* radius);
b3g_status b3g_particle_set_friction(b3g_cloth* cloth, uint32_t vertex, float friction);
b3g_status b3g_particle_get_friction(const b3g_cloth* cloth, uint32_t vertex, float* friction);

/* Whole-cloth forms of the particle calls: arrays of 3 * vertex_count floats
 * (xyz per vertex) or vertex_count types, host memory. */
b3g_status b3g_cloth_set_types(b3g_cloth* cloth, const uint8_t* types);
b3g_status b3g_cloth_apply_forces(b3g_cloth* cloth, const float* forces);
b3g_status b3g_cloth_apply_translations(b3g_cloth* cloth, const float* translations);

/* ---- step ----------------------------------------------------------------- */

/* b3Cloth::Step (cloth.cpp:551-601): body-contact update, force/Jacobian
 * assembly, S-filtered Jacobi-preconditioned CG, contact velocity and position
 * iterations, AABB sync, new body contacts; at thickness > 0 also the
 * particle-triangle contacts (self-collision).  stats may be NULL.  The step
 * is enqueued and waited for.  At most B3G_MAX_POSITION_ITERATIONS position
 * iterations (the reference takes any number; more than that returns
 * B3G_ERR_INVALID_ARGUMENT, here and in every other step call). */
#define B3G_MAX_POSITION_ITERATIONS 16
b3g_status b3g_cloth_step(b3g_cloth* cloth, float dt, uint32_t velocity_iterations,
                          uint32_t position_iterations, b3g_step_stats* stats);

/* How one cloth's CG runs on the GPU.  LAUNCHES (default): three kernels
 * per iteration inside a CUDA-graph while loop.  PERSISTENT: one cooperative
 * launch for the whole solve, two grid reductions per iteration, separated by
 * grid barriers with bounded waits (B3G_ERR_TIMEOUT if one gives up); for
 * large cloths.  PERSISTENT_FUSED: as PERSISTENT with one grid reduction per
 * iteration.  Each vertex publishes r, s and p once per iteration, and every
 * row forms its neighbours' next direction from them.  The reduction returns
 * p.s, s.z, s.P^-1 s and r.z (z = S P^-1 r) of the iterate: alpha = r.z / p.s
 * as the reference's, and the next r.z expanded as
 * r.z - 2 alpha s.z + alpha^2 s.P^-1 s gives beta and the stop test.  So x, r,
 * z and p follow the reference's expressions and only beta's numerator
 * rounds differently; the next iteration recomputes r.z exactly, and a pass
 * whose exact r.z already meets the stop rule is discarded.  It needs a
 * device buffer of 96 bytes per vertex, allocated when the strategy is set. */
typedef enum { B3G_CG_LAUNCHES = 0, B3G_CG_PERSISTENT = 1, B3G_CG_PERSISTENT_FUSED = 2 } b3g_cg_strategy;
b3g_status b3g_cloth_set_cg_strategy(b3g_cloth* cloth, b3g_cg_strategy strategy);

/* How one cloth's system (b3ClothForceSolver::Solve's forces, Jacobians, A,
 * b and P^-1, cloth_force_solver.cpp:142-204) is assembled on the GPU; both
 * forms give the same floats.  ELEMENT_RECORDS (the default where the layout
 * allows it: rows of at most 16 blocks, under 2^26 triangles and springs):
 * every element evaluated once a step into a record, then each block of A
 * summed from the terms of the elements that couple its row and column, in
 * the reference's order.  ROWS: each row recomputes its incident elements,
 * in two passes.  The records and term lists take about 240 bytes a
 * triangle, 48 a spring and 4 a block term of the cloth's arena.
 * b3g_cloth_get_assembly returns the form in use (ROWS where the layout
 * does not allow the records).  A batch (and a server) assembles with the
 * records when every cloth it steps has them and their records take at
 * most 64 MB, so that they stay in L2 between the launch that writes them
 * and the launches that read them; otherwise row by row.  A server lays its
 * cloths out without the records (row by row), which leaves more of its HBM
 * budget for cloths. */
typedef enum { B3G_ASSEMBLY_ELEMENT_RECORDS = 0, B3G_ASSEMBLY_ROWS = 1 } b3g_assembly;
b3g_status b3g_cloth_set_assembly(b3g_cloth* cloth, b3g_assembly form);
b3g_assembly b3g_cloth_get_assembly(const b3g_cloth* cloth);
/* Diagnostic of the bounded waits: runs the persistent CG once with a grid
 * barrier that can never complete and a wait limit of spin_limit polls;
 * *result receives the solve status (B3G_ERR_TIMEOUT when the limit works).
 * The cloth's state is not changed. */
b3g_status b3g_debug_cg_barrier_timeout(b3g_cloth* cloth, uint32_t spin_limit, b3g_status* result);

/* Device time per kernel of one step, for roofline accounting: the same step
 * as b3g_cloth_step, launched kernel by kernel (no graph) with CUDA events
 * around each launch on the cloth's stream.  Sums over the step's launches. */
typedef struct {
    float contacts_update_ms;
    float assemble_ms;
    float cg_init_ms;
    float cg_spmv_ms;       /* all iterations */
    float cg_update_ms;     /* all iterations */
    float cg_direction_ms;  /* all iterations */
    float finalize_ms;
    float contact_position_ms;
    float post_ms;
    uint32_t cg_iterations;
    uint32_t contact_position_launches;
} b3g_phase_times;

b3g_status b3g_cloth_step_profiled(b3g_cloth* cloth, float dt, uint32_t velocity_iterations,
                                   uint32_t position_iterations, b3g_phase_times* times,
                                   b3g_step_stats* stats);

/* Bytes of the device-resident system: padded SELL-32 entries, unpadded
 * blocks, vertices, triangles, springs. */
typedef struct {
    uint32_t vertices, triangles, springs, blocks, sell_entries, max_degree;
} b3g_cloth_info;
b3g_status b3g_cloth_get_info(const b3g_cloth* cloth, b3g_cloth_info* info);

/* ---- state ---------------------------------------------------------------- */

uint32_t b3g_cloth_vertex_count(const b3g_cloth* cloth);
/* positions / velocities / last CG solution (b3Particle::m_x), 3 floats per
 * vertex; any pointer may be NULL. */
b3g_status b3g_cloth_read_state(const b3g_cloth* cloth, float* positions, float* velocities,
                                float* cg_solution);
b3g_status b3g_cloth_write_state(b3g_cloth* cloth, const float* positions, const float* velocities,
                                 const float* cg_solution);
b3g_status b3g_cloth_read_masses(const b3g_cloth* cloth, float* masses);
/* b3Cloth::GetEnergy (cloth.cpp:366-374) */
b3g_status b3g_cloth_get_energy(const b3g_cloth* cloth, float* energy);
/* Body contacts per vertex and collider: exists, active (vertex_count *
 * sphere_count bytes each), impulses (normal, tangent1, tangent2). */
b3g_status b3g_cloth_read_contacts(const b3g_cloth* cloth, uint8_t* exists, uint8_t* active,
                                   float* impulses);
/* The particles' broadphase proxies (b3Particle's fat AABB, cloth.cpp:
 * 312-317, moved by b3Particle::Synchronize as in b3ClothSolver, and read by
 * the body-contact lifetime test): lower and upper corners, 3 floats per
 * vertex; either pointer may be NULL. */
b3g_status b3g_cloth_read_proxies(const b3g_cloth* cloth, float* lo, float* hi);
/* Self-collision: the particle-triangle contacts of a cloth whose thickness
 * is above zero (b3ClothContactManager::m_particleTriangleContactList,
 * include/bounce/cloth/cloth_contact_manager.h; b3ParticleTriangleContact,
 * include/bounce/cloth/contacts/cloth_particle_triangle_contact.h), in list
 * order (head first).  *count gets the list length; each non-null array gets
 * per contact: the particle and triangle (2 u32), the active flag, the
 * barycentric weights m_w2, m_w3, m_w4 (zero while inactive) and the normal
 * and two tangent impulses.  A cloth of thickness 0 has no such contacts.
 * Cloths with self-collision take neither created particles nor mouse forces
 * (B3G_ERR_UNSUPPORTED), and cannot join a batch or a server. */
/* b3Cloth::RayCastSingle (cloth.cpp:466-491): the first triangle the
 * segment p1 -> p2 hits (b3RayCast, src/bounce/collision/collision.cpp:31-118),
 * its fraction along the segment and the normal facing p1.  *hit is 0 when
 * nothing is hit.  Equal fractions go to the lowest triangle index (the
 * reference takes the first its tree visits). */
b3g_status b3g_cloth_ray_cast_single(b3g_cloth* cloth, const float p1[3], const float p2[3], uint32_t* triangle,
                                     float* fraction, float normal[3], int* hit);
/* b3Cloth::RayCast (cloth.cpp:493-503): the segment against one triangle,
 * up to max_fraction. */
b3g_status b3g_cloth_ray_cast(b3g_cloth* cloth, const float p1[3], const float p2[3], float max_fraction,
                              uint32_t triangle, float* fraction, float normal[3], int* hit);
b3g_status b3g_cloth_read_tri_contacts(const b3g_cloth* cloth, uint32_t* count, uint32_t* pairs, uint8_t* active,
                                       float* weights, float* impulses);
/* Of the last step: particle-triangle contacts alive after it, active ones
 * handed to its contact solve, and the dependency levels that solve ran. */
b3g_status b3g_cloth_get_self_stats(const b3g_cloth* cloth, uint32_t* contacts, uint32_t* active,
                                    uint32_t* levels);
b3g_status b3g_cloth_last_stats(const b3g_cloth* cloth, b3g_step_stats* stats);

/* ---- inspection of the assembled system ----------------------------------- */

/* The block-sparse system of the last step (or b3g_cloth_assemble), A = M - h dfdv - h^2 dfdx and
 * b = h (f + h dfdx v + dfdx y) (cloth_force_solver.cpp:193-204), as
 * block CSR by vertex: rowptr (n + 1), cols (nnz), vals (9 floats per block,
 * column-major like b3Mat33), b (3 n), filter S (n, 1 or 0), warm start x0 (3 n).
 * Call with vals == NULL to get nnz only. */
b3g_status b3g_cloth_read_system(const b3g_cloth* cloth, uint32_t* nnz, uint32_t* rowptr,
                                 uint32_t* cols, float* vals, float* b, float* S, float* x0);

/* Assemble A, b and P^-1 from the current state for a step of dt without
 * changing the state (the first half of b3ClothForceSolver::Solve,
 * cloth_force_solver.cpp:142-204); read them with b3g_cloth_read_system. */
b3g_status b3g_cloth_assemble(b3g_cloth* cloth, float dt);

/* ---- standalone MPCG -------------------------------------------------------- */

/* b3SolveMPCG (cloth_force_solver.cpp:61-136) on a caller-supplied system in
 * DEVICE memory: block CSR (rowptr n + 1, cols nnz, vals 9 per block,
 * column-major), b (3 n), S (n floats, 1 or 0), x0 (3 n) -> x (3 n).  Device
 * scratch is allocated per call.  iterations and stats may be NULL. */
b3g_status b3g_mpcg_solve(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals,
                          const float* b, const float* S, const float* x0, const b3g_solver_opts* opts,
                          float* x, uint32_t* iterations, b3g_step_stats* stats, void* stream);

/* b3g_mpcg_solve without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc when they
 * solve -- a game or physics loop that reserves all device memory at level
 * load and forbids allocation inside a frame (cudaMalloc is slow and
 * synchronizes the device), a process whose device memory is already held by
 * another framework's caching allocator, or code running inside its own
 * allocator's callbacks.  Same arguments and results as b3g_mpcg_solve.
 *  - The scratch is one static device array in libb3g.so, sized for at most
 *    B3G_MPCG_NOALLOC_MAX_ROWS block rows (about 3.2 MB); every GPU that
 *    loads the library holds it until the process exits.  Larger systems
 *    return B3G_ERR_CAPACITY.
 *  - The first call on each device looks the array's device address up
 *    (cudaGetSymbolAddress) and keeps it for the life of the process.  A
 *    cudaDeviceReset after it is not supported (the library's module, and
 *    the array with it, may come back at another address).
 *  - Like b3g_mpcg_solve, it is synchronous: it waits for its work to
 *    finish before it returns (the iteration count and residual are read
 *    back to the host), so neither can be captured into a CUDA graph.
 *  - All calls share the one array: calls whose work overlaps on the GPU
 *    (other streams, other host threads) race and corrupt each other.  Each
 *    call clears the CG scalars it needs zeroed; other scratch contents are
 *    left from the previous call and overwritten before use. */
#define B3G_MPCG_NOALLOC_MAX_ROWS 65536
b3g_status b3g_mpcg_solve_noalloc(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals,
                                  const float* b, const float* S, const float* x0, const b3g_solver_opts* opts,
                                  float* x, uint32_t* iterations, b3g_step_stats* stats, void* stream);

/* ---- batches: many cloths per launch ---------------------------------------- */

/* No single reference counterpart: the reference steps each b3Cloth on its
 * own (b3Cloth::Step).  A batch advances many cloths -- of uneven sizes,
 * each with its own parameters, solver options and colliders -- by one
 * b3Cloth::Step each, in a fixed number of launches captured in a CUDA
 * graph: the per-row kernels cover every row of every cloth, the CG is one
 * persistent launch that runs one cloth per CTA (block-per-instance) or per
 * thread-block cluster (split-instance).  Each cloth's results are the same
 * as when it is stepped alone in the same batch object (fixed reduction
 * trees per cloth). */
typedef struct b3g_batch b3g_batch;

typedef struct {
    uint32_t cluster;          /* CTAs per cluster of the CG launch: 1, 2, 4 or 8 */
    uint8_t split_class[32];   /* per size class floor(log2(vertices)): 1 = split over a cluster */
    float tuned_cg_ms;         /* CG time the autotuner measured for this schedule */
} b3g_batch_schedule;

typedef struct {
    uint32_t count;                /* cloths stepped */
    uint32_t rows;                 /* their vertices */
    uint32_t tasks;                /* CG work items */
    uint32_t cg_iterations_total;
    uint32_t cg_iterations_max;
    float step_ms;                 /* device time of the whole batch step (CUDA events) */
    float cg_ms;                   /* device time of its batched CG launch */
} b3g_batch_stats;

/* capacity: most cloths one step call may pass */
b3g_status b3g_batch_create(int device, uint32_t capacity, b3g_batch** out);
b3g_status b3g_batch_destroy(b3g_batch* batch);
/* One b3Cloth::Step (dt, velocity and position iterations) of each listed
 * cloth; per_cloth (count entries) and stats may be NULL.  A cloth may be
 * listed once per call; all must live on the batch's device. */
b3g_status b3g_batch_step(b3g_batch* batch, b3g_cloth* const* cloths, uint32_t count, float dt,
                          uint32_t velocity_iterations, uint32_t position_iterations,
                          b3g_step_stats* per_cloth, b3g_batch_stats* stats);
b3g_status b3g_batch_set_schedule(b3g_batch* batch, const b3g_batch_schedule* schedule);
b3g_status b3g_batch_get_schedule(const b3g_batch* batch, b3g_batch_schedule* schedule);
/* Project autotuner: times the batched CG on these cloths' current systems
 * for cluster sizes 1/2/4/8, each with no class split and with every size
 * class at or above a threshold split over a cluster (block-per-instance
 * below it), for each threshold; keeps the fastest schedule.  Setting the
 * environment variable B3G_TRACE_AUTOTUNE=1 prints every timed candidate to
 * stderr.  Cloth state is not changed. */
b3g_status b3g_batch_autotune(b3g_batch* batch, b3g_cloth* const* cloths, uint32_t count, float dt,
                              b3g_batch_schedule* out);

/* ---- serving: continuous batching of cloth-step requests --------------------- */

/* No reference counterpart (the reference is a single-threaded library).
 * A server takes requests -- a cloth and a number of b3Cloth::Step calls --
 * builds their topology on host worker threads, admits them in arrival order
 * while an HBM budget and a slot limit allow, keeps their state resident on
 * the device, and on every tick advances all admitted cloths by one step in
 * one batched launch sequence.  Requests that arrive while others are in
 * flight join the next tick.  Finished cloths are copied back to the host
 * and their device memory returns to the server's pool.  Each request's
 * result is the same alone and in any mix (fixed batch schedule). */
typedef struct b3g_server b3g_server;

typedef struct {
    uint64_t hbm_budget_bytes;       /* admission cap on resident cloth memory */
    uint32_t max_active;             /* most cloths in flight */
    float dt;
    uint32_t velocity_iterations;
    uint32_t position_iterations;
    float gravity[3];
    b3g_solver_opts solver;          /* max_iterations 0: relative 1e-4, at most 200, FP64 dots */
    b3g_batch_schedule schedule;     /* cluster 0: block-per-instance */
    uint32_t host_threads;           /* topology worker threads, 0: one per core but one */
} b3g_server_config;

typedef struct {
    uint32_t admitted, stepped, completed, active, queued, rows;
    uint64_t bytes_used;
    float tick_ms;                   /* device time of this tick's batched step */
} b3g_server_tick_info;

/* state: 0 queued, 1 prepared, 2 active, 3 done, 4 failed */
typedef struct {
    uint32_t state;
    b3g_status status;
    uint32_t steps_done, steps_total, vertex_count;
    double arrival, admitted, finished;   /* in the caller's clock (submit / tick `now`) */
    uint64_t bytes;
} b3g_request_info;

typedef struct {
    uint64_t ticks, steps, vertex_steps, admitted, completed, rejected;
    double busy_ms;                  /* summed device time of all ticks */
    uint32_t active, queued, peak_active;
    uint64_t peak_bytes;
    float p50_step_ms, p99_step_ms, max_step_ms;  /* per request-step latency */
} b3g_server_statistics;

b3g_status b3g_server_create(int device, const b3g_server_config* config, b3g_server** out);
b3g_status b3g_server_destroy(b3g_server* server);
/* types: vertex_count particle types or NULL (all dynamic); spheres: 5 floats
 * each (center xyz, radius, friction).  Thread-safe. */
b3g_status b3g_server_submit(b3g_server* server, const b3g_mesh_desc* mesh, const b3g_cloth_def* def,
                             const uint8_t* types, const float* spheres, uint32_t sphere_count, uint32_t steps,
                             double arrival, uint64_t* request_id);
/* Step every active cloth once; while the device runs the step, admit what
 * fits the budget and the slots (admitted requests step from the next tick
 * on); then retire finished requests. */
b3g_status b3g_server_tick(b3g_server* server, double now, b3g_server_tick_info* info);
b3g_status b3g_server_poll(b3g_server* server, uint64_t request_id, b3g_request_info* info);
/* Final positions (3 floats per vertex) of a finished request. */
b3g_status b3g_server_result(b3g_server* server, uint64_t request_id, float* positions);
b3g_status b3g_server_release(b3g_server* server, uint64_t request_id);
b3g_status b3g_server_stats(const b3g_server* server, b3g_server_statistics* stats);

/* ---- soft bodies ---------------------------------------------------------- */

/* b3SoftBody (include/bounce/softbody/softbody.h, src/bounce/softbody/): a
 * tetrahedral mesh simulated by corotated linear FEM with plasticity and the
 * MPCG of softbody_force_solver.cpp.  The body has no world here, so it has
 * no contacts.  Vectors are 3 floats per node in mesh order. */
typedef struct b3g_softbody b3g_softbody;

/* b3SoftBodyDef (softbody.h:64-99): density, Young's modulus E, Poisson's
 * ratio nu, plastic yield, creep and maximum plastic strain. */
typedef struct {
    float density, E, nu, c_yield, c_creep, c_max;
} b3g_softbody_def;

/* b3SoftBody::b3SoftBody (softbody.cpp:436-553).  tets: 4 vertex ids each
 * (b3SoftBodyMeshTetrahedron).  Every node starts dynamic with zero
 * velocity and zero mass damping; each element's rotation starts at the
 * identity.  B3G_ERR_DEGENERATE_MESH for a zero-volume or repeated-vertex
 * tetrahedron, an id out of range or a vertex no tetrahedron uses. */
b3g_status b3g_softbody_create(uint32_t vertex_count, const float* vertices, uint32_t tet_count,
                               const uint32_t* tets, const b3g_softbody_def* def, int device, b3g_softbody** out);
b3g_status b3g_softbody_destroy(b3g_softbody* body);
uint32_t b3g_softbody_node_count(const b3g_softbody* body);
uint32_t b3g_softbody_element_count(const b3g_softbody* body);
/* b3SoftBody::SetGravity (softbody.h:192-195) */
b3g_status b3g_softbody_set_gravity(b3g_softbody* body, const float* gravity);
/* b3SoftBodyNode::SetType / SetMassDamping / ApplyForce / SetVelocity /
 * SetPosition (softbody_node.h:146-211); type 0 static, 1 kinematic,
 * 2 dynamic.  Applied in order with the steps. */
b3g_status b3g_softbody_set_node_type(b3g_softbody* body, uint32_t node, int type);
b3g_status b3g_softbody_set_mass_damping(b3g_softbody* body, uint32_t node, float damping);
b3g_status b3g_softbody_apply_force(b3g_softbody* body, uint32_t node, const float* force);
b3g_status b3g_softbody_set_velocity(b3g_softbody* body, uint32_t node, const float* velocity);
b3g_status b3g_softbody_set_position(b3g_softbody* body, uint32_t node, const float* position);
/* Default: the reference's MPCG (20 iterations, FLT_EPSILON^2, FP32 dots). */
b3g_status b3g_softbody_set_solver(b3g_softbody* body, const b3g_solver_opts* opts);
/* How the MPCG runs: B3G_CG_PERSISTENT (the default) is one cooperative
 * launch per solve with two grid reductions per iteration, on a copy of the
 * system in the cloth's SELL-32 layout with its rows ordered by degree;
 * B3G_CG_PERSISTENT_FUSED the same with one grid reduction per iteration;
 * B3G_CG_LAUNCHES three launches per iteration on the block-CSR system.
 * All solve the same system by the same rule; their dot products sum in
 * different orders. */
b3g_status b3g_softbody_set_cg_strategy(b3g_softbody* body, b3g_cg_strategy strategy);
/* b3SoftBody::Step (softbody.cpp:700-735) without a world.  stats->delta0 is
 * r.P^-1 r at the CG start, b_delta the soft body's delta_0 (Sb . diag(A) Sb).
 * At most B3G_MAX_POSITION_ITERATIONS position iterations. */
b3g_status b3g_softbody_step(b3g_softbody* body, float dt, uint32_t velocity_iterations,
                             uint32_t position_iterations, b3g_step_stats* stats);
/* b3SoftBody::SetWorld with static hulls (b3HullShape on a static body at the
 * origin; vertices and face planes in world coordinates, as for cloths):
 * node contacts follow b3NodeBodyContact::Update and b3SoftBodyContactSolver
 * (src/bounce/softbody/softbody_contact_manager.cpp,
 * src/bounce/softbody/contacts/softbody_contact_solver.cpp).  At most
 * B3G_MAX_SPHERES hulls per body. */
b3g_status b3g_softbody_add_static_hull(b3g_softbody* body, const float* vertices, uint32_t vertex_count,
                                        const float* planes, uint32_t face_count, float friction, uint32_t* shape_id);
/* b3SoftBodyNode::SetRadius / SetFriction (softbody_node.h:218-235); both 0
 * by default. */
b3g_status b3g_softbody_set_node_radius(b3g_softbody* body, uint32_t node, float radius);
b3g_status b3g_softbody_set_node_friction(b3g_softbody* body, uint32_t node, float friction);
/* Node contacts per (hull, node): exists, active (hull_count * node_count
 * bytes each), impulses (normal, tangent x, tangent y). */
b3g_status b3g_softbody_read_contacts(const b3g_softbody* body, uint8_t* exists, uint8_t* active, float* impulses);
b3g_status b3g_softbody_read_state(const b3g_softbody* body, float* positions, float* velocities);
b3g_status b3g_softbody_write_state(b3g_softbody* body, const float* positions, const float* velocities);
/* Element state: the rotation q (x, y, z, w per element) that the next
 * rotation extraction starts from, and the plastic strain (6 per element). */
b3g_status b3g_softbody_read_elements(const b3g_softbody* body, float* q, float* plastic_strain);
b3g_status b3g_softbody_write_elements(b3g_softbody* body, const float* q, const float* plastic_strain);
b3g_status b3g_softbody_read_masses(const b3g_softbody* body, float* masses);
/* b3SoftBody::GetEnergy (softbody.cpp:627-637) */
b3g_status b3g_softbody_energy(const b3g_softbody* body, float* energy);
/* The system A, b, S of one force solve from the current state, rows in the
 * reference's b3SparseMat33 list order; the state is not changed.  *count
 * receives the block count; nothing is written while capacity < *count. */
b3g_status b3g_softbody_export_system(b3g_softbody* body, float dt, uint32_t capacity, uint32_t* rowptr,
                                      uint32_t* cols, float* vals, float* b, float* S, uint32_t* count);

/* ---- misc ----------------------------------------------------------------- */

const char* b3g_status_string(b3g_status status);
/* Number of kernels this library has launched in this process. */
uint64_t b3g_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif
