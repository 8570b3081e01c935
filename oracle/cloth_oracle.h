/*
 * CPU restatement of Bounce's implicit cloth step (test infrastructure).
 *
 * This library is the parity oracle for the CUDA path in bounce_b200/.  Only
 * the tests, the smoke check and the CPU-baseline leg of bench.py load it; the
 * product never links or calls it.
 *
 * It restates, in plain C99, the reference's
 *   - cloth construction (src/bounce/cloth/cloth.cpp:96-266, :388-427),
 *   - force solve (src/bounce/cloth/cloth_force_solver.cpp:138-222) with the
 *     stretch / shear / spring elements (src/bounce/cloth/forces/strech_force.cpp,
 *     shear_force.cpp, spring_force.cpp),
 *   - MPCG (cloth_force_solver.cpp:61-136),
 *   - body-contact solve (src/bounce/cloth/contacts/cloth_contact_solver.cpp)
 *     and contact lifetime (src/bounce/cloth/cloth_contact_manager.cpp:64-123,
 *     :277-315; src/bounce/collision/broad_phase.cpp:99-149),
 * reproducing the reference's floating-point operation order (force-list
 * order, the row order the linked-list sparse matrices end up in, sequential
 * dot products), so that in reference mode its results are bit-identical to
 * the reference library compiled from source.  Beyond the reference it adds
 * a relative-residual stop rule, a configurable iteration cap, compensated
 * and FP64 dot products, and an FP64 solve of the same linear system.
 */
#ifndef CLOTH_ORACLE_H
#define CLOTH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oc_cloth oc_cloth;

enum { OC_STATIC = 0, OC_KINEMATIC = 1, OC_DYNAMIC = 2 };

/* CG stop rule: OC_STOP_REFERENCE is the reference's
 * delta <= FLT_EPSILON^2 * b_delta; OC_STOP_RELATIVE is
 * sqrt(delta / b_delta) <= tol. */
enum { OC_STOP_REFERENCE = 0, OC_STOP_RELATIVE = 1 };

/* Dot-product accumulation: sequential FP32 (the reference), compensated
 * FP32 (Neumaier), FP64. */
enum { OC_DOT_F32 = 0, OC_DOT_COMPENSATED = 1, OC_DOT_F64 = 2 };

typedef struct {
    uint32_t iterations;     /* CG iterations of the step */
    double delta0;           /* r^T P^-1 r at the start */
    double delta;            /* r^T P^-1 r at exit */
    double b_delta;          /* b^T P^-1 b, filtered */
    uint32_t active_contacts;/* body contacts handed to the solver */
    uint32_t contacts;       /* body contacts alive after the step */
    uint32_t active_tri_contacts; /* particle-triangle contacts handed to the solver */
    uint32_t tri_contacts;        /* particle-triangle contacts alive after the step */
} oc_step_info;

/* def: density, streching, shearing, bending, sewing, damping, thickness, friction */
oc_cloth* oc_create(const float* vertices, uint32_t vertex_count, const uint32_t* triangles,
                    uint32_t triangle_count, const uint32_t* sewing_lines, uint32_t sewing_count,
                    const float* def);
void oc_destroy(oc_cloth* c);

void oc_set_gravity(oc_cloth* c, const float* g);
void oc_set_state(oc_cloth* c, const float* x, const float* v, const float* dv);
/* Replace the body-contact list (tail to head; per contact its particle,
 * shape and 3 impulses) and the particles' fat AABBs (xyz triples). */
void oc_set_contacts(oc_cloth* c, uint32_t count, const uint32_t* particle, const uint32_t* shape,
                     const float* impulses);
void oc_set_proxies(oc_cloth* c, const float* lo, const float* hi);
/* Colliders on bodies: body state as 55 floats (see body_read); shapes with
 * geometry in the body's frame; the shapes' world-broadphase proxies. */
int oc_add_body(oc_cloth* c, const float* desc);
void oc_set_body(oc_cloth* c, uint32_t body, const float* desc);
void oc_get_body(const oc_cloth* c, uint32_t body, float* desc);
int oc_add_body_shape(oc_cloth* c, uint32_t body, int kind, const float* geom, uint32_t nv, uint32_t nf,
                      float radius, float friction);
void oc_set_shape_proxy(oc_cloth* c, uint32_t shape, const float* lo, const float* hi);
void oc_set_report_order(oc_cloth* c, const uint32_t* order, uint32_t count);
void oc_get_shape_proxy(const oc_cloth* c, uint32_t shape, float* lo, float* hi);
void oc_set_type(oc_cloth* c, uint32_t vertex, int type);
void oc_set_radius(oc_cloth* c, uint32_t vertex, float radius);
void oc_set_friction(oc_cloth* c, uint32_t vertex, float friction);
void oc_apply_force(oc_cloth* c, uint32_t vertex, const float* f);
void oc_apply_translation(oc_cloth* c, uint32_t vertex, const float* t);
void oc_set_position(oc_cloth* c, uint32_t vertex, const float* x);
void oc_set_velocity(oc_cloth* c, uint32_t vertex, const float* v);
int oc_add_sphere(oc_cloth* c, const float* center, float radius, float friction);
/* a static capsule collider, segment a-b in the world frame */
int oc_add_capsule(oc_cloth* c, const float* a, const float* b, float radius, float friction);
/* A static hull on a body at the origin: vertices (3 floats each) and face
 * planes (normal, offset: 4 floats each) in the world frame. */
int oc_add_hull(oc_cloth* c, const float* vertices, uint32_t vertex_count, const float* planes, uint32_t face_count,
                float friction);
void oc_set_solver(oc_cloth* c, int stop_rule, float tol, uint32_t max_iterations, int dot);

void oc_step(oc_cloth* c, float dt, uint32_t velocity_iterations, uint32_t position_iterations,
             oc_step_info* info);

void oc_get_state(const oc_cloth* c, float* x, float* v, float* dv, float* mass, uint8_t* type);
float oc_energy(const oc_cloth* c);
uint32_t oc_describe(const oc_cloth* c, float* tri_rest, float* fat_aabb, float* force_desc);
uint32_t oc_get_contacts(const oc_cloth* c, uint8_t* exists, uint8_t* active, float* impulses);
uint32_t oc_get_contact_list(const oc_cloth* c, uint32_t cap, uint32_t* particle, uint32_t* shape, uint8_t* active,
                             float* impulses);
int oc_ray_cast_single(const oc_cloth* c, const float* p1, const float* p2, uint32_t* triangle, float* fraction,
                       float* normal);
uint32_t oc_get_tri_contacts(const oc_cloth* c, uint32_t* pt, uint8_t* active, float* w, float* impulses);
uint32_t oc_force_count(const oc_cloth* c);
uint32_t oc_spring_count(const oc_cloth* c);
/* Springs in creation order: vertex pairs (2 per spring) and rest lengths. */
void oc_get_springs(const oc_cloth* c, uint32_t* pairs, float* rest_length, float* stiffness);

/* Created particles and forces (cloth.cpp:307-364).  A created particle
 * (b3ParticleDef: position, velocity, mass, radius, friction; mass 0 makes
 * it static) takes the index after every existing particle and heads the
 * particle list.  Destroying one (only created particles can be) removes its
 * forces and contacts; particles created after it move down one index.  A
 * mouse force (mouse_force.h:26-40) ties `particle` to the point
 * w2 x(v1) + w3 x(v2) + w4 x(v3) of `triangle` and heads the force list;
 * the returned id names it to oc_destroy_force.  Return 0 / -1 on error. */
uint32_t oc_create_particle(oc_cloth* c, const float* position, const float* velocity, float mass, float radius,
                            float friction);
int oc_destroy_particle(oc_cloth* c, uint32_t particle);
uint32_t oc_create_mouse_force(oc_cloth* c, uint32_t particle, uint32_t triangle, float w2, float w3, float w4,
                               float mouse, float damping);
int oc_destroy_force(oc_cloth* c, uint32_t id);
uint32_t oc_particle_count(const oc_cloth* c);

/* The system one force solve would build (cloth_force_solver.cpp:142-204),
 * rows in solver order, blocks in the reference's row-list order. */
uint32_t oc_build_system(oc_cloth* c, float dt);
void oc_get_system(const oc_cloth* c, uint32_t* rowptr, uint32_t* cols, float* vals, float* b,
                   float* S, float* x0, uint32_t* vertex_of_row);

/* MPCG on a given system (cloth_force_solver.cpp:61-136).  vals holds 9
 * floats per block, column-major; S one 0/1 per row; x0 the warm start.
 * stats (may be NULL): delta0, b_delta, delta.  Returns iterations. */
uint32_t oc_mpcg(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals,
                 const float* b, const float* S, const float* x0, int stop_rule, float tol,
                 uint32_t max_iterations, int dot, float* x, double* stats);

/* FP64 Jacobi-preconditioned filtered CG on the same system, run until
 * sqrt(delta / b_delta) <= tol.  Returns iterations. */
uint32_t oc_solve_f64(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals,
                      const float* b, const float* S, const float* x0, double tol,
                      uint32_t max_iterations, double* x);

#ifdef __cplusplus
}
#endif

#endif
