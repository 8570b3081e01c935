/* CPU restatement of Bounce's soft body step (test infrastructure only).
 *
 * Follows src/bounce/softbody/softbody.cpp (constructor, ComputeMass, Step),
 * softbody_force_solver.cpp (corotated linear FEM with plasticity, MPCG) and
 * softbody_solver.cpp (integration) in the reference's operation order, so
 * that its results equal the reference's bit for bit on the same inputs.
 * Node-body contacts are not restated: a body without a world has none.
 * Only tests and the CPU baseline use it; nothing in the product links it. */
#pragma once

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct os_body os_body;

typedef struct {
    uint32_t iterations;
    double delta0, delta, b_delta;
} os_stats;

/* vertices: 3 floats each; tets: 4 vertex ids each (b3SoftBodyMeshTetrahedron) */
os_body* os_create(uint32_t nv, const float* vertices, uint32_t nt, const uint32_t* tets, float density, float E,
                   float nu, float c_yield, float c_creep, float c_max);
void os_destroy(os_body* b);
uint32_t os_node_count(const os_body* b);
/* 0 static, 1 kinematic, 2 dynamic (b3SoftBodyNodeType) */
void os_set_type(os_body* b, uint32_t i, int type);
void os_set_mass_damping(os_body* b, uint32_t i, float damping);
void os_set_gravity(os_body* b, const float* g);
void os_apply_force(os_body* b, uint32_t i, const float* f);
void os_set_position(os_body* b, uint32_t i, const float* x);
void os_set_velocity(os_body* b, uint32_t i, const float* v);
/* stop_rule 0: the reference's (20 iterations, delta <= eps^2 delta_0);
 * 1: relative, sqrt(delta / delta_0) <= tol.  dot 0: sequential FP32 (the
 * reference's), 2: FP64 accumulation. */
void os_set_solver(os_body* b, int stop_rule, float tol, uint32_t max_iterations, int dot);
void os_step(os_body* b, float dt, uint32_t velocity_iterations, uint32_t position_iterations, os_stats* out);
void os_get_state(const os_body* b, float* x, float* v);
void os_set_state(os_body* b, const float* x, const float* v);
void os_get_masses(const os_body* b, float* m);
/* per element: q (4 floats, x y z w), plastic strain (6 floats) */
void os_get_elements(const os_body* b, float* q, float* eps);
void os_set_elements(os_body* b, const float* q, const float* eps);
/* per element: the 16 stiffness blocks (9 floats each, column-major b3Mat33,
 * block i + 4 j), invE (9), B (72), P (72) */
void os_get_element_data(const os_body* b, uint32_t e, float* K, float* invE, float* B, float* P);
float os_energy(const os_body* b);
/* The system of one force solve from the current state, without changing
 * it: A's rows in the reference's row-list order (rowptr n + 1, cols and
 * 9-float column-major blocks), b and S.  Returns the block count, or the
 * needed capacity when cap is too small (nothing written). */
uint32_t os_system(os_body* b, float dt, uint32_t cap, uint32_t* rowptr, uint32_t* cols, float* vals, float* rhs,
                   float* S);

#ifdef __cplusplus
}
/* contacts with static hulls (b3SoftBody::SetWorld, softbody_contact_manager.cpp) */
void os_set_node_radius(os_body* b, uint32_t i, float radius);
void os_set_node_friction(os_body* b, uint32_t i, float friction);
int os_add_hull(os_body* b, const float* vertices, uint32_t nv, const float* planes, uint32_t nf, float friction);
uint32_t os_get_contacts(const os_body* b, uint8_t* exists, uint8_t* active, float* impulses);
uint32_t os_get_contact_list(const os_body* b, uint32_t cap, uint32_t* node, uint32_t* shape, uint8_t* active,
                             float* impulses);

#endif
