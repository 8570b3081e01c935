/*
 * CPU restatement of Bounce's implicit cloth step -- test infrastructure only
 * (parity oracle; see cloth_oracle.h).  Every function names the reference
 * file and lines it follows.  Vector and matrix helpers evaluate in the same
 * order as the reference's inline operators (include/bounce/common/math/
 * vec3.h, mat33.h, vec2.h, mat22.h), which is what makes the results
 * bit-identical to the compiled reference in reference mode.
 */
#include "world_order.h"
#include "cloth_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* math helpers, same evaluation order as the reference's operators          */
/* ------------------------------------------------------------------------ */

typedef struct { float x, y, z; } v3;
typedef struct { v3 x, y, z; } m33; /* column-major, like b3Mat33 */
typedef struct { float x, y; } v2;

static const float kEps = FLT_EPSILON;         /* B3_EPSILON, settings.h:42 */
static const float kAabbExtension = 0.2f;       /* settings.h:54 */
static const float kAabbMultiplier = 2.0f;      /* settings.h:60 */
static const float kLinearSlop = 0.005f;        /* settings.h:63 */
static const float kMaxLinearCorrection = 0.2f; /* settings.h:95 */
static const float kBaumgarte = 0.1f;           /* settings.h:101 */

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vscale(float s, v3 v) { return V(s * v.x, s * v.y, s * v.z); }
static inline v3 vdiv(v3 v, float s) { return V(v.x / s, v.y / s, v.z / s); }
static inline v3 vneg(v3 v) { return V(-v.x, -v.y, -v.z); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b)
{
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vlength(v3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
static inline v3 vmin(v3 a, v3 b)
{
    return V(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z);
}
static inline v3 vmax(v3 a, v3 b)
{
    return V(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z);
}
static inline v3 vzero(void) { return V(0.0f, 0.0f, 0.0f); }

static inline m33 M3(v3 x, v3 y, v3 z) { m33 m = {x, y, z}; return m; }
static inline m33 mzero(void) { return M3(vzero(), vzero(), vzero()); }
static inline m33 mident(void)
{
    return M3(V(1.0f, 0.0f, 0.0f), V(0.0f, 1.0f, 0.0f), V(0.0f, 0.0f, 1.0f));
}
static inline m33 mdiag3(float x, float y, float z)
{
    return M3(V(x, 0.0f, 0.0f), V(0.0f, y, 0.0f), V(0.0f, 0.0f, z));
}
static inline m33 madd(m33 a, m33 b) { return M3(vadd(a.x, b.x), vadd(a.y, b.y), vadd(a.z, b.z)); }
static inline m33 msub(m33 a, m33 b) { return M3(vsub(a.x, b.x), vsub(a.y, b.y), vsub(a.z, b.z)); }
static inline m33 mscale(float s, m33 a) { return M3(vscale(s, a.x), vscale(s, a.y), vscale(s, a.z)); }
static inline m33 mouter(v3 a, v3 b) { return M3(vscale(b.x, a), vscale(b.y, a), vscale(b.z, a)); }
/* A * v = v.x * A.x + v.y * A.y + v.z * A.z (mat33.h:129-132) */
static inline v3 mmul(m33 a, v3 v)
{
    return vadd(vadd(vscale(v.x, a.x), vscale(v.y, a.y)), vscale(v.z, a.z));
}
static inline void madd_to(m33* a, m33 b)
{
    a->x = vadd(a->x, b.x);
    a->y = vadd(a->y, b.y);
    a->z = vadd(a->z, b.z);
}
static inline void msub_to(m33* a, m33 b)
{
    a->x = vsub(a->x, b.x);
    a->y = vsub(a->y, b.y);
    a->z = vsub(a->z, b.z);
}

static inline v2 W(float x, float y) { v2 r = {x, y}; return r; }

/* b3Perp (vec3.h:255-266): unnormalised perpendicular. */
static inline v3 vperp(v3 v)
{
    if (fabsf(v.x) >= 0.57735027f) return V(v.y, -v.x, 0.0f);
    return V(0.0f, v.z, -v.y);
}

/* ------------------------------------------------------------------------ */
/* sparse rows with the reference's list semantics                           */
/* ------------------------------------------------------------------------ */

/* One sparse row.  Blocks are kept in first-touch (append) order; the
 * reference's singly linked row (sparse_mat33.h:27-32, :194-216) pushes each
 * new block to the front, so its list order is the reverse of this array. */
typedef struct {
    uint32_t* cols;
    m33* vals;
    uint32_t count, cap;
} lrow;

static m33* lrow_at(lrow* r, uint32_t col)
{
    for (uint32_t k = 0; k < r->count; ++k)
        if (r->cols[k] == col) return r->vals + k;
    if (r->count == r->cap) {
        r->cap = r->cap ? 2 * r->cap : 8;
        r->cols = (uint32_t*)realloc(r->cols, r->cap * sizeof(uint32_t));
        r->vals = (m33*)realloc(r->vals, r->cap * sizeof(m33));
    }
    r->cols[r->count] = col;
    r->vals[r->count] = mzero();
    return r->vals + r->count++;
}

static int lrow_find(const lrow* r, uint32_t col)
{
    for (uint32_t k = 0; k < r->count; ++k)
        if (r->cols[k] == col) return (int)k;
    return -1;
}

static void lrows_clear(lrow* rows, uint32_t n)
{
    for (uint32_t i = 0; i < n; ++i) rows[i].count = 0;
}

static void lrows_free(lrow* rows, uint32_t n)
{
    if (!rows) return;
    for (uint32_t i = 0; i < n; ++i) {
        free(rows[i].cols);
        free(rows[i].vals);
    }
    free(rows);
}

/* ------------------------------------------------------------------------ */
/* cloth state                                                               */
/* ------------------------------------------------------------------------ */

enum { F_STRETCH = 0, F_SHEAR = 1, F_SPRING = 2, F_MOUSE = 3 };

typedef struct {
    int type;
    uint32_t a, b, c;    /* triangle index (a) for stretch/shear; vertices (a, b) for springs;
                            mouse: particle (a), triangle (b) */
    float ks, kd, p0, p1; /* stretch: bu, bv; spring: L0; mouse: km, kd, w2, w3 */
    float p2;             /* mouse: w4 */
    uint32_t id;          /* mouse: the handle oc_create_mouse_force returned */
} force_t;

enum { SHAPE_SPHERE = 0, SHAPE_CAPSULE = 1, SHAPE_HULL = 2 };

/* b3Quat (include/bounce/common/math/quat.h) */
typedef struct { float x, y, z, w; } quat;

/* The state of a b3Body a collider belongs to (include/bounce/dynamics/
 * body.h): type (0 static, 1 kinematic, 2 dynamic), transform m_xf, sweep
 * (local center, world centers and orientations at the start and end of
 * the world step), velocities, inverse mass, local and world inverse
 * inertia.  The caller's world owns it; the cloth step reads it and, as the
 * reference's contact solver does, writes velocities, the sweep's end state
 * and the synchronised transform back. */
typedef struct {
    int type;
    m33 R;
    v3 p;
    v3 lc, c0, c;
    quat q0, q;
    v3 v, w;
    float im;
    m33 ii, wii;
} body_t;

typedef struct {
    int kind;
    int body;          /* -1: a static shape given in the world frame, whose body sits at the
                          sphere's centre (spheres) or the origin (others); else the index of a
                          body, with the geometry below in that body's frame */
    v3 center;         /* sphere */
    v3 a, b;           /* capsule segment, world frame (the body at the origin) */
    v3* hv;            /* hull: vertices and face planes (normal, offset), world frame (body at the origin) */
    v3* hn;
    float* ho;
    uint32_t nhv, nhf;
    float radius, friction;
    v3 fat_lo, fat_hi; /* the shape's proxy in the world broadphase */
} sphere_t;

/* b3ParticleTriangleContact (cloth_particle_triangle_contact.h): particle p
 * against triangle t, whose vertices are b, cc, d (the contact's m_p2, m_p3,
 * m_p4). */
typedef struct {
    uint32_t p, t, b, cc, d;
    int active;
    float w2, w3, w4;
    float normal_impulse, tangent_impulse1, tangent_impulse2;
} tcontact_t;

typedef struct {
    uint32_t particle, shape;
    int active;
    v3 normal1, local_point2, tangent1, tangent2;
    float normal_impulse;
    v2 tangent_impulse;
} contact_t;

struct oc_cloth {
    uint32_t n, t;
    uint32_t n_mesh;      /* particles made from mesh vertices; created particles follow */
    uint32_t next_force_id;
    float def[8];
    uint32_t* tris;

    /* particles, by vertex index */
    v3 *x, *v, *f, *y, *mx;
    float *mass, *inv_mass, *radius, *friction;
    uint8_t* type;
    v3 *fat_lo, *fat_hi;
    /* particle list (cloth.cpp:319 PushFront): order[k] = vertex of list slot k */
    uint32_t* order;

    /* triangles rest state (cloth.cpp:155-191) */
    float *du1, *dv1, *du2, *dv2, *inv_det, *alpha;

    /* forces in list (application) order */
    force_t* forces;
    uint32_t nforce;
    uint32_t nspring;

    v3 gravity;
    sphere_t* spheres;
    uint32_t nsphere;
    body_t* bodies;
    uint32_t nbody;
    uint32_t report[WO_MAX]; /* shapes in a world query's report order, when given */
    int has_report;

    /* body-contact list stored tail first: element [ncontact-1] is the list head */
    contact_t* contacts;
    uint32_t ncontact, contact_cap;

    /* self-collision (thickness > 0): triangle proxies, the broadphase move
     * buffer as one flag per proxy, and the particle-triangle contact list,
     * stored tail first like the body contacts */
    v3 *tri_lo, *tri_hi;
    uint8_t *p_moved, *t_moved;
    tcontact_t* tcs;
    uint32_t ntc, tc_cap;

    int stop_rule, dot;
    float tol;
    uint32_t max_iter;

    /* solver scratch */
    lrow *dfdx, *dfdv;
    uint32_t *a_rowptr, *a_cols;
    m33* a_vals;
    uint32_t a_cap;
    v3 *sx, *sv, *sf, *sy, *sx0, *b, *dvsol;
    float* Sflag;
    uint32_t* solver_of_vertex;
    uint32_t sys_nnz;
};

/* ------------------------------------------------------------------------ */
/* construction                                                              */
/* ------------------------------------------------------------------------ */

typedef struct { uint32_t a, b, tri, slot; } dedge;

static int dedge_cmp(const void* pa, const void* pb)
{
    const dedge* x = (const dedge*)pa;
    const dedge* y = (const dedge*)pb;
    if (x->a != y->a) return x->a < y->a ? -1 : 1;
    if (x->b != y->b) return x->b < y->b ? -1 : 1;
    if (x->tri != y->tri) return x->tri < y->tri ? -1 : 1;
    if (x->slot != y->slot) return x->slot < y->slot ? -1 : 1;
    return 0;
}

static void push_force(oc_cloth* c, force_t f)
{
    c->forces[c->nforce++] = f;
}

/* b3Cloth::b3Cloth (cloth.cpp:96-266) with b3FindSharedEdges (:40-94)
 * restated over a sorted directed-edge table: same pairs, same order. */
oc_cloth* oc_create(const float* vertices, uint32_t n, const uint32_t* triangles, uint32_t t,
                    const uint32_t* sewing, uint32_t nsew, const float* def)
{
    oc_cloth* c = (oc_cloth*)calloc(1, sizeof(oc_cloth));
    c->n = n;
    c->n_mesh = n;
    c->t = t;
    memcpy(c->def, def, sizeof(c->def));
    c->tris = (uint32_t*)malloc(3 * (size_t)t * sizeof(uint32_t));
    memcpy(c->tris, triangles, 3 * (size_t)t * sizeof(uint32_t));

    c->x = (v3*)calloc(n, sizeof(v3));
    c->v = (v3*)calloc(n, sizeof(v3));
    c->f = (v3*)calloc(n, sizeof(v3));
    c->y = (v3*)calloc(n, sizeof(v3));
    c->mx = (v3*)calloc(n, sizeof(v3));
    c->mass = (float*)calloc(n, sizeof(float));
    c->inv_mass = (float*)calloc(n, sizeof(float));
    c->radius = (float*)calloc(n, sizeof(float));
    c->friction = (float*)calloc(n, sizeof(float));
    c->type = (uint8_t*)calloc(n, 1);
    c->fat_lo = (v3*)calloc(n, sizeof(v3));
    c->fat_hi = (v3*)calloc(n, sizeof(v3));
    c->order = (uint32_t*)calloc(n, sizeof(uint32_t));
    c->solver_of_vertex = (uint32_t*)calloc(n, sizeof(uint32_t));

    float thickness = def[6], fric = def[7];
    /* particles: mass 1 -> dynamic (particle.cpp:24-44), proxy fattened by
     * B3_AABB_EXTENSION (cloth.cpp:312-317, broad_phase.cpp:78-82) */
    for (uint32_t i = 0; i < n; ++i) {
        c->x[i] = V(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
        c->type[i] = OC_DYNAMIC;
        c->radius[i] = thickness;
        c->friction[i] = fric;
        v3 r = V(thickness, thickness, thickness);
        v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
        c->fat_lo[i] = vsub(vsub(c->x[i], r), ext);
        c->fat_hi[i] = vadd(vadd(c->x[i], r), ext);
        /* PushFront: the newest particle heads the list */
        c->order[n - 1 - i] = i;
    }

    /* ComputeMass (cloth.cpp:388-427) */
    const float inv3 = 1.0f / 3.0f;
    const float rho = def[0];
    for (uint32_t k = 0; k < t; ++k) {
        v3 a = c->x[triangles[3 * k]], b = c->x[triangles[3 * k + 1]], cc = c->x[triangles[3 * k + 2]];
        float area = 0.5f * vlength(vcross(vsub(b, a), vsub(cc, a)));
        float m = rho * area;
        c->mass[triangles[3 * k]] += inv3 * m;
        c->mass[triangles[3 * k + 1]] += inv3 * m;
        c->mass[triangles[3 * k + 2]] += inv3 * m;
    }
    for (uint32_t i = 0; i < n; ++i) c->inv_mass[i] = 1.0f / c->mass[i];

    /* triangle proxies (cloth.cpp:140-150): the triangle's AABB extended by
     * the thickness, fattened by B3_AABB_EXTENSION in CreateProxy
     * (broad_phase.cpp:78-90); every new proxy is in the move buffer */
    c->tri_lo = (v3*)malloc((t ? t : 1) * sizeof(v3));
    c->tri_hi = (v3*)malloc((t ? t : 1) * sizeof(v3));
    c->t_moved = (uint8_t*)malloc(t ? t : 1);
    c->p_moved = (uint8_t*)malloc(n ? n : 1);
    memset(c->t_moved, 1, t ? t : 1);
    memset(c->p_moved, 1, n ? n : 1);
    for (uint32_t k = 0; k < t; ++k) {
        v3 A = c->x[triangles[3 * k]], B = c->x[triangles[3 * k + 1]], C = c->x[triangles[3 * k + 2]];
        v3 r = V(thickness, thickness, thickness);
        v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
        c->tri_lo[k] = vsub(vsub(vmin(A, vmin(B, C)), r), ext);
        c->tri_hi[k] = vadd(vadd(vmax(A, vmax(B, C)), r), ext);
    }

    /* triangles (cloth.cpp:129-215) */
    c->du1 = (float*)malloc(t * sizeof(float));
    c->dv1 = (float*)malloc(t * sizeof(float));
    c->du2 = (float*)malloc(t * sizeof(float));
    c->dv2 = (float*)malloc(t * sizeof(float));
    c->inv_det = (float*)malloc(t * sizeof(float));
    c->alpha = (float*)malloc(t * sizeof(float));

    /* forces are created in this order and pushed to the front of the force
     * list (cloth.cpp:353-358); we build the creation order first. */
    size_t fcap = 2 * (size_t)t + 3 * (size_t)t + nsew + 1;
    force_t* created = (force_t*)calloc(fcap, sizeof(force_t));
    uint32_t ncreated = 0;

    for (uint32_t k = 0; k < t; ++k) {
        v3 A = c->x[triangles[3 * k]], B = c->x[triangles[3 * k + 1]], C = c->x[triangles[3 * k + 2]];
        v3 AB = vsub(B, A), AC = vsub(C, A);
        float u1 = 0.0f, v1 = 0.0f;
        float u2 = vlength(AB), v2_ = 0.0f;
        v3 n_AB = vdiv(AB, u2);
        float A2 = vlength(vcross(AB, AC));
        float u3 = vdot(AC, n_AB);
        float v3_ = A2 / u2;
        float du1 = u2 - u1, dv1 = v2_ - v1, du2 = u3 - u1, dv2 = v3_ - v1;
        c->du1[k] = du1;
        c->dv1[k] = dv1;
        c->du2[k] = du2;
        c->dv2[k] = dv2;
        float det = du1 * dv2 - du2 * dv1;
        c->inv_det[k] = 1.0f / det;
        c->alpha[k] = 0.5f * A2;
        if (def[1] > 0.0f) {
            force_t f = {F_STRETCH, k, 0, 0, def[1], def[5], 1.0f, 1.0f, 0.0f, 0u};
            created[ncreated++] = f;
        }
        if (def[2] > 0.0f) {
            force_t f = {F_SHEAR, k, 0, 0, def[2], def[5], 0.0f, 0.0f, 0.0f, 0u};
            created[ncreated++] = f;
        }
    }

    /* bending springs between non-shared vertices (cloth.cpp:218-245) */
    dedge* edges = (dedge*)malloc(3 * (size_t)t * sizeof(dedge) + 1);
    for (uint32_t k = 0; k < t; ++k) {
        for (uint32_t e = 0; e < 3; ++e) {
            dedge d = {triangles[3 * k + e], triangles[3 * k + (e + 1) % 3], k, e};
            edges[3 * k + e] = d;
        }
    }
    qsort(edges, 3 * (size_t)t, sizeof(dedge), dedge_cmp);
    c->nspring = 0;
    for (uint32_t i = 0; i < t; ++i) {
        const uint32_t* t1 = triangles + 3 * i;
        for (uint32_t j1 = 0; j1 < 3; ++j1) {
            uint32_t k1 = j1 + 1 < 3 ? j1 + 1 : 0;
            uint32_t a = t1[j1], b = t1[k1];
            /* lower bound of (b, a, i + 1, 0) */
            size_t lo = 0, hi = 3 * (size_t)t;
            dedge key = {b, a, i + 1, 0};
            while (lo < hi) {
                size_t mid = (lo + hi) / 2;
                if (dedge_cmp(edges + mid, &key) < 0) lo = mid + 1;
                else hi = mid;
            }
            uint32_t last = UINT32_MAX;
            for (size_t q = lo; q < 3 * (size_t)t && edges[q].a == b && edges[q].b == a; ++q) {
                if (edges[q].tri == last) continue;
                last = edges[q].tri;
                const uint32_t* t2 = triangles + 3 * edges[q].tri;
                uint32_t k2 = edges[q].slot + 1 < 3 ? edges[q].slot + 1 : 0;
                uint32_t k3 = k1 + 1 < 3 ? k1 + 1 : 0;
                uint32_t k4 = k2 + 1 < 3 ? k2 + 1 : 0;
                uint32_t p3 = t1[k3], p4 = t2[k4];
                /* b3SpringForceDef::Initialize (spring_force.cpp:25-35) */
                float L0 = vlength(vsub(c->x[p3], c->x[p4]));
                if (def[3] > 0.0f) {
                    force_t f = {F_SPRING, p3, p4, 0, def[3], def[5], L0, 0.0f, 0.0f, 0u};
                    if (ncreated == fcap) {
                        fcap *= 2;
                        created = (force_t*)realloc(created, fcap * sizeof(force_t));
                    }
                    created[ncreated++] = f;
                    c->nspring++;
                }
            }
        }
    }
    free(edges);

    /* sewing springs (cloth.cpp:248-262) */
    for (uint32_t s = 0; s < nsew; ++s) {
        uint32_t p1 = sewing[4 * s + 2], p2 = sewing[4 * s + 3];
        float L0 = vlength(vsub(c->x[p1], c->x[p2]));
        if (def[4] > 0.0f) {
            force_t f = {F_SPRING, p1, p2, 0, def[4], def[5], L0, 0.0f, 0.0f, 0u};
            if (ncreated == fcap) {
                fcap *= 2;
                created = (force_t*)realloc(created, fcap * sizeof(force_t));
            }
            created[ncreated++] = f;
            c->nspring++;
        }
    }

    c->forces = (force_t*)malloc((ncreated + 1) * sizeof(force_t));
    c->nforce = 0;
    for (uint32_t k = ncreated; k-- > 0;) push_force(c, created[k]);
    free(created);

    c->gravity = vzero();
    c->stop_rule = OC_STOP_REFERENCE;
    c->tol = 0.0f;
    c->max_iter = 20;
    c->dot = OC_DOT_F32;

    c->dfdx = (lrow*)calloc(n, sizeof(lrow));
    c->dfdv = (lrow*)calloc(n, sizeof(lrow));
    c->a_rowptr = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    c->sx = (v3*)calloc(n, sizeof(v3));
    c->sv = (v3*)calloc(n, sizeof(v3));
    c->sf = (v3*)calloc(n, sizeof(v3));
    c->sy = (v3*)calloc(n, sizeof(v3));
    c->sx0 = (v3*)calloc(n, sizeof(v3));
    c->b = (v3*)calloc(n, sizeof(v3));
    c->dvsol = (v3*)calloc(n, sizeof(v3));
    c->Sflag = (float*)calloc(n, sizeof(float));
    return c;
}

void oc_destroy(oc_cloth* c)
{
    if (!c) return;
    free(c->tris);
    free(c->tri_lo); free(c->tri_hi); free(c->t_moved); free(c->p_moved); free(c->tcs);
    free(c->x); free(c->v); free(c->f); free(c->y); free(c->mx);
    free(c->mass); free(c->inv_mass); free(c->radius); free(c->friction); free(c->type);
    free(c->fat_lo); free(c->fat_hi); free(c->order); free(c->solver_of_vertex);
    free(c->du1); free(c->dv1); free(c->du2); free(c->dv2); free(c->inv_det); free(c->alpha);
    for (uint32_t k = 0; k < c->nsphere; ++k) {
        free(c->spheres[k].hv); free(c->spheres[k].hn); free(c->spheres[k].ho);
    }
    free(c->forces); free(c->spheres); free(c->contacts); free(c->bodies);
    lrows_free(c->dfdx, c->n);
    lrows_free(c->dfdv, c->n);
    free(c->a_rowptr); free(c->a_cols); free(c->a_vals);
    free(c->sx); free(c->sv); free(c->sf); free(c->sy); free(c->sx0); free(c->b); free(c->dvsol);
    free(c->Sflag);
    free(c);
}

/* ------------------------------------------------------------------------ */
/* particle API (particle.cpp, particle.h)                                   */
/* ------------------------------------------------------------------------ */

/* b3BroadPhase::MoveProxy (broad_phase.cpp:99-149) for a particle proxy. */
static void move_proxy(oc_cloth* c, uint32_t i, v3 displacement)
{
    v3 r = V(c->radius[i], c->radius[i], c->radius[i]);
    v3 lo = vsub(c->x[i], r), hi = vadd(c->x[i], r);
    v3 flo = c->fat_lo[i], fhi = c->fat_hi[i];
    int contains = flo.x <= lo.x && lo.x <= fhi.x && flo.y <= lo.y && lo.y <= fhi.y &&
                   flo.z <= lo.z && lo.z <= fhi.z && flo.x <= hi.x && hi.x <= fhi.x &&
                   flo.y <= hi.y && hi.y <= fhi.y && flo.z <= hi.z && hi.z <= fhi.z;
    if (contains) return;
    v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
    lo = vsub(lo, ext);
    hi = vadd(hi, ext);
    v3 d = vscale(kAabbMultiplier, displacement);
    if (d.x < 0.0f) lo.x += d.x; else hi.x += d.x;
    if (d.y < 0.0f) lo.y += d.y; else hi.y += d.y;
    if (d.z < 0.0f) lo.z += d.z; else hi.z += d.z;
    c->fat_lo[i] = lo;
    c->fat_hi[i] = hi;
    c->p_moved[i] = 1; /* BufferMove */
}

static inline int self_collision(const oc_cloth* c) { return c->def[6] > 0.0f; }

/* b3ClothTriangle::Synchronize (cloth_triangle.cpp:24-40) with
 * b3BroadPhase::MoveProxy (broad_phase.cpp:99-149). */
static void move_triangle_proxy(oc_cloth* c, uint32_t k, v3 displacement)
{
    const float rad = c->def[6];
    v3 A = c->x[c->tris[3 * k]], B = c->x[c->tris[3 * k + 1]], C = c->x[c->tris[3 * k + 2]];
    v3 r = V(rad, rad, rad);
    v3 lo = vsub(vmin(A, vmin(B, C)), r), hi = vadd(vmax(A, vmax(B, C)), r);
    v3 flo = c->tri_lo[k], fhi = c->tri_hi[k];
    int contains = flo.x <= lo.x && lo.x <= fhi.x && flo.y <= lo.y && lo.y <= fhi.y &&
                   flo.z <= lo.z && lo.z <= fhi.z && flo.x <= hi.x && hi.x <= fhi.x &&
                   flo.y <= hi.y && hi.y <= fhi.y && flo.z <= hi.z && hi.z <= fhi.z;
    if (contains) return;
    v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
    lo = vsub(lo, ext);
    hi = vadd(hi, ext);
    v3 d = vscale(kAabbMultiplier, displacement);
    if (d.x < 0.0f) lo.x += d.x; else hi.x += d.x;
    if (d.y < 0.0f) lo.y += d.y; else hi.y += d.y;
    if (d.z < 0.0f) lo.z += d.z; else hi.z += d.z;
    c->tri_lo[k] = lo;
    c->tri_hi[k] = hi;
    c->t_moved[k] = 1;
}

/* b3Particle::SynchronizeTriangles (particle.cpp:66-82): every triangle of a
 * mesh vertex, with no displacement. */
static void sync_vertex_triangles(oc_cloth* c, uint32_t i)
{
    if (i >= c->n_mesh) return;
    for (uint32_t k = 0; k < c->t; ++k)
        if (c->tris[3 * k] == i || c->tris[3 * k + 1] == i || c->tris[3 * k + 2] == i)
            move_triangle_proxy(c, k, vzero());
}

/* The particle-triangle contacts whose particle is i (particle.cpp:103-118). */
static void destroy_particle_triangle_contacts(oc_cloth* c, uint32_t i)
{
    uint32_t w = 0;
    for (uint32_t k = 0; k < c->ntc; ++k)
        if (c->tcs[k].p != i) c->tcs[w++] = c->tcs[k];
    c->ntc = w;
}

/* Remove every body contact of particle i (particle.cpp:66-83). */
static void destroy_particle_contacts(oc_cloth* c, uint32_t i)
{
    uint32_t w = 0;
    for (uint32_t k = 0; k < c->ncontact; ++k)
        if (c->contacts[k].particle != i) c->contacts[w++] = c->contacts[k];
    c->ncontact = w;
}

/* Overwrite positions, velocities and the CG warm start of every particle
 * (no proxy update): used to start both solvers from identical inputs. */
void oc_set_state(oc_cloth* c, const float* x, const float* v, const float* dv)
{
    for (uint32_t i = 0; i < c->n; ++i) {
        if (x) c->x[i] = V(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
        if (v) c->v[i] = V(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        if (dv) c->mx[i] = V(dv[3 * i], dv[3 * i + 1], dv[3 * i + 2]);
    }
}

/* Replace the body-contact list (used to start the oracle from another
 * solver's state): `count` contacts in list order from the tail (the oldest)
 * to the head, each a (particle, shape) pair with its normal and two tangent
 * impulses (3 floats).  The contact update at the next step start recomputes
 * activity, normal, tangents and point from the positions, as
 * b3ClothContactManager::UpdateBodyContacts does (cloth_contact_manager.cpp:
 * 277-315); what persists between steps is the list and the impulses. */
void oc_set_contacts(oc_cloth* c, uint32_t count, const uint32_t* particle, const uint32_t* shape,
                     const float* impulses)
{
    if (count > c->contact_cap) {
        c->contact_cap = count;
        c->contacts = (contact_t*)realloc(c->contacts, c->contact_cap * sizeof(contact_t));
    }
    c->ncontact = count;
    for (uint32_t q = 0; q < count; ++q) {
        contact_t* k = c->contacts + q;
        memset(k, 0, sizeof(*k));
        k->particle = particle[q];
        k->shape = shape[q];
        k->normal_impulse = impulses[3 * q];
        k->tangent_impulse.x = impulses[3 * q + 1];
        k->tangent_impulse.y = impulses[3 * q + 2];
    }
}

/* Overwrite the particles' broadphase proxies (fat AABBs, xyz triples). */
void oc_set_proxies(oc_cloth* c, const float* lo, const float* hi)
{
    for (uint32_t i = 0; i < c->n; ++i) {
        c->fat_lo[i] = V(lo[3 * i], lo[3 * i + 1], lo[3 * i + 2]);
        c->fat_hi[i] = V(hi[3 * i], hi[3 * i + 1], hi[3 * i + 2]);
    }
}

void oc_set_gravity(oc_cloth* c, const float* g) { c->gravity = V(g[0], g[1], g[2]); }

/* b3Particle::SetType (particle.cpp:121-143) */
void oc_set_type(oc_cloth* c, uint32_t i, int type)
{
    if (c->type[i] == type) return;
    c->type[i] = (uint8_t)type;
    c->f[i] = vzero();
    if (type == OC_STATIC) {
        c->v[i] = vzero();
        c->y[i] = vzero();
        move_proxy(c, i, vzero());
        sync_vertex_triangles(c, i);
    }
    destroy_particle_contacts(c, i);
    destroy_particle_triangle_contacts(c, i);
    c->p_moved[i] = 1; /* TouchProxy */
}

/* b3Particle::SetRadius (particle.h:240-245): the new radius, then
 * Synchronize(0), which moves the particle's proxy (particle.cpp:58-64). */
void oc_set_radius(oc_cloth* c, uint32_t i, float radius)
{
    c->radius[i] = radius;
    move_proxy(c, i, vzero());
}

/* b3Particle::SetFriction (particle.h:252-255) */
void oc_set_friction(oc_cloth* c, uint32_t i, float friction) { c->friction[i] = friction; }

/* b3Particle::ApplyForce / ApplyTranslation / SetPosition / SetVelocity (particle.h:205-271) */
void oc_apply_force(oc_cloth* c, uint32_t i, const float* f)
{
    if (c->type[i] != OC_DYNAMIC) return;
    c->f[i] = vadd(c->f[i], V(f[0], f[1], f[2]));
}

void oc_apply_translation(oc_cloth* c, uint32_t i, const float* t)
{
    c->y[i] = vadd(c->y[i], V(t[0], t[1], t[2]));
}

void oc_set_position(oc_cloth* c, uint32_t i, const float* x)
{
    v3 p = V(x[0], x[1], x[2]);
    v3 d = vsub(p, c->x[i]);
    c->x[i] = p;
    c->y[i] = vzero();
    move_proxy(c, i, d);
    sync_vertex_triangles(c, i);
}

void oc_set_velocity(oc_cloth* c, uint32_t i, const float* v)
{
    if (c->type[i] == OC_STATIC) return;
    c->v[i] = V(v[0], v[1], v[2]);
}

/* A static body at `center` with one sphere shape: the shape proxy is the
 * sphere's AABB (sphere_shape.cpp:53-59) fattened by B3_AABB_EXTENSION. */
int oc_add_sphere(oc_cloth* c, const float* center, float radius, float friction)
{
    c->spheres = (sphere_t*)realloc(c->spheres, (c->nsphere + 1) * sizeof(sphere_t));
    sphere_t* s = c->spheres + c->nsphere;
    memset(s, 0, sizeof(*s));
    s->kind = SHAPE_SPHERE;
    s->body = -1;
    s->center = V(center[0], center[1], center[2]);
    s->radius = radius;
    s->friction = friction;
    v3 r = V(radius, radius, radius);
    v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
    s->fat_lo = vsub(vsub(s->center, r), ext);
    s->fat_hi = vadd(vadd(s->center, r), ext);
    return (int)c->nsphere++;
}

/* A static body at the origin with one capsule shape (capsule_shape.h):
 * segment a-b in the world frame; the proxy is ComputeAABB
 * (capsule_shape.cpp:130-137) fattened by B3_AABB_EXTENSION. */
int oc_add_capsule(oc_cloth* c, const float* a, const float* b, float radius, float friction)
{
    c->spheres = (sphere_t*)realloc(c->spheres, (c->nsphere + 1) * sizeof(sphere_t));
    sphere_t* s = c->spheres + c->nsphere;
    memset(s, 0, sizeof(*s));
    s->kind = SHAPE_CAPSULE;
    s->body = -1;
    s->a = V(a[0], a[1], a[2]);
    s->b = V(b[0], b[1], b[2]);
    s->radius = radius;
    s->friction = friction;
    v3 r = V(radius, radius, radius);
    v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
    s->fat_lo = vsub(vsub(vmin(s->a, s->b), r), ext);
    s->fat_hi = vadd(vadd(vmax(s->a, s->b), r), ext);
    return (int)c->nsphere++;
}

/* b3Mul(b3Transform, b3Vec3) and b3MulT for a static body at the origin
 * with the identity rotation (transform.h:74-110, mat33.h:129-160), written
 * out so that the float operations are the reference's. */
static const v3 kIdX = {1.0f, 0.0f, 0.0f}, kIdY = {0.0f, 1.0f, 0.0f}, kIdZ = {0.0f, 0.0f, 1.0f};
static inline v3 xf_mul(v3 v)
{
    v3 r = vadd(vadd(vscale(v.x, kIdX), vscale(v.y, kIdY)), vscale(v.z, kIdZ));
    return vadd(r, vzero());
}
static inline v3 xf_mult(v3 v)
{
    v3 d = vsub(v, vzero());
    return V(vdot(kIdX, d), vdot(kIdY, d), vdot(kIdZ, d));
}

/* A static b3HullShape (hull radius B3_HULL_RADIUS = 0) on a body at the
 * origin: its proxy is b3HullShape::ComputeAABB (hull_shape.cpp:162-166)
 * fattened by B3_AABB_EXTENSION. */
int oc_add_hull(oc_cloth* c, const float* vertices, uint32_t nv, const float* planes, uint32_t nf, float friction)
{
    c->spheres = (sphere_t*)realloc(c->spheres, (c->nsphere + 1) * sizeof(sphere_t));
    sphere_t* s = c->spheres + c->nsphere;
    memset(s, 0, sizeof(*s));
    s->kind = SHAPE_HULL;
    s->body = -1;
    s->radius = 0.0f;
    s->friction = friction;
    s->nhv = nv;
    s->nhf = nf;
    s->hv = (v3*)malloc((nv ? nv : 1) * sizeof(v3));
    s->hn = (v3*)malloc((nf ? nf : 1) * sizeof(v3));
    s->ho = (float*)malloc((nf ? nf : 1) * sizeof(float));
    for (uint32_t i = 0; i < nv; ++i) s->hv[i] = V(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
    for (uint32_t i = 0; i < nf; ++i) {
        s->hn[i] = V(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2]);
        s->ho[i] = planes[4 * i + 3];
    }
    v3 lo = xf_mul(s->hv[0]), hi = lo;
    for (uint32_t i = 1; i < nv; ++i) {
        v3 w = xf_mul(s->hv[i]);
        lo = vmin(lo, w);
        hi = vmax(hi, w);
    }
    v3 r = V(s->radius, s->radius, s->radius);
    v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
    s->fat_lo = vsub(vsub(lo, r), ext);
    s->fat_hi = vadd(vadd(hi, r), ext);
    return (int)c->nsphere++;
}

/* ---- b3GJK between a hull and a point (gjk.cpp) ------------------------ */

typedef struct {
    v3 point1, point2, point;
    float weight;
    uint32_t index1, index2;
} gjk_vertex;

typedef struct {
    gjk_vertex v[4];
    uint32_t count;
} gjk_simplex;

/* b3Barycentric for a segment, a triangle, a tetrahedron (gjk.cpp:32-99) */
static void gbary2(float out[3], v3 A, v3 B, v3 Q)
{
    v3 AB = vsub(B, A), QA = vsub(A, Q), QB = vsub(B, Q);
    out[0] = vdot(QB, AB);
    out[1] = -vdot(QA, AB);
    out[2] = out[0] + out[1];
}

static void gbary3(float out[4], v3 A, v3 B, v3 C, v3 Q)
{
    v3 AB = vsub(B, A), AC = vsub(C, A), QA = vsub(A, Q), QB = vsub(B, Q), QC = vsub(C, Q);
    v3 QB_x_QC = vcross(QB, QC), QC_x_QA = vcross(QC, QA), QA_x_QB = vcross(QA, QB);
    v3 AB_x_AC = vcross(AB, AC);
    out[0] = vdot(QB_x_QC, AB_x_AC);
    out[1] = vdot(QC_x_QA, AB_x_AC);
    out[2] = vdot(QA_x_QB, AB_x_AC);
    out[3] = out[0] + out[1] + out[2];
}

static inline float gdet(v3 a, v3 b, v3 c) { return vdot(a, vcross(b, c)); }
static inline float gsign(float x) { return (float)(0.0f < x) - (float)(x < 0.0f); }

static void gbary4(float out[5], v3 A, v3 B, v3 C, v3 D, v3 Q)
{
    v3 AB = vsub(B, A), AC = vsub(C, A), AD = vsub(D, A);
    v3 QA = vsub(A, Q), QB = vsub(B, Q), QC = vsub(C, Q), QD = vsub(D, Q);
    float divisor = gdet(AB, AC, AD);
    float sign = gsign(divisor);
    out[0] = sign * gdet(QB, QC, QD);
    out[1] = sign * gdet(QA, QD, QC);
    out[2] = sign * gdet(QA, QB, QD);
    out[3] = sign * gdet(QA, QC, QB);
    out[4] = sign * divisor;
}

static void gset1(gjk_simplex* s, gjk_vertex a)
{
    s->count = 1;
    s->v[0] = a;
    s->v[0].weight = 1.0f;
}

static void gset2(gjk_simplex* s, gjk_vertex a, float wa, gjk_vertex b, float wb)
{
    s->count = 2;
    s->v[0] = a;
    s->v[0].weight = wa;
    s->v[1] = b;
    s->v[1].weight = wb;
}

static void gset3(gjk_simplex* s, gjk_vertex a, float wa, gjk_vertex b, float wb, gjk_vertex c, float wc)
{
    s->count = 3;
    s->v[0] = a;
    s->v[0].weight = wa;
    s->v[1] = b;
    s->v[1].weight = wb;
    s->v[2] = c;
    s->v[2].weight = wc;
}

/* b3Simplex::Solve2 (gjk.cpp:201-236) */
static void gsolve2(gjk_simplex* s, v3 Q)
{
    gjk_vertex A = s->v[0], B = s->v[1];
    float wAB[3];
    gbary2(wAB, A.point, B.point, Q);
    if (wAB[1] <= 0.0f) { gset1(s, A); return; }
    if (wAB[0] <= 0.0f) { gset1(s, B); return; }
    float sc = 1.0f / wAB[2];
    gset2(s, A, sc * wAB[0], B, sc * wAB[1]);
}

/* b3Simplex::Solve3 (gjk.cpp:240-346) */
static void gsolve3(gjk_simplex* s, v3 Q)
{
    gjk_vertex A = s->v[0], B = s->v[1], C = s->v[2];
    float wAB[3], wBC[3], wCA[3];
    gbary2(wAB, A.point, B.point, Q);
    gbary2(wBC, B.point, C.point, Q);
    gbary2(wCA, C.point, A.point, Q);
    if (wAB[1] <= 0.0f && wCA[0] <= 0.0f) { gset1(s, A); return; }
    if (wAB[0] <= 0.0f && wBC[1] <= 0.0f) { gset1(s, B); return; }
    if (wBC[0] <= 0.0f && wCA[1] <= 0.0f) { gset1(s, C); return; }
    float wABC[4];
    gbary3(wABC, A.point, B.point, C.point, Q);
    float area = wABC[3];
    if (wAB[0] > 0.0f && wAB[1] > 0.0f && area * wABC[2] <= 0.0f) {
        float sc = 1.0f / wAB[2];
        gset2(s, A, sc * wAB[0], B, sc * wAB[1]);
        return;
    }
    if (wBC[0] > 0.0f && wBC[1] > 0.0f && area * wABC[0] <= 0.0f) {
        float sc = 1.0f / wBC[2];
        gset2(s, B, sc * wBC[0], C, sc * wBC[1]);
        return;
    }
    if (wCA[0] > 0.0f && wCA[1] > 0.0f && area * wABC[1] <= 0.0f) {
        float sc = 1.0f / wCA[2];
        gset2(s, C, sc * wCA[0], A, sc * wCA[1]);
        return;
    }
    float divisor = wABC[3];
    if (divisor <= 0.0f) return; /* give up: the simplex and its weights stay */
    float sc = 1.0f / divisor;
    gset3(s, A, sc * wABC[0], B, sc * wABC[1], C, sc * wABC[2]);
}

/* b3Simplex::Solve4 (gjk.cpp:349-575) */
static void gsolve4(gjk_simplex* s, v3 Q)
{
    gjk_vertex A = s->v[0], B = s->v[1], C = s->v[2], D = s->v[3];
    float wAB[3], wAC[3], wAD[3], wBC[3], wCD[3], wDB[3];
    gbary2(wAB, A.point, B.point, Q);
    gbary2(wBC, B.point, C.point, Q);
    gbary2(wAC, A.point, C.point, Q);
    gbary2(wAD, A.point, D.point, Q);
    gbary2(wCD, C.point, D.point, Q);
    gbary2(wDB, D.point, B.point, Q);
    if (wAB[1] <= 0.0f && wAC[1] <= 0.0f && wAD[1] <= 0.0f) { gset1(s, A); return; }
    if (wAB[0] <= 0.0f && wDB[0] <= 0.0f && wBC[1] <= 0.0f) { gset1(s, B); return; }
    if (wAC[0] <= 0.0f && wBC[0] <= 0.0f && wCD[1] <= 0.0f) { gset1(s, C); return; }
    if (wAD[0] <= 0.0f && wCD[0] <= 0.0f && wDB[1] <= 0.0f) { gset1(s, D); return; }
    float wACB[4], wABD[4], wADC[4], wBCD[4];
    gbary3(wACB, A.point, C.point, B.point, Q);
    gbary3(wABD, A.point, B.point, D.point, Q);
    gbary3(wADC, A.point, D.point, C.point, Q);
    gbary3(wBCD, B.point, C.point, D.point, Q);
    if (wABD[2] <= 0.0f && wACB[1] <= 0.0f && wAB[0] > 0.0f && wAB[1] > 0.0f) {
        float sc = 1.0f / wAB[2];
        gset2(s, A, sc * wAB[0], B, sc * wAB[1]);
        return;
    }
    if (wACB[2] <= 0.0f && wADC[1] <= 0.0f && wAC[0] > 0.0f && wAC[1] > 0.0f) {
        float sc = 1.0f / wAC[2];
        gset2(s, A, sc * wAC[0], C, sc * wAC[1]);
        return;
    }
    if (wADC[2] <= 0.0f && wABD[1] <= 0.0f && wAD[0] > 0.0f && wAD[1] > 0.0f) {
        float sc = 1.0f / wAD[2];
        gset2(s, A, sc * wAD[0], D, sc * wAD[1]);
        return;
    }
    if (wACB[0] <= 0.0f && wBCD[2] <= 0.0f && wBC[0] > 0.0f && wBC[1] > 0.0f) {
        float sc = 1.0f / wBC[2];
        gset2(s, B, sc * wBC[0], C, sc * wBC[1]);
        return;
    }
    if (wADC[0] <= 0.0f && wBCD[0] <= 0.0f && wCD[0] > 0.0f && wCD[1] > 0.0f) {
        float sc = 1.0f / wCD[2];
        gset2(s, C, sc * wCD[0], D, sc * wCD[1]);
        return;
    }
    if (wABD[0] <= 0.0f && wBCD[1] <= 0.0f && wDB[0] > 0.0f && wDB[1] > 0.0f) {
        float sc = 1.0f / wDB[2];
        gset2(s, D, sc * wDB[0], B, sc * wDB[1]);
        return;
    }
    float wABCD[5];
    gbary4(wABCD, A.point, B.point, C.point, D.point, Q);
    if (wABCD[3] <= 0.0f && wACB[0] > 0.0f && wACB[1] > 0.0f && wACB[2] > 0.0f) {
        float sc = 1.0f / (wACB[0] + wACB[1] + wACB[2]);
        gset3(s, A, sc * wACB[0], C, sc * wACB[1], B, sc * wACB[2]);
        return;
    }
    if (wABCD[2] <= 0.0f && wABD[0] > 0.0f && wABD[1] > 0.0f && wABD[2] > 0.0f) {
        float sc = 1.0f / (wABD[0] + wABD[1] + wABD[2]);
        gset3(s, A, sc * wABD[0], B, sc * wABD[1], D, sc * wABD[2]);
        return;
    }
    if (wABCD[1] <= 0.0f && wADC[0] > 0.0f && wADC[1] > 0.0f && wADC[2] > 0.0f) {
        float sc = 1.0f / (wADC[0] + wADC[1] + wADC[2]);
        gset3(s, A, sc * wADC[0], D, sc * wADC[1], C, sc * wADC[2]);
        return;
    }
    if (wABCD[0] <= 0.0f && wBCD[0] > 0.0f && wBCD[1] > 0.0f && wBCD[2] > 0.0f) {
        float sc = 1.0f / (wBCD[0] + wBCD[1] + wBCD[2]);
        gset3(s, B, sc * wBCD[0], C, sc * wBCD[1], D, sc * wBCD[2]);
        return;
    }
    float divisor = wABCD[0] + wABCD[1] + wABCD[2] + wABCD[3];
    if (divisor <= 0.0f) return;
    float sc = 1.0f / divisor;
    s->count = 4;
    s->v[0].weight = sc * wABCD[0];
    s->v[1].weight = sc * wABCD[1];
    s->v[2].weight = sc * wABCD[2];
    s->v[3].weight = sc * wABCD[3];
}

/* b3Simplex::GetSearchDirection and GetClosestPoint(s) (gjk.cpp:101-199) */
static v3 gsearch(const gjk_simplex* s, v3 Q)
{
    if (s->count == 1) return vsub(Q, s->v[0].point);
    if (s->count == 2) {
        v3 A = s->v[0].point, B = s->v[1].point;
        v3 AB = vsub(B, A), AQ = vsub(Q, A);
        return vcross(vcross(AB, AQ), AB);
    }
    v3 A = s->v[0].point, B = s->v[1].point, C = s->v[2].point;
    v3 AB = vsub(B, A), AC = vsub(C, A), AQ = vsub(Q, A);
    v3 AB_x_AC = vcross(AB, AC);
    return vdot(AB_x_AC, AQ) > 0.0f ? AB_x_AC : vneg(AB_x_AC);
}

static v3 gclosest(const gjk_simplex* s)
{
    const gjk_vertex* v = s->v;
    if (s->count == 1) return v[0].point;
    if (s->count == 2) return vadd(vscale(v[0].weight, v[0].point), vscale(v[1].weight, v[1].point));
    if (s->count == 3)
        return vadd(vadd(vscale(v[0].weight, v[0].point), vscale(v[1].weight, v[1].point)),
                    vscale(v[2].weight, v[2].point));
    return vzero();
}

static void gwitness(const gjk_simplex* s, v3* p1, v3* p2)
{
    const gjk_vertex* v = s->v;
    switch (s->count) {
        case 1:
            *p1 = v[0].point1;
            *p2 = v[0].point2;
            break;
        case 2:
            *p1 = vadd(vscale(v[0].weight, v[0].point1), vscale(v[1].weight, v[1].point1));
            *p2 = vadd(vscale(v[0].weight, v[0].point2), vscale(v[1].weight, v[1].point2));
            break;
        case 3:
            *p1 = vadd(vadd(vscale(v[0].weight, v[0].point1), vscale(v[1].weight, v[1].point1)),
                       vscale(v[2].weight, v[2].point1));
            *p2 = vadd(vadd(vscale(v[0].weight, v[0].point2), vscale(v[1].weight, v[1].point2)),
                       vscale(v[2].weight, v[2].point2));
            break;
        default:
            *p1 = vadd(vadd(vadd(vscale(v[0].weight, v[0].point1), vscale(v[1].weight, v[1].point1)),
                            vscale(v[2].weight, v[2].point1)),
                       vscale(v[3].weight, v[3].point1));
            *p2 = *p1;
            break;
    }
}

/* b3GJK (gjk.cpp:579-740, no cache, no radius) between the hull (proxy 1,
 * body at the origin) and the point Q (proxy 2, identity frame). */
static float gjk_hull_point(const sphere_t* h, v3 Q, v3* p1, v3* p2)
{
    gjk_simplex s;
    memset(&s, 0, sizeof(s));
    /* ReadCache with an empty cache (gjk.cpp:743-795): vertex 0 of both */
    s.v[0].point1 = xf_mul(h->hv[0]);
    s.v[0].point2 = xf_mul(Q);
    s.v[0].point = vsub(s.v[0].point2, s.v[0].point1);
    s.v[0].weight = 1.0f;
    s.count = 1;
    uint32_t save1[4], save2[4], saveCount = 0;
    const v3 origin = vzero();
    uint32_t iter = 0;
    while (iter < 20) {
        saveCount = s.count;
        for (uint32_t i = 0; i < saveCount; ++i) {
            save1[i] = s.v[i].index1;
            save2[i] = s.v[i].index2;
        }
        if (s.count == 2) gsolve2(&s, origin);
        else if (s.count == 3) gsolve3(&s, origin);
        else if (s.count == 4) gsolve4(&s, origin);
        if (s.count == 4) break;
        (void)gclosest(&s);
        v3 d = gsearch(&s, origin);
        if (vdot(d, d) < kEps * kEps) break;
        gjk_vertex* vx = s.v + s.count;
        /* proxy 1: the hull's support in -d (b3GJKProxy::GetSupportIndex) */
        v3 dl = xf_mult(vneg(d));
        uint32_t best = 0;
        float bestp = vdot(dl, h->hv[0]);
        for (uint32_t i = 1; i < h->nhv; ++i) {
            float pr = vdot(dl, h->hv[i]);
            if (pr > bestp) {
                best = i;
                bestp = pr;
            }
        }
        vx->index1 = best;
        vx->point1 = xf_mul(h->hv[best]);
        vx->index2 = 0;
        vx->point2 = xf_mul(Q);
        vx->point = vsub(vx->point2, vx->point1);
        ++iter;
        int duplicate = 0;
        for (uint32_t i = 0; i < saveCount; ++i)
            if (vx->index1 == save1[i] && vx->index2 == save2[i]) {
                duplicate = 1;
                break;
            }
        if (duplicate) break;
        ++s.count;
    }
    gwitness(&s, p1, p2);
    return vlength(vsub(*p1, *p2));
}

/* b3HullShape::TestSphere (hull_shape.cpp:187-254) for a hull on a static
 * body at the origin, shared with the soft body oracle: vertices (3 floats
 * each), planes (normal and offset), the sphere's centre q and radius
 * (particle radius plus hull radius).  On contact: the normal (hull to
 * sphere) and the contact point on the hull; returns 1. */
int oc_hull_test_sphere(const float* vertices, uint32_t nv, const float* planes, uint32_t nf, float radius,
                        const float* q, float* normal_out, float* point_out)
{
    sphere_t h;
    memset(&h, 0, sizeof(h));
    h.nhv = nv;
    h.nhf = nf;
    h.hv = (v3*)malloc((nv ? nv : 1) * sizeof(v3));
    h.hn = (v3*)malloc((nf ? nf : 1) * sizeof(v3));
    h.ho = (float*)malloc((nf ? nf : 1) * sizeof(float));
    for (uint32_t i = 0; i < nv; ++i) h.hv[i] = V(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
    for (uint32_t i = 0; i < nf; ++i) {
        h.hn[i] = V(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2]);
        h.ho[i] = planes[4 * i + 3];
    }
    v3 Q = V(q[0], q[1], q[2]), c1, c2, normal, point;
    int hit = 1;
    float distance = gjk_hull_point(&h, Q, &c1, &c2);
    if (distance > radius) {
        hit = 0;
    } else if (distance > 0.0f) {
        normal = vdiv(vsub(c2, c1), distance);
        point = c1;
    } else {
        v3 support = xf_mult(Q);
        uint32_t maxIndex = ~0u;
        float maxSeparation = -FLT_MAX;
        for (uint32_t f = 0; f < nf && hit; ++f) {
            float separation = vdot(h.hn[f], support) - h.ho[f];
            if (separation > radius) hit = 0;
            else if (separation > maxSeparation) {
                maxIndex = f;
                maxSeparation = separation;
            }
        }
        if (hit) {
            v3 pn = vadd(vadd(vscale(h.hn[maxIndex].x, kIdX), vscale(h.hn[maxIndex].y, kIdY)),
                         vscale(h.hn[maxIndex].z, kIdZ));
            float po = h.ho[maxIndex] + vdot(pn, vzero());
            float fraction = vdot(pn, Q) - po;
            point = vsub(Q, vscale(fraction, pn));
            normal = pn;
        }
    }
    if (hit) {
        normal_out[0] = normal.x; normal_out[1] = normal.y; normal_out[2] = normal.z;
        v3 lp = xf_mult(point); /* body->GetLocalPoint */
        point_out[0] = lp.x; point_out[1] = lp.y; point_out[2] = lp.z;
    }
    free(h.hv); free(h.hn); free(h.ho);
    return hit;
}

void oc_set_solver(oc_cloth* c, int stop_rule, float tol, uint32_t max_iterations, int dot)
{
    c->stop_rule = stop_rule;
    c->tol = tol;
    c->max_iter = max_iterations;
    c->dot = dot;
}

/* ------------------------------------------------------------------------ */
/* force elements                                                            */
/* ------------------------------------------------------------------------ */

static void add9(lrow* rows, const uint32_t* ids, m33 K[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) madd_to(lrow_at(rows + ids[i], ids[j]), K[i][j]);
}

/* b3StrechForce::Apply (strech_force.cpp:59-329) */
static void apply_stretch(oc_cloth* c, const force_t* fo)
{
    uint32_t t = fo->a;
    float alpha = c->alpha[t], du1 = c->du1[t], dv1 = c->dv1[t], du2 = c->du2[t], dv2 = c->dv2[t];
    float inv_det = c->inv_det[t];
    uint32_t ids[3] = {c->solver_of_vertex[c->tris[3 * t]], c->solver_of_vertex[c->tris[3 * t + 1]],
                       c->solver_of_vertex[c->tris[3 * t + 2]]};
    float ks = fo->ks, kd = fo->kd, bu = fo->p0, bv = fo->p1;
    v3 x1 = c->sx[ids[0]], x2 = c->sx[ids[1]], x3 = c->sx[ids[2]];
    v3 vs[3] = {c->sv[ids[0]], c->sv[ids[1]], c->sv[ids[2]]};
    m33 I = mident();
    v3 dx1 = vsub(x2, x1), dx2 = vsub(x3, x1);
    v3 wu = vscale(inv_det, vsub(vscale(dv2, dx1), vscale(dv1, dx2)));
    float len_wu = vlength(wu);
    v3 wv = vscale(inv_det, vadd(vscale(-du2, dx1), vscale(du1, dx2)));
    float len_wv = vlength(wv);
    float dwudx[3] = {inv_det * (dv1 - dv2), inv_det * dv2, -inv_det * dv1};
    float dwvdx[3] = {inv_det * (du2 - du1), -inv_det * du2, inv_det * du1};
    v3 f[3] = {vzero(), vzero(), vzero()};
    m33 K[3][3];

    for (int dir = 0; dir < 2; ++dir) {
        v3 w = dir == 0 ? wu : wv;
        float len = dir == 0 ? len_wu : len_wv;
        const float* dw = dir == 0 ? dwudx : dwvdx;
        float bdir = dir == 0 ? bu : bv;
        if (!(len > 0.0f)) continue;
        float inv_len = 1.0f / len;
        v3 nw = vscale(inv_len, w);
        v3 dC[3];
        for (int i = 0; i < 3; ++i) dC[i] = vscale(alpha * dw[i], nw);
        if (ks > 0.0f && len > bdir) {
            float C = alpha * (len - bdir);
            for (int i = 0; i < 3; ++i) f[i] = vadd(f[i], vscale(-ks * C, dC[i]));
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    m33 d2 = mscale(alpha * inv_len * dw[i] * dw[j], msub(I, mouter(nw, nw)));
                    K[i][j] = mscale(-ks, madd(mouter(dC[i], dC[j]), mscale(C, d2)));
                }
            add9(c->dfdx, ids, K);
        }
        if (kd > 0.0f) {
            float dCdt = 0.0f;
            for (int i = 0; i < 3; ++i) dCdt += vdot(dC[i], vs[i]);
            for (int i = 0; i < 3; ++i) f[i] = vadd(f[i], vscale(-kd * dCdt, dC[i]));
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) K[i][j] = mscale(-kd, mouter(dC[i], dC[j]));
            add9(c->dfdv, ids, K);
        }
    }
    for (int i = 0; i < 3; ++i) c->sf[ids[i]] = vadd(c->sf[ids[i]], f[i]);
}

/* b3ShearForce::Apply (shear_force.cpp:57-212); the second-derivative term
 * is left out as in the reference (:142-144). */
static void apply_shear(oc_cloth* c, const force_t* fo)
{
    uint32_t t = fo->a;
    float alpha = c->alpha[t], du1 = c->du1[t], dv1 = c->dv1[t], du2 = c->du2[t], dv2 = c->dv2[t];
    float inv_det = c->inv_det[t];
    uint32_t ids[3] = {c->solver_of_vertex[c->tris[3 * t]], c->solver_of_vertex[c->tris[3 * t + 1]],
                       c->solver_of_vertex[c->tris[3 * t + 2]]};
    float ks = fo->ks, kd = fo->kd;
    v3 x1 = c->sx[ids[0]], x2 = c->sx[ids[1]], x3 = c->sx[ids[2]];
    v3 vs[3] = {c->sv[ids[0]], c->sv[ids[1]], c->sv[ids[2]]};
    v3 dx1 = vsub(x2, x1), dx2 = vsub(x3, x1);
    v3 wu = vscale(inv_det, vsub(vscale(dv2, dx1), vscale(dv1, dx2)));
    v3 wv = vscale(inv_det, vadd(vscale(-du2, dx1), vscale(du1, dx2)));
    float dwudx[3] = {inv_det * (dv1 - dv2), inv_det * dv2, -inv_det * dv1};
    float dwvdx[3] = {inv_det * (du2 - du1), -inv_det * du2, inv_det * du1};
    v3 f[3] = {vzero(), vzero(), vzero()};
    m33 K[3][3];
    v3 dC[3];
    for (int i = 0; i < 3; ++i) dC[i] = vscale(alpha, vadd(vscale(dwudx[i], wv), vscale(dwvdx[i], wu)));
    if (ks > 0.0f) {
        float C = alpha * vdot(wu, wv);
        for (int i = 0; i < 3; ++i) f[i] = vadd(f[i], vscale(-ks * C, dC[i]));
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) K[i][j] = mscale(-ks, mouter(dC[i], dC[j]));
        add9(c->dfdx, ids, K);
    }
    if (kd > 0.0f) {
        float dCdt = 0.0f;
        for (int i = 0; i < 3; ++i) dCdt += vdot(dC[i], vs[i]);
        for (int i = 0; i < 3; ++i) f[i] = vadd(f[i], vscale(-kd * dCdt, dC[i]));
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) K[i][j] = mscale(-kd, mouter(dC[i], dC[j]));
        add9(c->dfdv, ids, K);
    }
    for (int i = 0; i < 3; ++i) c->sf[ids[i]] = vadd(c->sf[ids[i]], f[i]);
}

/* b3SpringForce::Apply (spring_force.cpp:53-120), including the reference's
 * unnormalised outer product in K11 (:88). */
static void apply_spring(oc_cloth* c, const force_t* fo)
{
    uint32_t i1 = c->solver_of_vertex[fo->a], i2 = c->solver_of_vertex[fo->b];
    float ks = fo->ks, kd = fo->kd, L0 = fo->p0;
    v3 x1 = c->sx[i1], v1 = c->sv[i1], x2 = c->sx[i2], v2_ = c->sv[i2];
    m33 I = mident();
    v3 f = vzero();
    if (ks > 0.0f) {
        v3 dx = vsub(x1, x2);
        float L = vlength(dx);
        if (L > L0) {
            v3 dCdx = vdiv(dx, L);
            f = vadd(f, vscale(-ks * (L - L0), dCdx));
            m33 K11 = mscale(-ks, madd(mouter(dx, dx), mscale(1.0f - L0 / L, msub(I, mouter(dx, dx)))));
            m33 K12 = mscale(-1.0f, K11);
            madd_to(lrow_at(c->dfdx + i1, i1), K11);
            madd_to(lrow_at(c->dfdx + i1, i2), K12);
            madd_to(lrow_at(c->dfdx + i2, i1), K12);
            madd_to(lrow_at(c->dfdx + i2, i2), K11);
        }
    }
    if (kd > 0.0f) {
        v3 dv = vsub(v1, v2_);
        f = vadd(f, vscale(-kd, dv));
        m33 K11 = mscale(-kd, I);
        m33 K12 = mscale(-1.0f, K11);
        madd_to(lrow_at(c->dfdv + i1, i1), K11);
        madd_to(lrow_at(c->dfdv + i1, i2), K12);
        madd_to(lrow_at(c->dfdv + i2, i1), K12);
        madd_to(lrow_at(c->dfdv + i2, i2), K11);
    }
    c->sf[i1] = vadd(c->sf[i1], f);
    c->sf[i2] = vsub(c->sf[i2], f);
}

/* b3MouseForce::Apply (mouse_force.cpp:63-227): particle 1 tied to the point
 * w2 x2 + w3 x3 + w4 x4 of a triangle, C = |x1 - c2|, no second-derivative
 * term; rows receive their blocks in the reference's (i, j) order. */
static void apply_mouse(oc_cloth* c, const force_t* fo)
{
    const uint32_t* tv = c->tris + 3 * (size_t)fo->b;
    const uint32_t ids[4] = {c->solver_of_vertex[fo->a], c->solver_of_vertex[tv[0]], c->solver_of_vertex[tv[1]],
                             c->solver_of_vertex[tv[2]]};
    const float km = fo->ks, kd = fo->kd, w2 = fo->p0, w3 = fo->p1, w4 = fo->p2;
    v3 xs[4], vs[4], mf[4];
    for (int i = 0; i < 4; ++i) {
        xs[i] = c->sx[ids[i]];
        vs[i] = c->sv[ids[i]];
        mf[i] = vzero();
    }
    v3 c2 = vadd(vadd(vscale(w2, xs[1]), vscale(w3, xs[2])), vscale(w4, xs[3]));
    v3 d = vsub(xs[0], c2);
    float len = vlength(d);
    if (len > 0.0f) {
        v3 nrm = vdiv(d, len);
        v3 dCdx[4] = {nrm, vscale(-w2, nrm), vscale(-w3, nrm), vscale(-w4, nrm)};
        if (km > 0.0f) {
            float C = len;
            for (int i = 0; i < 4; ++i) mf[i] = vadd(mf[i], vscale(-km * C, dCdx[i]));
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j)
                    madd_to(lrow_at(c->dfdx + ids[i], ids[j]), mscale(-km, mouter(dCdx[i], dCdx[j])));
        }
        if (kd > 0.0f) {
            float dCdt = 0.0f;
            for (int i = 0; i < 4; ++i) dCdt += vdot(dCdx[i], vs[i]);
            for (int i = 0; i < 4; ++i) mf[i] = vadd(mf[i], vscale(-kd * dCdt, dCdx[i]));
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j)
                    madd_to(lrow_at(c->dfdv + ids[i], ids[j]), mscale(-kd, mouter(dCdx[i], dCdx[j])));
        }
    }
    for (int i = 0; i < 4; ++i) c->sf[ids[i]] = vadd(c->sf[ids[i]], mf[i]);
}

/* ------------------------------------------------------------------------ */
/* created particles and forces (cloth.cpp:307-364)                          */
/* ------------------------------------------------------------------------ */

/* Every per-particle array (state, proxies, list order, solver scratch) to
 * n_new entries; new entries zeroed. */
static void resize_particles(oc_cloth* c, uint32_t n_new)
{
    uint32_t n_old = c->n;
#define GROW(ptr, T)                                                                   \
    do {                                                                               \
        ptr = (T*)realloc(ptr, (size_t)(n_new ? n_new : 1) * sizeof(T));               \
        if (n_new > n_old) memset(ptr + n_old, 0, (size_t)(n_new - n_old) * sizeof(T)); \
    } while (0)
    GROW(c->x, v3); GROW(c->v, v3); GROW(c->f, v3); GROW(c->y, v3); GROW(c->mx, v3);
    GROW(c->mass, float); GROW(c->inv_mass, float); GROW(c->radius, float); GROW(c->friction, float);
    GROW(c->type, uint8_t); GROW(c->fat_lo, v3); GROW(c->fat_hi, v3); GROW(c->p_moved, uint8_t);
    GROW(c->order, uint32_t); GROW(c->solver_of_vertex, uint32_t);
    GROW(c->sx, v3); GROW(c->sv, v3); GROW(c->sf, v3); GROW(c->sy, v3); GROW(c->sx0, v3);
    GROW(c->b, v3); GROW(c->dvsol, v3); GROW(c->Sflag, float);
#undef GROW
    c->a_rowptr = (uint32_t*)realloc(c->a_rowptr, (size_t)(n_new + 1) * sizeof(uint32_t));
    for (uint32_t i = n_new; i < n_old; ++i) {  /* the rows that go: their buffers only */
        free(c->dfdx[i].cols); free(c->dfdx[i].vals);
        free(c->dfdv[i].cols); free(c->dfdv[i].vals);
    }
    c->dfdx = (lrow*)realloc(c->dfdx, (size_t)(n_new ? n_new : 1) * sizeof(lrow));
    c->dfdv = (lrow*)realloc(c->dfdv, (size_t)(n_new ? n_new : 1) * sizeof(lrow));
    if (n_new > n_old) {
        memset(c->dfdx + n_old, 0, (size_t)(n_new - n_old) * sizeof(lrow));
        memset(c->dfdv + n_old, 0, (size_t)(n_new - n_old) * sizeof(lrow));
    }
}

/* b3Cloth::CreateParticle (cloth.cpp:307-322) with b3Particle::b3Particle
 * (particle.cpp:24-51): mass 0 makes a static particle of mass 1; the proxy
 * is the particle's AABB fattened by B3_AABB_EXTENSION; the particle heads
 * the particle list.  Returns its index, after every existing particle. */
uint32_t oc_create_particle(oc_cloth* c, const float* position, const float* velocity, float mass, float radius,
                            float friction)
{
    uint32_t i = c->n;
    resize_particles(c, i + 1);
    c->n = i + 1;
    c->x[i] = V(position[0], position[1], position[2]);
    c->v[i] = velocity ? V(velocity[0], velocity[1], velocity[2]) : vzero();
    if (mass == 0.0f) {
        c->type[i] = OC_STATIC;
        c->mass[i] = 1.0f;
        c->inv_mass[i] = 1.0f;
    } else {
        c->type[i] = OC_DYNAMIC;
        c->mass[i] = mass;
        c->inv_mass[i] = 1.0f / mass;
    }
    c->radius[i] = radius;
    c->friction[i] = friction;
    v3 r = V(radius, radius, radius);
    v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
    c->fat_lo[i] = vsub(vsub(c->x[i], r), ext);
    c->fat_hi[i] = vadd(vadd(c->x[i], r), ext);
    c->p_moved[i] = 1;
    memmove(c->order + 1, c->order, (size_t)i * sizeof(uint32_t));
    c->order[0] = i;
    return i;
}

/* b3Cloth::DestroyParticle (cloth.cpp:324-351) of a created particle: its
 * forces, its contacts and its list entry go; particles created after it
 * move down one index. */
int oc_destroy_particle(oc_cloth* c, uint32_t i)
{
    if (i < c->n_mesh || i >= c->n) return -1;
    uint32_t w = 0;
    for (uint32_t q = 0; q < c->nforce; ++q) {
        const force_t* fo = c->forces + q;
        int has = 0;
        if (fo->type == F_MOUSE) {
            const uint32_t* tv = c->tris + 3 * (size_t)fo->b;
            has = fo->a == i || tv[0] == i || tv[1] == i || tv[2] == i;
        } else if (fo->type == F_SPRING) {
            has = fo->a == i || fo->b == i;
        }
        if (!has) c->forces[w++] = *fo;
    }
    c->nforce = w;
    destroy_particle_contacts(c, i);
    uint32_t k = 0;
    for (uint32_t q = 0; q < c->n; ++q)
        if (c->order[q] != i) c->order[k++] = c->order[q] > i ? c->order[q] - 1 : c->order[q];
    for (uint32_t q = 0; q < c->nforce; ++q)
        if (c->forces[q].type == F_MOUSE && c->forces[q].a > i) c->forces[q].a -= 1;
    for (uint32_t q = 0; q < c->ncontact; ++q)
        if (c->contacts[q].particle > i) c->contacts[q].particle -= 1;
    destroy_particle_triangle_contacts(c, i);
    for (uint32_t q = 0; q < c->ntc; ++q)
        if (c->tcs[q].p > i) c->tcs[q].p -= 1;
    uint32_t tail = c->n - i - 1;
#define SHIFT(ptr) memmove(ptr + i, ptr + i + 1, (size_t)tail * sizeof(*ptr))
    SHIFT(c->x); SHIFT(c->v); SHIFT(c->f); SHIFT(c->y); SHIFT(c->mx);
    SHIFT(c->mass); SHIFT(c->inv_mass); SHIFT(c->radius); SHIFT(c->friction); SHIFT(c->type);
    SHIFT(c->fat_lo); SHIFT(c->fat_hi); SHIFT(c->p_moved);
#undef SHIFT
    resize_particles(c, c->n - 1);
    c->n -= 1;
    return 0;
}

/* b3Cloth::CreateForce (cloth.cpp:353-358) of a b3MouseForceDef
 * (mouse_force.h:26-40): the new force heads the force list. */
uint32_t oc_create_mouse_force(oc_cloth* c, uint32_t particle, uint32_t triangle, float w2, float w3, float w4,
                               float mouse, float damping)
{
    c->forces = (force_t*)realloc(c->forces, (size_t)(c->nforce + 1) * sizeof(force_t));
    memmove(c->forces + 1, c->forces, (size_t)c->nforce * sizeof(force_t));
    force_t f;
    memset(&f, 0, sizeof(f));
    f.type = F_MOUSE;
    f.a = particle;
    f.b = triangle;
    f.ks = mouse;
    f.kd = damping;
    f.p0 = w2;
    f.p1 = w3;
    f.p2 = w4;
    f.id = ++c->next_force_id;
    c->forces[0] = f;
    c->nforce += 1;
    return f.id;
}

/* b3Cloth::DestroyForce (cloth.cpp:360-364) */
int oc_destroy_force(oc_cloth* c, uint32_t id)
{
    for (uint32_t q = 0; q < c->nforce; ++q) {
        if (c->forces[q].type == F_MOUSE && c->forces[q].id == id) {
            memmove(c->forces + q, c->forces + q + 1, (size_t)(c->nforce - q - 1) * sizeof(force_t));
            c->nforce -= 1;
            return 0;
        }
    }
    return -1;
}

uint32_t oc_particle_count(const oc_cloth* c) { return c->n; }

/* ------------------------------------------------------------------------ */
/* system formation                                                          */
/* ------------------------------------------------------------------------ */

/* out = A * v over rows stored in append order, summed in the reference's
 * list order (reverse of append), sparse_mat33.h:264-282. */
static void lrows_mul(const lrow* rows, uint32_t n, const v3* v, v3* out)
{
    for (uint32_t i = 0; i < n; ++i) {
        v3 acc = vzero();
        for (uint32_t k = rows[i].count; k-- > 0;) acc = vadd(acc, mmul(rows[i].vals[k], v[rows[i].cols[k]]));
        out[i] = acc;
    }
}

/* Gather + forces + A and b (cloth_force_solver.cpp:142-204).  A is left in
 * a_rowptr / a_cols / a_vals in the order its linked rows end up in after
 * `M - h * dfdv - (h * h) * dfdx`: blocks that only dfdx touches (in reverse
 * first-touch order), the diagonal, then the dfdv blocks in first-touch
 * order (sparse_mat33.h:153-174 copies reverse a row; :194-216 and :235-250
 * push new blocks to the front). */
static void form_system(oc_cloth* c, float h)
{
    uint32_t n = c->n;
    for (uint32_t k = 0; k < n; ++k) c->solver_of_vertex[c->order[k]] = k;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t i = c->order[k];
        c->sx[k] = c->x[i];
        c->sv[k] = c->v[i];
        c->sf[k] = c->f[i];
        if (c->type[i] == OC_DYNAMIC) {
            c->sf[k] = vadd(c->sf[k], vscale(c->mass[i], c->gravity));
            c->Sflag[k] = 1.0f;
        } else {
            c->Sflag[k] = 0.0f;
        }
        c->sy[k] = c->y[i];
        c->sx0[k] = c->mx[i];
    }
    lrows_clear(c->dfdx, n);
    lrows_clear(c->dfdv, n);
    for (uint32_t q = 0; q < c->nforce; ++q) {
        const force_t* fo = c->forces + q;
        if (fo->type == F_STRETCH) apply_stretch(c, fo);
        else if (fo->type == F_SHEAR) apply_shear(c, fo);
        else if (fo->type == F_MOUSE) apply_mouse(c, fo);
        else apply_spring(c, fo);
    }

    /* A */
    uint32_t nnz = 0;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t cnt = 1;
        for (uint32_t e = 0; e < c->dfdv[k].count; ++e) cnt += c->dfdv[k].cols[e] != k;
        for (uint32_t e = 0; e < c->dfdx[k].count; ++e) {
            uint32_t j = c->dfdx[k].cols[e];
            if (j != k && lrow_find(c->dfdv + k, j) < 0) ++cnt;
        }
        nnz += cnt;
    }
    if (nnz > c->a_cap) {
        c->a_cap = nnz;
        c->a_cols = (uint32_t*)realloc(c->a_cols, nnz * sizeof(uint32_t));
        c->a_vals = (m33*)realloc(c->a_vals, nnz * sizeof(m33));
    }
    float hh = h * h;
    uint32_t w = 0;
    for (uint32_t k = 0; k < n; ++k) {
        c->a_rowptr[k] = w;
        const lrow* D = c->dfdv + k;
        const lrow* K = c->dfdx + k;
        /* dfdx-only blocks, newest first */
        for (uint32_t e = K->count; e-- > 0;) {
            uint32_t j = K->cols[e];
            if (j == k || lrow_find(D, j) >= 0) continue;
            m33 val = mzero();
            msub_to(&val, mscale(hh, K->vals[e]));
            c->a_cols[w] = j;
            c->a_vals[w++] = val;
        }
        /* diagonal */
        {
            m33 val = mdiag3(c->mass[c->order[k]], c->mass[c->order[k]], c->mass[c->order[k]]);
            int d = lrow_find(D, k);
            if (d >= 0) msub_to(&val, mscale(h, D->vals[d]));
            int kk = lrow_find(K, k);
            if (kk >= 0) msub_to(&val, mscale(hh, K->vals[kk]));
            c->a_cols[w] = k;
            c->a_vals[w++] = val;
        }
        /* dfdv blocks in first-touch order */
        for (uint32_t e = 0; e < D->count; ++e) {
            uint32_t j = D->cols[e];
            if (j == k) continue;
            m33 val = mzero();
            msub_to(&val, mscale(h, D->vals[e]));
            int kk = lrow_find(K, j);
            if (kk >= 0) msub_to(&val, mscale(hh, K->vals[kk]));
            c->a_cols[w] = j;
            c->a_vals[w++] = val;
        }
    }
    c->a_rowptr[n] = w;
    c->sys_nnz = w;

    /* b = h * (f + h * (dfdx * v) + dfdx * y) */
    v3* t1 = (v3*)malloc(n * sizeof(v3));
    v3* t2 = (v3*)malloc(n * sizeof(v3));
    lrows_mul(c->dfdx, n, c->sv, t1);
    lrows_mul(c->dfdx, n, c->sy, t2);
    for (uint32_t k = 0; k < n; ++k) {
        v3 s = vadd(vadd(c->sf[k], vscale(h, t1[k])), t2[k]);
        c->b[k] = vscale(h, s);
    }
    free(t1);
    free(t2);
}

/* ------------------------------------------------------------------------ */
/* MPCG                                                                      */
/* ------------------------------------------------------------------------ */

/* Accumulator for a dot product in one of the three precisions. */
typedef struct {
    int mode;
    float s32, c32;
    double s64;
} dacc;

static inline void dacc_init(dacc* a, int mode)
{
    a->mode = mode;
    a->s32 = 0.0f;
    a->c32 = 0.0f;
    a->s64 = 0.0;
}

static inline void dacc_add(dacc* a, v3 x, v3 y)
{
    if (a->mode == OC_DOT_F64) {
        a->s64 += (double)x.x * (double)y.x + (double)x.y * (double)y.y + (double)x.z * (double)y.z;
    } else if (a->mode == OC_DOT_COMPENSATED) {
        /* Neumaier's variant of Kahan summation over the per-row terms */
        float term = vdot(x, y);
        float t = a->s32 + term;
        if (fabsf(a->s32) >= fabsf(term)) a->c32 += (a->s32 - t) + term;
        else a->c32 += (term - t) + a->s32;
        a->s32 = t;
    } else {
        a->s32 += vdot(x, y);
    }
}

static inline double dacc_get(const dacc* a)
{
    if (a->mode == OC_DOT_F64) return a->s64;
    if (a->mode == OC_DOT_COMPENSATED) return (double)(a->s32 + a->c32);
    return (double)a->s32;
}

static void csr_mul(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const m33* vals, const v3* v,
                    v3* out)
{
    for (uint32_t i = 0; i < n; ++i) {
        v3 acc = vzero();
        for (uint32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) acc = vadd(acc, mmul(vals[k], v[cols[k]]));
        out[i] = acc;
    }
}

static uint32_t mpcg(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const m33* vals, const v3* b,
                     const float* Sflag, const v3* y, int stop_rule, float tol, uint32_t max_iter, int dot,
                     v3* x, double* stats)
{
    m33* S = (m33*)malloc(n * sizeof(m33));
    m33* IS = (m33*)malloc(n * sizeof(m33));
    m33* invP = (m33*)malloc(n * sizeof(m33));
    v3* r = (v3*)malloc(n * sizeof(v3));
    v3* p = (v3*)malloc(n * sizeof(v3));
    v3* s = (v3*)malloc(n * sizeof(v3));
    v3* hv = (v3*)malloc(n * sizeof(v3));
    v3* tmp = (v3*)calloc(n + 1, sizeof(v3));
    v3* tmp2 = (v3*)malloc(n * sizeof(v3));
    v3* bhat = (v3*)malloc(n * sizeof(v3));

    /* Jacobi preconditioner from the diagonal blocks (:70-88) */
    for (uint32_t i = 0; i < n; ++i) {
        m33 a = mzero();
        for (uint32_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (cols[k] == i) { a = vals[k]; break; }
        invP[i] = mdiag3(1.0f / a.x.x, 1.0f / a.y.y, 1.0f / a.z.z);
        S[i] = Sflag[i] != 0.0f ? mident() : mzero();
        IS[i] = msub(mident(), S[i]);
    }
    /* x = S y + (I - S) z with z = 0 (:90) */
    for (uint32_t i = 0; i < n; ++i) {
        tmp[i] = mmul(IS[i], vzero());
        x[i] = vadd(mmul(S[i], y[i]), tmp[i]);
    }
    /* b_hat = S (b - A (I - S) z) (:92) */
    csr_mul(n, rowptr, cols, vals, tmp, tmp2);
    for (uint32_t i = 0; i < n; ++i) bhat[i] = mmul(S[i], vsub(b[i], tmp2[i]));
    dacc acc;
    dacc_init(&acc, dot);
    for (uint32_t i = 0; i < n; ++i) dacc_add(&acc, bhat[i], mmul(invP[i], bhat[i]));
    double b_delta = dacc_get(&acc);
    /* r = S (b - A x), p = S P^-1 r, delta = r.p (:96-100) */
    csr_mul(n, rowptr, cols, vals, x, tmp2);
    for (uint32_t i = 0; i < n; ++i) r[i] = mmul(S[i], vsub(b[i], tmp2[i]));
    for (uint32_t i = 0; i < n; ++i) p[i] = mmul(S[i], mmul(invP[i], r[i]));
    dacc_init(&acc, dot);
    for (uint32_t i = 0; i < n; ++i) dacc_add(&acc, r[i], p[i]);
    double delta_new = dacc_get(&acc);
    if (dot == OC_DOT_F32 || dot == OC_DOT_COMPENSATED) {
        b_delta = (float)b_delta;
        delta_new = (float)delta_new;
    }
    double delta0 = delta_new;

    uint32_t it = 0;
    for (;;) {
        if (it == max_iter) break;
        if (stop_rule == OC_STOP_REFERENCE) {
            if (dot == OC_DOT_F64) {
                if (delta_new <= (double)(kEps * kEps) * b_delta) break;
            } else if ((float)delta_new <= kEps * kEps * (float)b_delta) {
                break;
            }
        } else if (delta_new <= (double)tol * (double)tol * b_delta) {
            break;
        }
        csr_mul(n, rowptr, cols, vals, p, tmp);
        for (uint32_t i = 0; i < n; ++i) s[i] = mmul(S[i], tmp[i]);
        dacc_init(&acc, dot);
        for (uint32_t i = 0; i < n; ++i) dacc_add(&acc, p[i], s[i]);
        float alpha;
        if (dot == OC_DOT_F64) alpha = (float)(delta_new / dacc_get(&acc));
        else alpha = (float)delta_new / (float)dacc_get(&acc);
        for (uint32_t i = 0; i < n; ++i) x[i] = vadd(x[i], vscale(alpha, p[i]));
        for (uint32_t i = 0; i < n; ++i) r[i] = vsub(r[i], vscale(alpha, s[i]));
        for (uint32_t i = 0; i < n; ++i) hv[i] = mmul(invP[i], r[i]);
        double delta_old = delta_new;
        dacc_init(&acc, dot);
        for (uint32_t i = 0; i < n; ++i) dacc_add(&acc, r[i], hv[i]);
        delta_new = dacc_get(&acc);
        float beta;
        if (dot == OC_DOT_F64) {
            beta = (float)(delta_new / delta_old);
        } else {
            delta_new = (float)delta_new;
            beta = (float)delta_new / (float)delta_old;
        }
        for (uint32_t i = 0; i < n; ++i) p[i] = mmul(S[i], vadd(hv[i], vscale(beta, p[i])));
        ++it;
    }
    if (stats) {
        stats[0] = delta0;
        stats[1] = b_delta;
        stats[2] = delta_new;
    }
    free(S); free(IS); free(invP); free(r); free(p); free(s); free(hv); free(tmp); free(tmp2); free(bhat);
    return it;
}

uint32_t oc_mpcg(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals, const float* b,
                 const float* S, const float* x0, int stop_rule, float tol, uint32_t max_iterations, int dot,
                 float* x, double* stats)
{
    return mpcg(n, rowptr, cols, (const m33*)vals, (const v3*)b, S, (const v3*)x0, stop_rule, tol,
                max_iterations, dot, (v3*)x, stats);
}

/* FP64 filtered Jacobi-PCG on the same system, for error reports. */
uint32_t oc_solve_f64(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals,
                      const float* b, const float* S, const float* x0, double tol, uint32_t max_iterations,
                      double* x)
{
    double* A = (double*)malloc((size_t)rowptr[n] * 9 * sizeof(double));
    for (size_t k = 0; k < (size_t)rowptr[n] * 9; ++k) A[k] = vals[k];
    double* invP = (double*)malloc(3 * (size_t)n * sizeof(double));
    double* r = (double*)malloc(3 * (size_t)n * sizeof(double));
    double* p = (double*)malloc(3 * (size_t)n * sizeof(double));
    double* s = (double*)malloc(3 * (size_t)n * sizeof(double));
    double* tmp = (double*)calloc(3 * (size_t)n, sizeof(double));
    for (uint32_t i = 0; i < n; ++i) {
        const double* a = NULL;
        for (uint32_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (cols[k] == i) { a = A + 9 * (size_t)k; break; }
        for (int d = 0; d < 3; ++d) invP[3 * i + d] = a ? 1.0 / a[4 * d] : 0.0;
        for (int d = 0; d < 3; ++d) x[3 * i + d] = S[i] != 0.0f ? (double)x0[3 * i + d] : 0.0;
    }
#define SPMV(in, out)                                                                  \
    for (uint32_t i = 0; i < n; ++i) {                                                 \
        double a0 = 0, a1 = 0, a2 = 0;                                                 \
        for (uint32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {                         \
            const double* m = A + 9 * (size_t)k;                                       \
            const double* v = in + 3 * (size_t)cols[k];                                \
            a0 += m[0] * v[0] + m[3] * v[1] + m[6] * v[2];                             \
            a1 += m[1] * v[0] + m[4] * v[1] + m[7] * v[2];                             \
            a2 += m[2] * v[0] + m[5] * v[1] + m[8] * v[2];                             \
        }                                                                              \
        out[3 * i] = a0; out[3 * i + 1] = a1; out[3 * i + 2] = a2;                     \
    }
    double b_delta = 0.0;
    for (uint32_t i = 0; i < n; ++i)
        if (S[i] != 0.0f)
            for (int d = 0; d < 3; ++d) b_delta += (double)b[3 * i + d] * b[3 * i + d] * invP[3 * i + d];
    SPMV(x, tmp);
    double delta = 0.0;
    for (uint32_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            size_t q = 3 * (size_t)i + d;
            r[q] = S[i] != 0.0f ? (double)b[q] - tmp[q] : 0.0;
            p[q] = invP[q] * r[q];
            delta += r[q] * p[q];
        }
    uint32_t it = 0;
    while (it < max_iterations && delta > tol * tol * b_delta) {
        SPMV(p, s);
        double ps = 0.0;
        for (uint32_t i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) {
                size_t q = 3 * (size_t)i + d;
                if (S[i] == 0.0f) s[q] = 0.0;
                ps += p[q] * s[q];
            }
        double alpha = delta / ps;
        double dn = 0.0;
        for (size_t q = 0; q < 3 * (size_t)n; ++q) {
            x[q] += alpha * p[q];
            r[q] -= alpha * s[q];
            dn += r[q] * r[q] * invP[q];
        }
        double beta = dn / delta;
        delta = dn;
        for (uint32_t i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) {
                size_t q = 3 * (size_t)i + d;
                p[q] = S[i] != 0.0f ? invP[q] * r[q] + beta * p[q] : 0.0;
            }
        ++it;
    }
#undef SPMV
    free(A); free(invP); free(r); free(p); free(s); free(tmp);
    return it;
}

/* ------------------------------------------------------------------------ */
/* body contacts                                                             */
/* ------------------------------------------------------------------------ */

static inline int aabb_overlap(v3 alo, v3 ahi, v3 blo, v3 bhi)
{
    /* b3TestOverlap (aabb3.h:247-251) */
    return alo.x <= bhi.x && alo.y <= bhi.y && alo.z <= bhi.z && ahi.x >= blo.x && ahi.y >= blo.y &&
           ahi.z >= blo.z;
}

/* b3ParticleBodyContact::Update (cloth_particle_body_contact.cpp:24-47) with
 * b3SphereShape::TestSphere (sphere_shape.cpp:71-95) for a static body whose
 * frame is the identity rotation at the sphere centre. */
static void contact_update(oc_cloth* c, contact_t* k)
{
    const sphere_t* sp = c->spheres + k->shape;
    uint32_t i = k->particle;
    float radius = sp->radius + c->radius[i];
    v3 Q = c->x[i];
    v3 normal, point;
    if (sp->kind == SHAPE_SPHERE) {
        /* b3SphereShape::TestSphere (sphere_shape.cpp:71-95) */
        float rr = radius * radius;
        v3 d = vsub(Q, sp->center);
        float dd = vdot(d, d);
        if (!(dd <= rr)) {
            k->active = 0;
            return;
        }
        float d_len = sqrtf(dd);
        normal = V(0.0f, 1.0f, 0.0f);
        if (d_len > kEps) normal = vdiv(d, d_len);
        point = sp->center;
    } else if (sp->kind == SHAPE_HULL) {
        /* b3HullShape::TestSphere (hull_shape.cpp:187-254): GJK between the
         * hull and the particle's point; inside the hull, the face of
         * largest separation */
        v3 c1, c2;
        float distance = gjk_hull_point(sp, Q, &c1, &c2);
        float total = sp->radius + c->radius[i];
        if (distance > total) {
            k->active = 0;
            return;
        }
        if (distance > 0.0f) {
            normal = vdiv(vsub(c2, c1), distance);
            point = c1;
        } else {
            v3 support = xf_mult(Q);
            uint32_t maxIndex = ~0u;
            float maxSeparation = -FLT_MAX;
            for (uint32_t f = 0; f < sp->nhf; ++f) {
                float separation = vdot(sp->hn[f], support) - sp->ho[f];
                if (separation > total) {
                    k->active = 0;
                    return;
                }
                if (separation > maxSeparation) {
                    maxIndex = f;
                    maxSeparation = separation;
                }
            }
            /* b3Mul(xf, plane) (geometry.h:77-81), b3ClosestPointOnPlane (:96-100) */
            v3 pn = vadd(vadd(vscale(sp->hn[maxIndex].x, kIdX), vscale(sp->hn[maxIndex].y, kIdY)),
                         vscale(sp->hn[maxIndex].z, kIdZ));
            float po = sp->ho[maxIndex] + vdot(pn, vzero());
            float fraction = vdot(pn, Q) - po;
            point = vsub(Q, vscale(fraction, pn));
            normal = pn;
        }
    } else {
        /* b3CapsuleShape::TestSphere (capsule_shape.cpp:186-284) */
        v3 A = sp->a, B = sp->b;
        v3 AB = vsub(B, A);
        float u = vdot(vsub(B, Q), AB);
        float v = vdot(vsub(Q, A), AB);
        if (v <= 0.0f || u <= 0.0f) {
            v3 P = v <= 0.0f ? A : B;
            v3 d = vsub(Q, P);
            float dd = vdot(d, d);
            if (dd > radius * radius) {
                k->active = 0;
                return;
            }
            normal = V(0.0f, 1.0f, 0.0f);
            float len = sqrtf(dd);
            if (len > kEps) normal = vdiv(d, len);
            point = P;
        } else {
            float ss = vdot(AB, AB);
            v3 P;
            if (ss < kLinearSlop * kLinearSlop) P = A;
            else P = vdiv(vadd(vscale(u, A), vscale(v, B)), ss);
            v3 d = vsub(Q, P);
            float dd = vdot(d, d);
            if (dd > radius * radius) {
                k->active = 0;
                return;
            }
            v3 QA = vsub(A, Q);
            v3 e = vcross(AB, QA);
            v3 nn = vcross(AB, e);
            if (vdot(nn, QA) < 0.0f) nn = vneg(nn);
            float len = sqrtf(nn.x * nn.x + nn.y * nn.y + nn.z * nn.z); /* b3Vec3::Normalize (vec3.h:93-104) */
            if (len > kEps) {
                float s1 = 1.0f / len;
                nn = V(nn.x * s1, nn.y * s1, nn.z * s1);
            }
            normal = vneg(nn);
            point = P;
        }
    }
    k->active = 1;
    k->normal1 = vneg(normal);
    /* body->GetLocalPoint(point) for a static body: the sphere's body sits at
     * its centre, the capsule's at the origin */
    k->local_point2 = sp->kind == SHAPE_SPHERE ? vzero() : sp->kind == SHAPE_HULL ? xf_mult(point) : point;
    k->tangent1 = vperp(k->normal1);
    k->tangent2 = vcross(k->tangent1, k->normal1);
}

/* ------------------------------------------------------------------------ */
/* colliders on bodies: transforms, shape tests, the body API               */
/* ------------------------------------------------------------------------ */

/* b3Mul / b3MulT of a matrix, a transform, a quaternion (mat33.h:129-160,
 * transform.h:74-110, quat.h:225-238), in the reference's float order. */
static inline v3 mmul_t(m33 a, v3 v) { return V(vdot(a.x, v), vdot(a.y, v), vdot(a.z, v)); }
static inline v3 xmul(m33 R, v3 p, v3 v) { return vadd(mmul(R, v), p); }
static inline v3 xmul_t(m33 R, v3 p, v3 v) { return mmul_t(R, vsub(v, p)); }
static inline m33 mmul3(m33 a, m33 b) { return M3(mmul(a, b.x), mmul(a, b.y), mmul(a, b.z)); }
static inline m33 mtrans(m33 a) { return M3(V(a.x.x, a.y.x, a.z.x), V(a.x.y, a.y.y, a.z.y), V(a.x.z, a.y.z, a.z.z)); }
static inline quat Qt(float x, float y, float z, float w) { quat q = {x, y, z, w}; return q; }
static inline quat qmul(quat a, quat b) /* quat.h:172-180 */
{
    return Qt(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
              a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
static inline void qnormalize(quat* q) /* b3Quat::Normalize (quat.h:88-100) */
{
    float length = sqrtf(q->x * q->x + q->y * q->y + q->z * q->z + q->w * q->w);
    if (length > kEps) {
        float s = 1.0f / length;
        q->x *= s; q->y *= s; q->z *= s; q->w *= s;
    }
}
static inline m33 qmat(quat q) /* b3QuatMat33 (quat.h:306-318) */
{
    float x = q.x, y = q.y, z = q.z, w = q.w;
    float x2 = x + x, y2 = y + y, z2 = z + z;
    float xx = x * x2, xy = x * y2, xz = x * z2;
    float yy = y * y2, yz = y * z2, zz = z * z2;
    float wx = w * x2, wy = w * y2, wz = w * z2;
    return M3(V(1.0f - (yy + zz), xy + wz, xz - wy), V(xy - wz, 1.0f - (xx + zz), yz + wx),
              V(xz + wy, yz - wx, 1.0f - (xx + yy)));
}
static inline v3 qrot(quat q, v3 v) /* b3Mul(b3Quat, b3Vec3) (quat.h:225-232) */
{
    v3 qv = V(q.x, q.y, q.z);
    v3 t = vscale(2.0f, vcross(qv, v));
    return vadd(vadd(v, vscale(q.w, t)), vcross(qv, t));
}
static inline quat qderiv(quat q, v3 w) /* b3Derivative (time_step.h:105-109) */
{
    return qmul(Qt(0.5f * w.x, 0.5f * w.y, 0.5f * w.z, 0.0f), q);
}

/* The body a shape sits on; a world-frame shape's implicit static body. */
static body_t shape_body(const oc_cloth* c, const sphere_t* sp)
{
    if (sp->body >= 0) return c->bodies[sp->body];
    body_t b;
    memset(&b, 0, sizeof(b));
    b.R = mident();
    b.p = sp->kind == SHAPE_SPHERE ? sp->center : vzero();
    b.c0 = b.c = b.p;
    b.q0 = b.q = Qt(0.0f, 0.0f, 0.0f, 1.0f);
    return b;
}

/* b3Shape::ComputeAABB with a transform (sphere_shape.cpp:53-59,
 * capsule_shape.cpp:130-137, hull_shape.cpp:162-166 with b3AABB3::Set). */
static void shape_aabb(const sphere_t* sp, m33 R, v3 p, v3* lo, v3* hi)
{
    v3 r = V(sp->radius, sp->radius, sp->radius);
    if (sp->kind == SHAPE_SPHERE) {
        v3 ctr = xmul(R, p, sp->center);
        *lo = vsub(ctr, r);
        *hi = vadd(ctr, r);
    } else if (sp->kind == SHAPE_CAPSULE) {
        v3 c1 = xmul(R, p, sp->a), c2 = xmul(R, p, sp->b);
        *lo = vsub(vmin(c1, c2), r);
        *hi = vadd(vmax(c1, c2), r);
    } else {
        v3 l = xmul(R, p, sp->hv[0]), h = l;
        for (uint32_t i = 1; i < sp->nhv; ++i) {
            v3 w = xmul(R, p, sp->hv[i]);
            l = vmin(l, w);
            h = vmax(h, w);
        }
        *lo = vsub(l, r);
        *hi = vadd(h, r);
    }
}

/* b3GJK (gjk.cpp:579-740) between a hull on a body (transform R, p) and a
 * point in the world frame: supports in the hull's frame
 * (b3MulT(xf1.rotation, -d)), vertices mapped by b3Mul(xf1, v). */
static float gjk_hull_point_xf(const sphere_t* h, m33 R, v3 p, v3 Q, v3* p1, v3* p2)
{
    gjk_simplex s;
    memset(&s, 0, sizeof(s));
    s.v[0].point1 = xmul(R, p, h->hv[0]);
    s.v[0].point2 = xf_mul(Q);
    s.v[0].point = vsub(s.v[0].point2, s.v[0].point1);
    s.v[0].weight = 1.0f;
    s.count = 1;
    uint32_t save1[4], save2[4], saveCount = 0;
    const v3 origin = vzero();
    uint32_t iter = 0;
    while (iter < 20) {
        saveCount = s.count;
        for (uint32_t i = 0; i < saveCount; ++i) {
            save1[i] = s.v[i].index1;
            save2[i] = s.v[i].index2;
        }
        if (s.count == 2) gsolve2(&s, origin);
        else if (s.count == 3) gsolve3(&s, origin);
        else if (s.count == 4) gsolve4(&s, origin);
        if (s.count == 4) break;
        (void)gclosest(&s);
        v3 d = gsearch(&s, origin);
        if (vdot(d, d) < kEps * kEps) break;
        gjk_vertex* vx = s.v + s.count;
        v3 dl = mmul_t(R, vneg(d));
        uint32_t best = 0;
        float bestp = vdot(dl, h->hv[0]);
        for (uint32_t i = 1; i < h->nhv; ++i) {
            float pr = vdot(dl, h->hv[i]);
            if (pr > bestp) {
                best = i;
                bestp = pr;
            }
        }
        vx->index1 = best;
        vx->point1 = xmul(R, p, h->hv[best]);
        vx->index2 = 0;
        vx->point2 = xf_mul(Q);
        vx->point = vsub(vx->point2, vx->point1);
        ++iter;
        int duplicate = 0;
        for (uint32_t i = 0; i < saveCount; ++i)
            if (vx->index1 == save1[i] && vx->index2 == save2[i]) {
                duplicate = 1;
                break;
            }
        if (duplicate) break;
        ++s.count;
    }
    gwitness(&s, p1, p2);
    return vlength(vsub(*p1, *p2));
}

/* b3ParticleBodyContact::Update (cloth_particle_body_contact.cpp:24-47) for a
 * shape on a body: TestSphere with the body's transform m_xf, the contact
 * point stored in the body's frame (GetLocalPoint). */
static void contact_update_body(oc_cloth* c, contact_t* k)
{
    const sphere_t* sp = c->spheres + k->shape;
    const body_t* bd = c->bodies + sp->body;
    m33 R = bd->R;
    v3 p = bd->p;
    uint32_t i = k->particle;
    float radius = sp->radius + c->radius[i];
    v3 Q = c->x[i];
    v3 normal, point;
    if (sp->kind == SHAPE_SPHERE) {
        v3 center = xmul(R, p, sp->center);
        float rr = radius * radius;
        v3 d = vsub(Q, center);
        float dd = vdot(d, d);
        if (!(dd <= rr)) {
            k->active = 0;
            return;
        }
        float d_len = sqrtf(dd);
        normal = V(0.0f, 1.0f, 0.0f);
        if (d_len > kEps) normal = vdiv(d, d_len);
        point = center;
    } else if (sp->kind == SHAPE_HULL) {
        v3 c1, c2;
        float distance = gjk_hull_point_xf(sp, R, p, Q, &c1, &c2);
        float total = sp->radius + c->radius[i];
        if (distance > total) {
            k->active = 0;
            return;
        }
        if (distance > 0.0f) {
            normal = vdiv(vsub(c2, c1), distance);
            point = c1;
        } else {
            v3 support = xmul_t(R, p, Q);
            uint32_t maxIndex = ~0u;
            float maxSeparation = -FLT_MAX;
            for (uint32_t f = 0; f < sp->nhf; ++f) {
                float separation = vdot(sp->hn[f], support) - sp->ho[f];
                if (separation > total) {
                    k->active = 0;
                    return;
                }
                if (separation > maxSeparation) {
                    maxIndex = f;
                    maxSeparation = separation;
                }
            }
            v3 pn = mmul(R, sp->hn[maxIndex]);
            float po = sp->ho[maxIndex] + vdot(pn, p);
            float fraction = vdot(pn, Q) - po;
            point = vsub(Q, vscale(fraction, pn));
            normal = pn;
        }
    } else {
        v3 A = xmul(R, p, sp->a), B = xmul(R, p, sp->b);
        v3 AB = vsub(B, A);
        float u = vdot(vsub(B, Q), AB);
        float v = vdot(vsub(Q, A), AB);
        if (v <= 0.0f || u <= 0.0f) {
            v3 P = v <= 0.0f ? A : B;
            v3 d = vsub(Q, P);
            float dd = vdot(d, d);
            if (dd > radius * radius) {
                k->active = 0;
                return;
            }
            normal = V(0.0f, 1.0f, 0.0f);
            float len = sqrtf(dd);
            if (len > kEps) normal = vdiv(d, len);
            point = P;
        } else {
            float ss = vdot(AB, AB);
            v3 P;
            if (ss < kLinearSlop * kLinearSlop) P = A;
            else P = vdiv(vadd(vscale(u, A), vscale(v, B)), ss);
            v3 d = vsub(Q, P);
            float dd = vdot(d, d);
            if (dd > radius * radius) {
                k->active = 0;
                return;
            }
            v3 QA = vsub(A, Q);
            v3 e = vcross(AB, QA);
            v3 nn = vcross(AB, e);
            if (vdot(nn, QA) < 0.0f) nn = vneg(nn);
            float len = sqrtf(nn.x * nn.x + nn.y * nn.y + nn.z * nn.z);
            if (len > kEps) {
                float s1 = 1.0f / len;
                nn = V(nn.x * s1, nn.y * s1, nn.z * s1);
            }
            normal = vneg(nn);
            point = P;
        }
    }
    k->active = 1;
    k->normal1 = vneg(normal);
    k->local_point2 = xmul_t(R, p, point);
    k->tangent1 = vperp(k->normal1);
    k->tangent2 = vcross(k->tangent1, k->normal1);
}

/* Body state as 55 floats: type, R (9, column-major), p, local center,
 * world center 0, world center, orientation 0 (x y z w), orientation,
 * linear and angular velocity, inverse mass, local inverse inertia (9),
 * world inverse inertia (9). */
static void body_read(body_t* b, const float* d)
{
    b->type = (int)d[0];
    b->R = M3(V(d[1], d[2], d[3]), V(d[4], d[5], d[6]), V(d[7], d[8], d[9]));
    b->p = V(d[10], d[11], d[12]);
    b->lc = V(d[13], d[14], d[15]);
    b->c0 = V(d[16], d[17], d[18]);
    b->c = V(d[19], d[20], d[21]);
    b->q0 = Qt(d[22], d[23], d[24], d[25]);
    b->q = Qt(d[26], d[27], d[28], d[29]);
    b->v = V(d[30], d[31], d[32]);
    b->w = V(d[33], d[34], d[35]);
    b->im = d[36];
    b->ii = M3(V(d[37], d[38], d[39]), V(d[40], d[41], d[42]), V(d[43], d[44], d[45]));
    b->wii = M3(V(d[46], d[47], d[48]), V(d[49], d[50], d[51]), V(d[52], d[53], d[54]));
}

static void put_v3(float* o, v3 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

static void body_write(const body_t* b, float* d)
{
    d[0] = (float)b->type;
    put_v3(d + 1, b->R.x); put_v3(d + 4, b->R.y); put_v3(d + 7, b->R.z);
    put_v3(d + 10, b->p); put_v3(d + 13, b->lc); put_v3(d + 16, b->c0); put_v3(d + 19, b->c);
    d[22] = b->q0.x; d[23] = b->q0.y; d[24] = b->q0.z; d[25] = b->q0.w;
    d[26] = b->q.x; d[27] = b->q.y; d[28] = b->q.z; d[29] = b->q.w;
    put_v3(d + 30, b->v); put_v3(d + 33, b->w);
    d[36] = b->im;
    put_v3(d + 37, b->ii.x); put_v3(d + 40, b->ii.y); put_v3(d + 43, b->ii.z);
    put_v3(d + 46, b->wii.x); put_v3(d + 49, b->wii.y); put_v3(d + 52, b->wii.z);
}

int oc_add_body(oc_cloth* c, const float* desc)
{
    c->bodies = (body_t*)realloc(c->bodies, (c->nbody + 1) * sizeof(body_t));
    body_read(c->bodies + c->nbody, desc);
    return (int)c->nbody++;
}

void oc_set_body(oc_cloth* c, uint32_t body, const float* desc) { body_read(c->bodies + body, desc); }
void oc_get_body(const oc_cloth* c, uint32_t body, float* desc) { body_write(c->bodies + body, desc); }

/* A shape on a body, its geometry in the body's frame (b3Body::CreateShape):
 * sphere: centre (3 floats); capsule: the segment's ends (6); hull: nv
 * vertices then nf planes (normal, offset).  Its proxy in the world
 * broadphase starts as ComputeAABB(m_xf) fattened (broad_phase.cpp:78-90). */
int oc_add_body_shape(oc_cloth* c, uint32_t body, int kind, const float* geom, uint32_t nv, uint32_t nf,
                      float radius, float friction)
{
    c->spheres = (sphere_t*)realloc(c->spheres, (c->nsphere + 1) * sizeof(sphere_t));
    sphere_t* s = c->spheres + c->nsphere;
    memset(s, 0, sizeof(*s));
    s->kind = kind;
    s->body = (int)body;
    s->radius = radius;
    s->friction = friction;
    if (kind == SHAPE_SPHERE) {
        s->center = V(geom[0], geom[1], geom[2]);
    } else if (kind == SHAPE_CAPSULE) {
        s->a = V(geom[0], geom[1], geom[2]);
        s->b = V(geom[3], geom[4], geom[5]);
    } else {
        s->nhv = nv;
        s->nhf = nf;
        s->hv = (v3*)malloc((nv ? nv : 1) * sizeof(v3));
        s->hn = (v3*)malloc((nf ? nf : 1) * sizeof(v3));
        s->ho = (float*)malloc((nf ? nf : 1) * sizeof(float));
        for (uint32_t i = 0; i < nv; ++i) s->hv[i] = V(geom[3 * i], geom[3 * i + 1], geom[3 * i + 2]);
        const float* pl = geom + 3 * (size_t)nv;
        for (uint32_t i = 0; i < nf; ++i) {
            s->hn[i] = V(pl[4 * i], pl[4 * i + 1], pl[4 * i + 2]);
            s->ho[i] = pl[4 * i + 3];
        }
    }
    const body_t* b = c->bodies + body;
    v3 lo, hi, ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
    shape_aabb(s, b->R, b->p, &lo, &hi);
    s->fat_lo = vsub(lo, ext);
    s->fat_hi = vadd(hi, ext);
    return (int)c->nsphere++;
}

/* The order in which the caller's world query reports the shapes (its
 * dynamic tree's order), replacing the one derived from inserting the
 * proxies in creation order; count 0 returns to the derived one. */
void oc_set_report_order(oc_cloth* c, const uint32_t* order, uint32_t count)
{
    c->has_report = count > 0;
    for (uint32_t s = 0; s < count && s < WO_MAX; ++s) c->report[s] = order[s];
}

void oc_set_shape_proxy(oc_cloth* c, uint32_t shape, const float* lo, const float* hi)
{
    c->spheres[shape].fat_lo = V(lo[0], lo[1], lo[2]);
    c->spheres[shape].fat_hi = V(hi[0], hi[1], hi[2]);
}

void oc_get_shape_proxy(const oc_cloth* c, uint32_t shape, float* lo, float* hi)
{
    put_v3(lo, c->spheres[shape].fat_lo);
    put_v3(hi, c->spheres[shape].fat_hi);
}

/* UpdateBodyContacts (cloth_contact_manager.cpp:277-315). */
static void update_body_contacts(oc_cloth* c)
{
    /* walk the list from its head (the array's end) and compact */
    uint32_t n = c->ncontact;
    uint8_t* keep = (uint8_t*)malloc(n + 1);
    for (uint32_t q = n; q-- > 0;) {
        contact_t* k = c->contacts + q;
        keep[q] = 0;
        const sphere_t* sp = c->spheres + k->shape;
        /* neither side dynamic: the pair must not collide */
        const int body_dynamic = sp->body >= 0 && c->bodies[sp->body].type == 2;
        if (c->type[k->particle] != OC_DYNAMIC && !body_dynamic) continue;
        if (!aabb_overlap(c->fat_lo[k->particle], c->fat_hi[k->particle], sp->fat_lo, sp->fat_hi)) continue;
        if (sp->body >= 0) contact_update_body(c, k);
        else contact_update(c, k);
        keep[q] = 1;
    }
    uint32_t w = 0;
    for (uint32_t q = 0; q < n; ++q)
        if (keep[q]) c->contacts[w++] = c->contacts[q];
    c->ncontact = w;
    free(keep);
}

/* FindNewBodyContacts + AddPSPair (cloth_contact_manager.cpp:64-123).  The
 * world broadphase reports every shape whose fat AABB overlaps the
 * particle's; a new contact is pushed to the list front. */
static void find_new_body_contacts(oc_cloth* c)
{
    if (c->nsphere == 0) return;
    /* which (particle, shape) pairs already have a contact */
    uint8_t* has = (uint8_t*)calloc((size_t)c->n * c->nsphere, 1);
    for (uint32_t q = 0; q < c->ncontact; ++q)
        has[(size_t)c->contacts[q].particle * c->nsphere + c->contacts[q].shape] = 1;
    /* the world query reports the shapes in its tree's order */
    float wlo[WO_MAX][3], whi[WO_MAX][3];
    uint32_t report[WO_MAX];
    for (uint32_t s = 0; s < c->nsphere && s < WO_MAX; ++s) {
        wlo[s][0] = c->spheres[s].fat_lo.x; wlo[s][1] = c->spheres[s].fat_lo.y; wlo[s][2] = c->spheres[s].fat_lo.z;
        whi[s][0] = c->spheres[s].fat_hi.x; whi[s][1] = c->spheres[s].fat_hi.y; whi[s][2] = c->spheres[s].fat_hi.z;
    }
    world_report_order(wlo, whi, c->nsphere, report);
    if (c->has_report)
        for (uint32_t s = 0; s < c->nsphere && s < WO_MAX; ++s) report[s] = c->report[s];
    for (uint32_t k = 0; k < c->n; ++k) {
        uint32_t i = c->order[k];
        if (c->type[i] != OC_DYNAMIC) continue;
        for (uint32_t r = 0; r < c->nsphere; ++r) {
            const uint32_t s = report[r];
            const sphere_t* sp = c->spheres + s;
            if (!aabb_overlap(c->fat_lo[i], c->fat_hi[i], sp->fat_lo, sp->fat_hi)) continue;
            if (has[(size_t)i * c->nsphere + s]) continue;
            has[(size_t)i * c->nsphere + s] = 1;
            if (c->ncontact == c->contact_cap) {
                c->contact_cap = c->contact_cap ? 2 * c->contact_cap : 1024;
                c->contacts = (contact_t*)realloc(c->contacts, c->contact_cap * sizeof(contact_t));
            }
            contact_t* nk = c->contacts + c->ncontact++;
            memset(nk, 0, sizeof(*nk));
            nk->particle = i;
            nk->shape = s;
            nk->active = 0;
        }
    }
    free(has);
}

/* ------------------------------------------------------------------------ */
/* self-collision: particle-triangle contacts                                */
/* ------------------------------------------------------------------------ */

/* b3BarycentricCoordinates for a segment and a triangle (geometry.h:105-145). */
static void bary2(float out[3], v3 A, v3 B, v3 Q)
{
    v3 AB = vsub(B, A), QA = vsub(A, Q), QB = vsub(B, Q);
    float divisor = vdot(AB, AB);
    out[0] = vdot(QB, AB);
    out[1] = -vdot(QA, AB);
    out[2] = divisor;
}

static void bary3(float out[4], v3 A, v3 B, v3 C, v3 Q)
{
    v3 AB = vsub(B, A), AC = vsub(C, A);
    v3 QA = vsub(A, Q), QB = vsub(B, Q), QC = vsub(C, Q);
    v3 QB_x_QC = vcross(QB, QC), QC_x_QA = vcross(QC, QA), QA_x_QB = vcross(QA, QB);
    v3 AB_x_AC = vcross(AB, AC);
    out[0] = vdot(QB_x_QC, AB_x_AC);
    out[1] = vdot(QC_x_QA, AB_x_AC);
    out[2] = vdot(QA_x_QB, AB_x_AC);
    out[3] = out[0] + out[1] + out[2];
}

/* b3Solve3 (cloth_particle_triangle_contact.cpp:26-122): the barycentric
 * coordinates of the point of ABC closest to Q. */
static void solve3(float out[3], v3 A, v3 B, v3 C, v3 Q)
{
    float wAB[3], wBC[3], wCA[3];
    bary2(wAB, A, B, Q);
    bary2(wBC, B, C, Q);
    bary2(wCA, C, A, Q);
    if (wAB[1] <= 0.0f && wCA[0] <= 0.0f) { out[0] = 1.0f; out[1] = 0.0f; out[2] = 0.0f; return; }
    if (wAB[0] <= 0.0f && wBC[1] <= 0.0f) { out[0] = 0.0f; out[1] = 1.0f; out[2] = 0.0f; return; }
    if (wBC[0] <= 0.0f && wCA[1] <= 0.0f) { out[0] = 0.0f; out[1] = 0.0f; out[2] = 1.0f; return; }
    float wABC[4];
    bary3(wABC, A, B, C, Q);
    if (wAB[0] > 0.0f && wAB[1] > 0.0f && wABC[3] * wABC[2] <= 0.0f) {
        float s = 1.0f / wAB[2];
        out[0] = s * wAB[0]; out[1] = s * wAB[1]; out[2] = 0.0f;
        return;
    }
    if (wBC[0] > 0.0f && wBC[1] > 0.0f && wABC[3] * wABC[0] <= 0.0f) {
        float s = 1.0f / wBC[2];
        out[0] = 0.0f; out[1] = s * wBC[0]; out[2] = s * wBC[1];
        return;
    }
    if (wCA[0] > 0.0f && wCA[1] > 0.0f && wABC[3] * wABC[1] <= 0.0f) {
        float s = 1.0f / wCA[2];
        out[0] = s * wCA[1]; out[1] = 0.0f; out[2] = s * wCA[0];
        return;
    }
    float divisor = wABC[3];
    if (divisor == 0.0f) {
        float s = 1.0f / 3.0f;
        out[0] = s; out[1] = s; out[2] = s;
        return;
    }
    float s = 1.0f / divisor;
    out[0] = s * wABC[0]; out[1] = s * wABC[1]; out[2] = s * wABC[2];
}

/* b3ParticleTriangleContact::Update (cloth_particle_triangle_contact.cpp:124-179). */
static void tcontact_update(oc_cloth* c, tcontact_t* k)
{
    v3 A = c->x[k->b], B = c->x[k->cc], C = c->x[k->d];
    v3 N = vcross(vsub(B, A), vsub(C, A));
    float len = sqrtf(N.x * N.x + N.y * N.y + N.z * N.z); /* b3Vec3::Normalize */
    if (len > kEps) {
        float s1 = 1.0f / len;
        N = V(N.x * s1, N.y * s1, N.z * s1);
    }
    if (len == 0.0f) {
        k->active = 0;
        return;
    }
    float totalRadius = c->radius[k->p] + c->def[6];
    v3 P1 = c->x[k->p];
    float distance = vdot(N, vsub(P1, A));
    if (distance < -totalRadius || distance > totalRadius) {
        k->active = 0;
        return;
    }
    float w[3];
    solve3(w, A, B, C, P1);
    v3 P2 = vadd(vadd(vscale(w[0], A), vscale(w[1], B)), vscale(w[2], C));
    v3 dd = vsub(P1, P2);
    if (vdot(dd, dd) > totalRadius * totalRadius) {
        k->active = 0;
        return;
    }
    k->active = 1;
    k->w2 = w[0];
    k->w3 = w[1];
    k->w4 = w[2];
}

static inline int tri_dynamic(const oc_cloth* c, const tcontact_t* k)
{
    return c->type[k->b] == OC_DYNAMIC || c->type[k->cc] == OC_DYNAMIC || c->type[k->d] == OC_DYNAMIC;
}

/* UpdateClothContacts (cloth_contact_manager.cpp:229-275). */
static void update_cloth_contacts(oc_cloth* c)
{
    uint32_t w = 0;
    for (uint32_t q = 0; q < c->ntc; ++q) {
        tcontact_t* k = c->tcs + q;
        if (c->type[k->p] != OC_DYNAMIC && !tri_dynamic(c, k)) continue;
        if (!aabb_overlap(c->fat_lo[k->p], c->fat_hi[k->p], c->tri_lo[k->t], c->tri_hi[k->t])) continue;
        tcontact_update(c, k);
        c->tcs[w++] = *k;
    }
    c->ntc = w;
}

/* FindNewClothContacts (cloth_contact_manager.cpp:43-48) through
 * b3BroadPhase::FindPairs (broad_phase.h:160-208) and AddPair (:125-199).
 * FindPairs reports each overlapping pair with at least one proxy in the
 * move buffer once, in ascending (proxy1, proxy2) order.  Proxy ids follow
 * creation order, particles (cloth.cpp:109-123) before triangles (:129-150),
 * so a particle-triangle pair is ordered by (particle, triangle).  AddPair
 * pushes each new contact to the list front. */
static void find_new_cloth_contacts(oc_cloth* c)
{
    const uint32_t n = c->n, t = c->t;
    uint8_t* has = (uint8_t*)calloc((size_t)n * t + 1, 1);
    for (uint32_t q = 0; q < c->ntc; ++q) has[(size_t)c->tcs[q].p * t + c->tcs[q].t] = 1;
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t k = 0; k < t; ++k) {
            if (!c->p_moved[i] && !c->t_moved[k]) continue;
            if (!aabb_overlap(c->fat_lo[i], c->fat_hi[i], c->tri_lo[k], c->tri_hi[k])) continue;
            if (has[(size_t)i * t + k]) continue;
            tcontact_t nk;
            memset(&nk, 0, sizeof(nk));
            nk.p = i;
            nk.t = k;
            nk.b = c->tris[3 * k];
            nk.cc = c->tris[3 * k + 1];
            nk.d = c->tris[3 * k + 2];
            if (c->type[i] != OC_DYNAMIC && !tri_dynamic(c, &nk)) continue;
            if (i == nk.b || i == nk.cc || i == nk.d) continue;
            if (c->ntc == c->tc_cap) {
                c->tc_cap = c->tc_cap ? 2 * c->tc_cap : 1024;
                c->tcs = (tcontact_t*)realloc(c->tcs, c->tc_cap * sizeof(tcontact_t));
            }
            c->tcs[c->ntc++] = nk;
        }
    }
    free(has);
    memset(c->p_moved, 0, n ? n : 1);
    memset(c->t_moved, 0, t ? t : 1);
}

/* The solver's view of one active particle-triangle contact
 * (b3ClothSolverTriangleContactVelocityConstraint / PositionConstraint). */
typedef struct {
    uint32_t ia, ib, ic, id; /* solver rows */
    float mA, mB, mC, mD;
    float radiusA, triangleRadius;
    float wB, wC, wD;
    v3 normal, tangent1, tangent2;
    float normalMass, tangentMass1, tangentMass2, friction;
    float normalImpulse, tangentImpulse1, tangentImpulse2;
    tcontact_t* src;
} tc_t;

static inline float tc_mass(const oc_cloth* c, uint32_t v)
{
    return c->type[v] == OC_STATIC ? 0.0f : c->inv_mass[v];
}

/* InitializeTriangleContactConstraints (cloth_contact_solver.cpp:179-262). */
static void tc_init(oc_cloth* c, tc_t* x, tcontact_t* k, const v3* pos)
{
    x->src = k;
    x->ia = c->solver_of_vertex[k->p];
    x->ib = c->solver_of_vertex[k->b];
    x->ic = c->solver_of_vertex[k->cc];
    x->id = c->solver_of_vertex[k->d];
    x->mA = tc_mass(c, k->p);
    x->mB = tc_mass(c, k->b);
    x->mC = tc_mass(c, k->cc);
    x->mD = tc_mass(c, k->d);
    x->radiusA = c->radius[k->p];
    x->triangleRadius = c->def[6];
    x->wB = k->w2;
    x->wC = k->w3;
    x->wD = k->w4;
    v3 xA = pos[x->ia], xB = pos[x->ib], xC = pos[x->ic], xD = pos[x->id];
    v3 cB = vadd(vadd(vscale(x->wB, xB), vscale(x->wC, xC)), vscale(x->wD, xD));
    v3 n = vsub(cB, xA);
    float len = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
    if (len > kEps) {
        float s1 = 1.0f / len;
        n = V(n.x * s1, n.y * s1, n.z * s1);
    }
    x->normal = n;
    float K = x->mA + x->mB * x->wB * x->wB + x->mC * x->wC * x->wC + x->mD * x->wD * x->wD;
    x->normalMass = K > 0.0f ? 1.0f / K : 0.0f;
    x->normalImpulse = k->normal_impulse;
    x->friction = sqrtf(c->friction[k->p] * c->def[7]);
    x->tangent1 = vperp(n);
    x->tangent2 = vcross(x->tangent1, n);
    x->tangentMass1 = x->normalMass;
    x->tangentMass2 = x->normalMass;
    x->tangentImpulse1 = k->tangent_impulse1;
    x->tangentImpulse2 = k->tangent_impulse2;
}

/* The impulse `lambda` along direction `u` on the four particles. */
static inline void tc_apply(const tc_t* x, float lambda, v3 u, v3* vA, v3* vB, v3* vC, v3* vD)
{
    v3 JA = vneg(u), JB = vscale(x->wB, u), JC = vscale(x->wC, u), JD = vscale(x->wD, u);
    v3 PA = vscale(lambda, JA), PB = vscale(lambda, JB), PC = vscale(lambda, JC), PD = vscale(lambda, JD);
    *vA = vadd(*vA, vscale(x->mA, PA));
    *vB = vadd(*vB, vscale(x->mB, PB));
    *vC = vadd(*vC, vscale(x->mC, PC));
    *vD = vadd(*vD, vscale(x->mD, PD));
}

/* WarmStartTriangleContactConstraints (cloth_contact_solver.cpp:309-386). */
static void tc_warm_start(const tc_t* x, v3* vel)
{
    v3 vA = vel[x->ia], vB = vel[x->ib], vC = vel[x->ic], vD = vel[x->id];
    tc_apply(x, x->normalImpulse, x->normal, &vA, &vB, &vC, &vD);
    tc_apply(x, x->tangentImpulse1, x->tangent1, &vA, &vB, &vC, &vD);
    tc_apply(x, x->tangentImpulse2, x->tangent2, &vA, &vB, &vC, &vD);
    vel[x->ia] = vA; vel[x->ib] = vB; vel[x->ic] = vC; vel[x->id] = vD;
}

/* SolveTriangleContactVelocityConstraints (cloth_contact_solver.cpp:474-596). */
static void tc_solve_velocity(tc_t* x, v3* vel)
{
    v3 vA = vel[x->ia], vB = vel[x->ib], vC = vel[x->ic], vD = vel[x->id];
    {
        v3 vCB = vadd(vadd(vscale(x->wB, vB), vscale(x->wC, vC)), vscale(x->wD, vD));
        float Cdot = vdot(vsub(vCB, vA), x->normal);
        float impulse = -x->normalMass * Cdot;
        float old = x->normalImpulse;
        float sum = x->normalImpulse + impulse;
        x->normalImpulse = sum > 0.0f ? sum : 0.0f;
        impulse = x->normalImpulse - old;
        tc_apply(x, impulse, x->normal, &vA, &vB, &vC, &vD);
    }
    for (int dir = 0; dir < 2; ++dir) {
        float hi = x->friction * x->normalImpulse;
        float lo = -hi;
        v3 u = dir == 0 ? x->tangent1 : x->tangent2;
        float* acc = dir == 0 ? &x->tangentImpulse1 : &x->tangentImpulse2;
        float tm = dir == 0 ? x->tangentMass1 : x->tangentMass2;
        v3 vCB = vadd(vadd(vscale(x->wB, vB), vscale(x->wC, vC)), vscale(x->wD, vD));
        float Cdot = vdot(vsub(vCB, vA), u);
        float impulse = -tm * Cdot;
        float old = *acc;
        float a = *acc + impulse;
        float m = a < hi ? a : hi;   /* b3Clamp = b3Max(lo, b3Min(a, hi)) */
        *acc = lo > m ? lo : m;
        impulse = *acc - old;
        tc_apply(x, impulse, u, &vA, &vB, &vC, &vD);
    }
    vel[x->ia] = vA; vel[x->ib] = vB; vel[x->ic] = vC; vel[x->id] = vD;
}

/* SolveTriangleContactPositionConstraints (cloth_contact_solver.cpp:720-794);
 * returns the contact's separation. */
static float tc_solve_position(const tc_t* x, v3* pos)
{
    v3 xA = pos[x->ia], xB = pos[x->ib], xC = pos[x->ic], xD = pos[x->id];
    v3 cB = vadd(vadd(vscale(x->wB, xB), vscale(x->wC, xC)), vscale(x->wD, xD));
    v3 n = vsub(cB, xA);
    float distance = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z); /* b3Vec3::Normalize */
    if (distance > kEps) {
        float s1 = 1.0f / distance;
        n = V(n.x * s1, n.y * s1, n.z * s1);
    }
    float separation = distance - x->radiusA - x->triangleRadius;
    float Cv = kBaumgarte * (separation + kLinearSlop);
    float m = Cv < 0.0f ? Cv : 0.0f;
    float C = -kMaxLinearCorrection > m ? -kMaxLinearCorrection : m;
    float K = x->mA + x->mB * x->wB * x->wB + x->mC * x->wC * x->wC + x->mD * x->wD * x->wD;
    float impulse = K > 0.0f ? -C / K : 0.0f;
    tc_apply(x, impulse, n, &xA, &xB, &xC, &xD);
    pos[x->ia] = xA; pos[x->ib] = xB; pos[x->ic] = xC; pos[x->id] = xD;
    return separation;
}

typedef struct {
    uint32_t index;     /* solver row */
    float inv_mass, friction, normal_mass;
    float tm_xx, tm_xy, tm_yx, tm_yy; /* tangent mass (mat22, column-major x=(xx,xy), y=(yx,yy)) */
    v3 normal, tangent1, tangent2;
    float normal_impulse;
    v2 tangent_impulse;
    /* position constraint */
    v3 normal_a, center_b;
    float radius_a, radius_b;
    contact_t* src;
} bc_t;

/* b3ClothSolver::Solve contact part (cloth_solver.cpp:103-182) with the
 * body-contact functions of cloth_contact_solver.cpp, for static bodies
 * (inverse mass and inertia 0, zero velocity). */
static void solve_contacts(oc_cloth* c, float h, uint32_t vel_iters, uint32_t pos_iters, v3* pos, v3* vel,
                           uint32_t* nactive, uint32_t* ntactive)
{
    /* active particle-triangle contacts in list order (cloth.cpp:532-538) */
    uint32_t nt = 0;
    for (uint32_t q = c->ntc; q-- > 0;) nt += c->tcs[q].active != 0;
    *ntactive = nt;
    tc_t* tc = (tc_t*)calloc(nt + 1, sizeof(tc_t));
    {
        uint32_t w = 0;
        for (uint32_t q = c->ntc; q-- > 0;)
            if (c->tcs[q].active) tc_init(c, tc + w++, c->tcs + q, pos);
    }
    uint32_t na = 0;
    for (uint32_t q = c->ncontact; q-- > 0;) na += c->contacts[q].active != 0;
    *nactive = na;
    bc_t* bc = (bc_t*)calloc(na + 1, sizeof(bc_t));
    uint32_t w = 0;
    /* contacts enter the solver in list order (cloth.cpp:539-545) */
    for (uint32_t q = c->ncontact; q-- > 0;) {
        contact_t* k = c->contacts + q;
        if (!k->active) continue;
        bc_t* x = bc + w++;
        const sphere_t* sp = c->spheres + k->shape;
        uint32_t i = k->particle;
        x->src = k;
        x->index = c->solver_of_vertex[i];
        x->inv_mass = c->type[i] == OC_STATIC ? 0.0f : c->inv_mass[i];
        x->friction = sqrtf(c->friction[i] * sp->friction); /* b3MixFriction */
        x->normal_a = k->normal1;
        x->center_b = sp->kind == SHAPE_SPHERE ? sp->center : k->local_point2;
        x->radius_a = c->radius[i];
        x->radius_b = sp->radius;
        /* InitializeBodyContactConstraints (:54-177) */
        x->normal = k->normal1;
        x->tangent1 = k->tangent1;
        x->tangent2 = k->tangent2;
        x->normal_impulse = k->normal_impulse;
        x->tangent_impulse = k->tangent_impulse;
        float mA = x->inv_mass, mB = 0.0f;
        float K = mA + mB + 0.0f + 0.0f;
        x->normal_mass = K > 0.0f ? 1.0f / K : 0.0f;
        /* b3Inverse(b3Mat22) (math.cpp:77-93) of [[k11, k12], [k12, k22]] */
        float k11 = mA + mB + 0.0f + 0.0f, k12 = 0.0f + 0.0f, k22 = mA + mB + 0.0f + 0.0f;
        float det = k11 * k22 - k12 * k12;
        if (det != 0.0f) det = 1.0f / det;
        x->tm_xx = det * k22;
        x->tm_yx = -det * k12;
        x->tm_xy = -det * k12;
        x->tm_yy = det * k11;
    }
    /* WarmStartBodyContactConstraints (:264-307) */
    for (uint32_t q = 0; q < na; ++q) {
        bc_t* x = bc + q;
        v3 vA = vel[x->index];
        float mA = x->inv_mass;
        v3 P = vscale(x->normal_impulse, x->normal);
        vA = vsub(vA, vscale(mA, P));
        v3 P1 = vscale(x->tangent_impulse.x, x->tangent1);
        v3 P2 = vscale(x->tangent_impulse.y, x->tangent2);
        vA = vsub(vA, vscale(mA, vadd(P1, P2)));
        vel[x->index] = vA;
    }
    for (uint32_t q = 0; q < nt; ++q) tc_warm_start(tc + q, vel);
    /* SolveBodyContactVelocityConstraints (:388-472), then the triangle contacts */
    for (uint32_t it = 0; it < vel_iters; ++it) {
        for (uint32_t q = 0; q < na; ++q) {
            bc_t* x = bc + q;
            v3 vA = vel[x->index];
            float mA = x->inv_mass;
            {
                /* dv = vB + wB x rB - vA - wA x rA with vB = wB = wA = 0 */
                v3 dv = vsub(vzero(), vA);
                float Cdot = vdot(x->normal, dv);
                float impulse = x->normal_mass * (-Cdot + 0.0f);
                float old = x->normal_impulse;
                float ni = old + impulse;
                x->normal_impulse = ni > 0.0f ? ni : 0.0f;
                impulse = x->normal_impulse - old;
                v3 P = vscale(impulse, x->normal);
                vA = vsub(vA, vscale(mA, P));
            }
            {
                v3 dv = vsub(vzero(), vA);
                v2 Cdot = W(vdot(dv, x->tangent1), vdot(dv, x->tangent2));
                v2 nc = W(-Cdot.x, -Cdot.y);
                /* Mat22 * Vec2 = v.x * A.x + v.y * A.y (mat22.h:56-59) */
                v2 impulse = W(nc.x * x->tm_xx + nc.y * x->tm_yx, nc.x * x->tm_xy + nc.y * x->tm_yy);
                v2 old = x->tangent_impulse;
                x->tangent_impulse.x += impulse.x;
                x->tangent_impulse.y += impulse.y;
                float maxImpulse = x->friction * x->normal_impulse;
                v2 ti = x->tangent_impulse;
                if (ti.x * ti.x + ti.y * ti.y > maxImpulse * maxImpulse) {
                    float sl = sqrtf(ti.x * ti.x + ti.y * ti.y);
                    if (sl > kEps) {
                        ti.x /= sl;
                        ti.y /= sl;
                    }
                    ti.x *= maxImpulse;
                    ti.y *= maxImpulse;
                    x->tangent_impulse = ti;
                }
                impulse = W(x->tangent_impulse.x - old.x, x->tangent_impulse.y - old.y);
                v3 P1 = vscale(impulse.x, x->tangent1);
                v3 P2 = vscale(impulse.y, x->tangent2);
                v3 P = vadd(P1, P2);
                vA = vsub(vA, vscale(mA, P));
            }
            vel[x->index] = vA;
        }
        for (uint32_t q = 0; q < nt; ++q) tc_solve_velocity(tc + q, vel);
    }
    /* StoreImpulses (:598-616) */
    for (uint32_t q = 0; q < na; ++q) {
        bc[q].src->normal_impulse = bc[q].normal_impulse;
        bc[q].src->tangent_impulse = bc[q].tangent_impulse;
    }
    for (uint32_t q = 0; q < nt; ++q) {
        tc[q].src->normal_impulse = tc[q].normalImpulse;
        tc[q].src->tangent_impulse1 = tc[q].tangentImpulse1;
        tc[q].src->tangent_impulse2 = tc[q].tangentImpulse2;
    }
    /* integrate positions (cloth_solver.cpp:143-147) */
    for (uint32_t k = 0; k < c->n; ++k) pos[k] = vadd(pos[k], vscale(h, vel[k]));
    /* SolveBodyContactPositionConstraints (:620-718), early out (cloth_solver.cpp:151-164) */
    for (uint32_t it = 0; it < pos_iters; ++it) {
        float minSeparation = 0.0f;
        for (uint32_t q = 0; q < na; ++q) {
            bc_t* x = bc + q;
            v3 cA = pos[x->index];
            v3 cB = x->center_b;
            v3 nA = x->normal_a;
            float separation = vdot(vsub(cB, cA), nA) - x->radius_a - x->radius_b;
            minSeparation = minSeparation < separation ? minSeparation : separation;
            float Cv = kBaumgarte * (separation + kLinearSlop);
            float C = Cv < 0.0f ? Cv : 0.0f;
            C = -kMaxLinearCorrection > C ? -kMaxLinearCorrection : C;
            float mA = x->inv_mass;
            float K = mA + 0.0f + 0.0f + 0.0f;
            float impulse = K > 0.0f ? -C / K : 0.0f;
            v3 P = vscale(impulse, nA);
            cA = vsub(cA, vscale(mA, P));
            pos[x->index] = cA;
        }
        float minTri = 0.0f;
        for (uint32_t q = 0; q < nt; ++q) {
            float sep = tc_solve_position(tc + q, pos);
            minTri = minTri < sep ? minTri : sep;
        }
        if (minSeparation >= -3.0f * kLinearSlop && minTri >= -3.0f * kLinearSlop) break;
    }
    free(bc);
    free(tc);
}

/* b3BroadPhase::MoveProxy (broad_phase.cpp:99-149) on a shape's proxy in the
 * world broadphase. */
static void move_shape_proxy(sphere_t* sp, v3 lo, v3 hi, v3 displacement)
{
    v3 flo = sp->fat_lo, fhi = sp->fat_hi;
    int contains = flo.x <= lo.x && lo.x <= fhi.x && flo.y <= lo.y && lo.y <= fhi.y && flo.z <= lo.z &&
                   lo.z <= fhi.z && flo.x <= hi.x && hi.x <= fhi.x && flo.y <= hi.y && hi.y <= fhi.y &&
                   flo.z <= hi.z && hi.z <= fhi.z;
    if (contains) return;
    v3 ext = V(kAabbExtension, kAabbExtension, kAabbExtension);
    lo = vsub(lo, ext);
    hi = vadd(hi, ext);
    v3 d = vscale(kAabbMultiplier, displacement);
    if (d.x < 0.0f) lo.x += d.x; else hi.x += d.x;
    if (d.y < 0.0f) lo.y += d.y; else hi.y += d.y;
    if (d.z < 0.0f) lo.z += d.z; else hi.z += d.z;
    sp->fat_lo = lo;
    sp->fat_hi = hi;
}

/* b3Sweep::GetTransform (transform.h:224-234) */
static void sweep_xf(const body_t* b, float t, m33* R, v3* p)
{
    v3 cc = vadd(vscale(1.0f - t, b->c0), vscale(t, b->c));
    quat q0 = b->q0, q1 = b->q;
    quat q = Qt((1.0f - t) * q0.x + t * q1.x, (1.0f - t) * q0.y + t * q1.y, (1.0f - t) * q0.z + t * q1.z,
                (1.0f - t) * q0.w + t * q1.w);
    qnormalize(&q);
    *R = qmat(q);
    *p = vsub(cc, qrot(q, b->lc));
}

/* After the position solve, each non-static body with an active contact
 * (cloth_solver.cpp:167-181): SynchronizeTransform (body.cpp:176-179), the
 * world inverse inertia (b3RotateToFrame, time_step.h:86-89) and
 * SynchronizeShapes (body.cpp:181-202) for its shapes. */
static void sync_body(oc_cloth* c, uint32_t body)
{
    body_t* b = c->bodies + body;
    if (b->type == 0) return;
    sweep_xf(b, 1.0f, &b->R, &b->p);
    b->wii = mmul3(mmul3(b->R, b->ii), mtrans(b->R));
    m33 R1;
    v3 p1;
    sweep_xf(b, 0.0f, &R1, &p1);
    v3 disp = vsub(b->p, p1);
    for (uint32_t s = 0; s < c->nsphere; ++s) {
        sphere_t* sp = c->spheres + s;
        if (sp->body != (int)body) continue;
        v3 lo1, hi1, lo2, hi2;
        shape_aabb(sp, R1, p1, &lo1, &hi1);
        shape_aabb(sp, b->R, b->p, &lo2, &hi2);
        move_shape_proxy(sp, vmin(lo1, lo2), vmax(hi1, hi2), disp);
    }
}

typedef struct {
    uint32_t index;
    int body;  /* -1: an implicit static body */
    float mA, mB, friction, normal_mass;
    m33 iA, iB;
    float tm_xx, tm_xy, tm_yx, tm_yy;
    v3 normal, tangent1, tangent2, point, rA, rB;
    float normal_impulse;
    v2 tangent_impulse;
    float radius_a, radius_b;
    v3 lcB, normal_a, lpA, lpB;
    body_t fixed;  /* the implicit static body */
    contact_t* src;
} gbc_t;

static inline body_t* gbody(oc_cloth* c, gbc_t* x) { return x->body >= 0 ? c->bodies + x->body : &x->fixed; }

/* b3Body::SetLinearVelocity / SetAngularVelocity (body.h) skip static bodies */
static inline void set_body_velocity(body_t* b, v3 v, v3 w)
{
    if (b->type == 0) return;
    b->v = v;
    b->w = w;
}

/* The contact part of b3ClothSolver::Solve (cloth_solver.cpp:103-182) with
 * b3ClothContactSolver's body-contact functions in full
 * (cloth_contact_solver.cpp:54-177, 264-307, 388-472, 598-718): body
 * velocities and sweeps are read and written per contact, in list order. */
static void solve_contacts_bodies(oc_cloth* c, float h, uint32_t vel_iters, uint32_t pos_iters, v3* pos,
                                  v3* vel, uint32_t* nactive, uint32_t* ntactive)
{
    uint32_t nt = 0;
    for (uint32_t q = c->ntc; q-- > 0;) nt += c->tcs[q].active != 0;
    *ntactive = nt;
    tc_t* tc = (tc_t*)calloc(nt + 1, sizeof(tc_t));
    {
        uint32_t w = 0;
        for (uint32_t q = c->ntc; q-- > 0;)
            if (c->tcs[q].active) tc_init(c, tc + w++, c->tcs + q, pos);
    }
    uint32_t na = 0;
    for (uint32_t q = c->ncontact; q-- > 0;) na += c->contacts[q].active != 0;
    *nactive = na;
    gbc_t* bc = (gbc_t*)calloc(na + 1, sizeof(gbc_t));
    uint32_t w = 0;
    for (uint32_t q = c->ncontact; q-- > 0;) {
        contact_t* k = c->contacts + q;
        if (!k->active) continue;
        gbc_t* x = bc + w++;
        const sphere_t* sp = c->spheres + k->shape;
        uint32_t i = k->particle;
        x->src = k;
        x->body = sp->body;
        x->fixed = shape_body(c, sp);
        const body_t* b = gbody(c, x);
        x->index = c->solver_of_vertex[i];
        x->mA = c->type[i] == OC_STATIC ? 0.0f : c->inv_mass[i];
        x->mB = b->im;
        x->iA = mzero();
        x->iB = b->wii;
        x->friction = sqrtf(c->friction[i] * sp->friction);
        x->radius_a = c->radius[i];
        x->radius_b = sp->radius;
        x->lcB = b->lc;
        x->normal_a = k->normal1;
        x->lpA = vzero();
        x->lpB = k->local_point2;
    }
    for (uint32_t q = 0; q < na; ++q) {
        gbc_t* x = bc + q;
        const body_t* b = gbody(c, x);
        float mA = x->mA, mB = x->mB;
        m33 iA = x->iA, iB = x->iB;
        v3 xA = pos[x->index], xB = b->c;
        m33 RA = qmat(Qt(0.0f, 0.0f, 0.0f, 1.0f));
        v3 pA = vsub(xA, mmul(RA, vzero()));
        m33 RB = qmat(b->q);
        v3 pB = vsub(xB, mmul(RB, x->lcB));
        /* b3ParticleBodyContactWorldPoint::Initialize (cloth_particle_body_contact.cpp:49-62) */
        v3 nA = x->src->normal1;
        v3 cA = xmul(RA, pA, x->lpA);
        v3 cB = xmul(RB, pB, x->lpB);
        v3 wA = vadd(cA, vscale(x->radius_a, nA));
        v3 wB = vsub(cB, vscale(x->radius_b, nA));
        x->point = vscale(0.5f, vadd(wA, wB));
        x->normal = nA;
        x->tangent1 = x->src->tangent1;
        x->tangent2 = x->src->tangent2;
        x->rA = vsub(x->point, xA);
        x->rB = vsub(x->point, xB);
        x->normal_impulse = x->src->normal_impulse;
        x->tangent_impulse = x->src->tangent_impulse;
        {
            v3 rnA = vcross(x->rA, x->normal), rnB = vcross(x->rB, x->normal);
            float K = mA + mB + vdot(mmul(iA, rnA), rnA) + vdot(mmul(iB, rnB), rnB);
            x->normal_mass = K > 0.0f ? 1.0f / K : 0.0f;
        }
        {
            v3 rn1A = vcross(x->rA, x->tangent1), rn1B = vcross(x->rB, x->tangent1);
            v3 rn2A = vcross(x->rA, x->tangent2), rn2B = vcross(x->rB, x->tangent2);
            float k11 = mA + mB + vdot(mmul(iA, rn1A), rn1A) + vdot(mmul(iB, rn1B), rn1B);
            float k12 = vdot(mmul(iA, rn1A), rn2A) + vdot(mmul(iB, rn1B), rn2B);
            float k22 = mA + mB + vdot(mmul(iA, rn2A), rn2A) + vdot(mmul(iB, rn2B), rn2B);
            float det = k11 * k22 - k12 * k12;
            if (det != 0.0f) det = 1.0f / det;
            x->tm_xx = det * k22;
            x->tm_yx = -det * k12;
            x->tm_xy = -det * k12;
            x->tm_yy = det * k11;
        }
    }
    /* WarmStartBodyContactConstraints (:264-307) */
    for (uint32_t q = 0; q < na; ++q) {
        gbc_t* x = bc + q;
        body_t* b = gbody(c, x);
        v3 vA = vel[x->index], vB = b->v, wA = vzero(), wB = b->w;
        float mA = x->mA, mB = x->mB;
        v3 P = vscale(x->normal_impulse, x->normal);
        vA = vsub(vA, vscale(mA, P));
        wA = vsub(wA, mmul(x->iA, vcross(x->rA, P)));
        vB = vadd(vB, vscale(mB, P));
        wB = vadd(wB, mmul(x->iB, vcross(x->rB, P)));
        v3 P1 = vscale(x->tangent_impulse.x, x->tangent1);
        v3 P2 = vscale(x->tangent_impulse.y, x->tangent2);
        vA = vsub(vA, vscale(mA, vadd(P1, P2)));
        wA = vsub(wA, mmul(x->iA, vcross(x->rA, vadd(P1, P2))));
        vB = vadd(vB, vscale(mB, vadd(P1, P2)));
        wB = vadd(wB, mmul(x->iB, vcross(x->rB, vadd(P1, P2))));
        vel[x->index] = vA;
        set_body_velocity(b, vB, wB);
    }
    for (uint32_t q = 0; q < nt; ++q) tc_warm_start(tc + q, vel);
    /* SolveBodyContactVelocityConstraints (:388-472), then the triangle contacts */
    for (uint32_t it = 0; it < vel_iters; ++it) {
        for (uint32_t q = 0; q < na; ++q) {
            gbc_t* x = bc + q;
            body_t* b = gbody(c, x);
            v3 vA = vel[x->index], vB = b->v, wA = vzero(), wB = b->w;
            float mA = x->mA, mB = x->mB;
            m33 iA = x->iA, iB = x->iB;
            v3 rA = x->rA, rB = x->rB;
            {
                v3 dv = vsub(vsub(vadd(vB, vcross(wB, rB)), vA), vcross(wA, rA));
                float Cdot = vdot(x->normal, dv);
                float impulse = x->normal_mass * (-Cdot + 0.0f);
                float old = x->normal_impulse;
                float ni = old + impulse;
                x->normal_impulse = ni > 0.0f ? ni : 0.0f;
                impulse = x->normal_impulse - old;
                v3 P = vscale(impulse, x->normal);
                vA = vsub(vA, vscale(mA, P));
                wA = vsub(wA, mmul(iA, vcross(rA, P)));
                vB = vadd(vB, vscale(mB, P));
                wB = vadd(wB, mmul(iB, vcross(rB, P)));
            }
            {
                v3 dv = vsub(vsub(vadd(vB, vcross(wB, rB)), vA), vcross(wA, rA));
                v2 Cdot = W(vdot(dv, x->tangent1), vdot(dv, x->tangent2));
                v2 nc = W(-Cdot.x, -Cdot.y);
                v2 impulse = W(nc.x * x->tm_xx + nc.y * x->tm_yx, nc.x * x->tm_xy + nc.y * x->tm_yy);
                v2 old = x->tangent_impulse;
                x->tangent_impulse.x += impulse.x;
                x->tangent_impulse.y += impulse.y;
                float maxImpulse = x->friction * x->normal_impulse;
                v2 ti = x->tangent_impulse;
                if (ti.x * ti.x + ti.y * ti.y > maxImpulse * maxImpulse) {
                    float sl = sqrtf(ti.x * ti.x + ti.y * ti.y);
                    if (sl > kEps) {
                        ti.x /= sl;
                        ti.y /= sl;
                    }
                    ti.x *= maxImpulse;
                    ti.y *= maxImpulse;
                    x->tangent_impulse = ti;
                }
                impulse = W(x->tangent_impulse.x - old.x, x->tangent_impulse.y - old.y);
                v3 P1 = vscale(impulse.x, x->tangent1);
                v3 P2 = vscale(impulse.y, x->tangent2);
                v3 P = vadd(P1, P2);
                vA = vsub(vA, vscale(mA, P));
                wA = vsub(wA, mmul(iA, vcross(rA, P)));
                vB = vadd(vB, vscale(mB, P));
                wB = vadd(wB, mmul(iB, vcross(rB, P)));
            }
            vel[x->index] = vA;
            set_body_velocity(b, vB, wB);
        }
        for (uint32_t q = 0; q < nt; ++q) tc_solve_velocity(tc + q, vel);
    }
    for (uint32_t q = 0; q < na; ++q) {
        bc[q].src->normal_impulse = bc[q].normal_impulse;
        bc[q].src->tangent_impulse = bc[q].tangent_impulse;
    }
    for (uint32_t q = 0; q < nt; ++q) {
        tc[q].src->normal_impulse = tc[q].normalImpulse;
        tc[q].src->tangent_impulse1 = tc[q].tangentImpulse1;
        tc[q].src->tangent_impulse2 = tc[q].tangentImpulse2;
    }
    for (uint32_t k = 0; k < c->n; ++k) pos[k] = vadd(pos[k], vscale(h, vel[k]));
    /* SolveBodyContactPositionConstraints (:620-718) */
    for (uint32_t it = 0; it < pos_iters; ++it) {
        float minSeparation = 0.0f;
        for (uint32_t q = 0; q < na; ++q) {
            gbc_t* x = bc + q;
            body_t* b = gbody(c, x);
            float mA = x->mA, mB = x->mB;
            m33 iA = x->iA, iB = x->iB;
            v3 cA = pos[x->index];
            quat qA = Qt(0.0f, 0.0f, 0.0f, 1.0f);
            v3 cB = b->c;
            quat qB = b->q;
            m33 RA = qmat(qA);
            v3 pA = vsub(cA, mmul(RA, vzero()));
            m33 RB = qmat(qB);
            v3 pB = vsub(cB, mmul(RB, x->lcB));
            v3 nA = x->normal_a;
            v3 wcA = xmul(RA, pA, x->lpA);
            v3 wcB = xmul(RB, pB, x->lpB);
            v3 point = wcB;
            float separation = vdot(vsub(wcB, wcA), nA) - x->radius_a - x->radius_b;
            minSeparation = minSeparation < separation ? minSeparation : separation;
            float Cv = kBaumgarte * (separation + kLinearSlop);
            float C = Cv < 0.0f ? Cv : 0.0f;
            C = -kMaxLinearCorrection > C ? -kMaxLinearCorrection : C;
            v3 rA = vsub(point, cA), rB = vsub(point, cB);
            v3 rnA = vcross(rA, nA), rnB = vcross(rB, nA);
            float K = mA + mB + vdot(rnA, mmul(iA, rnA)) + vdot(rnB, mmul(iB, rnB));
            float impulse = K > 0.0f ? -C / K : 0.0f;
            v3 P = vscale(impulse, nA);
            cA = vsub(cA, vscale(mA, P));
            quat dA = qderiv(qA, mmul(iA, vcross(rA, P)));
            qA = Qt(qA.x - dA.x, qA.y - dA.y, qA.z - dA.z, qA.w - dA.w);
            qnormalize(&qA);
            cB = vadd(cB, vscale(mB, P));
            quat dB = qderiv(qB, mmul(iB, vcross(rB, P)));
            qB = Qt(qB.x + dB.x, qB.y + dB.y, qB.z + dB.z, qB.w + dB.w);
            qnormalize(&qB);
            pos[x->index] = cA;
            b->c = cB;
            b->q = qB;
        }
        float minTri = 0.0f;
        for (uint32_t q = 0; q < nt; ++q) {
            float sep = tc_solve_position(tc + q, pos);
            minTri = minTri < sep ? minTri : sep;
        }
        if (minSeparation >= -3.0f * kLinearSlop && minTri >= -3.0f * kLinearSlop) break;
    }
    /* synchronize the bodies of the active contacts (cloth_solver.cpp:167-181) */
    for (uint32_t q = 0; q < na; ++q)
        if (bc[q].body >= 0) sync_body(c, (uint32_t)bc[q].body);
    free(bc);
    free(tc);
}

/* ------------------------------------------------------------------------ */
/* step                                                                      */
/* ------------------------------------------------------------------------ */

/* b3Cloth::Step (cloth.cpp:551-601), its self-collision pass run only when
 * the thickness is above zero (below that no particle-triangle contact can
 * become active), with
 * b3Cloth::Solve (:507-549), b3ClothSolver::Solve (cloth_solver.cpp:78-193)
 * and b3ClothForceSolver::Solve (cloth_force_solver.cpp:138-222). */
void oc_step(oc_cloth* c, float dt, uint32_t vel_iters, uint32_t pos_iters, oc_step_info* info)
{
    uint32_t n = c->n;
    oc_step_info local;
    memset(&local, 0, sizeof(local));

    if (self_collision(c)) update_cloth_contacts(c);
    update_body_contacts(c);

    if (dt > 0.0f) {
        float h = dt;
        form_system(c, h);
        double stats[3];
        local.iterations = mpcg(n, c->a_rowptr, c->a_cols, c->a_vals, c->b, c->Sflag, c->sx0, c->stop_rule, c->tol,
                                c->max_iter, c->dot, c->dvsol, stats);
        local.delta0 = stats[0];
        local.b_delta = stats[1];
        local.delta = stats[2];
        /* sv = sv + x; sx = sx + sy; copy back (:211-222) */
        v3* pos = (v3*)malloc(n * sizeof(v3));
        v3* vel = (v3*)malloc(n * sizeof(v3));
        for (uint32_t k = 0; k < n; ++k) {
            uint32_t i = c->order[k];
            vel[k] = vadd(c->sv[k], c->dvsol[k]);
            pos[k] = vadd(c->sx[k], c->sy[k]);
            c->mx[i] = c->dvsol[k];
        }
        if (c->nbody) solve_contacts_bodies(c, h, vel_iters, pos_iters, pos, vel, &local.active_contacts,
                                            &local.active_tri_contacts);
        else solve_contacts(c, h, vel_iters, pos_iters, pos, vel, &local.active_contacts, &local.active_tri_contacts);
        for (uint32_t k = 0; k < n; ++k) {
            uint32_t i = c->order[k];
            c->x[i] = pos[k];
            c->v[i] = vel[k];
        }
        free(pos);
        free(vel);
    }
    for (uint32_t i = 0; i < n; ++i) {
        c->f[i] = vzero();
        c->y[i] = vzero();
    }
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t i = c->order[k];
        move_proxy(c, i, vscale(dt, c->v[i]));
    }
    if (self_collision(c)) {
        /* triangle proxies (cloth.cpp:580-597), then FindNewClothContacts */
        for (uint32_t k = 0; k < c->t; ++k) {
            v3 v1 = c->v[c->tris[3 * k]], v2 = c->v[c->tris[3 * k + 1]], v3_ = c->v[c->tris[3 * k + 2]];
            v3 velocity = vdiv(vadd(vadd(v1, v2), v3_), 3.0f);
            move_triangle_proxy(c, k, vscale(dt, velocity));
        }
        find_new_cloth_contacts(c);
    }
    find_new_body_contacts(c);
    local.contacts = c->ncontact;
    local.tri_contacts = c->ntc;
    if (info) *info = local;
}

/* ------------------------------------------------------------------------ */
/* queries                                                                   */
/* ------------------------------------------------------------------------ */

void oc_get_state(const oc_cloth* c, float* x, float* v, float* dv, float* mass, uint8_t* type)
{
    for (uint32_t i = 0; i < c->n; ++i) {
        if (x) { x[3 * i] = c->x[i].x; x[3 * i + 1] = c->x[i].y; x[3 * i + 2] = c->x[i].z; }
        if (v) { v[3 * i] = c->v[i].x; v[3 * i + 1] = c->v[i].y; v[3 * i + 2] = c->v[i].z; }
        if (dv) { dv[3 * i] = c->mx[i].x; dv[3 * i + 1] = c->mx[i].y; dv[3 * i + 2] = c->mx[i].z; }
        if (mass) mass[i] = c->mass[i];
        if (type) type[i] = c->type[i];
    }
}

/* b3Cloth::GetEnergy (cloth.cpp:366-374), summed in particle-list order */
float oc_energy(const oc_cloth* c)
{
    float E = 0.0f;
    for (uint32_t k = 0; k < c->n; ++k) {
        uint32_t i = c->order[k];
        E += c->mass[i] * vdot(c->v[i], c->v[i]);
    }
    return 0.5f * E;
}

uint32_t oc_describe(const oc_cloth* c, float* tri_rest, float* fat_aabb, float* force_desc)
{
    if (tri_rest)
        for (uint32_t k = 0; k < c->t; ++k) {
            float* o = tri_rest + 6 * k;
            o[0] = c->du1[k]; o[1] = c->dv1[k]; o[2] = c->du2[k]; o[3] = c->dv2[k];
            o[4] = c->inv_det[k]; o[5] = c->alpha[k];
        }
    if (fat_aabb)
        for (uint32_t i = 0; i < c->n; ++i) {
            float* o = fat_aabb + 6 * i;
            o[0] = c->fat_lo[i].x; o[1] = c->fat_lo[i].y; o[2] = c->fat_lo[i].z;
            o[3] = c->fat_hi[i].x; o[4] = c->fat_hi[i].y; o[5] = c->fat_hi[i].z;
        }
    if (force_desc)
        for (uint32_t q = 0; q < c->nforce; ++q) {
            const force_t* f = c->forces + q;
            float* o = force_desc + 8 * q;
            memset(o, 0, 8 * sizeof(float));
            o[0] = (float)f->type;
            if (f->type == F_SPRING) {
                o[1] = (float)f->a; o[2] = (float)f->b; o[3] = -1.0f;
                o[4] = f->ks; o[5] = f->kd; o[6] = f->p0;
            } else if (f->type == F_MOUSE) {
                o[1] = (float)f->a; o[2] = (float)f->b; o[3] = -1.0f;
                o[4] = f->ks; o[5] = f->kd; o[6] = f->p0; o[7] = f->p1;
            } else {
                o[1] = (float)c->tris[3 * f->a]; o[2] = (float)c->tris[3 * f->a + 1];
                o[3] = (float)c->tris[3 * f->a + 2];
                o[4] = f->ks; o[5] = f->kd;
                if (f->type == F_STRETCH) { o[6] = f->p0; o[7] = f->p1; }
            }
        }
    return c->nforce;
}

uint32_t oc_force_count(const oc_cloth* c) { return c->nforce; }
uint32_t oc_spring_count(const oc_cloth* c) { return c->nspring; }

void oc_get_springs(const oc_cloth* c, uint32_t* pairs, float* rest_length, float* stiffness)
{
    /* the force list holds springs newest first; report creation order */
    uint32_t w = 0;
    for (uint32_t q = c->nforce; q-- > 0;) {
        const force_t* f = c->forces + q;
        if (f->type != F_SPRING) continue;
        if (pairs) { pairs[2 * w] = f->a; pairs[2 * w + 1] = f->b; }
        if (rest_length) rest_length[w] = f->p0;
        if (stiffness) stiffness[w] = f->ks;
        ++w;
    }
}

uint32_t oc_get_contacts(const oc_cloth* c, uint8_t* exists, uint8_t* active, float* impulses)
{
    if (exists) memset(exists, 0, c->n);
    if (active) memset(active, 0, c->n);
    if (impulses) memset(impulses, 0, 3 * (size_t)c->n * sizeof(float));
    for (uint32_t q = 0; q < c->ncontact; ++q) {
        const contact_t* k = c->contacts + q;
        uint32_t i = k->particle;
        if (exists) exists[i] = 1;
        if (active) active[i] = (uint8_t)(k->active != 0);
        if (impulses) {
            impulses[3 * i] = k->normal_impulse;
            impulses[3 * i + 1] = k->tangent_impulse.x;
            impulses[3 * i + 2] = k->tangent_impulse.y;
        }
    }
    return c->ncontact;
}

/* The body-contact list from its head: particle, shape, active flag and
 * impulses; at most `cap` written, the count returned. */
uint32_t oc_get_contact_list(const oc_cloth* c, uint32_t cap, uint32_t* particle, uint32_t* shape, uint8_t* active,
                             float* impulses)
{
    uint32_t k = 0;
    for (uint32_t q = c->ncontact; q-- > 0 && k < cap; ++k) {
        const contact_t* ct = c->contacts + q;
        particle[k] = ct->particle;
        shape[k] = ct->shape;
        active[k] = (uint8_t)(ct->active != 0);
        impulses[3 * k] = ct->normal_impulse;
        impulses[3 * k + 1] = ct->tangent_impulse.x;
        impulses[3 * k + 2] = ct->tangent_impulse.y;
    }
    return c->ncontact;
}

/* b3RayCast against one triangle (collision.cpp:31-118): the hit fraction
 * along p1 -> p2 and the normal facing the ray's start. */
static int ray_triangle(v3 p1, v3 p2, float maxFraction, v3 v1, v3 v2, v3 v3_, float* fraction_out, v3* normal)
{
    v3 d = vsub(p2, p1);
    if (d.x * d.x + d.y * d.y + d.z * d.z < kEps * kEps) return 0;
    v3 n = vcross(vsub(v2, v1), vsub(v3_, v1));
    float len = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
    if (len == 0.0f) return 0;
    float s1 = 1.0f / len; /* b3Vec3::operator/= */
    n = V(n.x * s1, n.y * s1, n.z * s1);
    float num = vdot(n, vsub(v1, p1));
    float den = vdot(n, d);
    if (den == 0.0f) return 0;
    float fraction = num / den;
    if (fraction < 0.0f || maxFraction < fraction) return 0;
    v3 Q = vadd(p1, vscale(fraction, d));
    v3 AB = vsub(v2, v1), AC = vsub(v3_, v1);
    v3 QA = vsub(v1, Q), QB = vsub(v2, Q), QC = vsub(v3_, Q);
    v3 AB_x_AC = vcross(AB, AC);
    float u = vdot(vcross(QB, QC), AB_x_AC);
    float v = vdot(vcross(QC, QA), AB_x_AC);
    float w = vdot(vcross(QA, QB), AB_x_AC);
    if (!(u >= 0.0f && v >= 0.0f && w >= 0.0f)) return 0;
    *fraction_out = fraction;
    *normal = num > 0.0f ? vneg(n) : n;
    return 1;
}

/* b3Cloth::RayCastSingle (cloth.cpp:466-491): the triangle hit first along
 * p1 -> p2.  Candidates are visited in triangle order (the reference visits
 * them in its tree's order; only exact ties of the fraction can tell the
 * two apart).  Returns 1 on a hit. */
int oc_ray_cast_single(const oc_cloth* c, const float* p1, const float* p2, uint32_t* triangle, float* fraction,
                       float* normal)
{
    v3 a = V(p1[0], p1[1], p1[2]), b = V(p2[0], p2[1], p2[2]);
    uint32_t best = ~0u;
    float best_f = FLT_MAX;
    v3 best_n = vzero();
    for (uint32_t k = 0; k < c->t; ++k) {
        float f;
        v3 n;
        if (ray_triangle(a, b, 1.0f, c->x[c->tris[3 * k]], c->x[c->tris[3 * k + 1]], c->x[c->tris[3 * k + 2]], &f,
                         &n) &&
            f < best_f) {
            best = k;
            best_f = f;
            best_n = n;
        }
    }
    if (best == ~0u) return 0;
    *triangle = best;
    *fraction = best_f;
    normal[0] = best_n.x; normal[1] = best_n.y; normal[2] = best_n.z;
    return 1;
}

/* Particle-triangle contacts in list order (head first): particle and
 * triangle (2 per contact), active flag, barycentric weights w2, w3, w4 and
 * the normal and two tangent impulses (3 each).  Any pointer may be null. */
uint32_t oc_get_tri_contacts(const oc_cloth* c, uint32_t* pt, uint8_t* active, float* w, float* impulses)
{
    uint32_t k = 0;
    for (uint32_t q = c->ntc; q-- > 0; ++k) {
        const tcontact_t* x = c->tcs + q;
        if (pt) { pt[2 * k] = x->p; pt[2 * k + 1] = x->t; }
        if (active) active[k] = (uint8_t)(x->active != 0);
        if (w) { w[3 * k] = x->w2; w[3 * k + 1] = x->w3; w[3 * k + 2] = x->w4; }
        if (impulses) {
            impulses[3 * k] = x->normal_impulse;
            impulses[3 * k + 1] = x->tangent_impulse1;
            impulses[3 * k + 2] = x->tangent_impulse2;
        }
    }
    return k;
}

uint32_t oc_build_system(oc_cloth* c, float dt)
{
    form_system(c, dt);
    return c->sys_nnz;
}

void oc_get_system(const oc_cloth* c, uint32_t* rowptr, uint32_t* cols, float* vals, float* b, float* S,
                   float* x0, uint32_t* vertex_of_row)
{
    uint32_t n = c->n;
    memcpy(rowptr, c->a_rowptr, (n + 1) * sizeof(uint32_t));
    memcpy(cols, c->a_cols, c->sys_nnz * sizeof(uint32_t));
    memcpy(vals, c->a_vals, (size_t)c->sys_nnz * sizeof(m33));
    memcpy(b, c->b, n * sizeof(v3));
    memcpy(S, c->Sflag, n * sizeof(float));
    memcpy(x0, c->sx0, n * sizeof(v3));
    memcpy(vertex_of_row, c->order, n * sizeof(uint32_t));
}
