/* CPU restatement of Bounce's soft body step.  Test infrastructure: the
 * parity tests and the CPU baseline call it; the product never does.
 *
 * Every function cites the reference code it restates and keeps its
 * floating-point operation order (compiled with -ffp-contract=off, no FMA):
 *   constructor, ComputeMass      src/bounce/softbody/softbody.cpp:436-553, :640-680
 *   b3ComputeD / b3ComputeB / b3SetK / b3Mul   softbody.cpp:26-155, :157-435
 *   force solve                   src/bounce/softbody/softbody_force_solver.cpp:189-388
 *   b3ExtractRotation             softbody_force_solver.cpp:53-91
 *   b3SolveMPCG                   softbody_force_solver.cpp:93-164
 *   integration                   src/bounce/softbody/softbody_solver.cpp:49-152
 *   Step                          softbody.cpp:700-735
 * Sparse rows follow b3SparseMat33 (include/bounce/sparse/sparse_mat33.h):
 * a new block goes to the front of its row list, a copy reverses a row,
 * products and sums walk the list from its head. */
#include "world_order.h"
#include "softbody_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float x, y, z; } v3;
typedef struct { v3 x, y, z; } m33; /* columns, like b3Mat33 */
typedef struct { float x, y, z, w; } quat;

static const float kEps = FLT_EPSILON; /* B3_EPSILON */

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vscale(float s, v3 v) { return V(s * v.x, s * v.y, s * v.z); }
static inline v3 vdiv(v3 v, float s) { return V(v.x / s, v.y / s, v.z / s); }
static inline v3 vneg(v3 v) { return V(-v.x, -v.y, -v.z); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float vlength(v3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
static inline v3 vzero(void) { return V(0.0f, 0.0f, 0.0f); }
static inline m33 M3(v3 x, v3 y, v3 z) { m33 m = {x, y, z}; return m; }
static inline m33 mzero(void) { return M3(vzero(), vzero(), vzero()); }
static inline m33 mdiag(float x, float y, float z) { return M3(V(x, 0.0f, 0.0f), V(0.0f, y, 0.0f), V(0.0f, 0.0f, z)); }
/* b3Mat33 * b3Vec3 (mat33.h:129-132) */
static inline v3 mmul(m33 a, v3 v) { return vadd(vadd(vscale(v.x, a.x), vscale(v.y, a.y)), vscale(v.z, a.z)); }
/* b3Mat33 * b3Mat33 (mat33.h:135-138) */
static inline m33 mmulm(m33 a, m33 b) { return M3(mmul(a, b.x), mmul(a, b.y), mmul(a, b.z)); }
static inline m33 mscale(float s, m33 a) { return M3(vscale(s, a.x), vscale(s, a.y), vscale(s, a.z)); }
static inline void madd_to(m33* a, m33 b)
{
    a->x = vadd(a->x, b.x);
    a->y = vadd(a->y, b.y);
    a->z = vadd(a->z, b.z);
}
static inline m33 mtranspose(m33 a) { return M3(V(a.x.x, a.y.x, a.z.x), V(a.x.y, a.y.y, a.z.y), V(a.x.z, a.y.z, a.z.z)); }

/* b3Det (vec3.h:171-174), b3Volume (vec3.h:226-233) with b3Sign (math.h:80-83) */
static inline float det3(v3 a, v3 b, v3 c) { return vdot(a, vcross(b, c)); }
static inline float volume(v3 a, v3 b, v3 c, v3 d)
{
    const float vol = det3(vsub(b, a), vsub(c, a), vsub(d, a));
    const float sign = (float)(0.0f < vol) - (float)(vol < 0.0f);
    const float inv6 = 1.0f / 6.0f;
    return sign * inv6 * vol;
}
/* b3Inverse: det^-1 * adjugate (src/bounce/common/math/math.cpp:111-133) */
static m33 minverse(m33 A)
{
    float det = det3(A.x, A.y, A.z);
    if (det != 0.0f) det = 1.0f / det;
    const v3 c1 = vcross(A.y, A.z), c2 = vcross(A.z, A.x), c3 = vcross(A.x, A.y);
    const m33 B = M3(V(c1.x, c2.x, c3.x), V(c1.y, c2.y, c3.y), V(c1.z, c2.z, c3.z));
    return mscale(det, B);
}

/* quaternion helpers (include/bounce/common/math/quat.h) */
static inline quat Q(float x, float y, float z, float w) { quat q = {x, y, z, w}; return q; }
static inline quat qmul(quat a, quat b) /* b3Mul, quat.h:170-178 */
{
    return Q(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
             a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
static inline void qnormalize(quat* q) /* quat.h:83-97 */
{
    const float length = sqrtf(q->x * q->x + q->y * q->y + q->z * q->z + q->w * q->w);
    if (length > kEps) {
        const float s = 1.0f / length;
        q->x *= s;
        q->y *= s;
        q->z *= s;
        q->w *= s;
    }
}
/* b3Quat::Set(axis, angle), quat.h:99-107.  Its sin and cos are the C
 * library's double functions of the float half angle, rounded to float. */
static inline quat qaxis_angle(v3 axis, float angle)
{
    const float theta = 0.5f * angle;
    const float sine = (float)sin((double)theta);
    return Q(sine * axis.x, sine * axis.y, sine * axis.z, (float)cos((double)theta));
}
static inline m33 qmat(quat q) /* b3QuatMat33, quat.h:306-318 */
{
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    const float x2 = x + x, y2 = y + y, z2 = z + z;
    const float xx = x * x2, xy = x * y2, xz = x * z2;
    const float yy = y * y2, yz = y * z2, zz = z * z2;
    const float wx = w * x2, wy = w * y2, wz = w * z2;
    return M3(V(1.0f - (yy + zz), xy + wz, xz - wy), V(xy - wz, 1.0f - (xx + zz), yz + wx),
              V(xz + wy, yz - wx, 1.0f - (xx + yy)));
}

/* b3ExtractRotation (softbody_force_solver.cpp:53-91) */
static m33 extract_rotation(quat* q, m33 A)
{
    for (uint32_t iteration = 0; iteration < 20; ++iteration) {
        const m33 R = qmat(*q);
        const float s = fabsf(vdot(R.x, A.x) + vdot(R.y, A.y) + vdot(R.z, A.z));
        if (s == 0.0f) break;
        const float inv_s = 1.0f / s + 1.0e-9f;
        const v3 v = vadd(vadd(vcross(R.x, A.x), vcross(R.y, A.y)), vcross(R.z, A.z));
        const v3 omega = vscale(inv_s, v);
        const float w = vlength(omega);
        if (w < 1.0e-9f) break;
        const quat omega_q = qaxis_angle(vdiv(omega, w), w);
        *q = qmul(omega_q, *q);
        qnormalize(q);
    }
    return qmat(*q);
}

/* b3Mul on column-major float arrays (softbody.cpp:26-42) */
static void fmul(float* C, const float* A, uint32_t AM, uint32_t AN, const float* B, uint32_t BM, uint32_t BN)
{
    for (uint32_t i = 0; i < AM; ++i)
        for (uint32_t j = 0; j < BN; ++j) {
            C[i + AM * j] = 0.0f;
            for (uint32_t k = 0; k < AN; ++k) C[i + AM * j] += A[i + AM * k] * B[k + BM * j];
        }
}
/* b3Length on a float array (softbody_force_solver.cpp:184-192) */
static float flength(const float* v, uint32_t n)
{
    float r = 0.0f;
    for (uint32_t i = 0; i < n; ++i) r += v[i] * v[i];
    return sqrtf(r);
}

typedef struct {
    m33 K[16]; /* block i + 4 j */
    m33 invE;
    quat q;
    float B[72]; /* 6 x 12 */
    float P[72]; /* 12 x 6 */
    float eps[6];
    float c_yield, c_creep, c_max;
} element;

/* A sparse row: blocks in append order; the reference's list order is the
 * reverse (PushFront). */
typedef struct {
    uint32_t n, cap;
    uint32_t* col;
    m33* val;
} lrow;

static m33* lrow_at(lrow* r, uint32_t col) /* b3SparseMat33::operator(), sparse_mat33.h:212-234 */
{
    for (uint32_t k = 0; k < r->n; ++k)
        if (r->col[k] == col) return &r->val[k];
    if (r->n == r->cap) {
        r->cap = r->cap ? 2 * r->cap : 16;
        r->col = (uint32_t*)realloc(r->col, r->cap * sizeof(uint32_t));
        r->val = (m33*)realloc(r->val, r->cap * sizeof(m33));
    }
    r->col[r->n] = col;
    r->val[r->n] = mzero();
    return &r->val[r->n++];
}

/* A static hull on a body at the origin (world frame), with its fattened
 * proxy in the world broadphase. */
typedef struct {
    float* verts;
    float* planes;
    uint32_t nv, nf;
    float friction;
    v3 lo, hi;
} os_hull;

/* b3NodeBodyContact (softbody_node_body_contact.h) */
typedef struct {
    uint32_t node, shape;
    int active;
    v3 normal1, local_point2, tangent1, tangent2;
    float normal_impulse, ti_x, ti_y;
} os_contact;

int oc_hull_test_sphere(const float* vertices, uint32_t nv, const float* planes, uint32_t nf, float radius,
                        const float* q, float* normal_out, float* point_out);

static const float kAabbExt = 0.2f;      /* B3_AABB_EXTENSION */
static const float kLinSlop = 0.005f;    /* B3_LINEAR_SLOP */
static const float kMaxCorr = 0.2f;      /* B3_MAX_LINEAR_CORRECTION */
static const float kBaum = 0.1f;         /* B3_BAUMGARTE */

struct os_body {
    uint32_t n, t;
    v3* rest; /* mesh vertices */
    uint32_t* tets;
    v3 *x, *v, *f;
    float *mass, *damping;
    int* type;
    element* el;
    v3 gravity;
    int stop_rule, dot;
    float tol;
    uint32_t max_iter;
    lrow* K; /* scratch rows */
    /* contacts with a world of static hulls (softbody_contact_manager.cpp) */
    float *radius, *friction;
    v3 *fat_lo, *fat_hi;
    os_hull hulls[4];
    uint32_t nhull;
    os_contact* contacts; /* tail first: element [ncontact - 1] is the list head */
    uint32_t ncontact, contact_cap;
    uint32_t active_contacts;
};

/* softbody.cpp:43-74 */
static void compute_D(float out[36], float E, float nu)
{
    const float lambda = (nu * E) / ((1 + nu) * (1 - 2 * nu));
    const float mu = E / (2 * (1 + nu));
    const float D[36] = {lambda + 2 * mu, lambda, lambda, 0, 0, 0, lambda, lambda + 2 * mu, lambda, 0, 0, 0,
                         lambda, lambda, lambda + 2 * mu, 0, 0, 0, 0, 0, 0, mu, 0, 0,
                         0, 0, 0, 0, mu, 0, 0, 0, 0, 0, 0, mu};
    memcpy(out, D, sizeof(D));
}

/* softbody.cpp:76-155 */
static void compute_B(float out[72], m33 invE)
{
    const m33 cof = mtranspose(invE);
    m33 mi;
    mi.x.x = cof.x.x; mi.x.y = -cof.x.y; mi.x.z = cof.x.z;
    mi.y.x = -cof.y.x; mi.y.y = cof.y.y; mi.y.z = -cof.y.z;
    mi.z.x = cof.z.x; mi.z.y = -cof.z.y; mi.z.z = cof.z.z;
    const float e11 = -mi.x.x, e12 = mi.y.x, e13 = -mi.z.x;
    const float e21 = mi.x.y, e22 = -mi.y.y, e23 = mi.z.y;
    const float e31 = -mi.x.z, e32 = mi.y.z, e33 = -mi.z.z;
    const float b1 = -e11 - e12 - e13, c1 = -e21 - e22 - e23, d1 = -e31 - e32 - e33;
    const float b2 = e11, c2 = e21, d2 = e31;
    const float b3 = e12, c3 = e22, d3 = e32;
    const float b4 = e13, c4 = e23, d4 = e33;
    const float B[72] = {b1, 0, 0, c1, d1, 0, 0, c1, 0, b1, 0, d1, 0, 0, d1, 0, b1, c1,
                         b2, 0, 0, c2, d2, 0, 0, c2, 0, b2, 0, d2, 0, 0, d2, 0, b2, c2,
                         b3, 0, 0, c3, d3, 0, 0, c3, 0, b3, 0, d3, 0, 0, d3, 0, b3, c3,
                         b4, 0, 0, c4, d4, 0, 0, c4, 0, b4, 0, d4, 0, 0, d4, 0, b4, c4};
    memcpy(out, B, sizeof(B));
}

/* b3SetK (softbody.cpp:157-435): upper and diagonal blocks read from the
 * 12 x 12 matrix, lower blocks the transposes of the upper ones. */
static void set_K(m33 K[16], const float* Ke)
{
    for (uint32_t bi = 0; bi < 4; ++bi)
        for (uint32_t bj = bi; bj < 4; ++bj) {
            m33* k = &K[bi + 4 * bj];
            float* cols[3] = {&k->x.x, &k->y.x, &k->z.x};
            for (uint32_t c = 0; c < 3; ++c)
                for (uint32_t r = 0; r < 3; ++r) cols[c][r] = Ke[3 * bi + r + 12 * (3 * bj + c)];
        }
    for (uint32_t bi = 1; bi < 4; ++bi)
        for (uint32_t bj = 0; bj < bi; ++bj) K[bi + 4 * bj] = mtranspose(K[bj + 4 * bi]);
}

os_body* os_create(uint32_t nv, const float* vertices, uint32_t nt, const uint32_t* tets, float density, float E,
                   float nu, float c_yield, float c_creep, float c_max)
{
    os_body* b = (os_body*)calloc(1, sizeof(os_body));
    b->n = nv;
    b->t = nt;
    b->rest = (v3*)malloc(nv * sizeof(v3));
    b->x = (v3*)malloc(nv * sizeof(v3));
    b->v = (v3*)calloc(nv, sizeof(v3));
    b->f = (v3*)calloc(nv, sizeof(v3));
    b->mass = (float*)calloc(nv, sizeof(float));
    b->damping = (float*)calloc(nv, sizeof(float));
    b->type = (int*)malloc(nv * sizeof(int));
    b->tets = (uint32_t*)malloc(4 * (size_t)nt * sizeof(uint32_t));
    b->el = (element*)calloc(nt, sizeof(element));
    b->K = (lrow*)calloc(nv, sizeof(lrow));
    memcpy(b->tets, tets, 4 * (size_t)nt * sizeof(uint32_t));
    for (uint32_t i = 0; i < nv; ++i) {
        b->rest[i] = V(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
        b->x[i] = b->rest[i];
        b->type[i] = 2;
    }
    /* node proxies (softbody.cpp:477-480): the point AABB fattened by
     * B3_AABB_EXTENSION in CreateProxy */
    b->radius = (float*)calloc(nv ? nv : 1, sizeof(float));
    b->friction = (float*)calloc(nv ? nv : 1, sizeof(float));
    b->fat_lo = (v3*)malloc((nv ? nv : 1) * sizeof(v3));
    b->fat_hi = (v3*)malloc((nv ? nv : 1) * sizeof(v3));
    for (uint32_t i = 0; i < nv; ++i) {
        v3 r = V(0.0f, 0.0f, 0.0f), e = V(kAabbExt, kAabbExt, kAabbExt);
        b->fat_lo[i] = vsub(vsub(b->x[i], r), e);
        b->fat_hi[i] = vadd(vadd(b->x[i], r), e);
    }
    b->stop_rule = 0;
    b->tol = 0.0f;
    b->max_iter = 20;
    b->dot = 0;
    /* ComputeMass (softbody.cpp:640-680) */
    const float inv4 = 1.0f / 4.0f;
    for (uint32_t e = 0; e < nt; ++e) {
        const uint32_t* tv = tets + 4 * (size_t)e;
        const float mass = density * volume(b->rest[tv[0]], b->rest[tv[1]], b->rest[tv[2]], b->rest[tv[3]]);
        for (int k = 0; k < 4; ++k) b->mass[tv[k]] += inv4 * mass;
    }
    /* elements (softbody.cpp:484-553) */
    for (uint32_t e = 0; e < nt; ++e) {
        element* el = &b->el[e];
        const uint32_t* tv = tets + 4 * (size_t)e;
        el->c_yield = c_yield;
        el->c_creep = c_creep;
        el->c_max = c_max;
        const v3 p1 = b->rest[tv[0]], p2 = b->rest[tv[1]], p3 = b->rest[tv[2]], p4 = b->rest[tv[3]];
        const float Vol = volume(p1, p2, p3, p4);
        el->invE = minverse(M3(vsub(p2, p1), vsub(p3, p1), vsub(p4, p1)));
        float D[36], BT[72], BT_D[72], BT_D_B[144];
        compute_D(D, E, nu);
        compute_B(el->B, el->invE);
        for (uint32_t i = 0; i < 6; ++i)
            for (uint32_t j = 0; j < 12; ++j) BT[j + 12 * i] = el->B[i + 6 * j];
        fmul(BT_D, BT, 12, 6, D, 6, 6);
        fmul(BT_D_B, BT_D, 12, 6, el->B, 6, 12);
        for (uint32_t i = 0; i < 144; ++i) BT_D_B[i] *= Vol;
        set_K(el->K, BT_D_B);
        fmul(el->P, BT, 12, 6, D, 6, 6);
        for (uint32_t i = 0; i < 72; ++i) el->P[i] *= Vol;
        /* the reference leaves q unset; the identity is the rotation of the
         * rest state (see the harness note on b3SoftBodyElement::q) */
        el->q = Q(0.0f, 0.0f, 0.0f, 1.0f);
    }
    return b;
}

void os_destroy(os_body* b)
{
    if (!b) return;
    for (uint32_t i = 0; i < b->n; ++i) {
        free(b->K[i].col);
        free(b->K[i].val);
    }
    free(b->K);
    free(b->rest);
    free(b->x);
    free(b->v);
    free(b->f);
    free(b->mass);
    free(b->damping);
    free(b->type);
    free(b->tets);
    free(b->el);
    free(b->radius); free(b->friction); free(b->fat_lo); free(b->fat_hi); free(b->contacts);
    for (uint32_t k = 0; k < b->nhull; ++k) {
        free(b->hulls[k].verts);
        free(b->hulls[k].planes);
    }
    free(b);
}

uint32_t os_node_count(const os_body* b) { return b->n; }

/* b3BroadPhase::MoveProxy (broad_phase.cpp:99-149) for node i's proxy
 * (b3SoftBodyNode::Synchronize, softbody_node.cpp:22-28). */
static void node_move_proxy(os_body* b, uint32_t i, v3 displacement)
{
    v3 r = V(b->radius[i], b->radius[i], b->radius[i]);
    v3 lo = vsub(b->x[i], r), hi = vadd(b->x[i], r);
    v3 flo = b->fat_lo[i], fhi = b->fat_hi[i];
    int contains = flo.x <= lo.x && lo.x <= fhi.x && flo.y <= lo.y && lo.y <= fhi.y && flo.z <= lo.z &&
                   lo.z <= fhi.z && flo.x <= hi.x && hi.x <= fhi.x && flo.y <= hi.y && hi.y <= fhi.y &&
                   flo.z <= hi.z && hi.z <= fhi.z;
    if (contains) return;
    v3 e = V(kAabbExt, kAabbExt, kAabbExt);
    lo = vsub(lo, e);
    hi = vadd(hi, e);
    v3 d = vscale(2.0f, displacement); /* B3_AABB_MULTIPLIER */
    if (d.x < 0.0f) lo.x += d.x; else hi.x += d.x;
    if (d.y < 0.0f) lo.y += d.y; else hi.y += d.y;
    if (d.z < 0.0f) lo.z += d.z; else hi.z += d.z;
    b->fat_lo[i] = lo;
    b->fat_hi[i] = hi;
}

/* b3SoftBodyNode::DestroyContacts (softbody_node.cpp:30-48) */
static void node_destroy_contacts(os_body* b, uint32_t i)
{
    uint32_t w = 0;
    for (uint32_t k = 0; k < b->ncontact; ++k)
        if (b->contacts[k].node != i) b->contacts[w++] = b->contacts[k];
    b->ncontact = w;
}

/* b3SoftBodyNode::SetType (softbody_node.h:146-163) */
void os_set_type(os_body* b, uint32_t i, int type)
{
    if (b->type[i] == type) return;
    b->type[i] = type;
    b->f[i] = vzero();
    if (type == 0) {
        b->v[i] = vzero();
        node_move_proxy(b, i, vzero());
    }
    node_destroy_contacts(b, i);
}

/* b3SoftBodyNode::SetRadius / SetFriction (softbody_node.h:218-235) */
void os_set_node_radius(os_body* b, uint32_t i, float radius)
{
    b->radius[i] = radius;
    node_move_proxy(b, i, vzero());
}
void os_set_node_friction(os_body* b, uint32_t i, float friction) { b->friction[i] = friction; }

/* A static b3HullShape on a body at the origin, in the soft body's world
 * (b3SoftBody::SetWorld): proxy as b3HullShape::ComputeAABB fattened. */
int os_add_hull(os_body* b, const float* vertices, uint32_t nv, const float* planes, uint32_t nf, float friction)
{
    if (b->nhull >= 4 || nv == 0) return -1;
    os_hull* h = b->hulls + b->nhull;
    h->verts = (float*)malloc(3 * (size_t)nv * sizeof(float));
    h->planes = (float*)malloc(4 * (size_t)(nf ? nf : 1) * sizeof(float));
    memcpy(h->verts, vertices, 3 * (size_t)nv * sizeof(float));
    memcpy(h->planes, planes, 4 * (size_t)nf * sizeof(float));
    h->nv = nv;
    h->nf = nf;
    h->friction = friction;
    /* b3Mul(xf, v) with the identity at the origin, then min / max */
    for (uint32_t k = 0; k < nv; ++k) {
        const float* v = vertices + 3 * k;
        v3 w = vadd(vadd(vadd(vscale(v[0], V(1.0f, 0.0f, 0.0f)), vscale(v[1], V(0.0f, 1.0f, 0.0f))),
                         vscale(v[2], V(0.0f, 0.0f, 1.0f))),
                    vzero());
        if (k == 0) {
            h->lo = w;
            h->hi = w;
        } else {
            h->lo = V(h->lo.x < w.x ? h->lo.x : w.x, h->lo.y < w.y ? h->lo.y : w.y, h->lo.z < w.z ? h->lo.z : w.z);
            h->hi = V(h->hi.x > w.x ? h->hi.x : w.x, h->hi.y > w.y ? h->hi.y : w.y, h->hi.z > w.z ? h->hi.z : w.z);
        }
    }
    v3 e = V(kAabbExt, kAabbExt, kAabbExt), r = vzero();
    h->lo = vsub(vsub(h->lo, r), e);
    h->hi = vadd(vadd(h->hi, r), e);
    return (int)b->nhull++;
}

static inline int sb_overlap(v3 alo, v3 ahi, v3 blo, v3 bhi)
{
    return alo.x <= bhi.x && alo.y <= bhi.y && alo.z <= bhi.z && ahi.x >= blo.x && ahi.y >= blo.y && ahi.z >= blo.z;
}

static inline v3 sb_perp(v3 v)
{
    if (fabsf(v.x) >= 0.57735027f) return V(v.y, -v.x, 0.0f);
    return V(0.0f, v.z, -v.y);
}

/* UpdateBodyContacts (softbody_contact_manager.cpp:109-150) with
 * b3NodeBodyContact::Update (softbody_node_body_contact.cpp:24-47). */
static void sb_update_contacts(os_body* b)
{
    uint32_t w = 0;
    for (uint32_t q = 0; q < b->ncontact; ++q) {
        os_contact k = b->contacts[q];
        if (b->type[k.node] != 2) continue;  /* the shape's body is static */
        const os_hull* h = b->hulls + k.shape;
        if (!sb_overlap(b->fat_lo[k.node], b->fat_hi[k.node], h->lo, h->hi)) continue;
        float q3[3] = {b->x[k.node].x, b->x[k.node].y, b->x[k.node].z}, nrm[3], pt[3];
        if (!oc_hull_test_sphere(h->verts, h->nv, h->planes, h->nf, 0.0f + b->radius[k.node], q3, nrm, pt)) {
            k.active = 0;
        } else {
            k.active = 1;
            k.normal1 = vneg(V(nrm[0], nrm[1], nrm[2]));
            k.local_point2 = V(pt[0], pt[1], pt[2]);
            k.tangent1 = sb_perp(k.normal1);
            k.tangent2 = vcross(k.tangent1, k.normal1);
        }
        b->contacts[w++] = k;
    }
    b->ncontact = w;
}

/* FindNewBodyContacts + AddNSPair (softbody_contact_manager.cpp:44-107):
 * dynamic nodes in index order, each against every overlapping shape in the
 * world query's report order. */
static void sb_find_new_contacts(os_body* b)
{
    /* the world query reports the hulls in its tree's order */
    float wlo[WO_MAX][3], whi[WO_MAX][3];
    uint32_t report[WO_MAX];
    for (uint32_t k = 0; k < b->nhull; ++k) {
        wlo[k][0] = b->hulls[k].lo.x; wlo[k][1] = b->hulls[k].lo.y; wlo[k][2] = b->hulls[k].lo.z;
        whi[k][0] = b->hulls[k].hi.x; whi[k][1] = b->hulls[k].hi.y; whi[k][2] = b->hulls[k].hi.z;
    }
    world_report_order(wlo, whi, b->nhull, report);
    for (uint32_t i = 0; i < b->n; ++i) {
        if (b->type[i] != 2) continue;
        for (uint32_t r = 0; r < b->nhull; ++r) {
            const uint32_t sh = report[r];
            if (!sb_overlap(b->fat_lo[i], b->fat_hi[i], b->hulls[sh].lo, b->hulls[sh].hi)) continue;
            int exists = 0;
            for (uint32_t q = 0; q < b->ncontact && !exists; ++q)
                exists = b->contacts[q].node == i && b->contacts[q].shape == sh;
            if (exists) continue;
            if (b->ncontact == b->contact_cap) {
                b->contact_cap = b->contact_cap ? 2 * b->contact_cap : 256;
                b->contacts = (os_contact*)realloc(b->contacts, b->contact_cap * sizeof(os_contact));
            }
            os_contact* c = b->contacts + b->ncontact++;
            memset(c, 0, sizeof(*c));
            c->node = i;
            c->shape = sh;
        }
    }
}

/* The contact part of b3SoftBodySolver::Solve (softbody_solver.cpp:62-126)
 * with b3SoftBodyContactSolver (softbody_contact_solver.cpp) for static
 * bodies (inverse mass and inertia 0, zero velocity). */
static void sb_solve_contacts(os_body* b, float h, uint32_t vel_iters, uint32_t pos_iters)
{
    uint32_t na = 0;
    for (uint32_t q = 0; q < b->ncontact; ++q) na += b->contacts[q].active != 0;
    b->active_contacts = na;
    os_contact** ac = (os_contact**)malloc((na + 1) * sizeof(os_contact*));
    float* nmass = (float*)malloc((na + 1) * sizeof(float));
    float* tm = (float*)malloc(4 * (na + 1) * sizeof(float));
    uint32_t w = 0;
    for (uint32_t q = b->ncontact; q-- > 0;) /* list order, head first */
        if (b->contacts[q].active) ac[w++] = b->contacts + q;
    for (uint32_t k = 0; k < na; ++k) {
        const uint32_t i = ac[k]->node;
        const float mA = b->type[i] == 0 ? 0.0f : 1.0f / b->mass[i];
        float K = mA + 0.0f + 0.0f + 0.0f;
        nmass[k] = K > 0.0f ? 1.0f / K : 0.0f;
        float k11 = mA + 0.0f + 0.0f + 0.0f, k12 = 0.0f + 0.0f, k22 = mA + 0.0f + 0.0f + 0.0f;
        float det = k11 * k22 - k12 * k12;
        if (det != 0.0f) det = 1.0f / det;
        tm[4 * k] = det * k22;
        tm[4 * k + 1] = -det * k12;
        tm[4 * k + 2] = -det * k12;
        tm[4 * k + 3] = det * k11;
    }
    /* WarmStart */
    for (uint32_t k = 0; k < na; ++k) {
        os_contact* c = ac[k];
        const uint32_t i = c->node;
        const float mA = b->type[i] == 0 ? 0.0f : 1.0f / b->mass[i];
        v3 vA = b->v[i];
        v3 P = vscale(c->normal_impulse, c->normal1);
        vA = vsub(vA, vscale(mA, P));
        v3 P1 = vscale(c->ti_x, c->tangent1), P2 = vscale(c->ti_y, c->tangent2);
        vA = vsub(vA, vscale(mA, vadd(P1, P2)));
        b->v[i] = vA;
    }
    for (uint32_t it = 0; it < vel_iters; ++it)
        for (uint32_t k = 0; k < na; ++k) {
            os_contact* c = ac[k];
            const uint32_t i = c->node;
            const float mA = b->type[i] == 0 ? 0.0f : 1.0f / b->mass[i];
            const float fr = sqrtf(b->friction[i] * b->hulls[c->shape].friction);
            v3 vA = b->v[i];
            {
                v3 dv = vsub(vzero(), vA);
                float Cdot = vdot(c->normal1, dv);
                float impulse = nmass[k] * (-Cdot + 0.0f);
                float old = c->normal_impulse;
                float sum = old + impulse;
                c->normal_impulse = sum > 0.0f ? sum : 0.0f;
                impulse = c->normal_impulse - old;
                vA = vsub(vA, vscale(mA, vscale(impulse, c->normal1)));
            }
            {
                v3 dv = vsub(vzero(), vA);
                float cx = vdot(dv, c->tangent1), cy = vdot(dv, c->tangent2);
                float ncx = -cx, ncy = -cy;
                float ix = ncx * tm[4 * k] + ncy * tm[4 * k + 1];
                float iy = ncx * tm[4 * k + 2] + ncy * tm[4 * k + 3];
                float ox = c->ti_x, oy = c->ti_y;
                c->ti_x += ix;
                c->ti_y += iy;
                float maxImpulse = fr * c->normal_impulse;
                if (c->ti_x * c->ti_x + c->ti_y * c->ti_y > maxImpulse * maxImpulse) {
                    float sl = sqrtf(c->ti_x * c->ti_x + c->ti_y * c->ti_y);
                    if (sl > kEps) {
                        c->ti_x /= sl;
                        c->ti_y /= sl;
                    }
                    c->ti_x *= maxImpulse;
                    c->ti_y *= maxImpulse;
                }
                float jx = c->ti_x - ox, jy = c->ti_y - oy;
                v3 P = vadd(vscale(jx, c->tangent1), vscale(jy, c->tangent2));
                vA = vsub(vA, vscale(mA, P));
            }
            b->v[i] = vA;
        }
    /* integrate positions */
    for (uint32_t i = 0; i < b->n; ++i) b->x[i] = vadd(b->x[i], vscale(h, b->v[i]));
    for (uint32_t it = 0; it < pos_iters; ++it) {
        float minSeparation = 0.0f;
        for (uint32_t k = 0; k < na; ++k) {
            os_contact* c = ac[k];
            const uint32_t i = c->node;
            const float mA = b->type[i] == 0 ? 0.0f : 1.0f / b->mass[i];
            v3 cA = b->x[i];
            float separation = vdot(vsub(c->local_point2, cA), c->normal1) - b->radius[i] - 0.0f;
            minSeparation = minSeparation < separation ? minSeparation : separation;
            float Cv = kBaum * (separation + kLinSlop);
            float C = Cv < 0.0f ? Cv : 0.0f;
            C = -kMaxCorr > C ? -kMaxCorr : C;
            float K = mA + 0.0f + 0.0f + 0.0f;
            float impulse = K > 0.0f ? -C / K : 0.0f;
            cA = vsub(cA, vscale(mA, vscale(impulse, c->normal1)));
            b->x[i] = cA;
        }
        if (minSeparation >= -3.0f * kLinSlop) break;
    }
    free(ac);
    free(nmass);
    free(tm);
}
void os_set_mass_damping(os_body* b, uint32_t i, float d) { b->damping[i] = d; }
void os_set_gravity(os_body* b, const float* g) { b->gravity = V(g[0], g[1], g[2]); }
/* b3SoftBodyNode::ApplyForce: m_force += force */
void os_apply_force(os_body* b, uint32_t i, const float* f) { b->f[i] = vadd(b->f[i], V(f[0], f[1], f[2])); }
void os_set_position(os_body* b, uint32_t i, const float* x)
{
    v3 p = V(x[0], x[1], x[2]);
    v3 d = vsub(p, b->x[i]);
    b->x[i] = p;
    node_move_proxy(b, i, d);
}
void os_set_velocity(os_body* b, uint32_t i, const float* v)
{
    if (b->type[i] == 0) return;
    b->v[i] = V(v[0], v[1], v[2]);
}
void os_set_solver(os_body* b, int stop_rule, float tol, uint32_t max_iterations, int dot)
{
    b->stop_rule = stop_rule;
    b->tol = tol;
    b->max_iter = max_iterations;
    b->dot = dot;
}

/* FP32 sequential (b3Dot of b3DenseVec3, dense_vec3.h:139-151) or FP64 */
static double dense_dot(const v3* a, const v3* c, uint32_t n, int dot)
{
    if (dot == 2) {
        double r = 0.0;
        for (uint32_t i = 0; i < n; ++i)
            r += (double)a[i].x * (double)c[i].x + (double)a[i].y * (double)c[i].y + (double)a[i].z * (double)c[i].z;
        return r;
    }
    float r = 0.0f;
    for (uint32_t i = 0; i < n; ++i) r += vdot(a[i], c[i]);
    return (double)r;
}

/* S v with S = I or 0 per row: b3DiagMat33 * b3Vec3 */
static inline v3 filt(int dyn, v3 v) { return mmul(dyn ? mdiag(1.0f, 1.0f, 1.0f) : mzero(), v); }

/* One force solve (softbody_force_solver.cpp:189-388) up to the system:
 * A in list order (arows: append order, the list is the reverse), b, S. */
static void form_system(os_body* b, float h, lrow* arows, v3* rhs)
{
    const uint32_t n = b->n;
    const float inv_h = 1.0f / h;
    v3* f0 = (v3*)calloc(n, sizeof(v3));
    v3* fpl = (v3*)calloc(n, sizeof(v3));
    v3* fe = (v3*)malloc(n * sizeof(v3));
    for (uint32_t i = 0; i < n; ++i) {
        b->K[i].n = 0;
        fe[i] = b->f[i];
        if (b->type[i] == 2) fe[i] = vadd(fe[i], vscale(b->mass[i], b->gravity));
    }
    for (uint32_t ei = 0; ei < b->t; ++ei) {
        element* e = &b->el[ei];
        const uint32_t* tv = b->tets + 4 * (size_t)ei;
        const v3 p1 = b->x[tv[0]], p2 = b->x[tv[1]], p3 = b->x[tv[2]], p4 = b->x[tv[3]];
        const m33 Em = M3(vsub(p2, p1), vsub(p3, p1), vsub(p4, p1));
        const m33 A = mmulm(Em, e->invE);
        const m33 R = extract_rotation(&e->q, A);
        const m33 RT = mtranspose(R);
        for (uint32_t i = 0; i < 4; ++i)
            for (uint32_t j = 0; j < 4; ++j) madd_to(lrow_at(&b->K[tv[i]], tv[j]), mmulm(mmulm(R, e->K[i + 4 * j]), RT));
        const v3 xs[4] = {b->rest[tv[0]], b->rest[tv[1]], b->rest[tv[2]], b->rest[tv[3]]};
        v3 f0s[4];
        for (uint32_t i = 0; i < 4; ++i) {
            f0s[i] = vzero();
            for (uint32_t j = 0; j < 4; ++j) f0s[i] = vadd(f0s[i], mmul(mmulm(R, e->K[i + 4 * j]), xs[j]));
        }
        for (uint32_t i = 0; i < 4; ++i) f0[tv[i]] = vadd(f0[tv[i]], f0s[i]);
        /* plasticity */
        const v3 ps[4] = {p1, p2, p3, p4};
        float rt_x_x0[12];
        for (uint32_t i = 0; i < 4; ++i) {
            const v3 d = vsub(mmul(RT, ps[i]), xs[i]);
            rt_x_x0[3 * i] = d.x;
            rt_x_x0[3 * i + 1] = d.y;
            rt_x_x0[3 * i + 2] = d.z;
        }
        float eps_total[6], eps_elastic[6];
        fmul(eps_total, e->B, 6, 12, rt_x_x0, 12, 1);
        for (uint32_t i = 0; i < 6; ++i) eps_elastic[i] = eps_total[i] - e->eps[i];
        if (flength(eps_elastic, 6) > e->c_yield) {
            const float amount = h * (e->c_creep < inv_h ? e->c_creep : inv_h);
            for (uint32_t i = 0; i < 6; ++i) e->eps[i] += amount * eps_elastic[i];
        }
        const float len_plastic = flength(e->eps, 6);
        if (len_plastic > e->c_max) {
            const float scale = e->c_max / len_plastic;
            for (uint32_t i = 0; i < 6; ++i) e->eps[i] *= scale;
        }
        float fs[12];
        fmul(fs, e->P, 12, 6, e->eps, 6, 1);
        for (uint32_t i = 0; i < 4; ++i) {
            const v3 fp = mmul(R, V(fs[3 * i], fs[3 * i + 1], fs[3 * i + 2]));
            fpl[tv[i]] = vadd(fpl[tv[i]], fp);
        }
    }
    for (uint32_t i = 0; i < n; ++i) f0[i] = vneg(f0[i]);
    /* A = M + h C + (h h) K (sparse_mat33.h:150-192, 236-251, 270-341) */
    const float hh = h * h;
    for (uint32_t i = 0; i < n; ++i) {
        lrow* ar = &arows[i];
        ar->n = 0;
        const m33 Mi = mdiag(b->mass[i], b->mass[i], b->mass[i]);
        const float cd = b->damping[i] * b->mass[i];
        const m33 hC = mscale(h, mdiag(cd, cd, cd));
        m33 d = Mi;
        madd_to(&d, hC);
        *lrow_at(ar, i) = d;
        /* hhK = copy of K (its list reversed: append order) scaled; added
         * head to tail, new blocks pushed to the front of A's row */
        const lrow* kr = &b->K[i];
        for (uint32_t k = 0; k < kr->n; ++k) madd_to(lrow_at(ar, kr->col[k]), mscale(hh, kr->val[k]));
        /* b = M v - h (K p + f0 - (f_plastic + fe)) */
        v3 kp = vzero();
        for (uint32_t k = kr->n; k-- > 0;) kp = vadd(kp, mmul(kr->val[k], b->x[kr->col[k]]));
        const v3 mv = vadd(vzero(), mmul(Mi, b->v[i]));
        rhs[i] = vsub(mv, vscale(h, vsub(vadd(kp, f0[i]), vadd(fpl[i], fe[i]))));
    }
    free(f0);
    free(fpl);
    free(fe);
}

/* b3SolveMPCG (softbody_force_solver.cpp:93-164) over rows in list order */
static uint32_t mpcg(os_body* b, lrow* arows, const v3* rhs, v3* x, os_stats* st)
{
    const uint32_t n = b->n;
    v3* invP = (v3*)malloc(n * sizeof(v3));
    v3* Pd = (v3*)malloc(n * sizeof(v3));
    v3* r = (v3*)malloc(n * sizeof(v3));
    v3* c = (v3*)malloc(n * sizeof(v3));
    v3* q = (v3*)malloc(n * sizeof(v3));
    v3* sb = (v3*)malloc(n * sizeof(v3));
    v3* psb = (v3*)malloc(n * sizeof(v3));
    for (uint32_t i = 0; i < n; ++i) {
        const m33 a = *lrow_at(&arows[i], i);
        Pd[i] = V(a.x.x, a.y.y, a.z.z);
        invP[i] = V(1.0f / a.x.x, 1.0f / a.y.y, 1.0f / a.z.z);
    }
#define SPMV(out, vec)                                                                              \
    for (uint32_t i = 0; i < n; ++i) {                                                             \
        v3 acc = vzero();                                                                          \
        for (uint32_t k = arows[i].n; k-- > 0;) acc = vadd(acc, mmul(arows[i].val[k], (vec)[arows[i].col[k]])); \
        (out)[i] = acc;                                                                            \
    }
    for (uint32_t i = 0; i < n; ++i) x[i] = b->v[i]; /* x = z */
    for (uint32_t i = 0; i < n; ++i) {
        sb[i] = filt(b->type[i] == 2, rhs[i]);
        psb[i] = mmul(mdiag(Pd[i].x, Pd[i].y, Pd[i].z), sb[i]);
    }
    const double delta_0 = dense_dot(sb, psb, n, b->dot);
    SPMV(q, x);
    for (uint32_t i = 0; i < n; ++i) r[i] = filt(b->type[i] == 2, vsub(rhs[i], q[i]));
    for (uint32_t i = 0; i < n; ++i) c[i] = filt(b->type[i] == 2, mmul(mdiag(invP[i].x, invP[i].y, invP[i].z), r[i]));
    double delta_new = dense_dot(r, c, n, b->dot);
    st->delta0 = delta_new;
    st->b_delta = delta_0;
    uint32_t iteration = 0;
    for (;;) {
        if (iteration == b->max_iter) break;
        if (b->stop_rule == 0) {
            if (b->dot == 2 ? delta_new <= (double)(kEps * kEps) * delta_0
                            : (float)delta_new <= kEps * kEps * (float)delta_0)
                break;
        } else if (delta_new <= (double)b->tol * (double)b->tol * delta_0) {
            break;
        }
        SPMV(q, c);
        for (uint32_t i = 0; i < n; ++i) q[i] = filt(b->type[i] == 2, q[i]);
        const double cq = dense_dot(c, q, n, b->dot);
        const float alpha = b->dot == 2 ? (float)(delta_new / cq) : (float)delta_new / (float)cq;
        for (uint32_t i = 0; i < n; ++i) {
            x[i] = vadd(x[i], vscale(alpha, c[i]));
            r[i] = vsub(r[i], vscale(alpha, q[i]));
        }
        for (uint32_t i = 0; i < n; ++i) sb[i] = mmul(mdiag(invP[i].x, invP[i].y, invP[i].z), r[i]);
        const double delta_old = delta_new;
        delta_new = dense_dot(r, sb, n, b->dot);
        const float beta = b->dot == 2 ? (float)(delta_new / delta_old) : (float)delta_new / (float)delta_old;
        for (uint32_t i = 0; i < n; ++i) c[i] = filt(b->type[i] == 2, vadd(sb[i], vscale(beta, c[i])));
        ++iteration;
    }
#undef SPMV
    st->delta = delta_new;
    st->iterations = iteration;
    free(invP);
    free(Pd);
    free(r);
    free(c);
    free(q);
    free(sb);
    free(psb);
    return iteration;
}

static void free_rows(lrow* rows, uint32_t n)
{
    for (uint32_t i = 0; i < n; ++i) {
        free(rows[i].col);
        free(rows[i].val);
    }
    free(rows);
}

/* b3SoftBody::Step without a world (softbody.cpp:700-735): force solve,
 * x += h v (softbody_solver.cpp:105-110), forces cleared. */
void os_step(os_body* b, float dt, uint32_t velocity_iterations, uint32_t position_iterations, os_stats* out)
{
    os_stats st;
    memset(&st, 0, sizeof(st));
    b->active_contacts = 0;
    if (b->nhull) sb_update_contacts(b);
    if (dt > 0.0f) {
        const uint32_t n = b->n;
        lrow* arows = (lrow*)calloc(n, sizeof(lrow));
        v3* rhs = (v3*)malloc(n * sizeof(v3));
        v3* sx = (v3*)malloc(n * sizeof(v3));
        form_system(b, dt, arows, rhs);
        mpcg(b, arows, rhs, sx, &st);
        for (uint32_t i = 0; i < n; ++i) b->v[i] = sx[i];
        if (b->nhull) sb_solve_contacts(b, dt, velocity_iterations, position_iterations);
        else
            for (uint32_t i = 0; i < n; ++i) b->x[i] = vadd(b->x[i], vscale(dt, b->v[i]));
        free_rows(arows, n);
        free(rhs);
        free(sx);
    }
    for (uint32_t i = 0; i < b->n; ++i) b->f[i] = vzero();
    if (b->nhull) {
        /* node proxies (softbody.cpp:764-775), then FindNewBodyContacts */
        for (uint32_t i = 0; i < b->n; ++i)
            if (b->type[i] != 0) node_move_proxy(b, i, vscale(dt, b->v[i]));
        sb_find_new_contacts(b);
    }
    if (out) *out = st;
}

/* Node contacts (one shape): per node exists, active, impulses (normal,
 * tangent x, tangent y); returns the contact count. */
uint32_t os_get_contacts(const os_body* b, uint8_t* exists, uint8_t* active, float* impulses)
{
    memset(exists, 0, b->n);
    memset(active, 0, b->n);
    memset(impulses, 0, 3 * (size_t)b->n * sizeof(float));
    for (uint32_t q = 0; q < b->ncontact; ++q) {
        const os_contact* c = b->contacts + q;
        exists[c->node] = 1;
        active[c->node] = (uint8_t)(c->active != 0);
        impulses[3 * c->node] = c->normal_impulse;
        impulses[3 * c->node + 1] = c->ti_x;
        impulses[3 * c->node + 2] = c->ti_y;
    }
    return b->ncontact;
}

/* The contact list from its head: per contact its node, hull, active flag
 * and impulses (normal, tangent x, tangent y); at most `cap` are written,
 * the count is returned. */
uint32_t os_get_contact_list(const os_body* b, uint32_t cap, uint32_t* node, uint32_t* shape, uint8_t* active,
                             float* impulses)
{
    uint32_t k = 0;
    for (uint32_t q = b->ncontact; q-- > 0 && k < cap; ++k) {
        const os_contact* c = b->contacts + q;
        node[k] = c->node;
        shape[k] = c->shape;
        active[k] = (uint8_t)(c->active != 0);
        impulses[3 * k] = c->normal_impulse;
        impulses[3 * k + 1] = c->ti_x;
        impulses[3 * k + 2] = c->ti_y;
    }
    return b->ncontact;
}

void os_get_state(const os_body* b, float* x, float* v)
{
    for (uint32_t i = 0; i < b->n; ++i) {
        if (x) {
            x[3 * i] = b->x[i].x;
            x[3 * i + 1] = b->x[i].y;
            x[3 * i + 2] = b->x[i].z;
        }
        if (v) {
            v[3 * i] = b->v[i].x;
            v[3 * i + 1] = b->v[i].y;
            v[3 * i + 2] = b->v[i].z;
        }
    }
}

void os_set_state(os_body* b, const float* x, const float* v)
{
    for (uint32_t i = 0; i < b->n; ++i) {
        if (x) b->x[i] = V(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
        if (v) b->v[i] = V(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    }
}

void os_get_masses(const os_body* b, float* m) { memcpy(m, b->mass, b->n * sizeof(float)); }

void os_get_elements(const os_body* b, float* q, float* eps)
{
    for (uint32_t e = 0; e < b->t; ++e) {
        if (q) {
            q[4 * e] = b->el[e].q.x;
            q[4 * e + 1] = b->el[e].q.y;
            q[4 * e + 2] = b->el[e].q.z;
            q[4 * e + 3] = b->el[e].q.w;
        }
        if (eps) memcpy(eps + 6 * (size_t)e, b->el[e].eps, 6 * sizeof(float));
    }
}

void os_set_elements(os_body* b, const float* q, const float* eps)
{
    for (uint32_t e = 0; e < b->t; ++e) {
        if (q) b->el[e].q = Q(q[4 * e], q[4 * e + 1], q[4 * e + 2], q[4 * e + 3]);
        if (eps) memcpy(b->el[e].eps, eps + 6 * (size_t)e, 6 * sizeof(float));
    }
}

void os_get_element_data(const os_body* b, uint32_t e, float* K, float* invE, float* B, float* P)
{
    const element* el = &b->el[e];
    if (K) memcpy(K, el->K, sizeof(el->K));
    if (invE) memcpy(invE, &el->invE, sizeof(m33));
    if (B) memcpy(B, el->B, sizeof(el->B));
    if (P) memcpy(P, el->P, sizeof(el->P));
}

/* b3SoftBody::GetEnergy (softbody.cpp:627-637) */
float os_energy(const os_body* b)
{
    float E = 0.0f;
    for (uint32_t i = 0; i < b->n; ++i) E += b->mass[i] * vdot(b->v[i], b->v[i]);
    return 0.5f * E;
}

uint32_t os_system(os_body* b, float dt, uint32_t cap, uint32_t* rowptr, uint32_t* cols, float* vals, float* rhs,
                   float* S)
{
    const uint32_t n = b->n;
    /* the solve updates the elements' rotation and plastic state: keep them */
    element* saved = (element*)malloc(b->t * sizeof(element));
    memcpy(saved, b->el, b->t * sizeof(element));
    lrow* arows = (lrow*)calloc(n, sizeof(lrow));
    v3* r = (v3*)malloc(n * sizeof(v3));
    form_system(b, dt, arows, r);
    memcpy(b->el, saved, b->t * sizeof(element));
    free(saved);
    uint32_t total = 0;
    for (uint32_t i = 0; i < n; ++i) total += arows[i].n;
    if (total <= cap) {
        uint32_t k = 0;
        for (uint32_t i = 0; i < n; ++i) {
            rowptr[i] = k;
            for (uint32_t q = arows[i].n; q-- > 0; ++k) {
                cols[k] = arows[i].col[q];
                memcpy(vals + 9 * (size_t)k, &arows[i].val[q], 9 * sizeof(float));
            }
            rhs[3 * i] = r[i].x;
            rhs[3 * i + 1] = r[i].y;
            rhs[3 * i + 2] = r[i].z;
            S[i] = b->type[i] == 2 ? 1.0f : 0.0f;
        }
        rowptr[n] = k;
    }
    free_rows(arows, n);
    free(r);
    return total;
}
