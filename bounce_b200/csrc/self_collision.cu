// Cloth self-collision on the GPU (see self_collision.cuh): the
// particle-triangle contact list of one cloth, kept in the reference's list
// order, and its contact solve interleaved with the body contacts.
//
//   k_sc_update   UpdateClothContacts (cloth_contact_manager.cpp:229-275) with
//                 b3ParticleTriangleContact::Update
//                 (contacts/cloth_particle_triangle_contact.cpp:124-179); one
//                 block compacts the list in order and lists the active
//                 contacts
//   k_sc_solve    b3ClothSolver::Solve's contact part (cloth_solver.cpp:95-164)
//                 with both contact kinds: one block; body contacts one
//                 thread per particle, triangle contacts by dependency level
//   k_sc_tri_sync triangle proxies (cloth.cpp:580-597)
//   k_sc_hash, k_sc_pairs, k_sc_scan, k_sc_prepend
//                 FindNewClothContacts: b3BroadPhase::FindPairs
//                 (broad_phase.h:160-208) and AddPair
//                 (cloth_contact_manager.cpp:125-199).  FindPairs reports each
//                 overlapping pair with a proxy in the move buffer once, in
//                 ascending (proxy1, proxy2) order; proxy ids follow creation
//                 order, particles before triangles, so the new contacts come
//                 in ascending (particle, triangle) order and each is pushed
//                 to the list front.
//
// Everything follows the reference's float order (-fmad=false), so the
// trajectory, the list and its impulses are the reference's bit for bit.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/b3g.h"
#include "cloth_internal.h"
#include "self_collision.cuh"

namespace b3g {

namespace {

constexpr float kSlop = 0.005f;           // B3_LINEAR_SLOP
constexpr float kMaxCorrection = 0.2f;    // B3_MAX_LINEAR_CORRECTION
constexpr float kBaum = 0.1f;             // B3_BAUMGARTE
constexpr float kEpsilon = 1.1920929e-7f; // B3_EPSILON (FLT_EPSILON)
constexpr int kSolveThreads = 1024;
constexpr uint32_t kMaxBodyContacts = kMaxSpheres;

__device__ __forceinline__ f3 neg(f3 v) { return mk(-v.x, -v.y, -v.z); }

// b3Vec3::Normalize (vec3.h:93-104): returns the length, scales when it is
// above B3_EPSILON
__device__ __forceinline__ float normalize(f3& v)
{
    const float len = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    if (len > kEpsilon) {
        const float s = 1.0f / len;
        v = mk(v.x * s, v.y * s, v.z * s);
    }
    return len;
}

__device__ __forceinline__ bool overlap_pt(const ClothDev& c, uint32_t p, uint32_t k)
{
    // b3TestOverlap (aabb3.h:247-251) of the particle's and the triangle's fat AABBs
    const uint32_t n = c.n, t = c.t;
    return c.fat_lo[p] <= c.tri_hi[k] && c.fat_lo[n + p] <= c.tri_hi[t + k] &&
           c.fat_lo[2 * n + p] <= c.tri_hi[2 * t + k] && c.fat_hi[p] >= c.tri_lo[k] &&
           c.fat_hi[n + p] >= c.tri_lo[t + k] && c.fat_hi[2 * n + p] >= c.tri_lo[2 * t + k];
}

__device__ __forceinline__ bool dyn(const ClothDev& c, uint32_t i) { return c.type[i] == 2; }

// b3BarycentricCoordinates (geometry.h:105-145)
__device__ __forceinline__ void bary2(float out[3], f3 A, f3 B, f3 Q)
{
    const f3 AB = B - A, QA = A - Q, QB = B - Q;
    const float divisor = dot(AB, AB);
    out[0] = dot(QB, AB);
    out[1] = -dot(QA, AB);
    out[2] = divisor;
}

__device__ __forceinline__ void bary3(float out[4], f3 A, f3 B, f3 C, f3 Q)
{
    const f3 AB = B - A, AC = C - A, QA = A - Q, QB = B - Q, QC = C - Q;
    const f3 QB_x_QC = cross(QB, QC), QC_x_QA = cross(QC, QA), QA_x_QB = cross(QA, QB);
    const f3 AB_x_AC = cross(AB, AC);
    out[0] = dot(QB_x_QC, AB_x_AC);
    out[1] = dot(QC_x_QA, AB_x_AC);
    out[2] = dot(QA_x_QB, AB_x_AC);
    out[3] = out[0] + out[1] + out[2];
}

// b3Solve3 (cloth_particle_triangle_contact.cpp:26-122): barycentric
// coordinates of the point of ABC closest to Q
__device__ void solve3(float out[3], f3 A, f3 B, f3 C, f3 Q)
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
        const float s = 1.0f / wAB[2];
        out[0] = s * wAB[0]; out[1] = s * wAB[1]; out[2] = 0.0f;
        return;
    }
    if (wBC[0] > 0.0f && wBC[1] > 0.0f && wABC[3] * wABC[0] <= 0.0f) {
        const float s = 1.0f / wBC[2];
        out[0] = 0.0f; out[1] = s * wBC[0]; out[2] = s * wBC[1];
        return;
    }
    if (wCA[0] > 0.0f && wCA[1] > 0.0f && wABC[3] * wABC[1] <= 0.0f) {
        const float s = 1.0f / wCA[2];
        out[0] = s * wCA[1]; out[1] = 0.0f; out[2] = s * wCA[0];
        return;
    }
    const float divisor = wABC[3];
    if (divisor == 0.0f) {
        const float s = 1.0f / 3.0f;
        out[0] = s; out[1] = s; out[2] = s;
        return;
    }
    const float s = 1.0f / divisor;
    out[0] = s * wABC[0]; out[1] = s * wABC[1]; out[2] = s * wABC[2];
}

// b3ParticleTriangleContact::Update: the active flag and the weights
__device__ bool contact_update(const ClothDev& c, uint32_t p, uint4 tv, float4& w)
{
    const uint32_t n = c.n;
    const f3 A = ld3(c.x, n, tv.x), B = ld3(c.x, n, tv.y), C = ld3(c.x, n, tv.z);
    f3 N = cross(B - A, C - A);
    const float len = normalize(N);
    if (len == 0.0f) return false;
    const float total = c.p_radius[p] + c.thickness;  // particle radius + triangle radius
    const f3 P1 = ld3(c.x, n, p);
    const float distance = dot(N, P1 - A);
    if (distance < -total) return false;
    if (distance > total) return false;
    float wt[3];
    solve3(wt, A, B, C, P1);
    const f3 P2 = (wt[0] * A + wt[1] * B) + wt[2] * C;
    const f3 d = P1 - P2;
    if (d.x * d.x + d.y * d.y + d.z * d.z > total * total) return false;
    w = make_float4(wt[0], wt[1], wt[2], 0.0f);
    return true;
}

// Exclusive scan of one value per thread over the block; `total` gets the sum.
__device__ uint32_t block_scan(uint32_t v, uint32_t& total)
{
    __shared__ uint32_t warp_sum[32];
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = (blockDim.x + 31u) >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31u) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < nw ? warp_sum[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= (uint32_t)o) s += y;
        }
        warp_sum[lane] = s;
    }
    __syncthreads();
    const uint32_t before = (wid ? warp_sum[wid - 1] : 0u) + x - v;
    total = warp_sum[nw - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(1024) k_sc_update(ClothDev c, SelfDev s, int src, uint32_t m)
{
    const int dst = 1 - src;
    uint32_t out_base = 0, act_base = 0;
    for (uint32_t base = 0; base < m; base += blockDim.x) {
        const uint32_t k = base + threadIdx.x;
        uint32_t keep = 0, on = 0;
        uint2 key = make_uint2(0u, 0u);
        float4 w = make_float4(0.0f, 0.0f, 0.0f, 0.0f), imp = w;
        if (k < m) {
            key = s.key[src][k];
            const uint4 tv = c.tri[key.y];
            const bool alive = dyn(c, key.x) || dyn(c, tv.x) || dyn(c, tv.y) || dyn(c, tv.z);
            if (!c.p_purge[key.x] && alive && overlap_pt(c, key.x, key.y)) {
                keep = 1;
                w = s.w[src][k];
                on = contact_update(c, key.x, tv, w) ? 1u : 0u;
                imp = s.imp[src][k];
            }
        }
        uint32_t kept, acts;
        const uint32_t pos = block_scan(keep, kept);
        const uint32_t apos = block_scan(on, acts);
        if (keep) {
            const uint32_t j = out_base + pos;
            s.key[dst][j] = key;
            s.act[dst][j] = (uint8_t)on;
            s.w[dst][j] = w;
            s.imp[dst][j] = imp;
            if (on) s.active_idx[act_base + apos] = j;
        }
        out_base += kept;
        act_base += acts;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < c.n; i += blockDim.x) c.p_purge[i] = 0;
    if (threadIdx.x == 0) {
        s.counts[kCountList] = out_base;
        s.counts[kCountActive] = act_base;
    }
}

// ---- body contacts, one particle (the arithmetic of k_finalize) ----------

__device__ int body_order(const ClothDev& c, uint32_t i, int* order)
{
    int k = 0;
    const uint32_t n = c.n;
    for (uint32_t s = 0; s < c.nsph; ++s) {
        const uint32_t q = s * n + i;
        if (c.c_exists[q] && c.c_active[q]) order[k++] = (int)s;
    }
    for (int a = 1; a < k; ++a) {  // newest first
        const int v = order[a];
        int b = a - 1;
        while (b >= 0 && c.c_key[order[b] * n + i] < c.c_key[v * n + i]) {
            order[b + 1] = order[b];
            --b;
        }
        order[b + 1] = v;
    }
    return k;
}

// WarmStartBodyContactConstraints (cloth_contact_solver.cpp:264-307)
__device__ void body_warm_start(const ClothDev& c, uint32_t i, const int* order, int k)
{
    const uint32_t n = c.n, nn = c.nsph * n;
    const float mA = 1.0f / c.mass[i];
    f3 vel = ld3(c.v, n, i);
    for (int a = 0; a < k; ++a) {
        const uint32_t q = order[a] * n + i;
        const f3 nrm = ld3(c.c_normal, nn, q), t1 = ld3(c.c_t1, nn, q), t2 = ld3(c.c_t2, nn, q);
        const f3 P = c.c_imp[q] * nrm;
        vel = vel - mA * P;
        const f3 P1 = c.c_imp[nn + q] * t1, P2 = c.c_imp[2 * nn + q] * t2;
        vel = vel - mA * (P1 + P2);
    }
    st3(c.v, n, i, vel);
}

// SolveBodyContactVelocityConstraints (cloth_contact_solver.cpp:388-472)
__device__ void body_velocity(const ClothDev& c, uint32_t i, const int* order, int k)
{
    const uint32_t n = c.n, nn = c.nsph * n;
    const float mA = 1.0f / c.mass[i];
    f3 vel = ld3(c.v, n, i);
    for (int a = 0; a < k; ++a) {
        const int sidx = order[a];
        const uint32_t q = sidx * n + i;
        const float K = mA + 0.0f + 0.0f + 0.0f;
        const float nmass = K > 0.0f ? 1.0f / K : 0.0f;
        const float k11 = mA + 0.0f + 0.0f + 0.0f, k12 = 0.0f + 0.0f, k22 = mA + 0.0f + 0.0f + 0.0f;
        float det = k11 * k22 - k12 * k12;
        if (det != 0.0f) det = 1.0f / det;
        const float tm_xx = det * k22, tm_yx = -det * k12, tm_xy = -det * k12, tm_yy = det * k11;
        const float fr = sqrtf(c.p_friction[i] * c.sph[sidx].friction);
        float ni = c.c_imp[q], tix = c.c_imp[nn + q], tiy = c.c_imp[2 * nn + q];
        const f3 nrm = ld3(c.c_normal, nn, q), t1 = ld3(c.c_t1, nn, q), t2 = ld3(c.c_t2, nn, q);
        {
            const f3 dvv = zero3() - vel;
            const float Cdot = dot(nrm, dvv);
            float impulse = nmass * (-Cdot + 0.0f);
            const float old = ni;
            const float sum = old + impulse;
            ni = sum > 0.0f ? sum : 0.0f;
            impulse = ni - old;
            const f3 P = impulse * nrm;
            vel = vel - mA * P;
        }
        {
            const f3 dvv = zero3() - vel;
            const float cx = dot(dvv, t1), cy = dot(dvv, t2);
            const float ncx = -cx, ncy = -cy;
            const float ix = ncx * tm_xx + ncy * tm_yx;
            const float iy = ncx * tm_xy + ncy * tm_yy;
            const float ox = tix, oy = tiy;
            tix += ix;
            tiy += iy;
            const float maxImpulse = fr * ni;
            if (tix * tix + tiy * tiy > maxImpulse * maxImpulse) {
                const float sl = sqrtf(tix * tix + tiy * tiy);
                if (sl > kEpsilon) {
                    tix /= sl;
                    tiy /= sl;
                }
                tix *= maxImpulse;
                tiy *= maxImpulse;
            }
            const float jx = tix - ox, jy = tiy - oy;
            const f3 P = jx * t1 + jy * t2;
            vel = vel - mA * P;
        }
        c.c_imp[q] = ni;
        c.c_imp[nn + q] = tix;
        c.c_imp[2 * nn + q] = tiy;
    }
    st3(c.v, n, i, vel);
}

// SolveBodyContactPositionConstraints (cloth_contact_solver.cpp:620-718);
// returns the smallest separation
__device__ float body_position(const ClothDev& c, uint32_t i, const int* order, int k)
{
    const uint32_t n = c.n, nn = c.nsph * n;
    const float mA = 1.0f / c.mass[i];
    f3 pos = ld3(c.x, n, i);
    float min_sep = 0.0f;
    for (int a = 0; a < k; ++a) {
        const int sidx = order[a];
        const SphereDev& sp = c.sph[sidx];
        const f3 nA = ld3(c.c_normal, nn, sidx * n + i);
        const f3 cB = sp.kind == 0 ? mk(sp.cx, sp.cy, sp.cz) : ld3(c.c_point, nn, sidx * n + i);
        const float separation = dot(cB - pos, nA) - c.p_radius[i] - sp.radius;
        min_sep = min_sep < separation ? min_sep : separation;
        const float Cv = kBaum * (separation + kSlop);
        float C = Cv < 0.0f ? Cv : 0.0f;
        C = -kMaxCorrection > C ? -kMaxCorrection : C;
        const float K = mA + 0.0f + 0.0f + 0.0f;
        const float impulse = K > 0.0f ? -C / K : 0.0f;
        const f3 P = impulse * nA;
        pos = pos - mA * P;
    }
    st3(c.x, n, i, pos);
    return min_sep;
}

// ---- triangle contacts ---------------------------------------------------

__device__ __forceinline__ float inv_mass(const ClothDev& c, uint32_t i)
{
    return c.type[i] == 0 ? 0.0f : 1.0f / c.mass[i];
}

// InitializeTriangleContactConstraints (cloth_contact_solver.cpp:179-262)
__device__ void tri_init(const ClothDev& c, TriCon& x, uint2 key, float4 w, float4 imp)
{
    const uint32_t n = c.n;
    const uint4 tv = c.tri[key.y];
    x.ia = key.x; x.ib = tv.x; x.ic = tv.y; x.id = tv.z;
    x.mA = inv_mass(c, x.ia); x.mB = inv_mass(c, x.ib); x.mC = inv_mass(c, x.ic); x.mD = inv_mass(c, x.id);
    x.radius_a = c.p_radius[x.ia];
    x.radius_t = c.thickness;  // the triangle's radius (cloth.cpp:136)
    x.wB = w.x; x.wC = w.y; x.wD = w.z;
    const f3 xA = ld3(c.x, n, x.ia), xB = ld3(c.x, n, x.ib), xC = ld3(c.x, n, x.ic), xD = ld3(c.x, n, x.id);
    const f3 cB = (x.wB * xB + x.wC * xC) + x.wD * xD;
    f3 nrm = cB - xA;
    normalize(nrm);
    x.nx = nrm.x; x.ny = nrm.y; x.nz = nrm.z;
    const float K = ((x.mA + x.mB * x.wB * x.wB) + x.mC * x.wC * x.wC) + x.mD * x.wD * x.wD;
    x.normal_mass = K > 0.0f ? 1.0f / K : 0.0f;
    x.friction = sqrtf(c.p_friction[x.ia] * c.friction);  // b3MixFriction(particle, triangle)
    const f3 t1 = perp(nrm), t2 = cross(t1, nrm);
    x.t1x = t1.x; x.t1y = t1.y; x.t1z = t1.z;
    x.t2x = t2.x; x.t2y = t2.y; x.t2z = t2.z;
    x.ni = imp.x; x.ti1 = imp.y; x.ti2 = imp.z;
}

struct Quad {
    f3 a, b, c, d;
};

__device__ __forceinline__ Quad load_quad(const float* p, uint32_t n, const TriCon& x)
{
    return Quad{ld3(p, n, x.ia), ld3(p, n, x.ib), ld3(p, n, x.ic), ld3(p, n, x.id)};
}

__device__ __forceinline__ void store_quad(float* p, uint32_t n, const TriCon& x, const Quad& q)
{
    st3(p, n, x.ia, q.a);
    st3(p, n, x.ib, q.b);
    st3(p, n, x.ic, q.c);
    st3(p, n, x.id, q.d);
}

// vA += mA (lambda JA), ... with JA = -u, JB = wB u, JC = wC u, JD = wD u
__device__ __forceinline__ void apply(const TriCon& x, float lambda, f3 u, Quad& q)
{
    const f3 JA = neg(u), JB = x.wB * u, JC = x.wC * u, JD = x.wD * u;
    const f3 PA = lambda * JA, PB = lambda * JB, PC = lambda * JC, PD = lambda * JD;
    q.a = q.a + x.mA * PA;
    q.b = q.b + x.mB * PB;
    q.c = q.c + x.mC * PC;
    q.d = q.d + x.mD * PD;
}

// WarmStartTriangleContactConstraints (cloth_contact_solver.cpp:309-386)
__device__ void tri_warm_start(const ClothDev& c, const TriCon& x)
{
    Quad q = load_quad(c.v, c.n, x);
    apply(x, x.ni, mk(x.nx, x.ny, x.nz), q);
    apply(x, x.ti1, mk(x.t1x, x.t1y, x.t1z), q);
    apply(x, x.ti2, mk(x.t2x, x.t2y, x.t2z), q);
    store_quad(c.v, c.n, x, q);
}

// SolveTriangleContactVelocityConstraints (cloth_contact_solver.cpp:474-596)
__device__ void tri_velocity(const ClothDev& c, TriCon& x)
{
    Quad q = load_quad(c.v, c.n, x);
    {
        const f3 nrm = mk(x.nx, x.ny, x.nz);
        const f3 vCB = (x.wB * q.b + x.wC * q.c) + x.wD * q.d;
        const float Cdot = dot(vCB - q.a, nrm);
        float impulse = -x.normal_mass * Cdot;
        const float old = x.ni;
        const float sum = x.ni + impulse;
        x.ni = sum > 0.0f ? sum : 0.0f;
        impulse = x.ni - old;
        apply(x, impulse, nrm, q);
    }
    for (int dir = 0; dir < 2; ++dir) {
        const float hi = x.friction * x.ni;
        const float lo = -hi;
        const f3 u = dir == 0 ? mk(x.t1x, x.t1y, x.t1z) : mk(x.t2x, x.t2y, x.t2z);
        float& acc = dir == 0 ? x.ti1 : x.ti2;
        const f3 vCB = (x.wB * q.b + x.wC * q.c) + x.wD * q.d;
        const float Cdot = dot(vCB - q.a, u);
        float impulse = -x.normal_mass * Cdot;  // tangent masses equal the normal mass
        const float old = acc;
        const float a = acc + impulse;
        const float m = a < hi ? a : hi;  // b3Clamp = b3Max(lo, b3Min(a, hi))
        acc = lo > m ? lo : m;
        impulse = acc - old;
        apply(x, impulse, u, q);
    }
    store_quad(c.v, c.n, x, q);
}

// SolveTriangleContactPositionConstraints (cloth_contact_solver.cpp:720-794)
__device__ float tri_position(const ClothDev& c, const TriCon& x)
{
    Quad q = load_quad(c.x, c.n, x);
    const f3 cB = (x.wB * q.b + x.wC * q.c) + x.wD * q.d;
    f3 nrm = cB - q.a;
    const float distance = normalize(nrm);
    const float separation = (distance - x.radius_a) - x.radius_t;
    const float Cv = kBaum * (separation + kSlop);
    const float m = Cv < 0.0f ? Cv : 0.0f;
    const float C = -kMaxCorrection > m ? -kMaxCorrection : m;
    const float K = ((x.mA + x.mB * x.wB * x.wB) + x.mC * x.wC * x.wC) + x.mD * x.wD * x.wD;
    const float impulse = K > 0.0f ? -C / K : 0.0f;
    apply(x, impulse, nrm, q);
    store_quad(c.x, c.n, x, q);
    return separation;
}

__device__ __forceinline__ int enc_min(float f)
{
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float dec_min(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// The whole contact phase of one step in one block: v += dv, x += y, m_x =
// dv; initialize, warm start, velocity iterations (body contacts, then
// triangle contacts), store, x += h v, position iterations with the early
// out.  Triangle contacts run level by level: a contact's level is one more
// than the highest level of an earlier active contact sharing a particle, so
// each particle's updates come in list order.
__global__ void __launch_bounds__(kSolveThreads) k_sc_solve(ClothDev c, SelfDev s, int cur)
{
    extern __shared__ uint32_t last[];  // per particle: level of its latest contact
    __shared__ int s_min[2];
    __shared__ uint32_t s_levels, s_width;
    const uint32_t n = c.n, tid = threadIdx.x, nt = blockDim.x;
    StepScalars* sc = c.sc;
    const float h = sc->dt;
    const uint32_t A = s.counts[kCountActive];
    const uint32_t* ls = s.level_start;

    for (uint32_t i = tid; i < n; i += nt) {
        const f3 dv = ld3(c.dv, n, i);
        st3(c.v, n, i, ld3(c.v, n, i) + dv);
        st3(c.x, n, i, ld3(c.x, n, i) + ld3(c.y, n, i));
        st3(c.mx, n, i, dv);
        last[i] = 0;
    }
    __syncthreads();
    for (uint32_t a = tid; a < A; a += nt) {
        const uint32_t k = s.active_idx[a];
        tri_init(c, s.con[a], s.key[cur][k], s.w[cur][k], s.imp[cur][k]);
    }
    __syncthreads();
    if (tid == 0) {
        // levels, then the contacts grouped by level (ascending within a level)
        uint32_t top = 0;
        for (uint32_t a = 0; a < A; ++a) {
            TriCon& x = s.con[a];
            uint32_t L = last[x.ia];
            L = last[x.ib] > L ? last[x.ib] : L;
            L = last[x.ic] > L ? last[x.ic] : L;
            L = last[x.id] > L ? last[x.id] : L;
            L += 1;
            last[x.ia] = last[x.ib] = last[x.ic] = last[x.id] = L;
            x.pad = __uint_as_float(L);
            top = L > top ? L : top;
        }
        uint32_t* lsw = s.level_start;
        for (uint32_t L = 0; L <= top + 1; ++L) lsw[L] = 0;
        for (uint32_t a = 0; a < A; ++a) lsw[__float_as_uint(s.con[a].pad)] += 1;
        uint32_t width = 0;
        for (uint32_t L = 1; L <= top; ++L) width = lsw[L] > width ? lsw[L] : width;
        s_width = width;
        for (uint32_t L = 1; L <= top; ++L) lsw[L] += lsw[L - 1];
        lsw[top + 1] = A;
        for (uint32_t a = A; a-- > 0;) s.by_level[--lsw[__float_as_uint(s.con[a].pad)]] = a;
        s_levels = top;
        s.counts[kCountLevels] = top;
    }
    __syncthreads();
    const uint32_t top = s_levels;
    // Levels of at most 32 contacts run in warp 0 alone, with warp
    // barriers between levels; wider ones use the whole block.
    const bool narrow = s_width <= 32u;
    const uint32_t lane = tid & 31u;
    auto sweep = [&](auto&& fn) {
        if (narrow) {
            if (tid < 32u) {
                for (uint32_t L = 1; L <= top; ++L) {
                    const uint32_t j = ls[L] + lane;
                    if (j < ls[L + 1]) fn(j);
                    __syncwarp();
                }
            }
            __syncthreads();
        } else {
            for (uint32_t L = 1; L <= top; ++L) {
                for (uint32_t j = ls[L] + tid; j < ls[L + 1]; j += nt) fn(j);
                __syncthreads();
            }
        }
    };

    // warm start: body contacts, then triangle contacts
    uint32_t body_active = 0;
    for (uint32_t i = tid; i < n; i += nt) {
        int order[kMaxBodyContacts];
        const int k = c.nsph ? body_order(c, i, order) : 0;
        body_active += (uint32_t)k;
        if (k) body_warm_start(c, i, order, k);
    }
    if (body_active) atomicAdd(&sc->active_contacts, body_active);
    __syncthreads();
    sweep([&](uint32_t j) { tri_warm_start(c, s.con[s.by_level[j]]); });
    // velocity iterations
    for (uint32_t it = 0; it < sc->vel_iters; ++it) {
        for (uint32_t i = tid; i < n; i += nt) {
            int order[kMaxBodyContacts];
            const int k = c.nsph ? body_order(c, i, order) : 0;
            if (k) body_velocity(c, i, order, k);
        }
        __syncthreads();
        sweep([&](uint32_t j) { tri_velocity(c, s.con[s.by_level[j]]); });
    }
    // store impulses (body impulses live in c_imp already); integrate positions
    for (uint32_t a = tid; a < A; a += nt) {
        const TriCon& x = s.con[a];
        s.imp[cur][s.active_idx[a]] = make_float4(x.ni, x.ti1, x.ti2, 0.0f);
    }
    for (uint32_t i = tid; i < n; i += nt) st3(c.x, n, i, ld3(c.x, n, i) + h * ld3(c.v, n, i));
    __syncthreads();
    // position iterations with the early out (cloth_solver.cpp:149-164)
    for (uint32_t it = 0; it < sc->pos_iters; ++it) {
        if (tid == 0) s_min[0] = s_min[1] = enc_min(0.0f);
        __syncthreads();
        float mb = 0.0f;
        for (uint32_t i = tid; i < n; i += nt) {
            int order[kMaxBodyContacts];
            const int k = c.nsph ? body_order(c, i, order) : 0;
            if (k) {
                const float ms = body_position(c, i, order, k);
                mb = mb < ms ? mb : ms;
            }
        }
        if (mb < 0.0f) atomicMin(&s_min[0], enc_min(mb));
        __syncthreads();
        float mt = 0.0f;
        sweep([&](uint32_t j) {
            const float sep = tri_position(c, s.con[s.by_level[j]]);
            mt = mt < sep ? mt : sep;
        });
        if (mt < 0.0f) atomicMin(&s_min[1], enc_min(mt));
        __syncthreads();
        const bool solved = dec_min(s_min[0]) >= -3.0f * kSlop && dec_min(s_min[1]) >= -3.0f * kSlop;
        __syncthreads();
        if (solved) break;
    }
}

// Triangle proxies after the step (cloth.cpp:580-597): displacement dt times
// the mean of the three vertex velocities.
__global__ void k_sc_tri_sync(ClothDev c)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.t) return;
    const uint32_t n = c.n;
    const uint4 tv = c.tri[k];
    const f3 velocity = ((ld3(c.v, n, tv.x) + ld3(c.v, n, tv.y)) + ld3(c.v, n, tv.z)) / 3.0f;
    tri_move_proxy_dev(c, k, c.sc->dt * velocity);
}

__device__ __forceinline__ unsigned long long pair_key(uint32_t p, uint32_t t)
{
    return ((unsigned long long)p << 32) | t;
}

__device__ __forceinline__ uint32_t hash_slot(unsigned long long key, uint32_t mask)
{
    key ^= key >> 33;
    key *= 0xff51afd7ed558ccdull;
    key ^= key >> 33;
    return (uint32_t)key & mask;
}

__global__ void k_sc_hash(SelfDev s, int cur, uint32_t m_bound)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m_bound || k >= s.counts[kCountList]) return;
    const uint2 pk = s.key[cur][k];
    const unsigned long long key = pair_key(pk.x, pk.y);
    uint32_t slot = hash_slot(key, s.hash_mask);
    for (uint32_t probe = 0; probe <= s.hash_mask; ++probe) {
        const unsigned long long prev = atomicCAS(&s.table[slot], ~0ull, key);
        if (prev == ~0ull || prev == key) return;
        slot = (slot + 1) & s.hash_mask;
    }
}

__device__ __forceinline__ bool listed(const SelfDev& s, uint32_t p, uint32_t t)
{
    const unsigned long long key = pair_key(p, t);
    uint32_t slot = hash_slot(key, s.hash_mask);
    for (uint32_t probe = 0; probe <= s.hash_mask; ++probe) {
        const unsigned long long v = s.table[slot];
        if (v == key) return true;
        if (v == ~0ull) return false;
        slot = (slot + 1) & s.hash_mask;
    }
    return false;
}

// One warp per particle over every triangle in index order: the pairs
// FindPairs + AddPair would add, counted (write = 0) or written at the
// particle's offset in ascending triangle order (write = 1).
__global__ void k_sc_pairs(ClothDev c, SelfDev s, int write)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < c.n; p += warps) {
        const bool moved_p = c.p_moved[p] != 0, dyn_p = dyn(c, p);
        uint32_t running = write ? s.pair_off[p] : 0u;
        for (uint32_t t0 = 0; t0 < c.t; t0 += 32u) {
            const uint32_t t = t0 + lane;
            bool cand = false;
            if (t < c.t && (moved_p || c.t_moved[t]) && overlap_pt(c, p, t)) {
                const uint4 tv = c.tri[t];
                cand = p != tv.x && p != tv.y && p != tv.z && (dyn_p || dyn(c, tv.x) || dyn(c, tv.y) || dyn(c, tv.z)) &&
                       !listed(s, p, t);
            }
            const uint32_t mask = __ballot_sync(0xffffffffu, cand);
            if (write && cand) s.fresh[running + __popc(mask & ((1u << lane) - 1u))] = make_uint2(p, t);
            running += __popc(mask);
        }
        if (!write && lane == 0) s.pair_off[p] = running;
    }
}

// Exclusive scan of pair_off[0, n) in place; pair_off[n] and counts[fresh]
// get the total.
__global__ void __launch_bounds__(1024) k_sc_scan(SelfDev s, uint32_t n)
{
    uint32_t base_sum = 0;
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n ? s.pair_off[i] : 0u;
        uint32_t tot;
        const uint32_t before = block_scan(v, tot);
        if (i < n) s.pair_off[i] = base_sum + before;
        base_sum += tot;
    }
    if (threadIdx.x == 0) {
        s.pair_off[n] = base_sum;
        s.counts[kCountFresh] = base_sum;
    }
}

// The new list: this step's pairs, newest first (each AddPair pushes to the
// front), then the old list.
__global__ void k_sc_prepend(SelfDev s, int cur, uint32_t fresh, uint32_t old)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const int dst = 1 - cur;
    if (j < fresh) {
        s.key[dst][j] = s.fresh[fresh - 1 - j];
        s.act[dst][j] = 0;
        s.w[dst][j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        s.imp[dst][j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else if (j < fresh + old) {
        const uint32_t k = j - fresh;
        s.key[dst][j] = s.key[cur][k];
        s.act[dst][j] = s.act[cur][k];
        s.w[dst][j] = s.w[cur][k];
        s.imp[dst][j] = s.imp[cur][k];
    }
}

// The move buffer is empty after FindPairs (broad_phase.h:181-182).
__global__ void k_sc_finish(ClothDev c, SelfDev s, uint32_t total)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) s.counts[kCountList] = total;
    if (i < c.n) c.p_moved[i] = 0;
    if (i < c.t) c.t_moved[i] = 0;
}

// Triangle proxies at creation (cloth.cpp:140-150): the triangle's AABB
// extended by the thickness, then by B3_AABB_EXTENSION in CreateProxy.
__global__ void k_sc_init_proxies(ClothDev c)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.t) return;
    const uint32_t n = c.n, t = c.t;
    const uint4 tv = c.tri[k];
    const f3 A = ld3(c.x, n, tv.x), B = ld3(c.x, n, tv.y), C = ld3(c.x, n, tv.z);
    const float r = c.thickness;
    const f3 mn = mk(B.x < C.x ? B.x : C.x, B.y < C.y ? B.y : C.y, B.z < C.z ? B.z : C.z);
    const f3 mx = mk(B.x > C.x ? B.x : C.x, B.y > C.y ? B.y : C.y, B.z > C.z ? B.z : C.z);
    c.tri_lo[k] = ((A.x < mn.x ? A.x : mn.x) - r) - 0.2f;
    c.tri_lo[t + k] = ((A.y < mn.y ? A.y : mn.y) - r) - 0.2f;
    c.tri_lo[2 * t + k] = ((A.z < mn.z ? A.z : mn.z) - r) - 0.2f;
    c.tri_hi[k] = ((A.x > mx.x ? A.x : mx.x) + r) + 0.2f;
    c.tri_hi[t + k] = ((A.y > mx.y ? A.y : mx.y) + r) + 0.2f;
    c.tri_hi[2 * t + k] = ((A.z > mx.z ? A.z : mx.z) + r) + 0.2f;
    c.t_moved[k] = 1;
}

__global__ void k_sc_fill_u8(uint8_t* p, uint32_t n, uint8_t v)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

inline uint32_t blocks(uint32_t n, uint32_t b) { return n ? (n + b - 1) / b : 1u; }

b3g_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return B3G_OK;
    return e == cudaErrorMemoryAllocation ? B3G_ERR_OUT_OF_MEMORY : B3G_ERR_CUDA;
}

#define SC_TRY(expr)                                   \
    do {                                               \
        cudaError_t e_ = (expr);                       \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

}  // namespace

// Host state of one cloth's self-collision.
struct SelfState {
    SelfDev d{};
    int cur = 0;
    uint32_t count = 0;      // list length after the last step
    uint32_t active = 0;     // active contacts of the last solve
    uint32_t levels = 0;     // dependency levels of the last solve
    uint32_t* h_counts = nullptr;
    std::vector<void*> list_bufs;  // buffers sized by the capacity
    void* fixed[6] = {};           // tri_lo, tri_hi, t_moved, p_moved, p_purge, counts / pair_off
};

namespace {

void free_list(SelfState* s)
{
    for (void* p : s->list_bufs) cudaFree(p);
    s->list_bufs.clear();
}

// Buffers sized by the capacity; the current list (count entries) is copied
// into the new current buffer.
b3g_status alloc_list(SelfState* s, uint32_t cap, cudaStream_t st)
{
    SelfDev nd = s->d;
    std::vector<void*> bufs;
    auto take = [&](auto*& p, size_t count) -> cudaError_t {
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(*p));
        if (e == cudaSuccess) bufs.push_back((void*)p);
        return e;
    };
    uint32_t slots = 1;
    while (slots < 2u * cap) slots <<= 1;
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        if (e == cudaSuccess) e = take(nd.key[b], cap);
        if (e == cudaSuccess) e = take(nd.act[b], cap);
        if (e == cudaSuccess) e = take(nd.w[b], cap);
        if (e == cudaSuccess) e = take(nd.imp[b], cap);
    }
    if (e == cudaSuccess) e = take(nd.fresh, cap);
    if (e == cudaSuccess) e = take(nd.table, slots);
    if (e == cudaSuccess) e = take(nd.active_idx, cap);
    if (e == cudaSuccess) e = take(nd.by_level, cap);
    if (e == cudaSuccess) e = take(nd.level_start, (size_t)cap + 2);
    if (e == cudaSuccess) e = take(nd.con, cap);
    if (e == cudaSuccess && s->count) {
        const int c = s->cur;
        const size_t m = s->count;
        e = cudaMemcpyAsync(nd.key[c], s->d.key[c], m * sizeof(uint2), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(nd.act[c], s->d.act[c], m * sizeof(uint8_t), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(nd.w[c], s->d.w[c], m * sizeof(float4), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(nd.imp[c], s->d.imp[c], m * sizeof(float4), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        for (void* p : bufs) cudaFree(p);
        return cuda_status(e);
    }
    free_list(s);
    s->list_bufs = bufs;
    nd.cap = cap;
    nd.hash_mask = slots - 1;
    s->d = nd;
    return B3G_OK;
}

}  // namespace

// Sets up self-collision for a cloth whose thickness is above zero: triangle
// proxies from the current positions, every proxy in the move buffer, an
// empty contact list.
b3g_status self_attach(b3g_cloth* c)
{
    const uint32_t n = c->dev.n, t = c->dev.t;
    if (n > kSelfMaxParticles) return B3G_ERR_UNSUPPORTED;
    SelfState* s = new (std::nothrow) SelfState();
    if (!s) return B3G_ERR_OUT_OF_MEMORY;
    s->d.n = n;
    s->d.t = t;
    cudaStream_t st = c->stream;
    float *lo = nullptr, *hi = nullptr;
    uint8_t *tm = nullptr, *pm = nullptr, *pp = nullptr;
    uint32_t* words = nullptr;
    cudaError_t e = cudaMalloc(&lo, 3 * (size_t)std::max(t, 1u) * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&hi, 3 * (size_t)std::max(t, 1u) * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&tm, std::max(t, 1u));
    if (e == cudaSuccess) e = cudaMalloc(&pm, n);
    if (e == cudaSuccess) e = cudaMalloc(&pp, n);
    if (e == cudaSuccess) e = cudaMalloc(&words, (kCountWords + (size_t)n + 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_counts, kCountWords * sizeof(uint32_t));
    s->fixed[0] = lo; s->fixed[1] = hi; s->fixed[2] = tm; s->fixed[3] = pm; s->fixed[4] = pp; s->fixed[5] = words;
    b3g_status r = cuda_status(e);
    if (r == B3G_OK) {
        s->d.counts = words;
        s->d.pair_off = words + kCountWords;
        r = alloc_list(s, std::max<uint32_t>(1024u, 4u * n), st);
    }
    if (r != B3G_OK) {
        c->self = s;
        self_free(c);
        return r;
    }
    c->dev.tri_lo = lo;
    c->dev.tri_hi = hi;
    c->dev.t_moved = tm;
    c->dev.p_moved = pm;
    c->dev.p_purge = pp;
    c->self = s;
    SC_TRY(cudaMemsetAsync(words, 0, (kCountWords + (size_t)n + 1) * sizeof(uint32_t), st));
    SC_TRY(cudaMemsetAsync(pp, 0, n, st));
    k_sc_fill_u8<<<blocks(n, 256), 256, 0, st>>>(pm, n, 1);
    if (t) k_sc_init_proxies<<<blocks(t, 256), 256, 0, st>>>(c->dev);
    count_launches(t ? 2 : 1);
    SC_TRY(cudaGetLastError());
    SC_TRY(cudaFuncSetAttribute(k_sc_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kSelfMaxParticles * sizeof(uint32_t))));
    SC_TRY(cudaStreamSynchronize(st));
    return B3G_OK;
}

void self_free(b3g_cloth* c)
{
    SelfState* s = c->self;
    if (!s) return;
    free_list(s);
    for (void* p : s->fixed)
        if (p) cudaFree(p);
    if (s->h_counts) cudaFreeHost(s->h_counts);
    delete s;
    c->self = nullptr;
    c->dev.tri_lo = c->dev.tri_hi = nullptr;
    c->dev.t_moved = c->dev.p_moved = c->dev.p_purge = nullptr;
}

// Step start: UpdateClothContacts.
b3g_status self_update(b3g_cloth* c, cudaStream_t st)
{
    SelfState* s = c->self;
    k_sc_update<<<1, 1024, 0, st>>>(c->dev, s->d, s->cur, s->count);
    count_launches(1);
    SC_TRY(cudaGetLastError());
    s->cur = 1 - s->cur;
    return B3G_OK;
}

// After the CG: the contact solve of both contact kinds (replaces the body
// contact kernels of the plain step).
b3g_status self_solve(b3g_cloth* c, cudaStream_t st)
{
    SelfState* s = c->self;
    const size_t smem = (size_t)c->dev.n * sizeof(uint32_t);
    if (c->dev.n > kSelfMaxParticles) return B3G_ERR_UNSUPPORTED;
    k_sc_solve<<<1, kSolveThreads, smem, st>>>(c->dev, s->d, s->cur);
    count_launches(1);
    SC_TRY(cudaGetLastError());
    return B3G_OK;
}

// Step end, after the particle proxies moved: triangle proxies, then
// FindNewClothContacts.  Reads the pair count back to size the list.
b3g_status self_find(b3g_cloth* c, cudaStream_t st)
{
    SelfState* s = c->self;
    const uint32_t n = c->dev.n, t = c->dev.t;
    if (t) k_sc_tri_sync<<<blocks(t, 256), 256, 0, st>>>(c->dev);
    SC_TRY(cudaMemsetAsync(s->d.table, 0xff, ((size_t)s->d.hash_mask + 1) * sizeof(unsigned long long), st));
    if (s->count) k_sc_hash<<<blocks(s->count, 256), 256, 0, st>>>(s->d, s->cur, s->count);
    const uint32_t pair_blocks = blocks(n * 32u, 256);
    k_sc_pairs<<<pair_blocks, 256, 0, st>>>(c->dev, s->d, 0);
    k_sc_scan<<<1, 1024, 0, st>>>(s->d, n);
    count_launches((t ? 1 : 0) + (s->count ? 1 : 0) + 2);
    SC_TRY(cudaGetLastError());
    SC_TRY(cudaMemcpyAsync(s->h_counts, s->d.counts, kCountWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    SC_TRY(cudaStreamSynchronize(st));
    const uint32_t old = s->h_counts[kCountList], fresh = s->h_counts[kCountFresh];
    s->active = s->h_counts[kCountActive];
    s->levels = s->h_counts[kCountLevels];
    s->count = old;
    if ((uint64_t)old + fresh > s->d.cap) {
        uint64_t want = std::max<uint64_t>(2ull * s->d.cap, (uint64_t)old + fresh);
        if (want > 0x7fffffffull) return B3G_ERR_CAPACITY;
        b3g_status r = alloc_list(s, (uint32_t)want, st);
        if (r != B3G_OK) return r;
        // the write pass must see the same table as the count pass
        SC_TRY(cudaMemsetAsync(s->d.table, 0xff, ((size_t)s->d.hash_mask + 1) * sizeof(unsigned long long), st));
        if (old) k_sc_hash<<<blocks(old, 256), 256, 0, st>>>(s->d, s->cur, old);
        count_launches(old ? 1 : 0);
    }
    if (fresh) k_sc_pairs<<<pair_blocks, 256, 0, st>>>(c->dev, s->d, 1);
    if (fresh + old) k_sc_prepend<<<blocks(fresh + old, 256), 256, 0, st>>>(s->d, s->cur, fresh, old);
    k_sc_finish<<<blocks(std::max(n, t), 256), 256, 0, st>>>(c->dev, s->d, fresh + old);
    count_launches((fresh ? 1 : 0) + (fresh + old ? 1 : 0) + 1);
    SC_TRY(cudaGetLastError());
    if (fresh + old) s->cur = 1 - s->cur;
    s->count = fresh + old;
    return B3G_OK;
}

// The list in list order (head first): see b3g_cloth_read_tri_contacts.
b3g_status self_read(const b3g_cloth* c, uint32_t* count, uint32_t* pt, uint8_t* active, float* w, float* impulses)
{
    const SelfState* s = c->self;
    if (!s) {
        *count = 0;
        return B3G_OK;
    }
    const uint32_t m = s->count;
    *count = m;
    if (!m) return B3G_OK;
    cudaStream_t st = c->stream;
    SC_TRY(cudaStreamSynchronize(st));
    const int k = s->cur;
    std::vector<uint2> key(m);
    std::vector<uint8_t> act(m);
    std::vector<float4> ww(m), imp(m);
    SC_TRY(cudaMemcpy(key.data(), s->d.key[k], m * sizeof(uint2), cudaMemcpyDeviceToHost));
    SC_TRY(cudaMemcpy(act.data(), s->d.act[k], m, cudaMemcpyDeviceToHost));
    SC_TRY(cudaMemcpy(ww.data(), s->d.w[k], m * sizeof(float4), cudaMemcpyDeviceToHost));
    SC_TRY(cudaMemcpy(imp.data(), s->d.imp[k], m * sizeof(float4), cudaMemcpyDeviceToHost));
    for (uint32_t j = 0; j < m; ++j) {
        if (pt) { pt[2 * j] = key[j].x; pt[2 * j + 1] = key[j].y; }
        if (active) active[j] = act[j];
        if (w) {
            const bool on = act[j] != 0;
            w[3 * j] = on ? ww[j].x : 0.0f;
            w[3 * j + 1] = on ? ww[j].y : 0.0f;
            w[3 * j + 2] = on ? ww[j].z : 0.0f;
        }
        if (impulses) { impulses[3 * j] = imp[j].x; impulses[3 * j + 1] = imp[j].y; impulses[3 * j + 2] = imp[j].z; }
    }
    return B3G_OK;
}

void self_stats(const b3g_cloth* c, uint32_t* contacts, uint32_t* active, uint32_t* levels)
{
    const SelfState* s = c->self;
    *contacts = s ? s->count : 0;
    *active = s ? s->active : 0;
    *levels = s ? s->levels : 0;
}

}  // namespace b3g
