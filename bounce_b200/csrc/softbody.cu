// Soft body step on the GPU: b3SoftBody::Step (src/bounce/softbody/
// softbody.cpp:700-735) without a world.
//
//   k_sb_elements   one thread per tetrahedron: the element rotation by
//                   b3ExtractRotation from the element's previous rotation
//                   (softbody_force_solver.cpp:53-91), the element's f0 terms
//                   R Ke x0 and its plastic strain update and plastic forces
//                   (:256-357)
//   k_sb_assemble   one warp per node: the node's row of K summed over its
//                   elements in element order (the reference's K(vi, vj) +=
//                   R Ke RT), then b = M v - h (K p + f0 - (f_plastic + f_ext))
//                   and A = M + h C + h^2 K (:359-377) in the reference's
//                   float order; K p runs in the row list's order
//   MPCG            the block-CSR MPCG in its soft body mode (x0 = v,
//                   delta_0 = Sb . diag(A) Sb; softbody_force_solver.cpp:93-164)
//   k_sb_integrate  v = solution, x += h v, forces cleared
//                   (softbody_solver.cpp:105-110, softbody.cpp:716-720)
//
// Node vectors are xyz per node (b3DenseVec3 layout).  With -fmad=false the
// element and assembly arithmetic is the reference's; the one difference is
// the C library's double sin and cos in b3Quat::Set against CUDA's, which can
// differ in the last bit of the rounded float in rare cases.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/b3g.h"
#include "cloth_dev.cuh"
#include "grid_cg.cuh"
#include "mpcg_solve.cuh"
#include "hull_gjk.cuh"
#include "softbody_prep.h"
#include "vec.cuh"

namespace b3g {

struct SoftDev {
    uint32_t n, t, nnz;
    const float* rest;
    float *x, *v, *f;
    const float* mass;
    float* damping;
    uint8_t* type;
    const uint4* tets;
    const float *Ke, *invE, *B, *P;
    float4* q;
    float* eps;
    float *R, *f0s, *fps;
    float c_yield, c_creep, c_max;
    const uint32_t *rowptr, *cols, *diag;
    float* vals;
    const uint32_t *inc_ptr, *inc_elem, *inc_meta;
    float *b, *S, *xsol;
    float gx, gy, gz;

    // contacts with static hulls (b3SoftBody::SetWorld): node radius and
    // friction, node proxies (fat AABBs, 3 floats per node for lo and hi),
    // and per (hull, node) contact slots; the proxies are kept from creation
    float *radius, *friction, *fat_lo, *fat_hi;
    uint32_t nhull, step_index;
    SphereDev hull[kMaxSpheres];
    uint8_t *c_exists, *c_active;
    uint32_t* c_key;                // creation key: step index * kMaxSpheres + hull
    float *c_normal, *c_t1, *c_t2, *c_point, *c_imp;  // 3 planes of nhull * n each
    int* min_sep;                   // per position iteration, order-preserving ints
    uint32_t* active_count;
    uint32_t vel_iters, pos_iters;

    // The system again in the cloth's SELL-32 layout for the persistent CG
    // (null until the first persistent solve): slot k of row r at
    // sell_off[r / 32] + 32 k + r % 32 of each of the 9 value planes; slot 0
    // is the diagonal block, as in the cloth's layout (the fused CG relies on
    // it), the other slots follow in the row list's order; b, x0 (= v), P^-1
    // and diag(A) as 3 planes of n.
    // The rows are reordered by degree there (sell_inv: node -> row), so
    // that every slice holds rows of one width; sb_type is the node types in
    // that order.
    float* sell_vals;
    const uint32_t *sell_off, *sell_inv;
    uint32_t sell_E;
    float *sb_b, *sb_x0, *sb_pinv, *sb_diag;
    uint8_t* sb_type;
};

namespace {

__device__ __forceinline__ f3 ldv(const float* p, uint32_t i) { return f3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void stv(float* p, uint32_t i, f3 v)
{
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
__device__ __forceinline__ m3 ldm(const float* p)
{
    return m3{f3{p[0], p[1], p[2]}, f3{p[3], p[4], p[5]}, f3{p[6], p[7], p[8]}};
}
__device__ __forceinline__ void stm(float* p, const m3& a)
{
    p[0] = a.x.x, p[1] = a.x.y, p[2] = a.x.z;
    p[3] = a.y.x, p[4] = a.y.y, p[5] = a.y.z;
    p[6] = a.z.x, p[7] = a.z.y, p[8] = a.z.z;
}
__device__ __forceinline__ m3 mmul(const m3& a, const m3& b) { return m3{a * b.x, a * b.y, a * b.z}; }
__device__ __forceinline__ m3 transpose(const m3& a)
{
    return m3{f3{a.x.x, a.y.x, a.z.x}, f3{a.x.y, a.y.y, a.z.y}, f3{a.x.z, a.y.z, a.z.z}};
}
__device__ __forceinline__ m3 diag3(float s) { return m3{f3{s, 0.0f, 0.0f}, f3{0.0f, s, 0.0f}, f3{0.0f, 0.0f, s}}; }

// include/bounce/common/math/quat.h: b3QuatMat33 (:306-318), b3Mul (:170-178),
// Normalize (:83-97), Set(axis, angle) (:99-107)
__device__ __forceinline__ m3 quat_mat(float4 q)
{
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    const float x2 = x + x, y2 = y + y, z2 = z + z;
    const float xx = x * x2, xy = x * y2, xz = x * z2;
    const float yy = y * y2, yz = y * z2, zz = z * z2;
    const float wx = w * x2, wy = w * y2, wz = w * z2;
    return m3{f3{1.0f - (yy + zz), xy + wz, xz - wy}, f3{xy - wz, 1.0f - (xx + zz), yz + wx},
              f3{xz + wy, yz - wx, 1.0f - (xx + yy)}};
}
__device__ __forceinline__ float4 quat_mul(float4 a, float4 b)
{
    return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
                       a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}

// b3ExtractRotation (softbody_force_solver.cpp:53-91): at most 20 steps of
// the rotation update from the previous rotation q
__device__ m3 extract_rotation(float4& q, const m3& A)
{
    for (int iteration = 0; iteration < 20; ++iteration) {
        const m3 R = quat_mat(q);
        const float s = fabsf(dot(R.x, A.x) + dot(R.y, A.y) + dot(R.z, A.z));
        if (s == 0.0f) break;
        const float inv_s = 1.0f / s + 1.0e-9f;
        const f3 v = (cross(R.x, A.x) + cross(R.y, A.y)) + cross(R.z, A.z);
        const f3 omega = inv_s * v;
        const float w = length(omega);
        if (w < 1.0e-9f) break;
        const f3 axis = omega / w;
        const float theta = 0.5f * w;
        const float sine = (float)sin((double)theta);
        const float4 oq = make_float4(sine * axis.x, sine * axis.y, sine * axis.z, (float)cos((double)theta));
        q = quat_mul(oq, q);
        const float len = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        if (len > 1.1920929e-07f) {
            const float sc = 1.0f / len;
            q.x *= sc;
            q.y *= sc;
            q.z *= sc;
            q.w *= sc;
        }
    }
    return quat_mat(q);
}

__device__ __forceinline__ float len6(const float* v)
{
    float r = 0.0f;
    for (int i = 0; i < 6; ++i) r += v[i] * v[i];
    return sqrtf(r);
}

__global__ void k_sb_elements(SoftDev d, float h, float inv_h)
{
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= d.t) return;
    const uint4 tv = d.tets[e];
    const uint32_t vs[4] = {tv.x, tv.y, tv.z, tv.w};
    f3 ps[4], xs[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        ps[k] = ldv(d.x, vs[k]);
        xs[k] = ldv(d.rest, vs[k]);
    }
    const m3 E = m3{ps[1] - ps[0], ps[2] - ps[0], ps[3] - ps[0]};
    const m3 A = mmul(E, ldm(d.invE + 9 * (size_t)e));
    float4 q = d.q[e];
    const m3 R = extract_rotation(q, A);
    d.q[e] = q;
    const m3 RT = transpose(R);
    stm(d.R + 9 * (size_t)e, R);
    // f0 terms: sum_j (R Ke_ij) x0_j.  Ke is read in memory order, 16 bytes
    // per load: block (i, j) sits at 9 (i + 4 j), so the four blocks of one j
    // are 36 consecutive floats; each of the four sums still runs over j in
    // order.
    const float4* Ke4 = reinterpret_cast<const float4*>(d.Ke + 144 * (size_t)e);
    f3 f0acc[4] = {zero3(), zero3(), zero3(), zero3()};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float kb[36];
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const float4 t4 = Ke4[9 * j + q];
            kb[4 * q] = t4.x, kb[4 * q + 1] = t4.y, kb[4 * q + 2] = t4.z, kb[4 * q + 3] = t4.w;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) f0acc[i] = f0acc[i] + mmul(R, ldm(kb + 9 * i)) * xs[j];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) stv(d.f0s + 12 * (size_t)e, i, f0acc[i]);
    // plasticity: total strain B (R^T p - x0), elastic = total - plastic
    float rx[12];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const f3 dd = RT * ps[i] - xs[i];
        rx[3 * i] = dd.x, rx[3 * i + 1] = dd.y, rx[3 * i + 2] = dd.z;
    }
    // B (6 x 12, entry (i, k) at i + 6 k) in memory order, 16 bytes per load
    const float4* B4 = reinterpret_cast<const float4*>(d.B + 72 * (size_t)e);
    float* ep = d.eps + 6 * (size_t)e;
    float plastic[6], elastic[6], bacc[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k2 = 0; k2 < 6; ++k2) {  // two columns k = 2 k2, 2 k2 + 1: 12 floats
        float bb[12];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const float4 t4 = B4[3 * k2 + q];
            bb[4 * q] = t4.x, bb[4 * q + 1] = t4.y, bb[4 * q + 2] = t4.z, bb[4 * q + 3] = t4.w;
        }
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2)
#pragma unroll
            for (int i = 0; i < 6; ++i) bacc[i] += bb[6 * h2 + i] * rx[2 * k2 + h2];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        plastic[i] = ep[i];
        elastic[i] = bacc[i] - plastic[i];
    }
    if (len6(elastic) > d.c_yield) {
        const float amount = h * (d.c_creep < inv_h ? d.c_creep : inv_h);
#pragma unroll
        for (int i = 0; i < 6; ++i) plastic[i] += amount * elastic[i];
    }
    const float lp = len6(plastic);
    if (lp > d.c_max) {
        const float scale = d.c_max / lp;
#pragma unroll
        for (int i = 0; i < 6; ++i) plastic[i] *= scale;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) ep[i] = plastic[i];
    // P (12 x 6, entry (3 i + r, k) at 3 i + r + 12 k) in memory order
    const float4* P4 = reinterpret_cast<const float4*>(d.P + 72 * (size_t)e);
    float pc[12] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        float pp[12];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const float4 t4 = P4[3 * k + q];
            pp[4 * q] = t4.x, pp[4 * q + 1] = t4.y, pp[4 * q + 2] = t4.z, pp[4 * q + 3] = t4.w;
        }
#pragma unroll
        for (int m = 0; m < 12; ++m) pc[m] += pp[m] * plastic[k];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) stv(d.fps + 12 * (size_t)e, i, R * mk(pc[3 * i], pc[3 * i + 1], pc[3 * i + 2]));
}

// One warp per node.  The node's incidences are taken 32 at a time: each
// lane forms its element's four R Ke_ij R^T blocks (and f0, f_plastic terms)
// into shared memory; then each lane owns up to four of the row's slots and
// adds, in incidence (= element) order, every block that lands on them --
// the reference's K(vi, vj) += R Ke R^T order, so the row is the same float
// for float.  K p, b and A follow as in the reference (:359-377), the serial
// sums on lane 0.
constexpr int kAsmWarps = 4;
constexpr uint32_t kMaxRowSlots = 128;  // slot ids are 7 bits wide

__global__ void __launch_bounds__(32 * kAsmWarps, 8) k_sb_assemble(SoftDev d, float h)
{
    __shared__ __align__(16) float sX[kAsmWarps][32 * 4 * 9];   // element blocks of one chunk
    __shared__ uint8_t sSlot[kAsmWarps][32 * 4];
    __shared__ float sF[kAsmWarps][32 * 6];       // f0 and f_plastic terms of one chunk
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t i = blockIdx.x * kAsmWarps + w;
    if (i >= d.n) return;  // whole warps leave together
    float* X = sX[w];
    uint8_t* SL = sSlot[w];
    float* F = sF[w];
    const uint32_t r0 = d.rowptr[i], deg = d.rowptr[i + 1] - r0;
    const float m = d.mass[i];
    const m3 M = diag3(m);
    // A = (M + h C) + (h h) K on the diagonal, 0 + (h h) K elsewhere
    const float hh = h * h;
    const float cd = d.damping[i] * m;
    const uint32_t dg = d.diag[i] - r0;
    float* vals = d.vals + 9 * (size_t)r0;
    f3 f0 = zero3(), fp = zero3(), kp = zero3();
    const uint32_t q0 = d.inc_ptr[i], q1 = d.inc_ptr[i + 1];
    // Each lane owns one slot of a group of 32; a row wider than 32 slots
    // (rare) takes the incidences again for each further group, so one
    // accumulator suffices and the kernel keeps to 64 registers.  Groups run
    // from the last down, so lane 0 can add K p in the row list's order
    // (newest first touch first: slot deg-1 down to 0) as they finish.
    for (uint32_t g = (deg + 31u) / 32u; g-- > 0;) {
        const uint32_t slot = lane + 32u * g;
        m3 acc = mzero();
        for (uint32_t qb = q0; qb < q1; qb += 32u) {
            const uint32_t cnt = min(32u, q1 - qb);
            if (lane < cnt) {
                const uint32_t e = d.inc_elem[qb + lane], meta = d.inc_meta[qb + lane];
                const uint32_t li = meta & 3u;
                const m3 R = ldm(d.R + 9 * (size_t)e);
                const m3 RT = transpose(R);
                // Ke is symmetric and stored so: a block below the diagonal
                // is the exact transpose of the one above it.  So the node's
                // blocks Ke(li, j) are the transposes of Ke(j, li), j != li,
                // which lie together, 144 bytes from 36 li on: nine 16-byte
                // loads instead of four scattered 36-byte blocks.
                // They are staged in the lane's own 36 floats of X and
                // replaced there by the products, block by block.
                const float4* K4 = reinterpret_cast<const float4*>(d.Ke + 144 * (size_t)e + 36 * li);
                float4* X4 = reinterpret_cast<float4*>(X + 36 * lane);
#pragma unroll 3
                for (int q = 0; q < 9; ++q) X4[q] = K4[q];
#pragma unroll
                for (uint32_t j = 0; j < 4; ++j) {
                    SL[4 * lane + j] = (uint8_t)((meta >> (4 + 7 * j)) & 127u);
                    float* xb = X + 36 * lane + 9 * j;
                    // Ke(li, j): Ke(j, li) itself on the diagonal, else its transpose
                    if (j == li) stm(xb, mmul(mmul(R, ldm(xb)), RT));
                    else stm(xb, mmul(mmul(R, transpose(ldm(xb))), RT));
                }
                if (g == 0) {
                    const f3 a = ldv(d.f0s + 12 * (size_t)e, li), b = ldv(d.fps + 12 * (size_t)e, li);
                    F[6 * lane] = a.x; F[6 * lane + 1] = a.y; F[6 * lane + 2] = a.z;
                    F[6 * lane + 3] = b.x; F[6 * lane + 4] = b.y; F[6 * lane + 5] = b.z;
                }
            }
            __syncwarp();
            // every block that lands on this slot, in incidence (= element) order
            if (slot < deg)
                for (uint32_t q = 0; q < cnt; ++q)
#pragma unroll
                    for (uint32_t j = 0; j < 4; ++j)
                        if (SL[4 * q + j] == slot) acc = acc + ldm(X + 9 * (4 * q + j));
            if (g == 0 && lane == 0)
                for (uint32_t q = 0; q < cnt; ++q) {
                    f0 = f0 + mk(F[6 * q], F[6 * q + 1], F[6 * q + 2]);
                    fp = fp + mk(F[6 * q + 3], F[6 * q + 4], F[6 * q + 5]);
                }
            __syncwarp();
        }
        f3 kx = zero3();
        if (slot < deg) kx = acc * ldv(d.x, d.cols[r0 + slot]);  // this slot's K_k x_col
        for (uint32_t l = min(31u, deg - 1u - 32u * g) + 1u; l-- > 0;) {
            const f3 t = mk(__shfl_sync(0xffffffffu, kx.x, l), __shfl_sync(0xffffffffu, kx.y, l),
                            __shfl_sync(0xffffffffu, kx.z, l));
            if (lane == 0) kp = kp + t;
        }
        if (slot < deg) {
            m3 a;
            if (slot == dg) a = (M + h * diag3(cd)) + hh * acc;
            else a = mzero() + hh * acc;
            stm(vals + 9 * slot, a);
            if (d.sell_vals) {
                // the SELL copy keeps the diagonal block in slot 0, then the rest in order
                const uint32_t ri = d.sell_inv[i];
                const uint32_t ss = slot == dg ? 0u : slot < dg ? slot + 1u : slot;
                float* sv = d.sell_vals + d.sell_off[ri >> 5] + 32u * ss + (ri & 31u);
                const size_t E = d.sell_E;
                sv[0] = a.x.x, sv[E] = a.x.y, sv[2 * E] = a.x.z;
                sv[3 * E] = a.y.x, sv[4 * E] = a.y.y, sv[5 * E] = a.y.z;
                sv[6 * E] = a.z.x, sv[7 * E] = a.z.y, sv[8 * E] = a.z.z;
                if (slot == dg) {
                    st3(d.sb_pinv, d.n, ri, mk(1.0f / a.x.x, 1.0f / a.y.y, 1.0f / a.z.z));
                    st3(d.sb_diag, d.n, ri, mk(a.x.x, a.y.y, a.z.z));
                }
            }
        }
    }
    if (lane == 0) {
        const bool dyn = d.type[i] == 2;
        const f3 f0n = mk(-f0.x, -f0.y, -f0.z);
        f3 fe = ldv(d.f, i);
        if (dyn) fe = fe + m * mk(d.gx, d.gy, d.gz);
        const f3 mv = zero3() + M * ldv(d.v, i);
        const f3 bi = mv - h * ((kp + f0n) - (fp + fe));
        stv(d.b, i, bi);
        d.S[i] = dyn ? 1.0f : 0.0f;
        if (d.sell_vals) {
            const uint32_t ri = d.sell_inv[i];
            st3(d.sb_b, d.n, ri, bi);
            st3(d.sb_x0, d.n, ri, ldv(d.v, i));
            d.sb_type[ri] = d.type[i];
        }
    }
}

// b3BroadPhase::MoveProxy for node i's proxy (b3SoftBodyNode::Synchronize,
// softbody_node.cpp:22-28; broad_phase.cpp:99-149)
__device__ void node_move_proxy(const SoftDev& d, uint32_t i, f3 disp)
{
    const f3 x = ldv(d.x, i);
    const float r = d.radius[i];
    float lo[3] = {d.fat_lo[3 * i], d.fat_lo[3 * i + 1], d.fat_lo[3 * i + 2]};
    float hi[3] = {d.fat_hi[3 * i], d.fat_hi[3 * i + 1], d.fat_hi[3 * i + 2]};
    const float tlo[3] = {x.x - r, x.y - r, x.z - r}, thi[3] = {x.x + r, x.y + r, x.z + r};
    bool contains = true;
    for (int k = 0; k < 3; ++k) contains = contains && lo[k] <= tlo[k] && tlo[k] <= hi[k] && lo[k] <= thi[k] && thi[k] <= hi[k];
    if (contains) return;
    const float dd[3] = {2.0f * disp.x, 2.0f * disp.y, 2.0f * disp.z};
    for (int k = 0; k < 3; ++k) {
        lo[k] = tlo[k] - 0.2f;
        hi[k] = thi[k] + 0.2f;
        if (dd[k] < 0.0f) lo[k] += dd[k];
        else hi[k] += dd[k];
        d.fat_lo[3 * i + k] = lo[k];
        d.fat_hi[3 * i + k] = hi[k];
    }
}

__device__ __forceinline__ bool node_overlap(const SoftDev& d, uint32_t i, const SphereDev& s)
{
    return d.fat_lo[3 * i] <= s.hi[0] && d.fat_lo[3 * i + 1] <= s.hi[1] && d.fat_lo[3 * i + 2] <= s.hi[2] &&
           d.fat_hi[3 * i] >= s.lo[0] && d.fat_hi[3 * i + 1] >= s.lo[1] && d.fat_hi[3 * i + 2] >= s.lo[2];
}

__device__ __forceinline__ int sb_enc(float f)
{
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float sb_dec(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// Without hulls: v = solution, x += h v, forces cleared, node proxies moved
// (softbody_solver.cpp:105-110, softbody.cpp:716-775)
__global__ void k_sb_integrate(SoftDev d, float h)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const f3 v = ldv(d.xsol, i);
    stv(d.v, i, v);
    stv(d.x, i, ldv(d.x, i) + h * v);
    stv(d.f, i, zero3());
    if (d.type[i] != 0) node_move_proxy(d, i, h * v);
}

// UpdateBodyContacts (softbody_contact_manager.cpp:109-150) with
// b3NodeBodyContact::Update and b3HullShape::TestSphere
__global__ void k_sb_contacts_update(SoftDev d)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const uint32_t n = d.n, nn = (uint32_t)kMaxSpheres * n;  // slot planes laid out for the hull capacity
    const f3 xi = ldv(d.x, i);
    for (uint32_t s = 0; s < d.nhull; ++s) {
        const uint32_t q = s * n + i;
        if (!d.c_exists[q]) continue;
        const SphereDev& sp = d.hull[s];
        if (d.type[i] != 2 || !node_overlap(d, i, sp)) {
            d.c_exists[q] = 0;
            d.c_active[q] = 0;
            continue;
        }
        f3 normal, P;
        if (!hull::test_sphere(sp.hull, sp.nhv, sp.hull + 3 * sp.nhv, sp.nhf, sp.radius + d.radius[i], mident(), zero3(),
                               xi, normal, P)) {
            d.c_active[q] = 0;
            continue;
        }
        const f3 n1 = mk(-normal.x, -normal.y, -normal.z);
        const f3 t1 = perp(n1);
        const f3 t2 = cross(t1, n1);
        d.c_active[q] = 1;
        st3(d.c_normal, nn, q, n1);
        st3(d.c_t1, nn, q, t1);
        st3(d.c_t2, nn, q, t2);
        st3(d.c_point, nn, q, hull::xf_mult(P));
    }
}

// Node i's active contacts in list order (newest first).
__device__ int sb_contact_order(const SoftDev& d, uint32_t i, int* order)
{
    int k = 0;
    const uint32_t n = d.n;
    for (uint32_t s = 0; s < d.nhull; ++s)
        if (d.c_exists[s * n + i] && d.c_active[s * n + i]) order[k++] = (int)s;
    for (int a = 1; a < k; ++a) {
        const int v = order[a];
        int b = a - 1;
        while (b >= 0 && d.c_key[order[b] * n + i] < d.c_key[v * n + i]) {
            order[b + 1] = order[b];
            --b;
        }
        order[b + 1] = v;
    }
    return k;
}

// One position iteration for node i (softbody_contact_solver.cpp:330-410);
// returns its smallest separation.
__device__ float sb_position_iteration(const SoftDev& d, uint32_t i, f3& pos, const int* order, int k, float mA)
{
    const uint32_t n = d.n, nn = (uint32_t)kMaxSpheres * n;  // slot planes laid out for the hull capacity
    float min_sep = 0.0f;
    for (int a = 0; a < k; ++a) {
        const uint32_t q = order[a] * n + i;
        const f3 nA = ld3(d.c_normal, nn, q);
        const f3 cB = ld3(d.c_point, nn, q);
        const float separation = dot(cB - pos, nA) - d.radius[i] - d.hull[order[a]].radius;
        min_sep = min_sep < separation ? min_sep : separation;
        const float Cv = 0.1f * (separation + 0.005f);
        float C = Cv < 0.0f ? Cv : 0.0f;
        C = -0.2f > C ? -0.2f : C;
        const float K = mA + 0.0f + 0.0f + 0.0f;
        const float impulse = K > 0.0f ? -C / K : 0.0f;
        pos = pos - mA * (impulse * nA);
    }
    return min_sep;
}

// With hulls: v = solution, then the contact solve of b3SoftBodySolver::Solve
// (softbody_solver.cpp:62-126) for node i -- warm start, velocity
// iterations, impulses stored, x += h v, first position iteration.  Contacts
// of different nodes are independent (static shapes), so each node runs its
// own sweep in list order.
__global__ void k_sb_contact_solve(SoftDev d, float h)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const uint32_t n = d.n, nn = (uint32_t)kMaxSpheres * n;  // slot planes laid out for the hull capacity
    f3 vel = ldv(d.xsol, i);
    int order[kMaxSpheres];
    const int k = sb_contact_order(d, i, order);
    const float mA = d.type[i] == 0 ? 0.0f : 1.0f / d.mass[i];
    if (k > 0) {
        atomicAdd(d.active_count, (uint32_t)k);
        for (int a = 0; a < k; ++a) {  // WarmStart
            const uint32_t q = order[a] * n + i;
            const f3 P = d.c_imp[q] * ld3(d.c_normal, nn, q);
            vel = vel - mA * P;
            const f3 P1 = d.c_imp[nn + q] * ld3(d.c_t1, nn, q), P2 = d.c_imp[2 * nn + q] * ld3(d.c_t2, nn, q);
            vel = vel - mA * (P1 + P2);
        }
        for (uint32_t it = 0; it < d.vel_iters; ++it)
            for (int a = 0; a < k; ++a) {
                const uint32_t q = order[a] * n + i;
                const float K = mA + 0.0f + 0.0f + 0.0f;
                const float nmass = K > 0.0f ? 1.0f / K : 0.0f;
                const float k11 = mA + 0.0f + 0.0f + 0.0f, k12 = 0.0f + 0.0f, k22 = mA + 0.0f + 0.0f + 0.0f;
                float det = k11 * k22 - k12 * k12;
                if (det != 0.0f) det = 1.0f / det;
                const float tm_xx = det * k22, tm_yx = -det * k12, tm_xy = -det * k12, tm_yy = det * k11;
                const float fr = sqrtf(d.friction[i] * d.hull[order[a]].friction);
                const f3 nrm = ld3(d.c_normal, nn, q), t1 = ld3(d.c_t1, nn, q), t2 = ld3(d.c_t2, nn, q);
                float ni = d.c_imp[q], tix = d.c_imp[nn + q], tiy = d.c_imp[2 * nn + q];
                {
                    const f3 dvv = zero3() - vel;
                    const float Cdot = dot(nrm, dvv);
                    float impulse = nmass * (-Cdot + 0.0f);
                    const float old = ni;
                    const float sum = old + impulse;
                    ni = sum > 0.0f ? sum : 0.0f;
                    impulse = ni - old;
                    vel = vel - mA * (impulse * nrm);
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
                        if (sl > 1.1920929e-7f) {
                            tix /= sl;
                            tiy /= sl;
                        }
                        tix *= maxImpulse;
                        tiy *= maxImpulse;
                    }
                    const float jx = tix - ox, jy = tiy - oy;
                    vel = vel - mA * (jx * t1 + jy * t2);
                }
                d.c_imp[q] = ni;
                d.c_imp[nn + q] = tix;
                d.c_imp[2 * nn + q] = tiy;
            }
    }
    f3 pos = ldv(d.x, i) + h * vel;
    if (k > 0 && d.pos_iters > 0) {
        const float ms = sb_position_iteration(d, i, pos, order, k, mA);
        if (ms < 0.0f) atomicMin(&d.min_sep[0], sb_enc(ms));
    }
    stv(d.v, i, vel);
    stv(d.x, i, pos);
}

// Position iteration `it` >= 1, run while the previous one left a
// separation below -3 slops (softbody_solver.cpp:114-126).
__global__ void k_sb_contact_position(SoftDev d, uint32_t it)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n || sb_dec(d.min_sep[it - 1]) >= -3.0f * 0.005f) return;
    int order[kMaxSpheres];
    const int k = sb_contact_order(d, i, order);
    if (k == 0) return;
    const float mA = d.type[i] == 0 ? 0.0f : 1.0f / d.mass[i];
    f3 pos = ldv(d.x, i);
    const float ms = sb_position_iteration(d, i, pos, order, k, mA);
    stv(d.x, i, pos);
    if (ms < 0.0f) atomicMin(&d.min_sep[it], sb_enc(ms));
}

// Forces cleared, node proxies moved, new contacts (softbody.cpp:757-778,
// FindNewBodyContacts and AddNSPair, softbody_contact_manager.cpp:44-107)
__global__ void k_sb_post(SoftDev d, float h)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const uint32_t n = d.n, nn = (uint32_t)kMaxSpheres * n;  // slot planes laid out for the hull capacity
    stv(d.f, i, zero3());
    if (d.type[i] != 0) node_move_proxy(d, i, h * ldv(d.v, i));
    if (d.type[i] != 2) return;
    for (uint32_t s = 0; s < d.nhull; ++s) {
        const uint32_t q = s * n + i;
        if (d.c_exists[q] || !node_overlap(d, i, d.hull[s])) continue;
        d.c_exists[q] = 1;
        d.c_active[q] = 0;
        d.c_key[q] = d.step_index * kMaxSpheres + d.hull[s].rank;
        d.c_imp[q] = 0.0f;
        d.c_imp[nn + q] = 0.0f;
        d.c_imp[2 * nn + q] = 0.0f;
    }
}

__global__ void k_sb_init_proxies(SoftDev d)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const f3 x = ldv(d.x, i);
    // aabb.Set(position, 0) fattened by B3_AABB_EXTENSION (softbody.cpp:477-480)
    d.fat_lo[3 * i] = (x.x - 0.0f) - 0.2f;
    d.fat_lo[3 * i + 1] = (x.y - 0.0f) - 0.2f;
    d.fat_lo[3 * i + 2] = (x.z - 0.0f) - 0.2f;
    d.fat_hi[3 * i] = (x.x + 0.0f) + 0.2f;
    d.fat_hi[3 * i + 1] = (x.y + 0.0f) + 0.2f;
    d.fat_hi[3 * i + 2] = (x.z + 0.0f) + 0.2f;
    d.radius[i] = 0.0f;
    d.friction[i] = 0.0f;
}

// Edits of one node, in stream order with the steps: 0 type, 1 mass damping,
// 2 force +=, 3 velocity (ignored on static nodes), 4 position.
__global__ void k_sb_node_op(SoftDev d, uint32_t i, int op, float a, float b, float c)
{
    if (op == 0) {
        const uint8_t t = (uint8_t)a;
        if (d.type[i] == t) return;
        d.type[i] = t;
        stv(d.f, i, zero3());
        if (t == 0) {
            stv(d.v, i, zero3());
            node_move_proxy(d, i, zero3());
        }
        for (uint32_t s = 0; s < d.nhull; ++s) {  // DestroyContacts
            d.c_exists[s * d.n + i] = 0;
            d.c_active[s * d.n + i] = 0;
        }
    } else if (op == 5) {  // SetRadius
        d.radius[i] = a;
        node_move_proxy(d, i, zero3());
    } else if (op == 6) {  // SetFriction
        d.friction[i] = a;
    } else if (op == 1) {
        d.damping[i] = a;
    } else if (op == 2) {
        stv(d.f, i, ldv(d.f, i) + mk(a, b, c));
    } else if (op == 3) {
        if (d.type[i] != 0) stv(d.v, i, mk(a, b, c));
    } else {
        const f3 p = mk(a, b, c);
        const f3 disp = p - ldv(d.x, i);
        stv(d.x, i, p);
        node_move_proxy(d, i, disp);
    }
}

constexpr uint32_t kBlock = 256;
inline uint32_t blocks_for(uint32_t n) { return (n + kBlock - 1) / kBlock; }

// The solution's planes, in row order, back to xyz per node, where the
// integration and the contact solve read it.
__global__ void k_sb_from_planes(const float* dv, const uint32_t* inv, float* xsol, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        stv(xsol, i, ld3(dv, n, inv[i]));
}

}  // namespace

}  // namespace b3g

using namespace b3g;

struct b3g_softbody {
    int device = 0;
    cudaStream_t stream = nullptr;
    char* arena = nullptr;
    SoftDev dev{};
    CsrSystem cs{};
    b3g_solver_opts opts{B3G_STOP_REFERENCE, 0.0f, 20, B3G_DOT_F32};
    uint32_t tets_count = 0;
    std::vector<uint32_t> rowptr, cols, diag;  // host copies for the export
    std::vector<float> mass;
    b3g_step_stats last{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void* cbuf = nullptr;                 // node radius, friction, proxies, position-iteration words
    void* slots = nullptr;                // contact slots for kMaxSpheres hulls
    std::vector<void*> hull_bufs;         // device copies of the hulls' vertices and planes
    bool persistent = true;               // the MPCG as one persistent launch (else three launches per iteration)
    void* pcg = nullptr;                  // its SELL copy of the system, vectors, partials and grid barrier
    b3g::ClothDev view{};                 // the system as the persistent CG sees it
    b3g::GridBarrier* bar = nullptr;
    float4* rec = nullptr;                // the fused form's per-row records
    bool fused = false;                   // one grid reduction per CG iteration
};

namespace {

b3g_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return B3G_OK;
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? B3G_ERR_OUT_OF_MEMORY : B3G_ERR_CUDA;
}
#define SB_TRY(expr)                                      \
    do {                                                  \
        b3g_status s_ = cuda_status(expr);                \
        if (s_ != B3G_OK) return s_;                      \
    } while (0)

bool ok(const b3g_softbody* b) { return b && b->dev.n > 0; }

// The soft body's system in the cloth's SELL-32 layout, for the persistent
// CG: the pattern built from the row lists on the host once, the buffers
// (values, the solve's vectors as planes, partials, grid barrier) made on
// first use.  The assembly then writes the values there as well.
b3g_status ensure_sell(b3g_softbody* b)
{
    if (b->pcg) return B3G_OK;
    const uint32_t n = b->dev.n;
    const uint32_t nslices = (n + 31) / 32;
    // rows by degree, widest first, node order within a degree
    std::vector<uint32_t> perm(n), inv(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    auto degree = [&](uint32_t i) { return b->rowptr[i + 1] - b->rowptr[i]; };
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t x, uint32_t y) { return degree(x) > degree(y); });
    for (uint32_t r = 0; r < n; ++r) inv[perm[r]] = r;
    std::vector<uint32_t> off(nslices + 1, 0);
    std::vector<uint8_t> deg(n);
    uint32_t max_deg = 0;
    for (uint32_t q = 0; q < nslices; ++q) {
        uint32_t w = 0;
        for (uint32_t r = 32 * q; r < std::min(n, 32 * q + 32); ++r) {
            const uint32_t d = degree(perm[r]);
            deg[r] = (uint8_t)d;
            w = std::max(w, d);
        }
        max_deg = std::max(max_deg, w);
        off[q + 1] = off[q] + 32 * w;
    }
    const uint32_t E = off[nslices];
    std::vector<uint32_t> cols(E);
    for (uint32_t r = 0; r < n; ++r) {
        const uint32_t i = perm[r];
        const uint32_t width = (off[r / 32 + 1] - off[r / 32]) / 32;  // the slice's widest row
        const uint32_t dg = b->diag[i] - b->rowptr[i];
        for (uint32_t k = 0; k < width; ++k) cols[off[r / 32] + 32 * k + (r & 31)] = r;  // padding
        for (uint32_t k = 0; k < deg[r]; ++k) {
            const uint32_t ss = k == dg ? 0u : k < dg ? k + 1u : k;  // the diagonal block first
            cols[off[r / 32] + 32 * ss + (r & 31)] = inv[b->cols[b->rowptr[i] + k]];
        }
    }
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t plane = al(3 * (size_t)n * sizeof(float));
    const size_t bytes = al((nslices + 1) * 4) + al(n) + al((size_t)E * 4) + al((size_t)E * 36) + 10 * plane +
                         al(kGridCgPartialBytes) + al(sizeof(GridBarrier)) + al((size_t)n * 4) + al(n) +
                         al(grid_cg_fused_rec_bytes(n));
    SB_TRY(cudaMalloc(&b->pcg, bytes));
    char* q = static_cast<char*>(b->pcg);
    auto take = [&](size_t x) {
        char* r = q;
        q += al(x);
        return r;
    };
    uint32_t* d_off = (uint32_t*)take((nslices + 1) * 4);
    uint8_t* d_deg = (uint8_t*)take(n);
    uint32_t* d_cols = (uint32_t*)take((size_t)E * 4);
    float* d_vals = (float*)take((size_t)E * 36);
    float* planes[10];
    for (float*& f : planes) f = (float*)take(3 * (size_t)n * sizeof(float));
    void* partials = take(kGridCgPartialBytes);
    GridBarrier* bar = (GridBarrier*)take(sizeof(GridBarrier));
    uint32_t* d_inv = (uint32_t*)take((size_t)n * 4);
    uint8_t* d_type = (uint8_t*)take(n);
    b->rec = (float4*)take(grid_cg_fused_rec_bytes(n));
    cudaStream_t s = b->stream;
    SB_TRY(cudaMemcpyAsync(d_inv, inv.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
    SB_TRY(cudaMemcpyAsync(d_off, off.data(), (nslices + 1) * 4, cudaMemcpyHostToDevice, s));
    SB_TRY(cudaMemcpyAsync(d_deg, deg.data(), n, cudaMemcpyHostToDevice, s));
    SB_TRY(cudaMemcpyAsync(d_cols, cols.data(), (size_t)E * 4, cudaMemcpyHostToDevice, s));
    SB_TRY(cudaMemsetAsync(d_vals, 0, (size_t)E * 36, s));
    SB_TRY(cudaStreamSynchronize(s));  // the host vectors go out of scope
    SoftDev& d = b->dev;
    d.sell_vals = d_vals;
    d.sell_off = d_off;
    d.sell_inv = d_inv;
    d.sb_type = d_type;
    d.sell_E = E;
    d.sb_b = planes[0];
    d.sb_x0 = planes[1];
    d.sb_pinv = planes[2];
    d.sb_diag = planes[3];
    ClothDev& v = b->view;
    v = ClothDev{};
    v.n = n;
    v.nslices = nslices;
    v.max_deg = max_deg;
    v.E = E;
    v.slice_off = d_off;
    v.row_deg = d_deg;
    v.cols = d_cols;
    v.vals = d_vals;
    v.b = planes[0];
    v.mx = planes[1];
    v.pinv = planes[2];
    v.cg_diag = planes[3];
    v.dv = planes[4];
    v.r = planes[5];
    v.p = planes[6];
    v.p2 = planes[7];
    v.s = planes[8];
    v.z = planes[9];
    v.type = d_type;
    v.sc = b->cs.sc;
    v.partials = partials;
    v.cg_soft = 1;
    b->bar = bar;
    return B3G_OK;
}

// The soft body's MPCG (softbody_force_solver.cpp:93-164) as the cloth's
// persistent cooperative CG in its soft body mode, on the SELL copy of the
// system the assembly just wrote.
b3g_status persistent_cg(b3g_softbody* b, cudaStream_t s, StepScalars* h)
{
    const ClothDev& v = b->view;
    StepScalars init;
    std::memset(&init, 0, sizeof(init));
    init.max_iter = b->opts.max_iterations;
    init.stop_rule = (int)b->opts.stop_rule;
    init.tol = b->opts.tolerance;
    init.dot = (int)b->opts.dot;
    SB_TRY(cudaMemcpyAsync(v.sc, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    SB_TRY(cudaMemsetAsync(b->bar, 0, sizeof(GridBarrier), s));
    SB_TRY(b->fused ? launch_grid_cg_fused(v, (int)b->opts.dot, b->bar, b->rec, s)
                    : launch_grid_cg(v, (int)b->opts.dot, b->bar, s));
    k_sb_from_planes<<<blocks_for(v.n), kBlock, 0, s>>>(v.dv, b->dev.sell_inv, b->cs.x, v.n);
    count_launches(1);
    SB_TRY(cudaGetLastError());
    SB_TRY(cudaMemcpyAsync(h, v.sc, sizeof(StepScalars), cudaMemcpyDeviceToHost, s));
    SB_TRY(cudaStreamSynchronize(s));
    return B3G_OK;
}

b3g_status node_op(b3g_softbody* b, uint32_t i, int op, float x, float y, float z)
{
    if (!ok(b) || i >= b->dev.n) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    k_sb_node_op<<<1, 1, 0, b->stream>>>(b->dev, i, op, x, y, z);
    count_launches(1);
    SB_TRY(cudaGetLastError());
    return B3G_OK;
}

}  // namespace

extern "C" {

b3g_status b3g_softbody_create(uint32_t vertex_count, const float* vertices, uint32_t tet_count,
                               const uint32_t* tets, const b3g_softbody_def* def, int device, b3g_softbody** out)
{
    if (!out || !vertices || !tets || !def || vertex_count == 0 || tet_count == 0) return B3G_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!(def->density > 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return B3G_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return B3G_ERR_INVALID_ARGUMENT;
    SoftBodyPrep P;
    const int st = prepare_softbody(vertex_count, vertices, tet_count, tets, def->density, def->E, def->nu, &P);
    if (st != 0) return (b3g_status)st;
    b3g_softbody* b = new (std::nothrow) b3g_softbody();
    if (!b) return B3G_ERR_OUT_OF_MEMORY;
    b->device = device;
    cudaSetDevice(device);
    const uint32_t n = vertex_count, t = tet_count, nnz = (uint32_t)P.cols.size();
    const size_t vec = 3 * (size_t)n * sizeof(float);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const uint32_t grid = csr_grid(n);
    size_t bytes = 0;
    const size_t sizes[] = {vec,       vec,       vec,       vec,          (size_t)n * 4, (size_t)n * 4, (size_t)n,
                            (size_t)t * 16, (size_t)t * 576, (size_t)t * 36, (size_t)t * 288, (size_t)t * 288,
                            (size_t)t * 16, (size_t)t * 24, (size_t)t * 36, (size_t)t * 48, (size_t)t * 48,
                            (size_t)(n + 1) * 4, (size_t)nnz * 4, (size_t)n * 4, (size_t)nnz * 36,
                            (size_t)(n + 1) * 4, (size_t)t * 16, (size_t)t * 16, vec, (size_t)n * 4, vec,
                            csr_scratch_bytes(n, grid)};
    for (size_t s : sizes) bytes += al(s);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->arena, bytes);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b3g_softbody_destroy(b);
        return e == cudaErrorMemoryAllocation ? B3G_ERR_OUT_OF_MEMORY : B3G_ERR_CUDA;
    }
    char* p = b->arena;
    auto take = [&](size_t s) {
        char* r = p;
        p += al(s);
        return r;
    };
    SoftDev& d = b->dev;
    d.n = n;
    d.t = t;
    d.nnz = nnz;
    float* rest = (float*)take(vec);
    d.rest = rest;
    d.x = (float*)take(vec);
    d.v = (float*)take(vec);
    d.f = (float*)take(vec);
    float* mass = (float*)take((size_t)n * 4);
    d.mass = mass;
    d.damping = (float*)take((size_t)n * 4);
    d.type = (uint8_t*)take(n);
    uint4* tv = (uint4*)take((size_t)t * 16);
    d.tets = tv;
    float* Ke = (float*)take((size_t)t * 576);
    d.Ke = Ke;
    float* invE = (float*)take((size_t)t * 36);
    d.invE = invE;
    float* Bm = (float*)take((size_t)t * 288);
    d.B = Bm;
    float* Pm = (float*)take((size_t)t * 288);
    d.P = Pm;
    d.q = (float4*)take((size_t)t * 16);
    d.eps = (float*)take((size_t)t * 24);
    d.R = (float*)take((size_t)t * 36);
    d.f0s = (float*)take((size_t)t * 48);
    d.fps = (float*)take((size_t)t * 48);
    uint32_t* rowptr = (uint32_t*)take((size_t)(n + 1) * 4);
    d.rowptr = rowptr;
    uint32_t* cols = (uint32_t*)take((size_t)nnz * 4);
    d.cols = cols;
    uint32_t* dg = (uint32_t*)take((size_t)n * 4);
    d.diag = dg;
    d.vals = (float*)take((size_t)nnz * 36);
    uint32_t* inc_ptr = (uint32_t*)take((size_t)(n + 1) * 4);
    d.inc_ptr = inc_ptr;
    uint32_t* inc_elem = (uint32_t*)take((size_t)t * 16);
    d.inc_elem = inc_elem;
    uint32_t* inc_meta = (uint32_t*)take((size_t)t * 16);
    d.inc_meta = inc_meta;
    d.b = (float*)take(vec);
    d.S = (float*)take((size_t)n * 4);
    d.xsol = (float*)take(vec);
    char* scratch = take(csr_scratch_bytes(n, grid));
    d.c_yield = def->c_yield;
    d.c_creep = def->c_creep;
    d.c_max = def->c_max;
    // uploads
    std::vector<uint4> tets4(t);
    for (uint32_t k = 0; k < t; ++k) tets4[k] = make_uint4(tets[4 * k], tets[4 * k + 1], tets[4 * k + 2], tets[4 * k + 3]);
    std::vector<float4> q0(t, make_float4(0.0f, 0.0f, 0.0f, 1.0f));  // the rest state's rotation
    std::vector<uint8_t> types(n, 2);
    cudaStream_t s = b->stream;
    struct Up {
        void* dst;
        const void* src;
        size_t bytes;
    } ups[] = {{rest, vertices, vec}, {d.x, vertices, vec}, {mass, P.mass.data(), (size_t)n * 4},
               {tv, tets4.data(), (size_t)t * 16}, {Ke, P.Ke.data(), (size_t)t * 576},
               {invE, P.invE.data(), (size_t)t * 36}, {Bm, P.B.data(), (size_t)t * 288},
               {Pm, P.P.data(), (size_t)t * 288}, {d.q, q0.data(), (size_t)t * 16},
               {rowptr, P.rowptr.data(), (size_t)(n + 1) * 4}, {cols, P.cols.data(), (size_t)nnz * 4},
               {dg, P.diag.data(), (size_t)n * 4}, {inc_ptr, P.inc_ptr.data(), (size_t)(n + 1) * 4},
               {inc_elem, P.inc_elem.data(), (size_t)t * 16}, {inc_meta, P.inc_meta.data(), (size_t)t * 16},
               {d.type, types.data(), (size_t)n}};
    for (const Up& u : ups)
        if (e == cudaSuccess) e = cudaMemcpyAsync(u.dst, u.src, u.bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.v, 0, vec, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.f, 0, vec, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.damping, 0, (size_t)n * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.eps, 0, (size_t)t * 24, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host vectors above go out of scope
    if (e != cudaSuccess) {
        cudaGetLastError();
        b3g_softbody_destroy(b);
        return B3G_ERR_CUDA;
    }
    CsrSystem& c = b->cs;
    c.n = n;
    c.rowptr = rowptr;
    c.cols = cols;
    c.vals = d.vals;
    c.b = d.b;
    c.S = d.S;
    c.x0 = d.v;
    c.x = d.xsol;
    c.block = 256;
    c.grid = grid;
    c.softbody_mode = 1;
    csr_bind_scratch(&c, scratch);
    b->tets_count = t;
    b->rowptr = P.rowptr;
    b->cols = P.cols;
    b->diag = P.diag;
    b->mass = P.mass;
    // node proxies from creation on, with radius and friction 0
    // (softbody.cpp:462-481)
    {
        const size_t words = 8 * (size_t)n + kMaxPosIters + 4;
        cudaError_t ce = cudaMalloc(&b->cbuf, words * sizeof(float));
        if (ce != cudaSuccess) {
            cudaGetLastError();
            b3g_softbody_destroy(b);
            return ce == cudaErrorMemoryAllocation ? B3G_ERR_OUT_OF_MEMORY : B3G_ERR_CUDA;
        }
        float* f = static_cast<float*>(b->cbuf);
        d.radius = f;
        d.friction = f + n;
        d.fat_lo = f + 2 * (size_t)n;
        d.fat_hi = f + 5 * (size_t)n;
        d.min_sep = reinterpret_cast<int*>(f + 8 * (size_t)n);
        d.active_count = reinterpret_cast<uint32_t*>(f + 8 * (size_t)n + kMaxPosIters);
        k_sb_init_proxies<<<blocks_for(n), kBlock, 0, b->stream>>>(d);
        count_launches(1);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(b->stream) != cudaSuccess) {
            b3g_softbody_destroy(b);
            return B3G_ERR_CUDA;
        }
    }
    *out = b;
    return B3G_OK;
}

b3g_status b3g_softbody_destroy(b3g_softbody* b)
{
    if (!b) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->arena) cudaFree(b->arena);
    if (b->cbuf) cudaFree(b->cbuf);
    if (b->slots) cudaFree(b->slots);
    if (b->pcg) cudaFree(b->pcg);
    for (void* p : b->hull_bufs) cudaFree(p);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return B3G_OK;
}

b3g_status b3g_softbody_set_cg_strategy(b3g_softbody* b, b3g_cg_strategy strategy)
{
    if (!ok(b) || (strategy != B3G_CG_LAUNCHES && strategy != B3G_CG_PERSISTENT &&
                   strategy != B3G_CG_PERSISTENT_FUSED))
        return B3G_ERR_INVALID_ARGUMENT;
    b->persistent = strategy != B3G_CG_LAUNCHES;
    b->fused = strategy == B3G_CG_PERSISTENT_FUSED;
    return B3G_OK;
}

uint32_t b3g_softbody_node_count(const b3g_softbody* b) { return ok(b) ? b->dev.n : 0u; }
uint32_t b3g_softbody_element_count(const b3g_softbody* b) { return ok(b) ? b->dev.t : 0u; }

b3g_status b3g_softbody_set_gravity(b3g_softbody* b, const float* g)
{
    if (!ok(b) || !g) return B3G_ERR_INVALID_ARGUMENT;
    b->dev.gx = g[0];
    b->dev.gy = g[1];
    b->dev.gz = g[2];
    return B3G_OK;
}

b3g_status b3g_softbody_set_node_type(b3g_softbody* b, uint32_t i, int type)
{
    if (type < 0 || type > 2) return B3G_ERR_INVALID_ARGUMENT;
    return node_op(b, i, 0, (float)type, 0.0f, 0.0f);
}

b3g_status b3g_softbody_set_mass_damping(b3g_softbody* b, uint32_t i, float damping)
{
    return node_op(b, i, 1, damping, 0.0f, 0.0f);
}

b3g_status b3g_softbody_apply_force(b3g_softbody* b, uint32_t i, const float* f)
{
    if (!f) return B3G_ERR_INVALID_ARGUMENT;
    return node_op(b, i, 2, f[0], f[1], f[2]);
}

b3g_status b3g_softbody_set_velocity(b3g_softbody* b, uint32_t i, const float* v)
{
    if (!v) return B3G_ERR_INVALID_ARGUMENT;
    return node_op(b, i, 3, v[0], v[1], v[2]);
}

b3g_status b3g_softbody_set_position(b3g_softbody* b, uint32_t i, const float* x)
{
    if (!x) return B3G_ERR_INVALID_ARGUMENT;
    return node_op(b, i, 4, x[0], x[1], x[2]);
}

b3g_status b3g_softbody_set_solver(b3g_softbody* b, const b3g_solver_opts* o)
{
    if (!ok(b) || !o || o->max_iterations < 1 ||
        (o->stop_rule != B3G_STOP_REFERENCE && o->stop_rule != B3G_STOP_RELATIVE) ||
        (o->dot != B3G_DOT_F32 && o->dot != B3G_DOT_COMPENSATED && o->dot != B3G_DOT_F64))
        return B3G_ERR_INVALID_ARGUMENT;
    b->opts = *o;
    return B3G_OK;
}

b3g_status b3g_softbody_step(b3g_softbody* b, float dt, uint32_t velocity_iterations, uint32_t position_iterations,
                             b3g_step_stats* stats)
{
    if (!ok(b) || !(dt >= 0.0f) || position_iterations > (uint32_t)kMaxPosIters) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    cudaStream_t s = b->stream;
    SoftDev& d = b->dev;
    d.vel_iters = velocity_iterations;
    d.pos_iters = position_iterations;
    d.step_index += 1;
    if (d.nhull) {
        // UpdateBodyContacts (softbody.cpp:752)
        SB_TRY(cudaMemsetAsync(d.min_sep, 0, (kMaxPosIters + 4) * sizeof(int), s));
        k_sb_contacts_update<<<blocks_for(d.n), kBlock, 0, s>>>(d);
        count_launches(1);
    }
    std::memset(&b->last, 0, sizeof(b->last));
    SB_TRY(cudaEventRecord(b->ev0, s));
    StepScalars h;
    std::memset(&h, 0, sizeof(h));
    if (dt > 0.0f) {
        if (b->persistent) {
            const b3g_status es = ensure_sell(b);
            if (es != B3G_OK) return es;
        }
        k_sb_elements<<<blocks_for(d.t), kBlock, 0, s>>>(d, dt, 1.0f / dt);
        k_sb_assemble<<<(d.n + kAsmWarps - 1) / kAsmWarps, 32 * kAsmWarps, 0, s>>>(d, dt);
        count_launches(2);
        SB_TRY(cudaGetLastError());
        const b3g_status r = b->persistent ? persistent_cg(b, s, &h) : csr_run(b->cs, &b->opts, s, &h);
        if (r != B3G_OK) return r;
        if (d.nhull) {
            k_sb_contact_solve<<<blocks_for(d.n), kBlock, 0, s>>>(d, dt);
            for (uint32_t it = 1; it < position_iterations && it < (uint32_t)kMaxPosIters; ++it)
                k_sb_contact_position<<<blocks_for(d.n), kBlock, 0, s>>>(d, it);
            k_sb_post<<<blocks_for(d.n), kBlock, 0, s>>>(d, dt);
            const uint32_t extra = position_iterations > 1 ? std::min<uint32_t>(position_iterations, kMaxPosIters) - 1 : 0;
            count_launches(2 + extra);
        } else {
            k_sb_integrate<<<blocks_for(d.n), kBlock, 0, s>>>(d, dt);
            count_launches(1);
        }
    } else {
        // no solve: forces cleared, proxies moved by no displacement, new contacts
        k_sb_post<<<blocks_for(d.n), kBlock, 0, s>>>(d, 0.0f);
        count_launches(1);
    }
    SB_TRY(cudaGetLastError());
    SB_TRY(cudaEventRecord(b->ev1, s));
    SB_TRY(cudaStreamSynchronize(s));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    csr_report(h, nullptr, &b->last);
    b->last.step_ms = ms;
    if (d.nhull) {
        uint32_t active = 0;
        SB_TRY(cudaMemcpy(&active, d.active_count, sizeof(active), cudaMemcpyDeviceToHost));
        b->last.active_contacts = active;
    }
    if (stats) *stats = b->last;
    return h.status ? (b3g_status)h.status : B3G_OK;
}

static b3g_status copy_nodes(b3g_softbody* b, float* dst, const float* src, size_t bytes, cudaMemcpyKind kind)
{
    SB_TRY(cudaMemcpyAsync(dst, src, bytes, kind, b->stream));
    SB_TRY(cudaStreamSynchronize(b->stream));
    return B3G_OK;
}

b3g_status b3g_softbody_set_node_radius(b3g_softbody* b, uint32_t node, float radius)
{
    if (!(radius >= 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    return node_op(b, node, 5, radius, 0.0f, 0.0f);
}

b3g_status b3g_softbody_set_node_friction(b3g_softbody* b, uint32_t node, float friction)
{
    if (!(friction >= 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    return node_op(b, node, 6, friction, 0.0f, 0.0f);
}

b3g_status b3g_softbody_add_static_hull(b3g_softbody* b, const float* vertices, uint32_t vertex_count,
                                        const float* planes, uint32_t face_count, float friction, uint32_t* shape_id)
{
    if (!ok(b) || !vertices || !planes || vertex_count == 0 || face_count == 0 || vertex_count > 4096 ||
        face_count > 4096 || !(friction >= 0.0f))
        return B3G_ERR_INVALID_ARGUMENT;
    SoftDev& d = b->dev;
    if (d.nhull >= (uint32_t)kMaxSpheres) return B3G_ERR_CAPACITY;
    cudaSetDevice(b->device);
    const uint32_t n = d.n;
    if (!b->slots) {
        // contact slots for every hull the body can take, zeroed
        const size_t nn = (size_t)kMaxSpheres * n;
        const size_t bytes = 2 * nn + 4 * nn + 15 * nn * sizeof(float);
        SB_TRY(cudaMalloc(&b->slots, bytes));
        SB_TRY(cudaMemsetAsync(b->slots, 0, bytes, b->stream));
    }
    const size_t nf = 3 * (size_t)vertex_count + 4 * (size_t)face_count;
    std::vector<float> img(nf);
    std::memcpy(img.data(), vertices, 3 * (size_t)vertex_count * sizeof(float));
    std::memcpy(img.data() + 3 * (size_t)vertex_count, planes, 4 * (size_t)face_count * sizeof(float));
    float* hd = nullptr;
    SB_TRY(cudaMalloc(&hd, nf * sizeof(float)));
    b->hull_bufs.push_back(hd);
    SB_TRY(cudaMemcpyAsync(hd, img.data(), nf * sizeof(float), cudaMemcpyHostToDevice, b->stream));
    SB_TRY(cudaStreamSynchronize(b->stream));
    SphereDev& h = d.hull[d.nhull];
    h = SphereDev{};
    h.kind = 2;
    h.radius = 0.0f;  // B3_HULL_RADIUS
    h.friction = friction;
    h.hull = hd;
    h.nhv = vertex_count;
    h.nhf = face_count;
    // b3HullShape::ComputeAABB with the identity at the origin, fattened
    float lo[3], hi[3];
    for (uint32_t k = 0; k < vertex_count; ++k) {
        const float* v = vertices + 3 * k;
        const float w[3] = {((v[0] * 1.0f + v[1] * 0.0f) + v[2] * 0.0f) + 0.0f,
                            ((v[0] * 0.0f + v[1] * 1.0f) + v[2] * 0.0f) + 0.0f,
                            ((v[0] * 0.0f + v[1] * 0.0f) + v[2] * 1.0f) + 0.0f};
        for (int q = 0; q < 3; ++q) {
            lo[q] = k == 0 ? w[q] : (lo[q] < w[q] ? lo[q] : w[q]);
            hi[q] = k == 0 ? w[q] : (hi[q] > w[q] ? hi[q] : w[q]);
        }
    }
    for (int q = 0; q < 3; ++q) {
        h.lo[q] = (lo[q] - h.radius) - 0.2f;
        h.hi[q] = (hi[q] + h.radius) + 0.2f;
    }
    // slot planes for the new hull count: every array is laid out per
    // (hull, node) with the body's hull capacity, so the layout is fixed
    const size_t nn = (size_t)kMaxSpheres * n;
    char* base = static_cast<char*>(b->slots);
    d.c_exists = reinterpret_cast<uint8_t*>(base);
    d.c_active = reinterpret_cast<uint8_t*>(base + nn);
    d.c_key = reinterpret_cast<uint32_t*>(base + 2 * nn);
    float* f = reinterpret_cast<float*>(base + 6 * nn);
    d.c_normal = f;
    d.c_t1 = f + 3 * nn;
    d.c_t2 = f + 6 * nn;
    d.c_point = f + 9 * nn;
    d.c_imp = f + 12 * nn;
    if (shape_id) *shape_id = d.nhull;
    d.nhull += 1;
    rank_colliders(d.hull, d.nhull);
    return B3G_OK;
}

b3g_status b3g_softbody_read_contacts(const b3g_softbody* cb, uint8_t* exists, uint8_t* active, float* impulses)
{
    b3g_softbody* b = const_cast<b3g_softbody*>(cb);
    if (!ok(b)) return B3G_ERR_INVALID_ARGUMENT;
    const SoftDev& d = b->dev;
    const size_t m = (size_t)d.nhull * d.n;
    if (!m) return B3G_OK;
    cudaSetDevice(b->device);
    SB_TRY(cudaStreamSynchronize(b->stream));
    if (exists) SB_TRY(cudaMemcpy(exists, d.c_exists, m, cudaMemcpyDeviceToHost));
    if (active) SB_TRY(cudaMemcpy(active, d.c_active, m, cudaMemcpyDeviceToHost));
    if (impulses) {
        // per slot: normal, tangent x, tangent y
        std::vector<float> planes(3 * m);
        const size_t nn = (size_t)kMaxSpheres * d.n;
        for (int k = 0; k < 3; ++k)
            SB_TRY(cudaMemcpy(planes.data() + k * m, d.c_imp + k * nn, m * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < m; ++q)
            for (int k = 0; k < 3; ++k) impulses[3 * q + k] = planes[k * m + q];
    }
    return B3G_OK;
}

b3g_status b3g_softbody_read_state(const b3g_softbody* cb, float* x, float* v)
{
    b3g_softbody* b = const_cast<b3g_softbody*>(cb);
    if (!ok(b)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    const size_t vec = 3 * (size_t)b->dev.n * sizeof(float);
    b3g_status r = B3G_OK;
    if (x && (r = copy_nodes(b, x, b->dev.x, vec, cudaMemcpyDeviceToHost)) != B3G_OK) return r;
    if (v && (r = copy_nodes(b, v, b->dev.v, vec, cudaMemcpyDeviceToHost)) != B3G_OK) return r;
    return B3G_OK;
}

b3g_status b3g_softbody_write_state(b3g_softbody* b, const float* x, const float* v)
{
    if (!ok(b)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    const size_t vec = 3 * (size_t)b->dev.n * sizeof(float);
    b3g_status r = B3G_OK;
    if (x && (r = copy_nodes(b, b->dev.x, x, vec, cudaMemcpyHostToDevice)) != B3G_OK) return r;
    if (v && (r = copy_nodes(b, b->dev.v, v, vec, cudaMemcpyHostToDevice)) != B3G_OK) return r;
    return B3G_OK;
}

b3g_status b3g_softbody_read_elements(const b3g_softbody* cb, float* q, float* eps)
{
    b3g_softbody* b = const_cast<b3g_softbody*>(cb);
    if (!ok(b)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    b3g_status r = B3G_OK;
    if (q && (r = copy_nodes(b, q, (const float*)b->dev.q, (size_t)b->dev.t * 16, cudaMemcpyDeviceToHost)) != B3G_OK)
        return r;
    if (eps && (r = copy_nodes(b, eps, b->dev.eps, (size_t)b->dev.t * 24, cudaMemcpyDeviceToHost)) != B3G_OK) return r;
    return B3G_OK;
}

b3g_status b3g_softbody_write_elements(b3g_softbody* b, const float* q, const float* eps)
{
    if (!ok(b)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    b3g_status r = B3G_OK;
    if (q && (r = copy_nodes(b, (float*)b->dev.q, q, (size_t)b->dev.t * 16, cudaMemcpyHostToDevice)) != B3G_OK) return r;
    if (eps && (r = copy_nodes(b, b->dev.eps, eps, (size_t)b->dev.t * 24, cudaMemcpyHostToDevice)) != B3G_OK) return r;
    return B3G_OK;
}

b3g_status b3g_softbody_read_masses(const b3g_softbody* b, float* m)
{
    if (!ok(b) || !m) return B3G_ERR_INVALID_ARGUMENT;
    std::memcpy(m, b->mass.data(), b->mass.size() * sizeof(float));
    return B3G_OK;
}

// b3SoftBody::GetEnergy (softbody.cpp:627-637): 0.5 sum m v.v in node order
b3g_status b3g_softbody_energy(const b3g_softbody* b, float* energy)
{
    if (!ok(b) || !energy) return B3G_ERR_INVALID_ARGUMENT;
    std::vector<float> v(3 * (size_t)b->dev.n);
    b3g_status r = b3g_softbody_read_state(b, nullptr, v.data());
    if (r != B3G_OK) return r;
    float E = 0.0f;
    for (uint32_t i = 0; i < b->dev.n; ++i) E += b->mass[i] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    *energy = 0.5f * E;
    return B3G_OK;
}

b3g_status b3g_softbody_export_system(b3g_softbody* b, float dt, uint32_t capacity, uint32_t* rowptr, uint32_t* cols,
                                      float* vals, float* rhs, float* S, uint32_t* count)
{
    if (!ok(b) || !count || !(dt > 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    const SoftDev& d = b->dev;
    *count = d.nnz;
    if (capacity < d.nnz) return B3G_OK;
    if (!rowptr || !cols || !vals || !rhs || !S) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    cudaStream_t s = b->stream;
    // the element pass updates rotations and plastic strains: keep them
    std::vector<float> q(4 * (size_t)d.t), eps(6 * (size_t)d.t);
    b3g_status r = b3g_softbody_read_elements(b, q.data(), eps.data());
    if (r != B3G_OK) return r;
    k_sb_elements<<<blocks_for(d.t), kBlock, 0, s>>>(d, dt, 1.0f / dt);
    k_sb_assemble<<<(d.n + kAsmWarps - 1) / kAsmWarps, 32 * kAsmWarps, 0, s>>>(d, dt);
    count_launches(2);
    SB_TRY(cudaGetLastError());
    std::vector<float> v(9 * (size_t)d.nnz);
    SB_TRY(cudaMemcpyAsync(v.data(), d.vals, v.size() * 4, cudaMemcpyDeviceToHost, s));
    SB_TRY(cudaMemcpyAsync(rhs, d.b, 3 * (size_t)d.n * 4, cudaMemcpyDeviceToHost, s));
    SB_TRY(cudaMemcpyAsync(S, d.S, (size_t)d.n * 4, cudaMemcpyDeviceToHost, s));
    SB_TRY(cudaStreamSynchronize(s));
    r = b3g_softbody_write_elements(b, q.data(), eps.data());
    if (r != B3G_OK) return r;
    // rows in the reference's list order: the off-diagonal blocks newest
    // first touch first, then the diagonal block
    uint32_t k = 0;
    for (uint32_t i = 0; i < d.n; ++i) {
        rowptr[i] = k;
        const uint32_t r0 = b->rowptr[i], r1 = b->rowptr[i + 1];
        for (uint32_t j = r1; j-- > r0;) {
            if (j == b->diag[i]) continue;
            cols[k] = b->cols[j];
            std::memcpy(vals + 9 * (size_t)k, &v[9 * (size_t)j], 36);
            ++k;
        }
        cols[k] = i;
        std::memcpy(vals + 9 * (size_t)k, &v[9 * (size_t)b->diag[i]], 36);
        ++k;
    }
    rowptr[d.n] = k;
    return B3G_OK;
}

}  // extern "C"
