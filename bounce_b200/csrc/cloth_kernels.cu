// Kernels of one implicit cloth step (single cloth, whole GPU).
//
//   contacts_update  b3ClothContactManager::UpdateBodyContacts
//                    (src/bounce/cloth/cloth_contact_manager.cpp:277-315)
//   assemble         forces + Jacobians + A, b, P^-1
//                    (src/bounce/cloth/cloth_force_solver.cpp:164-204,
//                     src/bounce/cloth/forces/{strech,shear,spring}_force.cpp)
//   cg_*             b3SolveMPCG (cloth_force_solver.cpp:61-136)
//   finalize         v += dv, x += y, contact warm start / velocity
//                    iterations / x += h v / first position iteration
//                    (cloth_force_solver.cpp:211-222, cloth_solver.cpp:95-164,
//                     contacts/cloth_contact_solver.cpp body functions)
//   contact_position later position iterations with the global early out
//   post             clear f and y, particle AABB sync, new body contacts
//                    (cloth.cpp:564-577, cloth_contact_manager.cpp:64-123)
//
// Everything is compiled with -fmad=false so element arithmetic matches the
// CPU reference operation for operation.  Grid reductions are deterministic:
// every block writes one partial, the last block to arrive (ticket counter)
// sums the partials in index order.
#include <atomic>
#include <cfloat>
#include <cstdio>

#include "cg_common.cuh"
#include "cloth_dev.cuh"
#include "hull_gjk.cuh"
#include "bodies.cuh"
#include "self_collision.cuh"
#include "sell_spmv.cuh"
#include "topology.h"
#include "vec.cuh"

namespace b3g {

static std::atomic<uint64_t> g_launches{0};
uint64_t kernel_launches() { return g_launches.load(); }
void count_launches(uint64_t k) { g_launches += k; }

namespace {

constexpr float kAabbExtension = 0.2f;           // B3_AABB_EXTENSION
constexpr float kAabbMultiplier = 2.0f;          // B3_AABB_MULTIPLIER
constexpr float kLinearSlop = 0.005f;            // B3_LINEAR_SLOP
constexpr float kMaxLinearCorrection = 0.2f;     // B3_MAX_LINEAR_CORRECTION
constexpr float kBaumgarte = 0.1f;               // B3_BAUMGARTE

// ---------------------------------------------------------------------------
// SELL access
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t row_base(const ClothDev& c, uint32_t row)
{
    return c.slice_off[row >> 5] + (row & 31u);
}

__device__ __forceinline__ m3 load_block(const ClothDev& c, uint32_t idx)
{
    const float* v = c.vals;
    const uint32_t E = c.E;
    return m3{f3{v[idx], v[E + idx], v[2 * E + idx]}, f3{v[3 * E + idx], v[4 * E + idx], v[5 * E + idx]},
              f3{v[6 * E + idx], v[7 * E + idx], v[8 * E + idx]}};
}

__device__ __forceinline__ void store_block(const ClothDev& c, uint32_t idx, const m3& m)
{
    float* v = c.vals;
    const uint32_t E = c.E;
    v[idx] = m.x.x; v[E + idx] = m.x.y; v[2 * E + idx] = m.x.z;
    v[3 * E + idx] = m.y.x; v[4 * E + idx] = m.y.y; v[5 * E + idx] = m.y.z;
    v[6 * E + idx] = m.z.x; v[7 * E + idx] = m.z.y; v[8 * E + idx] = m.z.z;
}

// (A q)_row for a vector q given as 3 planes.
__device__ __forceinline__ f3 spmv_row(const ClothDev& c, uint32_t row, const float* q)
{
    return sell_row_times<false>(c, row, q);
}

__device__ __forceinline__ bool is_dynamic(const ClothDev& c, uint32_t i) { return c.type[i] == 2; }

// ---------------------------------------------------------------------------
// one cloth or many: thread -> (cloth, row)
// ---------------------------------------------------------------------------

// The entry k of prefix sums with prefix[k] <= g < prefix[k + 1] (binary search).
__device__ __forceinline__ uint32_t span_find(const uint32_t* prefix, uint32_t count, uint32_t g)
{
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The same for every lane of a warp whose g are consecutive: lane 0 searches
// and the lanes whose g fall in its entry take its answer; a lane past the
// entry's end (the warp straddles two cloths) searches on its own.  Every
// lane of the warp must call it, converged (kernel entry).
__device__ __forceinline__ uint32_t span_find_warp(const uint32_t* prefix, uint32_t count, uint32_t total,
                                                   uint32_t g)
{
    const uint32_t g0 = __shfl_sync(0xffffffffu, g, 0);
    uint32_t k0 = 0;
    if ((threadIdx.x & 31u) == 0u) k0 = span_find(prefix, count, g0 < total ? g0 : total - 1u);
    k0 = __shfl_sync(0xffffffffu, k0, 0);
    if (g < total && !(__ldg(prefix + k0) <= g && g < __ldg(prefix + k0 + 1))) k0 = span_find(prefix, count, g);
    return k0;
}

// Single-cloth launches read the cloth from the kernel parameter; launches
// over many cloths find the cloth of global thread g in the span's prefix sums
// of row counts (prefix[k] <= g < prefix[k + 1]), one search per warp.
template <bool MULTI>
__device__ __forceinline__ bool resolve(const ClothDev& one, const RowSpan& sp, uint32_t g, const ClothDev*& c,
                                        uint32_t& row)
{
    if (!MULTI) {
        c = &one;
        row = g;
        return g < one.n;
    }
    const uint32_t k = span_find_warp(sp.prefix, sp.count, sp.total, g);
    if (g >= sp.total) return false;
    c = sp.descs + k;
    row = g - __ldg(sp.prefix + k);
    return true;
}

// Adds v to *addr once per group of lanes that share addr (warp-aggregated,
// integer, so the total does not depend on the order).  Every lane of the
// warp must call it; lanes with nothing to add pass addr == nullptr.
__device__ __forceinline__ void warp_add(uint32_t* addr, uint32_t v)
{
    const unsigned grp = __match_any_sync(0xffffffffu, (unsigned long long)addr);
    const uint32_t sum = __reduce_add_sync(grp, v);
    if (addr && sum && (threadIdx.x & 31u) == (unsigned)(__ffs(grp) - 1)) atomicAdd(addr, sum);
}

// Order-preserving float <-> int for atomicMin on separations.
__device__ __forceinline__ int ord_enc(float f)
{
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ord_dec(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// ---------------------------------------------------------------------------
// assembly
// ---------------------------------------------------------------------------

// The assembly runs in two passes over each row's incidences, so that a row
// needs one 3x3 accumulator per slot in shared memory instead of two (twice
// the resident rows):
//   kPassK  the forces and dfdx: the row's force goes to b and its dfdx
//           blocks to A's storage, with the order of the slots' first touch;
//   kPassD  dfdv, then A = (M - h dfdv) - h^2 dfdx and b from the stored
//           parts.
// Each sum still runs over the row's elements in the reference's order, so
// A and b are the same floats as with both accumulators at once.
constexpr int kPassK = 0, kPassD = 1;

// Per-thread accumulators for one row in shared memory, one block per slot,
// laid out [(slot * 9 + component) * B + thread] so that lanes never
// conflict.
struct RowAcc {
    float* base;
    uint8_t* touch;   // dfdx first-touch order, [k * B + thread]
    int B, tid;
    uint64_t touched;
    int ntouch;

    __device__ void clear(int deg)
    {
        for (int k = 0; k < deg; ++k)
            for (int q = 0; q < 9; ++q) base[(k * 9 + q) * B + tid] = 0.0f;
        touched = 0ull;
        ntouch = 0;
    }
    __device__ void mark(int slot)
    {
        if (!(touched & (1ull << slot))) {
            touched |= 1ull << slot;
            touch[ntouch * B + tid] = (uint8_t)slot;
            ++ntouch;
        }
    }
    __device__ void add(int slot, const m3& m)
    {
        float* p = base + (slot * 9) * B + tid;
        p[0 * B] += m.x.x; p[1 * B] += m.x.y; p[2 * B] += m.x.z;
        p[3 * B] += m.y.x; p[4 * B] += m.y.y; p[5 * B] += m.y.z;
        p[6 * B] += m.z.x; p[7 * B] += m.z.y; p[8 * B] += m.z.z;
    }
    // dfdx: the first touch of a slot is recorded
    __device__ void addK(int slot, const m3& m)
    {
        mark(slot);
        add(slot, m);
    }
    __device__ m3 get(int slot) const
    {
        const float* p = base + (slot * 9) * B + tid;
        return m3{f3{p[0], p[B], p[2 * B]}, f3{p[3 * B], p[4 * B], p[5 * B]}, f3{p[6 * B], p[7 * B], p[8 * B]}};
    }
    __device__ m3 touchK(int slot)
    {
        mark(slot);
        return get(slot);
    }
    __device__ void set(int slot, const m3& m)
    {
        float* p = base + (slot * 9) * B + tid;
        p[0 * B] = m.x.x; p[1 * B] = m.x.y; p[2 * B] = m.x.z;
        p[3 * B] = m.y.x; p[4 * B] = m.y.y; p[5 * B] = m.y.z;
        p[6 * B] = m.z.x; p[7 * B] = m.z.y; p[8 * B] = m.z.z;
    }
    // reuse of a slot's area once its block of A is stored: two vectors
    __device__ void set6(int slot, const f3& a, const f3& b)
    {
        float* p = base + (slot * 9) * B + tid;
        p[0] = a.x; p[B] = a.y; p[2 * B] = a.z;
        p[3 * B] = b.x; p[4 * B] = b.y; p[5 * B] = b.z;
    }
    __device__ void get6(int slot, f3& a, f3& b) const
    {
        const float* p = base + (slot * 9) * B + tid;
        a = f3{p[0], p[B], p[2 * B]};
        b = f3{p[3 * B], p[4 * B], p[5 * B]};
    }
};

// b3SpringForce::Apply (spring_force.cpp:53-120) restricted to one end.
template <int PASS>
__device__ void spring_row(const ClothDev& c, RowAcc& acc, uint32_t sid, int end, int slot_self, int slot_other,
                           f3& f_row)
{
    const uint2 pr = c.spr[sid];
    const float4 par = c.spr_par[sid];
    const float L0 = par.x, ks = par.y, kd = par.z;
    const uint32_t n = c.n;
    const m3 I = mident();
    if (PASS == kPassD) {
        if (kd > 0.0f) {
            const m3 K11 = -kd * I;
            const m3 K12 = -1.0f * K11;
            acc.add(slot_self, K11);
            acc.add(slot_other, K12);
        }
        return;
    }
    const f3 x1 = ld3(c.x, n, pr.x), x2 = ld3(c.x, n, pr.y);
    f3 mf = zero3();
    if (ks > 0.0f) {
        const f3 dx = x1 - x2;
        const float L = length(dx);
        if (L > L0) {
            const f3 dCdx = dx / L;
            mf = mf + (-ks * (L - L0)) * dCdx;
            const m3 K11 = -ks * (outer(dx, dx) + (1.0f - L0 / L) * (I - outer(dx, dx)));
            const m3 K12 = -1.0f * K11;
            if (end == 0) {
                acc.addK(slot_self, K11);
                acc.addK(slot_other, K12);
            } else {
                acc.addK(slot_other, K12);
                acc.addK(slot_self, K11);
            }
        }
    }
    if (kd > 0.0f) {
        const f3 v1 = ld3(c.v, n, pr.x), v2 = ld3(c.v, n, pr.y);
        const f3 dv = v1 - v2;
        mf = mf + (-kd) * dv;
    }
    f_row = end == 0 ? f_row + mf : f_row - mf;
}

// b3MouseForce::Apply (mouse_force.cpp:63-227) restricted to the row of the
// force's vertex `role` (0: the particle, 1-3: the triangle's vertices):
// C = |x1 - (w2 x2 + w3 x3 + w4 x4)|, dC/dx = (n, -w2 n, -w3 n, -w4 n), and
// no second-derivative term.  The row's blocks are added for the force's
// vertices in order.
template <int PASS>
__device__ void mouse_row(const ClothDev& c, RowAcc& acc, uint32_t m, int role, const int slot[4], f3& f_row)
{
    const uint4 mv = c.mouse_v[m];
    const float4 pa = c.mouse_par[2 * m], pb = c.mouse_par[2 * m + 1];
    const float w2 = pa.x, w3 = pa.y, w4 = pa.z, km = pa.w, kd = pb.x;
    const uint32_t n = c.n;
    const f3 x1 = ld3(c.x, n, mv.x), x2 = ld3(c.x, n, mv.y), x3 = ld3(c.x, n, mv.z), x4 = ld3(c.x, n, mv.w);
    const f3 c2 = (w2 * x2 + w3 * x3) + w4 * x4;
    const f3 d = x1 - c2;
    const float len = length(d);
    f3 mf = zero3();
    if (len > 0.0f) {
        const f3 nrm = d / len;
        const f3 dC[4] = {nrm, (-w2) * nrm, (-w3) * nrm, (-w4) * nrm};
        const f3 dCr = role == 0 ? dC[0] : role == 1 ? dC[1] : role == 2 ? dC[2] : dC[3];
        if (PASS == kPassK && km > 0.0f) {
            const float C = len;
            mf = mf + (-km * C) * dCr;
#pragma unroll
            for (int j = 0; j < 4; ++j) acc.addK(slot[j], -km * outer(dCr, dC[j]));
        }
        if (kd > 0.0f) {
            if (PASS == kPassK) {
                const f3 vs[4] = {ld3(c.v, n, mv.x), ld3(c.v, n, mv.y), ld3(c.v, n, mv.z), ld3(c.v, n, mv.w)};
                float dCdt = 0.0f;
#pragma unroll
                for (int i = 0; i < 4; ++i) dCdt += dot(dC[i], vs[i]);
                mf = mf + (-kd * dCdt) * dCr;
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) acc.add(slot[j], -kd * outer(dCr, dC[j]));
            }
        }
    }
    if (PASS == kPassK) f_row = f_row + mf;
}

// Element `cn` of a 3-array held in registers (a select, not local memory).
template <typename T>
__device__ __forceinline__ T corner(int cn, const T& a0, const T& a1, const T& a2)
{
    return cn == 0 ? a0 : (cn == 1 ? a1 : a2);
}

// b3ShearForce::Apply then b3StrechForce::Apply (the force list holds the
// shear element of a triangle before its stretch element) for corner `cn`.
//
// A slot of the row receives up to three dfdx terms from the triangle -- the
// shear term, then the stretch terms along u and along v -- and likewise
// three dfdv terms.  The reference adds them one by one in that order
// (shear_force.cpp:142-207, strech_force.cpp:151-325); here every factor is
// computed first, then each slot's accumulators are read once, the present
// terms added in the same order, and written back once.
template <int PASS>
__device__ void triangle_row(const ClothDev& c, RowAcc& acc, uint32_t t, int cn, const int slot[3], f3& f_row)
{
    const uint4 tv = c.tri[t];
    const float4 rs = c.tri_rest[t];
    const float2 rs2 = c.tri_rest2[t];
    const float du1 = rs.x, dv1 = rs.y, du2 = rs.z, dv2 = rs.w, inv_det = rs2.x, alpha = rs2.y;
    const uint32_t n = c.n;
    const f3 x1 = ld3(c.x, n, tv.x), x2 = ld3(c.x, n, tv.y), x3 = ld3(c.x, n, tv.z);
    f3 vs[3] = {zero3(), zero3(), zero3()};
    if (PASS == kPassK) vs[0] = ld3(c.v, n, tv.x), vs[1] = ld3(c.v, n, tv.y), vs[2] = ld3(c.v, n, tv.z);
    const f3 dx1 = x2 - x1, dx2 = x3 - x1;
    const f3 wu = inv_det * (dv2 * dx1 - dv1 * dx2);
    const f3 wv = inv_det * ((-du2) * dx1 + du1 * dx2);
    const float dwudx[3] = {inv_det * (dv1 - dv2), inv_det * dv2, -inv_det * dv1};
    const float dwvdx[3] = {inv_det * (du2 - du1), -inv_det * du2, inv_det * du1};
    const float kd = c.k_damp;

    // shear (shear_force.cpp:57-212)
    const bool sh = c.k_shear > 0.0f;
    const float ks_sh = c.k_shear;
    const bool shK = sh && ks_sh > 0.0f, shD = sh && kd > 0.0f;
    f3 dCs[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) dCs[i] = alpha * (dwudx[i] * wv + dwvdx[i] * wu);
    const f3 dCsc = corner(cn, dCs[0], dCs[1], dCs[2]);
    if (PASS == kPassK && sh) {
        f3 fe = zero3();
        if (shK) {
            const float C = alpha * dot(wu, wv);
            fe = fe + (-ks_sh * C) * dCsc;
        }
        if (shD) {
            float dCdt = 0.0f;
#pragma unroll
            for (int i = 0; i < 3; ++i) dCdt += dot(dCs[i], vs[i]);
            fe = fe + (-kd * dCdt) * dCsc;
        }
        f_row = f_row + fe;
    }

    // stretch along u (d = 0) and v (d = 1) (strech_force.cpp:59-329, bu = bv = 1, cloth.cpp:198-199)
    const bool st = c.k_stretch > 0.0f;
    const float ks = c.k_stretch;
    const m3 I = mident();
    bool K_on[2], D_on[2];
    f3 dCst[2][3], dCstc[2];
    float Cst[2], kfac[2][3];  // (alpha * inv_len * dw[cn] * dw[j]) of the second-derivative term
    m3 P[2];
    {
        f3 fe = zero3();
#pragma unroll
        for (int d = 0; d < 2; ++d) {
            const f3 w = d == 0 ? wu : wv;
            const float len = d == 0 ? length(wu) : length(wv);
            const float dw[3] = {d == 0 ? dwudx[0] : dwvdx[0], d == 0 ? dwudx[1] : dwvdx[1],
                                 d == 0 ? dwudx[2] : dwvdx[2]};
            const bool live = st && len > 0.0f;
            const float inv_len = 1.0f / len;
            const f3 nw = inv_len * w;
#pragma unroll
            for (int i = 0; i < 3; ++i) dCst[d][i] = (alpha * dw[i]) * nw;
            dCstc[d] = corner(cn, dCst[d][0], dCst[d][1], dCst[d][2]);
            K_on[d] = live && ks > 0.0f && len > 1.0f;
            D_on[d] = live && kd > 0.0f;
            Cst[d] = alpha * (len - 1.0f);
            const float dwc = corner(cn, dw[0], dw[1], dw[2]);
#pragma unroll
            for (int j = 0; j < 3; ++j) kfac[d][j] = alpha * inv_len * dwc * dw[j];
            P[d] = I - outer(nw, nw);
            if (PASS == kPassK) {
                if (K_on[d]) fe = fe + (-ks * Cst[d]) * dCstc[d];
                if (D_on[d]) {
                    float dCdt = 0.0f;
#pragma unroll
                    for (int i = 0; i < 3; ++i) dCdt += dot(dCst[d][i], vs[i]);
                    fe = fe + (-kd * dCdt) * dCstc[d];
                }
            }
        }
        if (PASS == kPassK && st) f_row = f_row + fe;
    }

    // per slot, in the reference's order: shear, stretch u, stretch v
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        if (PASS == kPassK && (shK || K_on[0] || K_on[1])) {
            m3 k = acc.touchK(slot[j]);
            if (shK) k = k + -ks_sh * outer(dCsc, dCs[j]);
#pragma unroll
            for (int d = 0; d < 2; ++d)
                if (K_on[d]) k = k + -ks * (outer(dCstc[d], dCst[d][j]) + Cst[d] * (kfac[d][j] * P[d]));
            acc.set(slot[j], k);
        }
        if (PASS == kPassD && (shD || D_on[0] || D_on[1])) {
            m3 dm = acc.get(slot[j]);
            if (shD) dm = dm + -kd * outer(dCsc, dCs[j]);
#pragma unroll
            for (int d = 0; d < 2; ++d)
                if (D_on[d]) dm = dm + -kd * outer(dCstc[d], dCst[d][j]);
            acc.set(slot[j], dm);
        }
    }
}

template <bool MULTI, int PASS>
__global__ void __launch_bounds__(256) k_assemble(const __grid_constant__ ClothDev one,
                                                  const __grid_constant__ RowSpan span)
{
    extern __shared__ float smem[];
    const int B = blockDim.x, tid = threadIdx.x;
    const ClothDev* cp;
    uint32_t row;
    if (!resolve<MULTI>(one, span, blockIdx.x * B + tid, cp, row)) return;
    const ClothDev& c = *cp;
    const uint32_t max_deg = MULTI ? span.max_deg : one.max_deg;
    const StepScalars* sc = c.sc;
    const float h = sc->dt;
    const float hh = h * h;
    const uint32_t n = c.n;

    RowAcc acc;
    acc.base = smem;
    acc.touch = reinterpret_cast<uint8_t*>(smem + (size_t)max_deg * 9 * B);
    acc.B = B;
    acc.tid = tid;
    const int deg = c.row_deg[row];
    acc.clear(deg);

    // sf = f_ext (+ m g for dynamic particles), cloth_force_solver.cpp:172-180
    const float m = c.mass[row];
    f3 f = zero3();
    if (PASS == kPassK) {
        f = ld3(c.fext, n, row);
        if (is_dynamic(c, row)) f = f + m * mk(sc->gx, sc->gy, sc->gz);
    }

    // the next incidence entry is loaded while the current element is computed
    const uint32_t e_end = c.inc_ptr[row + 1];
    uint32_t e = c.inc_ptr[row];
    uint32_t el_next = e < e_end ? c.inc_elem[e] : 0u, meta_next = e < e_end ? c.inc_meta[e] : 0u;
    for (; e < e_end; ++e) {
        const uint32_t el = el_next;
        const uint32_t meta = meta_next;
        if (e + 1 < e_end) {
            el_next = c.inc_elem[e + 1];
            meta_next = c.inc_meta[e + 1];
        }
        const int cn = meta & 3u;
        const int s0 = (meta >> 8) & 0xffu, s1 = (meta >> 16) & 0xffu, s2 = (meta >> 24) & 0xffu;
        if ((el & 0xc0000000u) == 0xc0000000u) {
            // mouse force: role in bits 0-1, the four slots 7 bits each from bit 4
            const int ms[4] = {(int)((meta >> 4) & 0x7fu), (int)((meta >> 11) & 0x7fu), (int)((meta >> 18) & 0x7fu),
                               (int)((meta >> 25) & 0x7fu)};
            mouse_row<PASS>(c, acc, el & 0x3fffffffu, cn, ms, f);
        } else if (el & 0x80000000u) {
            // springs: slot of p1 in s0, of p2 in s1; cn = end
            spring_row<PASS>(c, acc, el & 0x7fffffffu, cn, cn == 0 ? s0 : s1, cn == 0 ? s1 : s0, f);
        } else {
            const int slots[3] = {s0, s1, s2};
            triangle_row<PASS>(c, acc, el, cn, slots, f);
        }
    }

    const uint32_t base = row_base(c, row);
    if (PASS == kPassK) {
        // dfdx into A's storage, the first-touch order beside it, the force into b
        for (int k = 0; k < deg; ++k) store_block(c, base + 32u * k, acc.get(k));
        for (int q = 0; q < acc.ntouch; ++q) c.asm_touch[base + 32u * q] = acc.touch[q * B + tid];
        c.asm_ntouch[row] = (uint8_t)acc.ntouch;
        st3(c.b, n, row, f);
        return;
    }

    // A = (M - h dfdv) - h^2 dfdx, one row (cloth_force_solver.cpp:198).
    // Each slot's dfdx block is read back, and its products with the v and y
    // of the slot's column (for b) go to the slot's accumulator once its
    // block of A is stored.  The column loads are issued 8 slots at a time.
    m3 diag = mzero();
    for (int k0 = 0; k0 < deg; k0 += 8) {
        uint32_t cl[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) cl[k] = k0 + k < deg ? c.cols[base + 32u * (k0 + k)] : row;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k0 + k < deg) {
                const int s = k0 + k;
                const m3 K = load_block(c, base + 32u * s);
                const m3 M = s == 0 ? m3{f3{m, 0.0f, 0.0f}, f3{0.0f, m, 0.0f}, f3{0.0f, 0.0f, m}} : mzero();
                const m3 a = (M - h * acc.get(s)) - hh * K;
                if (s == 0) diag = a;
                store_block(c, base + 32u * s, a);
                const f3 vj = ld3(c.v, n, cl[k]), yj = ld3(c.y, n, cl[k]);
                acc.set6(s, K * vj, K * yj);
            }
        }
    }
    // Jacobi preconditioner (cloth_force_solver.cpp:70-88)
    st3(c.pinv, n, row, mk(1.0f / diag.x.x, 1.0f / diag.y.y, 1.0f / diag.z.z));

    // b = h (f + h dfdx v + dfdx y), dfdx summed in its row-list order
    // (reverse first touch, sparse_mat33.h:264-282)
    f3 t1 = zero3(), t2 = zero3();
    for (int q = (int)c.asm_ntouch[row] - 1; q >= 0; --q) {
        const int k = c.asm_touch[base + 32u * q];
        f3 kv, ky;
        acc.get6(k, kv, ky);
        t1 = t1 + kv;
        t2 = t2 + ky;
    }
    st3(c.b, n, row, h * ((ld3(c.b, n, row) + h * t1) + t2));
}

// ---------------------------------------------------------------------------
// slot-major assembly
// ---------------------------------------------------------------------------
//
// The row-centric kernel above evaluates each triangle once per corner and
// pass (six times a step), one thread per row.  The slot-major form runs
// three launches:
//   k_elem_records     one thread per element: its per-corner constraint
//                      gradients, stretch projectors, force scalars and
//                      liveness flags go to a record (each element once);
//   k_assemble_blocks  one thread per block of A (row, slot): the terms of
//                      the elements that couple the row to the slot's column
//                      (the block's term list, topology.h), in the row's
//                      force-list order, into a dfdx and a dfdv sum held in
//                      registers; it stores the block of A and the dfdx
//                      block's products with the column's v and y.  The
//                      diagonal block's thread also sums the row's force
//                      from the records in force-list order (into b) and
//                      notes the order in which the row's dfdx blocks are
//                      first touched (as the row-centric first pass does);
//   k_assemble_rhs     one thread per row: b = h (f + h dfdx v + dfdx y) with
//                      the products summed in reverse first-touch order, and
//                      P^-1.
// Each block's sums see the same terms in the same order as the row-centric
// sums, every term is the same float expression, and b's dfdx products are
// summed in reverse first-touch order as before, so A, b and P^-1 are the
// same floats.  (A spring whose two ends are one particle would add its two
// dfdv terms to the diagonal in the other order at its second end: -kd and
// kd in either order sum to +0, so even that case agrees.)  A warp of
// k_assemble_blocks holds one slot of 32 consecutive rows, which on a
// regular mesh share their term pattern; walking a row's blocks in
// first-touch order instead (which follows which springs happen to be
// stretched) left 13 of 32 lanes active.
//
// Records are planes of float4: component j of element e at rec[j * count + e],
// so the record writes of a warp and the reads of neighbouring rows'
// elements are coalesced.
//
// Triangle record, 15 components:
//   3k, 3k+1, 3k+2 (corner k): (dC_shear_k, dwu_k), (dC_u_k, dwv_k), (dC_v_k, 0)
//   9-11  the stretch projectors P_u = I - n_u n_u^T, P_v (symmetric: xx xy xz yy yz zz each)
//   12    (alpha / |wu|, alpha / |wv|, C_u, C_v)
//   13    (flags, -ks_shear C_shear, -kd dC_shear/dt, 0)
//   14    (-ks C_u, -ks C_v, -kd dC_u/dt, -kd dC_v/dt)
// Spring record, 3: (force on p1, K live), (K11: xx xy xz yy), (yz zz, kd, 0).
// Mouse force record, 5: (dC_k, ·) for k = 0..3 with flags, -km C, -kd dC/dt
// and km in the w of 0..3, then (kd, 0, 0, 0).
enum : uint32_t {
    kTriShear = 1u, kTriShearK = 2u, kTriShearD = 4u, kTriStretch = 8u,
    kTriKu = 16u, kTriKv = 32u, kTriDu = 64u, kTriDv = 128u
};

__device__ __forceinline__ float4 f4(f3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
__device__ __forceinline__ f3 xyz(float4 a) { return f3{a.x, a.y, a.z}; }
// symmetric 3x3 from (xx xy xz yy) (yz zz)
__device__ __forceinline__ m3 sym3(float xx, float xy, float xz, float yy, float yz, float zz)
{
    return m3{f3{xx, xy, xz}, f3{xy, yy, yz}, f3{xz, yz, zz}};
}
// component j of a record whose component 0 is at r, in planes of `count`
__device__ __forceinline__ float4 rec(const float4* r, uint32_t count, int j) { return __ldg(r + (size_t)j * count); }

// b3ShearForce::Apply and b3StrechForce::Apply (shear_force.cpp:57-212,
// strech_force.cpp:59-329) up to the per-block products, in the same
// expressions as triangle_row.
__device__ void tri_record(const ClothDev& c, uint32_t t)
{
    const uint4 tv = c.tri[t];
    const float4 rs = c.tri_rest[t];
    const float2 rs2 = c.tri_rest2[t];
    const float du1 = rs.x, dv1 = rs.y, du2 = rs.z, dv2 = rs.w, inv_det = rs2.x, alpha = rs2.y;
    const uint32_t n = c.n;
    const f3 x1 = ld3(c.x, n, tv.x), x2 = ld3(c.x, n, tv.y), x3 = ld3(c.x, n, tv.z);
    const f3 vs[3] = {ld3(c.v, n, tv.x), ld3(c.v, n, tv.y), ld3(c.v, n, tv.z)};
    const f3 dx1 = x2 - x1, dx2 = x3 - x1;
    const f3 wu = inv_det * (dv2 * dx1 - dv1 * dx2);
    const f3 wv = inv_det * ((-du2) * dx1 + du1 * dx2);
    const float dwudx[3] = {inv_det * (dv1 - dv2), inv_det * dv2, -inv_det * dv1};
    const float dwvdx[3] = {inv_det * (du2 - du1), -inv_det * du2, inv_det * du1};
    const float kd = c.k_damp;

    const float ks_sh = c.k_shear;
    const bool sh = ks_sh > 0.0f, shK = sh && ks_sh > 0.0f, shD = sh && kd > 0.0f;
    f3 dCs[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) dCs[i] = alpha * (dwudx[i] * wv + dwvdx[i] * wu);
    uint32_t flags = (sh ? kTriShear : 0u) | (shK ? kTriShearK : 0u) | (shD ? kTriShearD : 0u);
    float fKs = 0.0f, fDs = 0.0f;
    if (shK) {
        const float C = alpha * dot(wu, wv);
        fKs = -ks_sh * C;
    }
    if (shD) {
        float dCdt = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i) dCdt += dot(dCs[i], vs[i]);
        fDs = -kd * dCdt;
    }

    const float ks = c.k_stretch;
    const bool st = ks > 0.0f;
    if (st) flags |= kTriStretch;
    const m3 I = mident();
    f3 dCst[2][3];
    float ai[2], Cst[2], fK[2] = {0.0f, 0.0f}, fD[2] = {0.0f, 0.0f};
    m3 P[2];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        const f3 w = d == 0 ? wu : wv;
        const float len = d == 0 ? length(wu) : length(wv);
        const float dw[3] = {d == 0 ? dwudx[0] : dwvdx[0], d == 0 ? dwudx[1] : dwvdx[1],
                             d == 0 ? dwudx[2] : dwvdx[2]};
        const bool live = st && len > 0.0f;
        const float inv_len = 1.0f / len;
        const f3 nw = inv_len * w;
#pragma unroll
        for (int i = 0; i < 3; ++i) dCst[d][i] = (alpha * dw[i]) * nw;
        const bool Kon = live && ks > 0.0f && len > 1.0f, Don = live && kd > 0.0f;
        Cst[d] = alpha * (len - 1.0f);
        ai[d] = alpha * inv_len;
        P[d] = I - outer(nw, nw);
        if (Kon) {
            flags |= d == 0 ? kTriKu : kTriKv;
            fK[d] = -ks * Cst[d];
        }
        if (Don) {
            flags |= d == 0 ? kTriDu : kTriDv;
            float dCdt = 0.0f;
#pragma unroll
            for (int i = 0; i < 3; ++i) dCdt += dot(dCst[d][i], vs[i]);
            fD[d] = -kd * dCdt;
        }
    }

    float4* r = c.tri_rec + t;
    const size_t T = c.t;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r[(3 * k) * T] = f4(dCs[k], dwudx[k]);
        r[(3 * k + 1) * T] = f4(dCst[0][k], dwvdx[k]);
        r[(3 * k + 2) * T] = f4(dCst[1][k], 0.0f);
    }
    r[9 * T] = make_float4(P[0].x.x, P[0].x.y, P[0].x.z, P[0].y.y);
    r[10 * T] = make_float4(P[0].y.z, P[0].z.z, P[1].x.x, P[1].x.y);
    r[11 * T] = make_float4(P[1].x.z, P[1].y.y, P[1].y.z, P[1].z.z);
    r[12 * T] = make_float4(ai[0], ai[1], Cst[0], Cst[1]);
    r[13 * T] = make_float4(__uint_as_float(flags), fKs, fDs, 0.0f);
    r[14 * T] = make_float4(fK[0], fK[1], fD[0], fD[1]);
}

// b3SpringForce::Apply (spring_force.cpp:53-120), the expressions of spring_row.
__device__ void spring_record(const ClothDev& c, uint32_t sid)
{
    const uint2 pr = c.spr[sid];
    const float4 par = c.spr_par[sid];
    const float L0 = par.x, ks = par.y, kd = par.z;
    const uint32_t n = c.n;
    const m3 I = mident();
    f3 mf = zero3();
    m3 K11 = mzero();
    uint32_t live = 0u;
    if (ks > 0.0f) {
        const f3 x1 = ld3(c.x, n, pr.x), x2 = ld3(c.x, n, pr.y);
        const f3 dx = x1 - x2;
        const float L = length(dx);
        if (L > L0) {
            const f3 dCdx = dx / L;
            mf = mf + (-ks * (L - L0)) * dCdx;
            K11 = -ks * (outer(dx, dx) + (1.0f - L0 / L) * (I - outer(dx, dx)));
            live = 1u;
        }
    }
    if (kd > 0.0f) {
        const f3 v1 = ld3(c.v, n, pr.x), v2 = ld3(c.v, n, pr.y);
        const f3 dv = v1 - v2;
        mf = mf + (-kd) * dv;
    }
    float4* r = c.spr_rec + sid;
    const size_t S = c.ns;
    r[0] = f4(mf, __uint_as_float(live));
    r[S] = make_float4(K11.x.x, K11.x.y, K11.x.z, K11.y.y);
    r[2 * S] = make_float4(K11.y.z, K11.z.z, kd, 0.0f);
}

// b3MouseForce::Apply (mouse_force.cpp:63-227), the expressions of mouse_row.
__device__ void mouse_record(const ClothDev& c, uint32_t m)
{
    const uint4 mv = c.mouse_v[m];
    const float4 pa = c.mouse_par[2 * m], pb = c.mouse_par[2 * m + 1];
    const float w2 = pa.x, w3 = pa.y, w4 = pa.z, km = pa.w, kd = pb.x;
    const uint32_t n = c.n;
    const f3 x1 = ld3(c.x, n, mv.x), x2 = ld3(c.x, n, mv.y), x3 = ld3(c.x, n, mv.z), x4 = ld3(c.x, n, mv.w);
    const f3 c2 = (w2 * x2 + w3 * x3) + w4 * x4;
    const f3 d = x1 - c2;
    const float len = length(d);
    f3 dC[4] = {zero3(), zero3(), zero3(), zero3()};
    float fK = 0.0f, fD = 0.0f;
    uint32_t flags = 0u;
    if (len > 0.0f) {
        const f3 nrm = d / len;
        dC[0] = nrm;
        dC[1] = (-w2) * nrm;
        dC[2] = (-w3) * nrm;
        dC[3] = (-w4) * nrm;
        flags = 1u;
        if (km > 0.0f) {
            flags |= 2u;
            const float C = len;
            fK = -km * C;
        }
        if (kd > 0.0f) {
            flags |= 4u;
            const f3 vs[4] = {ld3(c.v, n, mv.x), ld3(c.v, n, mv.y), ld3(c.v, n, mv.z), ld3(c.v, n, mv.w)};
            float dCdt = 0.0f;
#pragma unroll
            for (int i = 0; i < 4; ++i) dCdt += dot(dC[i], vs[i]);
            fD = -kd * dCdt;
        }
    }
    float4* r = c.mouse_rec + m;
    const size_t M = c.nmouse;
    r[0] = f4(dC[0], __uint_as_float(flags));
    r[M] = f4(dC[1], fK);
    r[2 * M] = f4(dC[2], fD);
    r[3 * M] = f4(dC[3], km);
    r[4 * M] = make_float4(kd, 0.0f, 0.0f, 0.0f);
}

// The element of global thread g of a launch over one cloth's or many
// cloths' elements: triangles, then springs, then mouse forces.
template <bool MULTI>
__device__ __forceinline__ bool resolve_elem(const ClothDev& one, const RowSpan& sp, uint32_t g, const ClothDev*& c,
                                             uint32_t& e)
{
    if (!MULTI) {
        c = &one;
        e = g;
        return g < one.t + one.ns + one.nmouse;
    }
    const uint32_t k = span_find_warp(sp.eprefix, sp.count, sp.etotal, g);
    if (g >= sp.etotal) return false;
    c = sp.descs + k;
    e = g - __ldg(sp.eprefix + k);
    return true;
}

// Every element's record, one thread per element.
template <bool MULTI>
__global__ void __launch_bounds__(256) k_elem_records(const __grid_constant__ ClothDev one,
                                                      const __grid_constant__ RowSpan span)
{
    const ClothDev* cp;
    uint32_t e;
    if (!resolve_elem<MULTI>(one, span, blockIdx.x * blockDim.x + threadIdx.x, cp, e)) return;
    const ClothDev& c = *cp;
    if (e < c.t) tri_record(c, e);
    else if (e < c.t + c.ns) spring_record(c, e - c.t);
    else mouse_record(c, e - c.t - c.ns);
}

// Adds one element term (code: kind, row corner, column corner, id) to a
// block's dfdx (K) and dfdv (D) sums, in triangle_row / spring_row /
// mouse_row's order and expressions.
__device__ __forceinline__ void slot_term(const ClothDev& c, uint32_t code, m3& K, m3& D)
{
    const uint32_t id = code & ((1u << kTermIdBits) - 1u);
    const int cr = (int)((code >> 28) & 3u), cj = (int)((code >> 26) & 3u);
    const uint32_t kind = code >> 30;
    if (kind == 0u) {
        const float4* r = c.tri_rec + id;
        const uint32_t T = c.t;
        const uint32_t flags = __float_as_uint(rec(r, T, 13).x);
        const float4 a0 = rec(r, T, 3 * cr), a1 = rec(r, T, 3 * cr + 1), a2 = rec(r, T, 3 * cr + 2);
        const float4 b0 = rec(r, T, 3 * cj), b1 = rec(r, T, 3 * cj + 1), b2 = rec(r, T, 3 * cj + 2);
        const f3 sc = xyz(a0), sj = xyz(b0), uc = xyz(a1), uj = xyz(b1), vc = xyz(a2), vj = xyz(b2);
        const float kd = c.k_damp;
        if (flags & kTriShearK) K = K + -c.k_shear * outer(sc, sj);
        if (flags & (kTriKu | kTriKv)) {
            const float ks = c.k_stretch;
            const float4 p0 = rec(r, T, 9), p1 = rec(r, T, 10), p2 = rec(r, T, 11), q = rec(r, T, 12);
            if (flags & kTriKu) {
                const float kf = (q.x * a0.w) * b0.w;
                K = K + -ks * (outer(uc, uj) + q.z * (kf * sym3(p0.x, p0.y, p0.z, p0.w, p1.x, p1.y)));
            }
            if (flags & kTriKv) {
                const float kf = (q.y * a1.w) * b1.w;
                K = K + -ks * (outer(vc, vj) + q.w * (kf * sym3(p1.z, p1.w, p2.x, p2.y, p2.z, p2.w)));
            }
        }
        if (flags & kTriShearD) D = D + -kd * outer(sc, sj);
        if (flags & kTriDu) D = D + -kd * outer(uc, uj);
        if (flags & kTriDv) D = D + -kd * outer(vc, vj);
    } else if (kind == 2u) {
        const float4* r = c.spr_rec + id;
        const uint32_t S = c.ns;
        const float4 r1 = rec(r, S, 1), r2 = rec(r, S, 2);
        if (__float_as_uint(rec(r, S, 0).w)) {
            const m3 K11 = sym3(r1.x, r1.y, r1.z, r1.w, r2.x, r2.y);
            K = K + (cj == cr ? K11 : -1.0f * K11);
        }
        const float kd = r2.z;
        if (kd > 0.0f) {
            const m3 D11 = -kd * mident();
            D = D + (cj == cr ? D11 : -1.0f * D11);
        }
    } else {
        const float4* r = c.mouse_rec + id;
        const uint32_t M = c.nmouse;
        const uint32_t flags = __float_as_uint(rec(r, M, 0).w);
        const f3 a = xyz(rec(r, M, cr)), b = xyz(rec(r, M, cj));
        if ((flags & 3u) == 3u) K = K + -rec(r, M, 3).w * outer(a, b);
        if ((flags & 5u) == 5u) D = D + -rec(r, M, 4).x * outer(a, b);
    }
}

// The row's force from the element records in force-list order
// (cloth_force_solver.cpp:172-180, the forces' Apply), stored in b, and the
// order in which its dfdx blocks are first touched, stored as the row-centric
// first pass stores it (slot ids at the row's SELL positions, and the count).
__device__ void row_force(const ClothDev& c, uint32_t row, uint32_t base)
{
    const StepScalars* sc = c.sc;
    const uint32_t n = c.n;
    const float m = c.mass[row];
    f3 f = ld3(c.fext, n, row);
    if (is_dynamic(c, row)) f = f + m * mk(sc->gx, sc->gy, sc->gz);
    uint32_t touched = 0u, ntouch = 0u;
    auto mark = [&](uint32_t s) {
        if (!((touched >> s) & 1u)) {
            touched |= 1u << s;
            c.asm_touch[base + 32u * ntouch] = (uint8_t)s;
            ++ntouch;
        }
    };
    const uint32_t T = c.t, S = c.ns, M = c.nmouse;
    const uint32_t e_end = c.inc_ptr[row + 1];
    for (uint32_t e = c.inc_ptr[row]; e < e_end; ++e) {
        const uint32_t el = c.inc_elem[e], meta = c.inc_meta[e];
        const int cn = (int)(meta & 3u);
        if ((el & 0xc0000000u) == 0xc0000000u) {
            const float4* r = c.mouse_rec + (el & 0x3fffffffu);
            const float4 a = rec(r, M, cn), r0 = rec(r, M, 0), r1 = rec(r, M, 1), r2 = rec(r, M, 2);
            const uint32_t flags = __float_as_uint(r0.w);
            f3 mf = zero3();
            if (flags & 1u) {
                if (flags & 2u) mf = mf + r1.w * xyz(a);
                if (flags & 4u) mf = mf + r2.w * xyz(a);
            }
            f = f + mf;
            if ((flags & 3u) == 3u) {
#pragma unroll
                for (int q = 0; q < 4; ++q) mark((meta >> (4 + 7 * q)) & 0x7fu);
            }
        } else if (el & 0x80000000u) {
            const float4 r0 = rec(c.spr_rec + (el & 0x7fffffffu), S, 0);
            const f3 mf = xyz(r0);
            f = cn == 0 ? f + mf : f - mf;
            if (__float_as_uint(r0.w)) {
                mark((meta >> 8) & 0xffu);
                mark((meta >> 16) & 0xffu);
            }
        } else {
            const float4* r = c.tri_rec + el;
            const float4 g0 = rec(r, T, 3 * cn), g1 = rec(r, T, 3 * cn + 1), g2 = rec(r, T, 3 * cn + 2);
            const float4 s13 = rec(r, T, 13), s14 = rec(r, T, 14);
            const uint32_t flags = __float_as_uint(s13.x);
            if (flags & kTriShear) {
                f3 fe = zero3();
                if (flags & kTriShearK) fe = fe + s13.y * xyz(g0);
                if (flags & kTriShearD) fe = fe + s13.z * xyz(g0);
                f = f + fe;
            }
            f3 fe = zero3();
            if (flags & kTriKu) fe = fe + s14.x * xyz(g1);
            if (flags & kTriDu) fe = fe + s14.z * xyz(g1);
            if (flags & kTriKv) fe = fe + s14.y * xyz(g2);
            if (flags & kTriDv) fe = fe + s14.w * xyz(g2);
            if (flags & kTriStretch) f = f + fe;
            if (flags & (kTriShearK | kTriKu | kTriKv)) {
                mark((meta >> 8) & 0xffu);
                mark((meta >> 16) & 0xffu);
                mark((meta >> 24) & 0xffu);
            }
        }
    }
    c.asm_ntouch[row] = (uint8_t)ntouch;
    st3(c.b, n, row, f);
}

// One block of A per thread: thread (row, slot k) with k = blockIdx.y, so a
// warp handles the same slot of 32 consecutive rows (the same term pattern
// on a regular mesh): its term codes and its stores are coalesced SELL
// words.  Besides the block of A (cloth_force_solver.cpp:198) it stores its
// dfdx products with the column's v and y, which k_assemble_rhs sums in the
// row's order.
template <bool MULTI>
__global__ void __launch_bounds__(128) k_assemble_blocks(const __grid_constant__ ClothDev one,
                                                         const __grid_constant__ RowSpan span)
{
    const ClothDev* cp;
    uint32_t row;
    if (!resolve<MULTI>(one, span, blockIdx.x * blockDim.x + threadIdx.x, cp, row)) return;
    const ClothDev& c = *cp;
    const uint32_t k = blockIdx.y;
    if (k >= c.row_deg[row]) return;
    const float h = c.sc->dt;
    const float hh = h * h;
    const uint32_t base = row_base(c, row);
    const uint32_t idx = base + 32u * k;
    const uint32_t col = c.cols[idx];
    const uint32_t cnt = c.term_slot[idx];
    const uint32_t* tp = c.terms + c.term_qk[(base >> 5) + k] + (row & 31u);
    m3 K = mzero(), D = mzero();
    uint32_t code_next = cnt ? __ldg(tp) : 0u;
    for (uint32_t q = 0; q < cnt; ++q) {
        const uint32_t code = code_next;
        if (q + 1 < cnt) code_next = __ldg(tp + 32u * (q + 1));
        slot_term(c, code, K, D);
    }
    const float m = k == 0 ? c.mass[row] : 0.0f;
    const m3 M = k == 0 ? m3{f3{m, 0.0f, 0.0f}, f3{0.0f, m, 0.0f}, f3{0.0f, 0.0f, m}} : mzero();
    store_block(c, idx, (M - h * D) - hh * K);
    const f3 kv = K * ld3(c.v, c.n, col), ky = K * ld3(c.y, c.n, col);
    float* qv = c.asm_kv;
    const uint32_t E = c.E;
    qv[idx] = kv.x; qv[E + idx] = kv.y; qv[2 * E + idx] = kv.z;
    qv[3 * E + idx] = ky.x; qv[4 * E + idx] = ky.y; qv[5 * E + idx] = ky.z;
    if (k == 0) row_force(c, row, base);
}

// One row per thread: b = h (f + h dfdx v + dfdx y) with the blocks' dfdx
// products summed in reverse first-touch order (the dfdx row list order,
// sparse_mat33.h:264-282), and the Jacobi preconditioner from the diagonal
// block (cloth_force_solver.cpp:70-88, 172-204).
template <bool MULTI>
__global__ void __launch_bounds__(256) k_assemble_rhs(const __grid_constant__ ClothDev one,
                                                      const __grid_constant__ RowSpan span)
{
    const ClothDev* cp;
    uint32_t row;
    if (!resolve<MULTI>(one, span, blockIdx.x * blockDim.x + threadIdx.x, cp, row)) return;
    const ClothDev& c = *cp;
    const float h = c.sc->dt;
    const uint32_t n = c.n;
    const uint32_t base = row_base(c, row);
    const float* q = c.asm_kv;
    const uint32_t E = c.E;
    f3 t1 = zero3(), t2 = zero3();
    for (int i = (int)c.asm_ntouch[row] - 1; i >= 0; --i) {
        const uint32_t idx = base + 32u * c.asm_touch[base + 32u * i];
        t1 = t1 + f3{q[idx], q[E + idx], q[2 * E + idx]};
        t2 = t2 + f3{q[3 * E + idx], q[4 * E + idx], q[5 * E + idx]};
    }
    const float* v = c.vals;
    st3(c.pinv, n, row, mk(1.0f / v[base], 1.0f / v[4 * E + base], 1.0f / v[8 * E + base]));
    st3(c.b, n, row, h * ((ld3(c.b, n, row) + h * t1) + t2));
}

// ---------------------------------------------------------------------------
// MPCG
// ---------------------------------------------------------------------------

// x0 = S m_x; r = S (b - A x0); p = S P^-1 r; b_delta, delta
// (cloth_force_solver.cpp:90-100)
template <int DOT>
__global__ void k_cg_init(ClothDev c, cudaGraphConditionalHandle cond, int use_graph)
{
    typedef DotT<DOT> D;
    typename D::T v[2] = {D::zero(), D::zero()};
    const uint32_t n = c.n;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const bool Si = is_dynamic(c, row);
        // A x0 with x0_j = S_j m_x_j gathered on the fly
        const uint32_t base = row_base(c, row);
        const uint32_t deg = c.row_deg[row];
        f3 ax = zero3();
        for (uint32_t k = 0; k < deg; ++k) {
            const uint32_t idx = base + 32u * k;
            const uint32_t col = c.cols[idx];
            const f3 xj = is_dynamic(c, col) ? ld3(c.mx, n, col) : zero3();
            ax = ax + load_block(c, idx) * xj;
        }
        const f3 bi = ld3(c.b, n, row);
        const f3 pv = ld3(c.pinv, n, row);
        const f3 x0 = Si ? ld3(c.mx, n, row) : zero3();
        const f3 r = Si ? bi - ax : zero3();
        const f3 p = Si ? mk(r.x * pv.x, r.y * pv.y, r.z * pv.z) : zero3();
        const f3 bh = Si ? bi : zero3();
        st3(c.dv, n, row, x0);
        st3(c.r, n, row, r);
        st3(c.p, n, row, p);
        v[0] = D::add_term(v[0], bh, mk(bh.x * pv.x, bh.y * pv.y, bh.z * pv.z));
        v[1] = D::add_term(v[1], r, p);
    }
    if (grid_reduce<DOT, 2>(v, c.partials, &c.sc->ticket[0]) && threadIdx.x == 0) {
        StepScalars* sc = c.sc;
        double bd = D::value(v[0]), dl = D::value(v[1]);
        if (DOT != 2) {
            bd = (double)(float)bd;
            dl = (double)(float)dl;
        }
        sc->b_delta = bd;
        sc->delta = dl;
        sc->delta0 = dl;
        sc->iter = 0;
        sc->status = 0;
        uint32_t cont = (sc->max_iter > 0 && !cg_stop(sc, dl, bd)) ? 1u : 0u;
        if (!isfinite(dl) || !isfinite(bd)) {
            sc->status = kStatusNumerical;
            cont = 0;
        }
        sc->cont = cont;
        if (use_graph) cudaGraphSetConditional(cond, cont);
    }
}

// s = S A p, alpha = delta / p.s (cloth_force_solver.cpp:115-117)
template <int DOT>
__global__ void k_cg_spmv(ClothDev c)
{
    typedef DotT<DOT> D;
    if (c.sc->cont == 0u) return;
    typename D::T v[1] = {D::zero()};
    const uint32_t n = c.n;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const f3 ap = spmv_row(c, row, c.p);
        const f3 s = is_dynamic(c, row) ? ap : zero3();
        st3(c.s, n, row, s);
        v[0] = D::add_term(v[0], ld3(c.p, n, row), s);
    }
    if (grid_reduce<DOT, 1>(v, c.partials, &c.sc->ticket[1]) && threadIdx.x == 0) {
        StepScalars* sc = c.sc;
        const double pAp = D::value(v[0]);
        sc->pAp = pAp;
        float alpha;
        if (DOT == 2) alpha = (float)(sc->delta / pAp);
        else alpha = (float)sc->delta / (float)pAp;
        sc->alpha = alpha;
    }
}

// x += alpha p; r -= alpha s; h = P^-1 r; delta' = r.h; beta
// (cloth_force_solver.cpp:119-128); sets the loop condition.
template <int DOT>
__global__ void k_cg_update(ClothDev c, cudaGraphConditionalHandle cond, int use_graph)
{
    typedef DotT<DOT> D;
    if (c.sc->cont == 0u) return;
    typename D::T v[1] = {D::zero()};
    const uint32_t n = c.n;
    const float alpha = c.sc->alpha;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const f3 p = ld3(c.p, n, row);
        const f3 s = ld3(c.s, n, row);
        const f3 x = ld3(c.dv, n, row) + alpha * p;
        const f3 r = ld3(c.r, n, row) - alpha * s;
        const f3 pv = ld3(c.pinv, n, row);
        const f3 hv = mk(r.x * pv.x, r.y * pv.y, r.z * pv.z);
        st3(c.dv, n, row, x);
        st3(c.r, n, row, r);
        v[0] = D::add_term(v[0], r, hv);
    }
    if (grid_reduce<DOT, 1>(v, c.partials, &c.sc->ticket[2]) && threadIdx.x == 0) {
        StepScalars* sc = c.sc;
        double dn = D::value(v[0]);
        const double dold = sc->delta;
        float beta;
        if (DOT == 2) {
            beta = (float)(dn / dold);
        } else {
            dn = (double)(float)dn;
            beta = (float)dn / (float)dold;
        }
        sc->delta = dn;
        sc->beta = beta;
        sc->iter += 1;
        uint32_t cont = (sc->iter < sc->max_iter && !cg_stop(sc, dn, sc->b_delta)) ? 1u : 0u;
        if (!isfinite(dn) || !isfinite(sc->alpha) || !isfinite(beta)) {
            sc->status = kStatusNumerical;
            cont = 0;
        }
        sc->cont = cont;
        if (use_graph) cudaGraphSetConditional(cond, cont);
    }
}

// p = S (P^-1 r + beta p) (cloth_force_solver.cpp:130)
__global__ void k_cg_direction(ClothDev c)
{
    if (c.sc->cont == 0u) return;
    const uint32_t n = c.n;
    const float beta = c.sc->beta;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const f3 r = ld3(c.r, n, row);
        const f3 pv = ld3(c.pinv, n, row);
        const f3 hv = mk(r.x * pv.x, r.y * pv.y, r.z * pv.z);
        const f3 p = is_dynamic(c, row) ? hv + beta * ld3(c.p, n, row) : zero3();
        st3(c.p, n, row, p);
    }
}

// ---------------------------------------------------------------------------
// contacts
// ---------------------------------------------------------------------------

__device__ __forceinline__ bool overlap(const float* lo, const float* hi, const SphereDev& s)
{
    // b3TestOverlap (include/bounce/collision/shapes/aabb3.h:247-251)
    return lo[0] <= s.hi[0] && lo[1] <= s.hi[1] && lo[2] <= s.hi[2] && hi[0] >= s.lo[0] && hi[1] >= s.lo[1] &&
           hi[2] >= s.lo[2];
}

// The overlap of a particle's proxy with collider s: body shapes keep their
// proxy in device memory (the caller's world and the step's body sync move it).
__device__ __forceinline__ bool overlap_shape(const ClothDev& c, uint32_t s, const float* lo, const float* hi)
{
    const SphereDev& sp = c.sph[s];
    if (!sp.body1) return overlap(lo, hi, sp);
    const float* f = c.shape_fat + 6 * s;
    return lo[0] <= f[3] && lo[1] <= f[4] && lo[2] <= f[5] && hi[0] >= f[0] && hi[1] >= f[1] && hi[2] >= f[2];
}

// A pair of a non-dynamic particle and a collider whose body is not dynamic
// does not collide (cloth_contact_manager.cpp:286-298).
__device__ __forceinline__ bool body_dynamic(const ClothDev& c, uint32_t s)
{
    return c.sph[s].body1 && c.bodies[c.sph[s].body1 - 1].type == 2;
}

// TestSphere of a collider on a body, with the body's transform m_xf; the
// contact keeps its shape point in the body's frame (GetLocalPoint).
__device__ __forceinline__ bool body_contact(const ClothDev& c, uint32_t s, uint32_t q, uint32_t nn, f3 xi,
                                             float radius, f3& normal)
{
    const SphereDev& sp = c.sph[s];
    m3 R;
    f3 p, point;
    body::body_xf(c.bodies[sp.body1 - 1], R, p);
    if (!body::test_sphere(sp, R, p, xi, radius, normal, point)) return false;
    st3(c.c_point, nn, q, body::xmult(R, p, point));
    return true;
}

__device__ __forceinline__ void load_fat(const ClothDev& c, uint32_t i, float* lo, float* hi)
{
    const uint32_t n = c.n;
    lo[0] = c.fat_lo[i]; lo[1] = c.fat_lo[n + i]; lo[2] = c.fat_lo[2 * n + i];
    hi[0] = c.fat_hi[i]; hi[1] = c.fat_hi[n + i]; hi[2] = c.fat_hi[2 * n + i];
}

// UpdateBodyContacts + b3ParticleBodyContact::Update with TestSphere
// (cloth_contact_manager.cpp:277-315, cloth_particle_body_contact.cpp:24-47,
// sphere_shape.cpp:71-95)
template <bool MULTI>
__global__ void k_contacts_update(const __grid_constant__ ClothDev one, const __grid_constant__ RowSpan span)
{
    const ClothDev* cp;
    uint32_t i;
    if (!resolve<MULTI>(one, span, blockIdx.x * blockDim.x + threadIdx.x, cp, i)) return;
    const ClothDev& c = *cp;
    if (!c.nsph) return;
    const uint32_t n = c.n, nn = c.nsph * n;
    float lo[3], hi[3];
    load_fat(c, i, lo, hi);
    const f3 xi = ld3(c.x, n, i);
    for (uint32_t s = 0; s < c.nsph; ++s) {
        const uint32_t q = s * n + i;
        if (!c.c_exists[q] || c.sph[s].kind == 2) continue;  // hulls: k_hull_contacts_update
        const SphereDev& sp = c.sph[s];
        if ((!is_dynamic(c, i) && !body_dynamic(c, s)) || !overlap_shape(c, s, lo, hi)) {
            c.c_exists[q] = 0;
            c.c_active[q] = 0;
            continue;
        }
        const float radius = sp.radius + c.p_radius[i];
        f3 normal;
        if (sp.body1) {
            if (!body_contact(c, s, q, nn, xi, radius, normal)) {
                c.c_active[q] = 0;
                continue;
            }
        } else if (sp.kind == 0) {
            // b3SphereShape::TestSphere (sphere_shape.cpp:71-95)
            const float rr = radius * radius;
            const f3 d = xi - mk(sp.cx, sp.cy, sp.cz);
            const float dd = dot(d, d);
            if (!(dd <= rr)) {
                c.c_active[q] = 0;
                continue;
            }
            const float d_len = sqrtf(dd);
            normal = mk(0.0f, 1.0f, 0.0f);
            if (d_len > kEps) normal = d / d_len;
        } else {
            // b3CapsuleShape::TestSphere (capsule_shape.cpp:186-284)
            const f3 A = mk(sp.ax, sp.ay, sp.az), B = mk(sp.bx, sp.by, sp.bz);
            const f3 AB = B - A;
            const float u = dot(B - xi, AB);
            const float v = dot(xi - A, AB);
            f3 P;
            if (v <= 0.0f || u <= 0.0f) {
                P = v <= 0.0f ? A : B;
                const f3 d = xi - P;
                const float dd = dot(d, d);
                if (dd > radius * radius) {
                    c.c_active[q] = 0;
                    continue;
                }
                normal = mk(0.0f, 1.0f, 0.0f);
                const float len = sqrtf(dd);
                if (len > kEps) normal = d / len;
            } else {
                const float ss = dot(AB, AB);
                P = ss < kLinearSlop * kLinearSlop ? A : (u * A + v * B) / ss;
                const f3 d = xi - P;
                const float dd = dot(d, d);
                if (dd > radius * radius) {
                    c.c_active[q] = 0;
                    continue;
                }
                const f3 QA = A - xi;
                const f3 e = cross(AB, QA);
                f3 nn3 = cross(AB, e);
                if (dot(nn3, QA) < 0.0f) nn3 = mk(-nn3.x, -nn3.y, -nn3.z);
                // b3Vec3::Normalize (vec3.h:93-104)
                const float len = sqrtf(nn3.x * nn3.x + nn3.y * nn3.y + nn3.z * nn3.z);
                if (len > kEps) {
                    const float s1 = 1.0f / len;
                    nn3 = mk(nn3.x * s1, nn3.y * s1, nn3.z * s1);
                }
                normal = mk(-nn3.x, -nn3.y, -nn3.z);
            }
            st3(c.c_point, nn, q, P);
        }
        const f3 n1 = mk(-normal.x, -normal.y, -normal.z);
        const f3 t1 = perp(n1);
        const f3 t2 = cross(t1, n1);
        c.c_active[q] = 1;
        st3(c.c_normal, nn, q, n1);
        st3(c.c_t1, nn, q, t1);
        st3(c.c_t2, nn, q, t2);
    }
}

// The same update for the hull colliders (b3HullShape::TestSphere,
// hull_shape.cpp:187-254), in a kernel of its own so that the GJK's
// registers stay out of the sphere and capsule update.
template <bool MULTI>
__global__ void k_hull_contacts_update(const __grid_constant__ ClothDev one, const __grid_constant__ RowSpan span)
{
    const ClothDev* cp;
    uint32_t i;
    if (!resolve<MULTI>(one, span, blockIdx.x * blockDim.x + threadIdx.x, cp, i)) return;
    const ClothDev& c = *cp;
    const uint32_t n = c.n, nn = c.nsph * n;
    float lo[3], hi[3];
    load_fat(c, i, lo, hi);
    const f3 xi = ld3(c.x, n, i);
    for (uint32_t s = 0; s < c.nsph; ++s) {
        const uint32_t q = s * n + i;
        const SphereDev& sp = c.sph[s];
        if (sp.kind != 2 || !c.c_exists[q]) continue;
        if ((!is_dynamic(c, i) && !body_dynamic(c, s)) || !overlap_shape(c, s, lo, hi)) {
            c.c_exists[q] = 0;
            c.c_active[q] = 0;
            continue;
        }
        const float radius = sp.radius + c.p_radius[i];
        f3 normal, P;
        if (sp.body1) {
            if (!body_contact(c, s, q, nn, xi, radius, normal)) {
                c.c_active[q] = 0;
                continue;
            }
        } else {
            if (!hull::test_sphere(sp.hull, sp.nhv, sp.hull + 3 * sp.nhv, sp.nhf, radius, mident(), zero3(), xi,
                                   normal, P)) {
                c.c_active[q] = 0;
                continue;
            }
            st3(c.c_point, nn, q, hull::xf_mult(P));  // body->GetLocalPoint
        }
        const f3 n1 = mk(-normal.x, -normal.y, -normal.z);
        const f3 t1 = perp(n1);
        const f3 t2 = cross(t1, n1);
        c.c_active[q] = 1;
        st3(c.c_normal, nn, q, n1);
        st3(c.c_t1, nn, q, t1);
        st3(c.c_t2, nn, q, t2);
    }
}

// Active contacts of vertex i in list order (newest first).
__device__ int contact_order(const ClothDev& c, uint32_t i, int* order)
{
    int k = 0;
    const uint32_t n = c.n;
    for (uint32_t s = 0; s < c.nsph; ++s) {
        const uint32_t q = s * n + i;
        if (c.c_exists[q] && c.c_active[q]) order[k++] = (int)s;
    }
    // insertion sort by descending creation key
    for (int a = 1; a < k; ++a) {
        int v = order[a];
        int b = a - 1;
        while (b >= 0 && c.c_key[order[b] * n + i] < c.c_key[v * n + i]) {
            order[b + 1] = order[b];
            --b;
        }
        order[b + 1] = v;
    }
    return k;
}

// One position iteration for vertex i; returns its smallest separation
// (cloth_contact_solver.cpp:620-718).
__device__ float position_iteration(const ClothDev& c, uint32_t i, f3& pos, const int* order, int k)
{
    const uint32_t n = c.n, nn = c.nsph * n;
    const float mA = 1.0f / c.mass[i];
    float min_sep = 0.0f;
    for (int a = 0; a < k; ++a) {
        const int s = order[a];
        const SphereDev& sp = c.sph[s];
        const f3 nA = ld3(c.c_normal, nn, s * n + i);
        const f3 cB = sp.kind == 0 ? mk(sp.cx, sp.cy, sp.cz) : ld3(c.c_point, nn, s * n + i);
        const float separation = dot(cB - pos, nA) - c.p_radius[i] - sp.radius;
        min_sep = min_sep < separation ? min_sep : separation;
        const float Cv = kBaumgarte * (separation + kLinearSlop);
        float C = Cv < 0.0f ? Cv : 0.0f;
        C = -kMaxLinearCorrection > C ? -kMaxLinearCorrection : C;
        const float K = mA + 0.0f + 0.0f + 0.0f;
        const float impulse = K > 0.0f ? -C / K : 0.0f;
        const f3 P = impulse * nA;
        pos = pos - mA * P;
    }
    return min_sep;
}

// v += dv; x += y; m_x = dv; contact solve (cloth_solver.cpp:95-164).  The
// smallest separation of the first position iteration goes to
// StepScalars::min_sep[0] (atomicMin, order-independent).
template <bool MULTI>
__global__ void k_finalize(const __grid_constant__ ClothDev one, const __grid_constant__ RowSpan span)
{
    const ClothDev* cp;
    uint32_t i;
    uint32_t* count_addr = nullptr;
    uint32_t active = 0;
    if (resolve<MULTI>(one, span, blockIdx.x * blockDim.x + threadIdx.x, cp, i)) {
        const ClothDev& c = *cp;
        const uint32_t n = c.n, nn = c.nsph * n;
        StepScalars* sc = c.sc;
        const float h = sc->dt;
        const f3 dv = ld3(c.dv, n, i);
        f3 vel = ld3(c.v, n, i) + dv;
        f3 pos = ld3(c.x, n, i) + ld3(c.y, n, i);
        st3(c.mx, n, i, dv);
        int order[kMaxSpheres];
        const int k = c.nsph ? contact_order(c, i, order) : 0;
        if (k > 0) {
            active = (uint32_t)k;
            count_addr = &sc->active_contacts;
            const float mA = 1.0f / c.mass[i];
            // InitializeBodyContactConstraints (cloth_contact_solver.cpp:54-177), static body
            float nmass[kMaxSpheres], tm_xx[kMaxSpheres], tm_xy[kMaxSpheres], tm_yx[kMaxSpheres],
                tm_yy[kMaxSpheres], fr[kMaxSpheres], ni[kMaxSpheres], tix[kMaxSpheres], tiy[kMaxSpheres];
            for (int a = 0; a < k; ++a) {
                const int s = order[a];
                const uint32_t q = s * n + i;
                const float K = mA + 0.0f + 0.0f + 0.0f;
                nmass[a] = K > 0.0f ? 1.0f / K : 0.0f;
                const float k11 = mA + 0.0f + 0.0f + 0.0f, k12 = 0.0f + 0.0f, k22 = mA + 0.0f + 0.0f + 0.0f;
                float det = k11 * k22 - k12 * k12;
                if (det != 0.0f) det = 1.0f / det;
                tm_xx[a] = det * k22;
                tm_yx[a] = -det * k12;
                tm_xy[a] = -det * k12;
                tm_yy[a] = det * k11;
                fr[a] = sqrtf(c.p_friction[i] * c.sph[s].friction);
                ni[a] = c.c_imp[q];
                tix[a] = c.c_imp[nn + q];
                tiy[a] = c.c_imp[2 * nn + q];
            }
            // WarmStartBodyContactConstraints (:264-307)
            for (int a = 0; a < k; ++a) {
                const uint32_t q = order[a] * n + i;
                const f3 nrm = ld3(c.c_normal, nn, q), t1 = ld3(c.c_t1, nn, q), t2 = ld3(c.c_t2, nn, q);
                const f3 P = ni[a] * nrm;
                vel = vel - mA * P;
                const f3 P1 = tix[a] * t1, P2 = tiy[a] * t2;
                vel = vel - mA * (P1 + P2);
            }
            // SolveBodyContactVelocityConstraints (:388-472)
            for (uint32_t it = 0; it < sc->vel_iters; ++it) {
                for (int a = 0; a < k; ++a) {
                    const uint32_t q = order[a] * n + i;
                    const f3 nrm = ld3(c.c_normal, nn, q), t1 = ld3(c.c_t1, nn, q), t2 = ld3(c.c_t2, nn, q);
                    {
                        const f3 dvv = zero3() - vel;
                        const float Cdot = dot(nrm, dvv);
                        float impulse = nmass[a] * (-Cdot + 0.0f);
                        const float old = ni[a];
                        const float sum = old + impulse;
                        ni[a] = sum > 0.0f ? sum : 0.0f;
                        impulse = ni[a] - old;
                        const f3 P = impulse * nrm;
                        vel = vel - mA * P;
                    }
                    {
                        const f3 dvv = zero3() - vel;
                        const float cx = dot(dvv, t1), cy = dot(dvv, t2);
                        const float ncx = -cx, ncy = -cy;
                        const float ix = ncx * tm_xx[a] + ncy * tm_yx[a];
                        const float iy = ncx * tm_xy[a] + ncy * tm_yy[a];
                        const float ox = tix[a], oy = tiy[a];
                        tix[a] += ix;
                        tiy[a] += iy;
                        const float maxImpulse = fr[a] * ni[a];
                        if (tix[a] * tix[a] + tiy[a] * tiy[a] > maxImpulse * maxImpulse) {
                            const float sl = sqrtf(tix[a] * tix[a] + tiy[a] * tiy[a]);
                            if (sl > kEps) {
                                tix[a] /= sl;
                                tiy[a] /= sl;
                            }
                            tix[a] *= maxImpulse;
                            tiy[a] *= maxImpulse;
                        }
                        const float jx = tix[a] - ox, jy = tiy[a] - oy;
                        const f3 P = jx * t1 + jy * t2;
                        vel = vel - mA * P;
                    }
                }
            }
            // StoreImpulses (:598-607)
            for (int a = 0; a < k; ++a) {
                const uint32_t q = order[a] * n + i;
                c.c_imp[q] = ni[a];
                c.c_imp[nn + q] = tix[a];
                c.c_imp[2 * nn + q] = tiy[a];
            }
        }
        // integrate positions (cloth_solver.cpp:143-147)
        pos = pos + h * vel;
        if (k > 0 && sc->pos_iters > 0) {
            const float ms = position_iteration(c, i, pos, order, k);
            if (ms < 0.0f) atomicMin(&sc->min_sep[0], ord_enc(ms));
        }
        st3(c.x, n, i, pos);
        st3(c.v, n, i, vel);
    }
    warp_add(count_addr, active);
}

// Position iteration `it` (>= 1), run for a cloth only while iteration it - 1
// left a contact deeper than 3 slops (cloth_solver.cpp:151-164).
template <bool MULTI>
__global__ void k_contact_position(const __grid_constant__ ClothDev one, const __grid_constant__ RowSpan span,
                                   uint32_t it)
{
    const ClothDev* cp;
    uint32_t i;
    if (!resolve<MULTI>(one, span, blockIdx.x * blockDim.x + threadIdx.x, cp, i)) return;
    const ClothDev& c = *cp;
    StepScalars* sc = c.sc;
    if (!c.nsph || it >= sc->pos_iters || it >= kMaxPosIters) return;
    if (ord_dec(sc->min_sep[it - 1]) >= -3.0f * kLinearSlop) return;
    int order[kMaxSpheres];
    const int k = contact_order(c, i, order);
    if (k > 0) {
        f3 pos = ld3(c.x, c.n, i);
        const float ms = position_iteration(c, i, pos, order, k);
        st3(c.x, c.n, i, pos);
        if (ms < 0.0f) atomicMin(&sc->min_sep[it], ord_enc(ms));
    }
}

__device__ void move_proxy_dev(const ClothDev& c, uint32_t i, f3 disp)
{
    const uint32_t n = c.n;
    const f3 x = ld3(c.x, n, i);
    float lo[3], hi[3];
    load_fat(c, i, lo, hi);
    const float r = c.p_radius[i];
    float tlo[3] = {x.x - r, x.y - r, x.z - r}, thi[3] = {x.x + r, x.y + r, x.z + r};
    bool contains = true;
    for (int d = 0; d < 3; ++d)
        contains = contains && lo[d] <= tlo[d] && tlo[d] <= hi[d] && lo[d] <= thi[d] && thi[d] <= hi[d];
    if (contains) return;
    const float dd[3] = {kAabbMultiplier * disp.x, kAabbMultiplier * disp.y, kAabbMultiplier * disp.z};
    for (int d = 0; d < 3; ++d) {
        lo[d] = tlo[d] - kAabbExtension;
        hi[d] = thi[d] + kAabbExtension;
        if (dd[d] < 0.0f) lo[d] += dd[d];
        else hi[d] += dd[d];
    }
    c.fat_lo[i] = lo[0]; c.fat_lo[n + i] = lo[1]; c.fat_lo[2 * n + i] = lo[2];
    c.fat_hi[i] = hi[0]; c.fat_hi[n + i] = hi[1]; c.fat_hi[2 * n + i] = hi[2];
    if (c.p_moved) c.p_moved[i] = 1;  // BufferMove
}

// Clear f and y, sync the particle AABB (b3BroadPhase::MoveProxy,
// broad_phase.cpp:99-149), new body contacts (cloth_contact_manager.cpp:64-123).
template <bool MULTI>
__global__ void k_post(const __grid_constant__ ClothDev one, const __grid_constant__ RowSpan span)
{
    const ClothDev* cp;
    uint32_t i;
    uint32_t alive = 0;
    uint32_t* count_addr = nullptr;
    if (resolve<MULTI>(one, span, blockIdx.x * blockDim.x + threadIdx.x, cp, i)) {
        const ClothDev& c = *cp;
        const uint32_t n = c.n, nn = c.nsph * n;
        const StepScalars* sc = c.sc;
        st3(c.fext, n, i, zero3());
        st3(c.y, n, i, zero3());
        move_proxy_dev(c, i, sc->dt * ld3(c.v, n, i));
        float lo[3], hi[3];
        load_fat(c, i, lo, hi);
        const bool dyn = is_dynamic(c, i);
        for (uint32_t s = 0; s < c.nsph; ++s) {
            const uint32_t q = s * n + i;
            if (!c.c_exists[q] && dyn && overlap_shape(c, s, lo, hi)) {
                c.c_exists[q] = 1;
                c.c_active[q] = 0;
                c.c_key[q] = sc->step_index * kMaxSpheres + c.sph[s].rank;
                c.c_imp[q] = 0.0f;
                c.c_imp[nn + q] = 0.0f;
                c.c_imp[2 * nn + q] = 0.0f;
            }
            alive += c.c_exists[q];
        }
        if (alive) count_addr = &c.sc->contacts;
    }
    warp_add(count_addr, alive);
}

// ---------------------------------------------------------------------------
// ray casts (b3Cloth::RayCast / RayCastSingle)
// ---------------------------------------------------------------------------

// b3RayCast against triangle k (src/bounce/collision/collision.cpp:31-118)
__device__ bool ray_triangle(const ClothDev& c, uint32_t k, f3 p1, f3 p2, float max_fraction, float& fraction,
                             f3& normal)
{
    const uint32_t n = c.n;
    const uint4 tv = c.tri[k];
    const f3 v1 = ld3(c.x, n, tv.x), v2 = ld3(c.x, n, tv.y), v3 = ld3(c.x, n, tv.z);
    const f3 d = p2 - p1;
    if (d.x * d.x + d.y * d.y + d.z * d.z < kEps * kEps) return false;
    f3 nn = cross(v2 - v1, v3 - v1);
    const float len = sqrtf(nn.x * nn.x + nn.y * nn.y + nn.z * nn.z);
    if (len == 0.0f) return false;
    const float s1 = 1.0f / len;  // b3Vec3::operator/=
    nn = mk(nn.x * s1, nn.y * s1, nn.z * s1);
    const float num = dot(nn, v1 - p1);
    const float den = dot(nn, d);
    if (den == 0.0f) return false;
    const float f = num / den;
    if (f < 0.0f || max_fraction < f) return false;
    const f3 Q = p1 + f * d;
    const f3 AB = v2 - v1, AC = v3 - v1, QA = v1 - Q, QB = v2 - Q, QC = v3 - Q;
    const f3 AB_x_AC = cross(AB, AC);
    const float u = dot(cross(QB, QC), AB_x_AC);
    const float v = dot(cross(QC, QA), AB_x_AC);
    const float w = dot(cross(QA, QB), AB_x_AC);
    if (!(u >= 0.0f && v >= 0.0f && w >= 0.0f)) return false;
    fraction = f;
    normal = num > 0.0f ? mk(-nn.x, -nn.y, -nn.z) : nn;
    return true;
}

// Every triangle against the ray; the smallest (fraction, triangle) wins.
__global__ void k_ray_min(ClothDev c, RayQuery q)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.t) return;
    float f;
    f3 nrm;
    if (!ray_triangle(c, k, mk(q.p1[0], q.p1[1], q.p1[2]), mk(q.p2[0], q.p2[1], q.p2[2]), q.max_fraction, f, nrm))
        return;
    const unsigned long long key = ((unsigned long long)__float_as_uint(f + 0.0f) << 32) | k;
    atomicMin(q.best, key);
}

// The winner's fraction and normal, or no hit.
__global__ void k_ray_result(ClothDev c, RayQuery q)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    RayHit h{};
    const unsigned long long key = *q.best;
    if (key != ~0ull) {
        const uint32_t k = (uint32_t)(key & 0xffffffffull);
        float f;
        f3 nrm;
        if (ray_triangle(c, k, mk(q.p1[0], q.p1[1], q.p1[2]), mk(q.p2[0], q.p2[1], q.p2[2]), q.max_fraction, f, nrm)) {
            h.hit = 1;
            h.triangle = k;
            h.fraction = f;
            h.normal[0] = nrm.x;
            h.normal[1] = nrm.y;
            h.normal[2] = nrm.z;
        }
    }
    *q.out = h;
}

// ---------------------------------------------------------------------------
// particle edits
// ---------------------------------------------------------------------------

__device__ void destroy_contacts_dev(const ClothDev& c, uint32_t i)
{
    for (uint32_t s = 0; s < c.nsph; ++s) {
        c.c_exists[s * c.n + i] = 0;
        c.c_active[s * c.n + i] = 0;
    }
}

// b3Particle::SetType (particle.cpp:121-143)
__device__ void set_type_dev(const ClothDev& c, uint32_t i, uint8_t type)
{
    const uint32_t n = c.n;
    if (c.type[i] == type) return;
    c.type[i] = type;
    st3(c.fext, n, i, zero3());
    if (type == 0) {
        st3(c.v, n, i, zero3());
        st3(c.y, n, i, zero3());
        move_proxy_dev(c, i, zero3());
        if (c.p_moved) sync_vertex_triangles_dev(c, i);
    }
    destroy_contacts_dev(c, i);
    if (c.p_moved) {
        c.p_purge[i] = 1;   // DestroyContacts (particle.cpp:103-118)
        c.p_moved[i] = 1;   // TouchProxy
    }
}

__global__ void k_particle_ops(ClothDev c, const ParticleOp* ops, uint32_t count)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const uint32_t n = c.n;
    for (uint32_t k = 0; k < count; ++k) {
        const ParticleOp op = ops[k];
        const uint32_t i = op.vertex;
        if (i >= n) continue;
        const f3 a = mk(op.a[0], op.a[1], op.a[2]);
        switch (op.kind) {
            case OP_SET_TYPE: set_type_dev(c, i, (uint8_t)op.a[0]); break;
            case OP_SET_POSITION: {  // particle.h:205-214
                const f3 d = a - ld3(c.x, n, i);
                st3(c.x, n, i, a);
                st3(c.y, n, i, zero3());
                move_proxy_dev(c, i, d);
                if (c.p_moved) sync_vertex_triangles_dev(c, i);
                break;
            }
            case OP_SET_VELOCITY:  // particle.h:221-228
                if (c.type[i] != 0) st3(c.v, n, i, a);
                break;
            case OP_APPLY_FORCE:  // particle.h:260-267
                if (c.type[i] == 2) st3(c.fext, n, i, ld3(c.fext, n, i) + a);
                break;
            case OP_APPLY_TRANSLATION:  // particle.h:269-272
                st3(c.y, n, i, ld3(c.y, n, i) + a);
                break;
            case OP_SET_RADIUS:  // particle.h:240-245: the radius, then Synchronize(0)
                c.p_radius[i] = op.a[0];
                move_proxy_dev(c, i, zero3());
                break;
            case OP_SET_FRICTION:  // particle.h:252-255
                c.p_friction[i] = op.a[0];
                break;
        }
    }
}

__global__ void k_set_types(ClothDev c, const uint8_t* types)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < c.n) set_type_dev(c, i, types[i]);
}

__global__ void k_add_vectors(ClothDev c, float* dst, const float* src, int only_dynamic)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    if (only_dynamic && c.type[i] != 2) return;
    const f3 a = mk(src[3 * i], src[3 * i + 1], src[3 * i + 2]);
    st3(dst, c.n, i, ld3(dst, c.n, i) + a);
}

// Three planes of n floats to n xyz triples, and back (host buffers hold
// xyz per particle; the device keeps planes).
__global__ void k_planes_to_xyz(const float* planes, float* xyz, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    xyz[3 * i] = planes[i];
    xyz[3 * i + 1] = planes[n + i];
    xyz[3 * i + 2] = planes[2 * n + i];
}

__global__ void k_xyz_to_planes(const float* xyz, float* planes, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    planes[i] = xyz[3 * i];
    planes[n + i] = xyz[3 * i + 1];
    planes[2 * n + i] = xyz[3 * i + 2];
}

__global__ void k_clear_contacts(ClothDev c)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < c.n) destroy_contacts_dev(c, i);
}

inline uint32_t blocks_for(uint32_t n, uint32_t b) { return (n + b - 1) / b; }

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

size_t assemble_smem_bytes(uint32_t max_deg, int block)
{
    return (size_t)max_deg * 9 * sizeof(float) * block + (size_t)max_deg * block;
}

// Every launch raises the kernel's dynamic shared memory limit to the same
// maximum, so concurrent launches from several host threads never lower it
// under one another.
constexpr size_t kAssembleSmemLimit = 227 * 1024;

// The assembly keeps a row's accumulators in shared memory (37 bytes per
// slot), so shared memory bounds how many rows an SM holds.  Of the block
// sizes 32..256 take the one with the most resident rows per SM (the
// smaller on ties, for a finer tail), from the occupancy calculator.
int assemble_block_for(uint32_t max_deg, bool multi)
{
    static std::atomic<int> cache[2][256];  // 0: not computed yet
    if (max_deg > 255) max_deg = 255;
    std::atomic<int>& slot = cache[multi ? 1 : 0][max_deg];
    if (const int known = slot.load(std::memory_order_relaxed)) return known;
    const void* fn = multi ? (const void*)k_assemble<true, kPassK> : (const void*)k_assemble<false, kPassK>;
    int best = 32, best_rows = 0;
    for (int b = 32; b <= 256; b += 32) {
        const size_t smem = assemble_smem_bytes(max_deg, b);
        if (smem > kAssembleSmemLimit) break;
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAssembleSmemLimit) !=
            cudaSuccess) {
            cudaGetLastError();
            break;
        }
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, b, smem) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (per_sm * b > best_rows) {
            best_rows = per_sm * b;
            best = b;
        }
    }
    slot.store(best, std::memory_order_relaxed);
    return best;
}

static const RowSpan kNoSpan{};

cudaError_t launch_ray_cast(const ClothDev& c, const RayQuery& q, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(q.best, 0xff, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    if (c.t) k_ray_min<<<blocks_for(c.t, 256), 256, 0, st>>>(c, q);
    k_ray_result<<<1, 32, 0, st>>>(c, q);
    count_launches(c.t ? 2 : 1);
    return cudaGetLastError();
}

cudaError_t launch_ray_result(const ClothDev& c, const RayQuery& q, cudaStream_t st)
{
    k_ray_result<<<1, 32, 0, st>>>(c, q);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_contacts_update(const ClothDev& c, cudaStream_t st)
{
    if (!c.nsph) return cudaSuccess;
    k_contacts_update<false><<<blocks_for(c.n, 256), 256, 0, st>>>(c, kNoSpan);
    count_launches(1);
    bool hulls = false;
    for (uint32_t s = 0; s < c.nsph; ++s) hulls = hulls || c.sph[s].kind == 2;
    if (hulls) {
        k_hull_contacts_update<false><<<blocks_for(c.n, 128), 128, 0, st>>>(c, kNoSpan);
        count_launches(1);
    }
    return cudaGetLastError();
}

constexpr int kRecordBlock = 256, kSlotBlock = 128;

// The assembly: the element records and the slot-major rows where the
// cloth's layout has them, else the row-centric two passes (forces and dfdx,
// then dfdv, A and b).
cudaError_t launch_assemble(const ClothDev& c, int block, cudaStream_t st)
{
    if (c.slot_asm) {
        k_elem_records<false><<<blocks_for(c.t + c.ns + c.nmouse, kRecordBlock), kRecordBlock, 0, st>>>(c,
                                                                                                   kNoSpan);
        k_assemble_blocks<false><<<dim3(blocks_for(c.n, kSlotBlock), c.max_deg), kSlotBlock, 0, st>>>(c, kNoSpan);
        k_assemble_rhs<false><<<blocks_for(c.n, kRecordBlock), kRecordBlock, 0, st>>>(c, kNoSpan);
        count_launches(3);
        return cudaGetLastError();
    }
    if (block <= 0) block = assemble_block_for(c.max_deg, false);
    const size_t smem = assemble_smem_bytes(c.max_deg, block);
    if (smem > kAssembleSmemLimit) return cudaErrorInvalidValue;
    for (const void* fn : {(const void*)k_assemble<false, kPassK>, (const void*)k_assemble<false, kPassD>}) {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)kAssembleSmemLimit);
        if (e != cudaSuccess) return e;
    }
    k_assemble<false, kPassK><<<blocks_for(c.n, block), block, smem, st>>>(c, kNoSpan);
    k_assemble<false, kPassD><<<blocks_for(c.n, block), block, smem, st>>>(c, kNoSpan);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_cg_init(const ClothDev& c, int dot, cudaGraphConditionalHandle cond, int use_graph,
                           cudaStream_t st)
{
    if (dot == 0) k_cg_init<0><<<c.grid, c.block, 0, st>>>(c, cond, use_graph);
    else if (dot == 1) k_cg_init<1><<<c.grid, c.block, 0, st>>>(c, cond, use_graph);
    else k_cg_init<2><<<c.grid, c.block, 0, st>>>(c, cond, use_graph);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_cg_iteration(const ClothDev& c, int dot, cudaGraphConditionalHandle cond, int use_graph,
                                cudaStream_t st)
{
    if (dot == 0) {
        k_cg_spmv<0><<<c.grid, c.block, 0, st>>>(c);
        k_cg_update<0><<<c.grid, c.block, 0, st>>>(c, cond, use_graph);
    } else if (dot == 1) {
        k_cg_spmv<1><<<c.grid, c.block, 0, st>>>(c);
        k_cg_update<1><<<c.grid, c.block, 0, st>>>(c, cond, use_graph);
    } else {
        k_cg_spmv<2><<<c.grid, c.block, 0, st>>>(c);
        k_cg_update<2><<<c.grid, c.block, 0, st>>>(c, cond, use_graph);
    }
    k_cg_direction<<<c.grid, c.block, 0, st>>>(c);
    count_launches(3);
    return cudaGetLastError();
}

cudaError_t launch_cg_part(const ClothDev& c, int dot, int part, cudaStream_t st)
{
    cudaGraphConditionalHandle none = 0;
    if (part == 0) {
        if (dot == 0) k_cg_spmv<0><<<c.grid, c.block, 0, st>>>(c);
        else if (dot == 1) k_cg_spmv<1><<<c.grid, c.block, 0, st>>>(c);
        else k_cg_spmv<2><<<c.grid, c.block, 0, st>>>(c);
    } else if (part == 1) {
        if (dot == 0) k_cg_update<0><<<c.grid, c.block, 0, st>>>(c, none, 0);
        else if (dot == 1) k_cg_update<1><<<c.grid, c.block, 0, st>>>(c, none, 0);
        else k_cg_update<2><<<c.grid, c.block, 0, st>>>(c, none, 0);
    } else {
        k_cg_direction<<<c.grid, c.block, 0, st>>>(c);
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const ClothDev& c, cudaStream_t st)
{
    k_finalize<false><<<blocks_for(c.n, 256), 256, 0, st>>>(c, kNoSpan);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_contact_position(const ClothDev& c, uint32_t it, cudaStream_t st)
{
    if (!c.nsph) return cudaSuccess;
    k_contact_position<false><<<blocks_for(c.n, 256), 256, 0, st>>>(c, kNoSpan, it);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_post(const ClothDev& c, cudaStream_t st)
{
    k_post<false><<<blocks_for(c.n, 256), 256, 0, st>>>(c, kNoSpan);
    count_launches(1);
    return cudaGetLastError();
}

// ---- launches over many cloths ----
static ClothDev g_unused_one{};

cudaError_t launch_span_contacts_update(const RowSpan& sp, cudaStream_t st)
{
    if (!sp.total) return cudaSuccess;
    k_contacts_update<true><<<blocks_for(sp.total, 256), 256, 0, st>>>(g_unused_one, sp);
    count_launches(1);
    if (sp.hulls) {
        k_hull_contacts_update<true><<<blocks_for(sp.total, 128), 128, 0, st>>>(g_unused_one, sp);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_span_assemble(const RowSpan& sp, int block, cudaStream_t st)
{
    if (!sp.total) return cudaSuccess;
    if (sp.slot_asm) {
        k_elem_records<true><<<blocks_for(sp.etotal, kRecordBlock), kRecordBlock, 0, st>>>(g_unused_one, sp);
        k_assemble_blocks<true><<<dim3(blocks_for(sp.total, kSlotBlock), sp.max_deg), kSlotBlock, 0, st>>>(
            g_unused_one, sp);
        k_assemble_rhs<true><<<blocks_for(sp.total, kRecordBlock), kRecordBlock, 0, st>>>(g_unused_one, sp);
        count_launches(3);
        return cudaGetLastError();
    }
    if (block <= 0) block = assemble_block_for(sp.max_deg, true);
    const size_t smem = assemble_smem_bytes(sp.max_deg, block);
    if (smem > kAssembleSmemLimit) return cudaErrorInvalidValue;
    for (const void* fn : {(const void*)k_assemble<true, kPassK>, (const void*)k_assemble<true, kPassD>}) {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)kAssembleSmemLimit);
        if (e != cudaSuccess) return e;
    }
    k_assemble<true, kPassK><<<blocks_for(sp.total, block), block, smem, st>>>(g_unused_one, sp);
    k_assemble<true, kPassD><<<blocks_for(sp.total, block), block, smem, st>>>(g_unused_one, sp);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_span_finalize(const RowSpan& sp, cudaStream_t st)
{
    if (!sp.total) return cudaSuccess;
    k_finalize<true><<<blocks_for(sp.total, 256), 256, 0, st>>>(g_unused_one, sp);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_span_contact_position(const RowSpan& sp, uint32_t it, cudaStream_t st)
{
    if (!sp.total) return cudaSuccess;
    k_contact_position<true><<<blocks_for(sp.total, 256), 256, 0, st>>>(g_unused_one, sp, it);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_span_post(const RowSpan& sp, cudaStream_t st)
{
    if (!sp.total) return cudaSuccess;
    k_post<true><<<blocks_for(sp.total, 256), 256, 0, st>>>(g_unused_one, sp);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_particle_ops(const ClothDev& c, const ParticleOp* ops, uint32_t count, cudaStream_t st)
{
    k_particle_ops<<<1, 32, 0, st>>>(c, ops, count);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_set_types(const ClothDev& c, const uint8_t* types, cudaStream_t st)
{
    k_set_types<<<blocks_for(c.n, 256), 256, 0, st>>>(c, types);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_add_vectors(const ClothDev& c, float* dst, const float* src, int only_dynamic, cudaStream_t st)
{
    k_add_vectors<<<blocks_for(c.n, 256), 256, 0, st>>>(c, dst, src, only_dynamic);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_planes_to_xyz(const float* planes, float* xyz, uint32_t n, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    k_planes_to_xyz<<<blocks_for(n, 256), 256, 0, st>>>(planes, xyz, n);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_xyz_to_planes(const float* xyz, float* planes, uint32_t n, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    k_xyz_to_planes<<<blocks_for(n, 256), 256, 0, st>>>(xyz, planes, n);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_clear_contacts(const ClothDev& c, cudaStream_t st)
{
    if (!c.nsph) return cudaSuccess;
    k_clear_contacts<<<blocks_for(c.n, 256), 256, 0, st>>>(c);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace b3g
