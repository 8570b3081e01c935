// Persistent MPCG of one large cloth on the whole GPU.
//
// b3SolveMPCG (src/bounce/cloth/cloth_force_solver.cpp:61-136) as a single
// cooperative launch: every CTA stays resident, the two phases of an
// iteration (new direction + SpMV + p.s; update + r.P^-1 r) are separated by
// a software grid barrier instead of kernel boundaries, and each reduction
// is summed by every CTA from the per-CTA partials in index order, so all
// CTAs agree on alpha and beta without another barrier and the result is
// deterministic.  The launch is shaped so that rows spread evenly over the
// SMs (one CTA per SM, one row per thread, while that fits).
// Every wait on the barrier is bounded: after kSpinLimit polls the CTA sets
// the cloth's status to B3G_ERR_TIMEOUT and leaves, and so do the others.
#include <algorithm>

#include <cuda/atomic>

#include "cg_common.cuh"
#include "cloth_dev.cuh"
#include "grid_cg.cuh"
#include "sell_spmv.cuh"
#include "vec.cuh"

namespace b3g {

namespace {

constexpr int kMaxBlock = 512;
constexpr int kMaxWarps = kMaxBlock / 32;
constexpr int kPrefetch = 16;  // partials per lane loaded together (up to 512 CTAs)
constexpr int kPrefetchFused = 6;  // the fused form's 32-byte partials: up to 192 CTAs
constexpr size_t kSmemLimit = 227 * 1024;  // dynamic shared memory of one CTA on sm_100
constexpr uint64_t kSpinLimit = 1ull << 26;
constexpr uint32_t kStatusTimeout = 7;

__device__ __forceinline__ uint32_t rbase(const ClothDev& c, uint32_t row)
{
    return c.slice_off[row >> 5] + (row & 31u);
}

__device__ __forceinline__ bool dyn(const ClothDev& c, uint32_t i) { return c.type[i] == 2; }

// z and the previous direction are written by other CTAs inside the launch:
// read them around L1.
__device__ __forceinline__ f3 ld3_l2(const float* p, uint32_t n, uint32_t i)
{
    return f3{__ldcg(p + i), __ldcg(p + n + i), __ldcg(p + 2 * n + i)};
}

__device__ __forceinline__ m3 block_at(const ClothDev& c, uint32_t idx)
{
    const float* v = c.vals;
    const uint32_t E = c.E;
    return m3{f3{v[idx], v[E + idx], v[2 * E + idx]}, f3{v[3 * E + idx], v[4 * E + idx], v[5 * E + idx]},
              f3{v[6 * E + idx], v[7 * E + idx], v[8 * E + idx]}};
}

// Block k of a thread's row kept in shared memory, [slot][component][thread].
__device__ __forceinline__ m3 smem_block(const float* sa, uint32_t k, uint32_t B, uint32_t tid)
{
    const uint32_t o = k * 9u * B + tid;
    return m3{f3{sa[o], sa[o + B], sa[o + 2 * B]}, f3{sa[o + 3 * B], sa[o + 4 * B], sa[o + 5 * B]},
              f3{sa[o + 6 * B], sa[o + 7 * B], sa[o + 8 * B]}};
}

// Copies the blocks of a one-row thread's row into its shared-memory column
// (once per solve; only the thread itself reads them later).
__device__ __forceinline__ void stage_row_blocks(const ClothDev& c, uint32_t base, uint32_t deg, float* sa,
                                                 uint32_t B, uint32_t tid)
{
#pragma unroll 1
    for (uint32_t k = 0; k < deg; ++k) {
        const uint32_t g = base + 32u * k, o = k * 9u * B + tid;
#pragma unroll
        for (uint32_t q = 0; q < 9; ++q) sa[o + q * B] = c.vals[(size_t)q * c.E + g];
    }
}

// Row `row` of s = A p, where the direction p = z + beta p_old is formed on
// the fly from the neighbours' z = S P^-1 r and previous direction (first
// iteration: p = z).  That is the same float expression the owner of each
// row evaluates for its own p, so every row sees bit-identical p values and
// the new direction needs no grid barrier of its own.  Blocks are summed in
// slot order, acc = acc + A_k p_k (b3Mat33 * b3Vec3,
// include/bounce/common/math/mat33.h:129-132).
__device__ __forceinline__ f3 row_times_direction(const ClothDev& c, uint32_t row, const float* z,
                                                  const float* pold, float beta, bool first)
{
    constexpr int W = 8;
    const uint32_t base = rbase(c, row);
    const uint32_t deg = c.row_deg[row];
    const uint32_t n = c.n;
    f3 acc = zero3();
    for (uint32_t k0 = 0; k0 < deg; k0 += W) {
        uint32_t cl[W];
#pragma unroll
        for (int k = 0; k < W; ++k) cl[k] = (k0 + k < deg) ? c.cols[base + 32u * (k0 + k)] : 0u;
#pragma unroll
        for (int k = 0; k < W; ++k) {
            if (k0 + k < deg) {
                const m3 a = block_at(c, base + 32u * (k0 + k));
                const uint32_t j = cl[k];
                const f3 zj = ld3_l2(z, n, j);
                const f3 pj = first ? zj : zj + beta * ld3_l2(pold, n, j);
                acc = acc + a * pj;
            }
        }
    }
    return acc;
}

__device__ __forceinline__ void bar_arrive(uint32_t* p)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(p) : "memory");
}

__device__ __forceinline__ uint32_t bar_poll(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier on a monotonic arrival counter (zeroed before the launch):
// the e-th barrier of the launch is complete once the counter has reached
// e * nblocks.  Arrival is one release reduction, so the last CTA to arrive
// completes the barrier without a second round trip.  The wait is bounded:
// after the spin limit the CTA raises the error word, which the others see
// and leave too.  Returns false (in every thread of the CTA) on error.
__device__ bool grid_sync(GridBarrier* b, uint32_t nblocks, uint32_t& epoch)
{
    __shared__ int ok;
    ++epoch;
    __syncthreads();  // the CTA's writes of this phase precede thread 0's release
    if (threadIdx.x == 0) {
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> err(b->error);
        const uint32_t target = epoch * nblocks;
        const uint64_t limit = b->spin_limit ? (uint64_t)b->spin_limit : kSpinLimit;
        int good = err.load(cuda::memory_order_relaxed) == 0;
        bar_arrive(&b->count);
        uint64_t spins = 0;
        while (good && (int32_t)(bar_poll(&b->count) - target) < 0) {
            if ((++spins & 63u) == 0 && err.load(cuda::memory_order_relaxed) != 0) good = 0;
            else if (spins > limit) {
                err.store(1u, cuda::memory_order_relaxed);
                good = 0;
            } else {
                __nanosleep(20);
            }
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// CTA-level sum, then the grid total from all CTAs' partials: every CTA sums
// the same partials in the same order (lane l takes CTAs l, l + 32, ... in
// order, then a fixed shuffle tree), so all agree without another barrier.
// A lane's partials are loaded together before they are summed.
template <class D, int NV, int PF = kPrefetch>
__device__ bool grid_total_of(typename D::T (&v)[NV], typename D::T* part, GridBarrier* bar, uint32_t nblocks,
                              uint32_t& epoch)
{
    typedef typename D::T T;
    __shared__ T wsum[NV][kMaxWarps];
    __shared__ T tot[NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int off = 16; off > 0; off >>= 1) v[k] = D::combine(v[k], D::shfl(v[k], off));
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) wsum[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            T a = wsum[k][0];
            for (int w = 1; w < nwarps; ++w) a = D::combine(a, wsum[k][w]);
            part[blockIdx.x * NV + k] = a;
        }
    }
    if (!grid_sync(bar, nblocks, epoch)) return false;
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            T buf[PF];
#pragma unroll
            for (int m = 0; m < PF; ++m) {
                const uint32_t b = lane + 32u * m;
                buf[m] = b < nblocks ? D::load(part + b * NV + k) : D::zero();
            }
            T a = D::zero();
#pragma unroll
            for (int m = 0; m < PF; ++m)
                if (lane + 32u * m < nblocks) a = D::combine(a, buf[m]);
            for (uint32_t b = lane + 32u * PF; b < nblocks; b += 32) a = D::combine(a, D::load(part + b * NV + k));
            for (int off = 16; off > 0; off >>= 1) a = D::combine(a, D::shfl(a, off));
            if (lane == 0) tot[k] = a;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = tot[k];
    return true;
}

template <int DOT, int NV>
__device__ __forceinline__ bool grid_total(typename DotT<DOT>::T (&v)[NV], typename DotT<DOT>::T* part,
                                           GridBarrier* bar, uint32_t nblocks, uint32_t& epoch)
{
    return grid_total_of<DotT<DOT>, NV>(v, part, bar, nblocks, epoch);
}

// The row of a one-row thread, kept in registers for the whole solve: its
// SELL base, degree and column indices (they never change during a solve).
constexpr int kRegCols = 16;
struct RegRow {
    uint32_t base, deg;
    uint32_t col[kRegCols];
};

__device__ __forceinline__ void load_reg_row(const ClothDev& c, uint32_t row, RegRow& rr)
{
    rr.base = rbase(c, row);
    rr.deg = c.row_deg[row];
#pragma unroll
    for (int k = 0; k < kRegCols; ++k) rr.col[k] = (uint32_t)k < rr.deg ? c.cols[rr.base + 32u * k] : row;
}

// row_times_direction with the row's columns already in registers: every
// load of the row (blocks, neighbours' z and p_old) is issued at once.
// SMEM_A: the row's blocks come from the thread's shared-memory column.
template <bool SMEM_A>
__device__ __forceinline__ f3 reg_row_times_direction(const ClothDev& c, const RegRow& rr, const float* z,
                                                      const float* pold, float beta, bool first, const float* sa,
                                                      uint32_t B, uint32_t tid)
{
    const uint32_t n = c.n;
    f3 acc = zero3();
#pragma unroll
    for (int k = 0; k < kRegCols; ++k) {
        if ((uint32_t)k < rr.deg) {
            const m3 a = SMEM_A ? smem_block(sa, (uint32_t)k, B, tid) : block_at(c, rr.base + 32u * k);
            const uint32_t j = rr.col[k];
            const f3 zj = ld3_l2(z, n, j);
            const f3 pj = first ? zj : zj + beta * ld3_l2(pold, n, j);
            acc = acc + a * pj;
        }
    }
    return acc;
}

// One CG iteration is two phases, each ended by a grid reduction:
//   A: p = z + beta p_old (own rows, stored), s = S A p (neighbours' p formed
//      on the fly), p.s                                   -> alpha
//   B: x += alpha p, r -= alpha s, z = S P^-1 r, r.z     -> delta', beta
// p alternates between two buffers so that phase A of one iteration never
// overwrites a direction another CTA is still reading.  ONE_ROW: every
// thread owns at most one row of at most kRegCols blocks and keeps its
// columns and its x, r, z, p and P^-1 in registers for the whole solve;
// only what neighbours read (z, p) and the solution go to memory.
// SMEM_A (one-row form only): the CTA's rows' blocks are copied into shared
// memory at the start, [slot][component][thread], and every later product
// reads them there; only the neighbours' z and p come from L2.
template <int DOT, bool ONE_ROW, bool SMEM_A>
__global__ void __launch_bounds__(kMaxBlock) k_grid_cg(const __grid_constant__ ClothDev c, GridBarrier* bar)
{
    extern __shared__ float smem_a[];
    const uint32_t B = blockDim.x, tid = threadIdx.x;
    typedef DotT<DOT> D;
    typedef typename D::T T;
    StepScalars* sc = c.sc;
    const uint32_t n = c.n;
    const uint32_t nb = gridDim.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t first_row = blockIdx.x * blockDim.x + threadIdx.x;
    // two alternating partial buffers: one is read while the next is written
    T* part0 = reinterpret_cast<T*>(c.partials);
    T* part1 = part0 + 2 * nb;
    const uint32_t max_iter = sc->max_iter;
    uint32_t epoch = 0;

    const bool act = first_row < n;
    bool Si = false;
    RegRow rr;
    f3 x = zero3(), r = zero3(), z = zero3(), pv = zero3(), p = zero3();
    if (ONE_ROW && act) load_reg_row(c, first_row, rr);
    if (SMEM_A && act) stage_row_blocks(c, rr.base, rr.deg, smem_a, B, tid);

    // x0 = S m_x, r = S (b - A x0), z = S P^-1 r (cloth_force_solver.cpp:90-100);
    // the soft body's MPCG (cg_soft) starts from x0 on every row and takes
    // b_delta = Sb . diag(A) Sb (softbody_force_solver.cpp:93-127)
    T v2[2] = {D::zero(), D::zero()};
    for (uint32_t row = first_row; row < n; row += stride) {
        const bool Sr = dyn(c, row);
        f3 ax = zero3();
        if (ONE_ROW) {
#pragma unroll
            for (int k = 0; k < kRegCols; ++k) {
                if ((uint32_t)k < rr.deg) {
                    const uint32_t col = rr.col[k];
                    const f3 xj = (c.cg_soft || dyn(c, col)) ? ld3(c.mx, n, col) : zero3();
                    ax = ax + block_at(c, rr.base + 32u * k) * xj;
                }
            }
        } else {
            const uint32_t base = rbase(c, row);
            const uint32_t deg = c.row_deg[row];
            for (uint32_t k = 0; k < deg; ++k) {
                const uint32_t idx = base + 32u * k;
                const uint32_t col = c.cols[idx];
                const f3 xj = (c.cg_soft || dyn(c, col)) ? ld3(c.mx, n, col) : zero3();
                ax = ax + block_at(c, idx) * xj;
            }
        }
        const f3 bi = ld3(c.b, n, row);
        const f3 pvr = ld3(c.pinv, n, row);
        const f3 rv = Sr ? bi - ax : zero3();
        const f3 zv = Sr ? mk(rv.x * pvr.x, rv.y * pvr.y, rv.z * pvr.z) : zero3();
        const f3 bh = Sr ? bi : zero3();
        const f3 x0 = (c.cg_soft || Sr) ? ld3(c.mx, n, row) : zero3();
        st3(c.z, n, row, zv);
        if (ONE_ROW) {
            Si = Sr, x = x0, r = rv, z = zv, pv = pvr;
        } else {
            st3(c.dv, n, row, x0);
            st3(c.r, n, row, rv);
        }
        const f3 w = c.cg_soft ? ld3(c.cg_diag, n, row) : pvr;
        v2[0] = D::add_term(v2[0], bh, mk(bh.x * w.x, bh.y * w.y, bh.z * w.z));
        v2[1] = D::add_term(v2[1], rv, zv);
        if (ONE_ROW) break;
    }
    if (!grid_total<DOT, 2>(v2, part0, bar, nb, epoch)) goto timeout;
    {
        double b_delta = D::value(v2[0]), delta = D::value(v2[1]);
        if (DOT != 2) {
            b_delta = (double)(float)b_delta;
            delta = (double)(float)delta;
        }
        const double delta0 = delta;
        uint32_t status = (!isfinite(delta) || !isfinite(b_delta)) ? kStatusNumerical : 0u;
        uint32_t it = 0;
        float beta = 0.0f;
        bool cont = status == 0 && max_iter > 0 && !cg_stop(sc, delta, b_delta);
        while (cont) {
            const bool first = it == 0;
            float* pnew = (it & 1u) ? c.p2 : c.p;
            const float* pold = (it & 1u) ? c.p : c.p2;
            // A: p = S (P^-1 r + beta p) (cloth_force_solver.cpp:130-131, folded
            // into the next SpMV), s = S A p, alpha = delta / p.s
            T v1[1] = {D::zero()};
            f3 s = zero3();
            if (ONE_ROW) {
                if (act) {
                    p = first ? z : z + beta * p;
                    const f3 ap = reg_row_times_direction<SMEM_A>(c, rr, c.z, pold, beta, first, smem_a, B, tid);
                    s = Si ? ap : zero3();
                    st3(pnew, n, first_row, p);
                    v1[0] = D::add_term(v1[0], p, s);
                }
            } else {
                for (uint32_t row = first_row; row < n; row += stride) {
                    const f3 zi = ld3(c.z, n, row);
                    const f3 pr = first ? zi : zi + beta * ld3(pold, n, row);
                    const f3 ap = row_times_direction(c, row, c.z, pold, beta, first);
                    const f3 sr = dyn(c, row) ? ap : zero3();
                    st3(pnew, n, row, pr);
                    st3(c.s, n, row, sr);
                    v1[0] = D::add_term(v1[0], pr, sr);
                }
            }
            if (!grid_total<DOT, 1>(v1, part1, bar, nb, epoch)) goto timeout;
            const double pAp = D::value(v1[0]);
            const float alpha = DOT == 2 ? (float)(delta / pAp) : (float)delta / (float)pAp;
            // B: x += alpha p, r -= alpha s, z = S P^-1 r, delta' = r.P^-1 r
            T u1[1] = {D::zero()};
            if (ONE_ROW) {
                if (act) {
                    x = x + alpha * p;
                    r = r - alpha * s;
                    const f3 h = mk(r.x * pv.x, r.y * pv.y, r.z * pv.z);
                    z = Si ? h : zero3();
                    st3(c.z, n, first_row, z);
                    u1[0] = D::add_term(u1[0], r, h);
                }
            } else {
                for (uint32_t row = first_row; row < n; row += stride) {
                    const f3 xr = ld3(c.dv, n, row) + alpha * ld3(pnew, n, row);
                    const f3 rv = ld3(c.r, n, row) - alpha * ld3(c.s, n, row);
                    const f3 pvr = ld3(c.pinv, n, row);
                    const f3 h = mk(rv.x * pvr.x, rv.y * pvr.y, rv.z * pvr.z);
                    st3(c.dv, n, row, xr);
                    st3(c.r, n, row, rv);
                    st3(c.z, n, row, dyn(c, row) ? h : zero3());
                    u1[0] = D::add_term(u1[0], rv, h);
                }
            }
            if (!grid_total<DOT, 1>(u1, part0, bar, nb, epoch)) goto timeout;
            double dn = D::value(u1[0]);
            if (DOT == 2) {
                beta = (float)(dn / delta);
            } else {
                dn = (double)(float)dn;
                beta = (float)dn / (float)delta;
            }
            delta = dn;
            ++it;
            if (!isfinite(dn) || !isfinite(alpha) || !isfinite(beta)) status = kStatusNumerical;
            cont = status == 0 && it < max_iter && !cg_stop(sc, dn, b_delta);
        }
        if (ONE_ROW && act) st3(c.dv, n, first_row, x);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            sc->b_delta = b_delta;
            sc->delta0 = delta0;
            sc->delta = delta;
            sc->iter = it;
            sc->status = status;
            sc->cont = 0;
        }
        return;
    }
timeout:
    if (threadIdx.x == 0) {
        sc->status = kStatusTimeout;
        sc->cont = 0;
    }
}

template <int DOT>
const void* grid_kernel(bool one_row, bool smem_a)
{
    if (!one_row) return (const void*)k_grid_cg<DOT, false, false>;
    return smem_a ? (const void*)k_grid_cg<DOT, true, true> : (const void*)k_grid_cg<DOT, true, false>;
}

// ---------------------------------------------------------------------------
// The fused form: one grid reduction per iteration
// ---------------------------------------------------------------------------
//
// Every vertex publishes, once per iteration, a record of its r, s and p and
// its S P^-1 (zero on rows that are not dynamic) as three float4:
// (r.xyz, s.x) (s.yz, p.xy) (p.z, SP^-1.xyz).  Records alternate between two
// buffers by iteration parity.
//
// A pass starts from everyone's record of the previous pass and that pass's
// alpha and beta.  Each row applies the previous update to itself,
//   x += alpha p,  r -= alpha s,  z = S P^-1 r,  p = z + beta p
// (cloth_force_solver.cpp:115-131), forms the same p for each neighbour it
// multiplies from the neighbour's record (the same float expressions, so
// every row sees bit-identical p), and computes s = S A p.  One reduction then
// gives four sums of the new iterate: p.s, s.z, s.P^-1 s and r.z.
//  - r.z is the reference's delta_new of this iterate, recomputed, not carried;
//    when it meets the stop rule the pass is discarded, as the reference would
//    stop before it.
//  - alpha = r.z / p.s, the reference's expression.
//  - The next delta is r'.z' for r' = r - alpha s, expanded:
//    r.z - 2 alpha s.z + alpha^2 s.P^-1 s.  It sets beta = delta' / r.z and
//    the stop test; the next pass recomputes it exactly.  So x, r, z and p
//    follow the reference's expressions, and only beta's numerator rounds
//    differently (by one iteration's rounding, never accumulated).
// The pass after the last accepted one applies nothing; the solution takes
// the last update itself.

struct Rec {
    f3 r, s, p, sp;
};

__device__ __forceinline__ Rec ld_rec(const float4* rec, uint32_t j)
{
    const float4 a = __ldcg(rec + 3 * (size_t)j), b = __ldcg(rec + 3 * (size_t)j + 1),
                 c = __ldcg(rec + 3 * (size_t)j + 2);
    return Rec{f3{a.x, a.y, a.z}, f3{a.w, b.x, b.y}, f3{b.z, b.w, c.x}, f3{c.y, c.z, c.w}};
}

__device__ __forceinline__ void st_rec(float4* rec, uint32_t j, f3 r, f3 s, f3 p, f3 sp)
{
    rec[3 * (size_t)j] = make_float4(r.x, r.y, r.z, s.x);
    rec[3 * (size_t)j + 1] = make_float4(s.y, s.z, p.x, p.y);
    rec[3 * (size_t)j + 2] = make_float4(p.z, sp.x, sp.y, sp.z);
}

__device__ __forceinline__ f3 hadamard(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }



// The direction of this pass at a vertex, from its record of the previous
// pass: the owner evaluates exactly this for its own row.
__device__ __forceinline__ f3 rec_direction(const Rec& q, float alpha, float beta, bool first)
{
    if (first) return hadamard(q.r, q.sp);
    const f3 rn = q.r - alpha * q.s;
    return hadamard(rn, q.sp) + beta * q.p;
}

// The sums of a fused pass, reduced together: p.s and r.z in the solve's
// dot precision (they give alpha and the exact delta, as the reference's
// float32 b3Dot would), s.z and s.P^-1 s always in FP64.  Those two only
// enter the expanded next delta, whose terms cancel; summed in FP32 their
// rounding would be magnified into beta.  The expansion also needs r.z to
// that accuracy: with FP32 dots an FP64 copy of it rides along (the
// compensated and FP64 sums carry it already).  32 bytes per CTA in every
// precision.
template <int DOT>
struct FusedStore {
    typename DotT<DOT>::T ps, rz;
    double sz, sps;
};
template <>
struct FusedStore<0> {
    float ps, rz;
    double sz, sps, rz64;
};

template <int DOT>
struct FusedSums {
    typedef DotT<DOT> P;
    typedef FusedStore<DOT> T;
    static __device__ T zero()
    {
        T a;
        a.ps = P::zero();
        a.rz = P::zero();
        a.sz = 0.0;
        a.sps = 0.0;
        if constexpr (DOT == 0) a.rz64 = 0.0;
        return a;
    }
    static __device__ T combine(T a, const T& b)
    {
        a.ps = P::combine(a.ps, b.ps);
        a.rz = P::combine(a.rz, b.rz);
        a.sz += b.sz;
        a.sps += b.sps;
        if constexpr (DOT == 0) a.rz64 += b.rz64;
        return a;
    }
    static __device__ T shfl(T a, int off)
    {
        a.ps = P::shfl(a.ps, off);
        a.rz = P::shfl(a.rz, off);
        a.sz = __shfl_down_sync(0xffffffffu, a.sz, off);
        a.sps = __shfl_down_sync(0xffffffffu, a.sps, off);
        if constexpr (DOT == 0) a.rz64 = __shfl_down_sync(0xffffffffu, a.rz64, off);
        return a;
    }
    static __device__ T load(const T* p)
    {
        T a;
        a.ps = P::load(&p->ps);
        a.rz = P::load(&p->rz);
        a.sz = __ldcg(&p->sz);
        a.sps = __ldcg(&p->sps);
        if constexpr (DOT == 0) a.rz64 = __ldcg(&p->rz64);
        return a;
    }
    static __device__ double dot64(f3 a, f3 b)
    {
        return (double)a.x * (double)b.x + (double)a.y * (double)b.y + (double)a.z * (double)b.z;
    }
    static __device__ void add(T& acc, f3 p, f3 s, f3 z, f3 r, f3 sp)
    {
        acc.ps = P::add_term(acc.ps, p, s);
        acc.rz = P::add_term(acc.rz, r, z);
        acc.sz += dot64(s, z);
        acc.sps += dot64(s, hadamard(s, sp));
        if constexpr (DOT == 0) acc.rz64 += dot64(r, z);
    }
    // r.z to FP64-like accuracy, for the expansion
    static __device__ double rz_exact(const T& a)
    {
        if constexpr (DOT == 0) return a.rz64;
        else return P::value(a.rz);
    }
};
static_assert(sizeof(FusedStore<0>) == 32 && sizeof(FusedStore<1>) == 32 && sizeof(FusedStore<2>) == 32,
              "fused partials: 32 bytes per CTA and parity");

// The scalars of one pass from its four sums.  Returns false when the true
// delta of the iterate (r.z) already meets the stop rule: the pass is then
// discarded.  DOT 0 and 1 round every scalar to float, as the reference's
// float32 b3Dot does.
template <int DOT>
__device__ __forceinline__ bool fused_scalars(const StepScalars* sc, double ps, double sz, double sps, double rz,
                                              double rz_exact, double b_delta, float& alpha, float& beta,
                                              double& delta_next, double& delta_true)
{
    if (DOT != 2) {
        ps = (double)(float)ps;
        rz = (double)(float)rz;
    }
    delta_true = rz;
    if (cg_stop(sc, rz, b_delta)) return false;
    alpha = DOT == 2 ? (float)(rz / ps) : (float)rz / (float)ps;
    const double a = (double)alpha;
    double dn = rz_exact - 2.0 * a * sz + a * a * sps;
    if (DOT != 2) dn = (double)(float)dn;
    delta_next = dn;
    beta = DOT == 2 ? (float)(dn / rz) : (float)dn / (float)rz;
    return true;
}

// SMEM_A (one-row form only): the CTA's rows' blocks are copied into shared
// memory at the start, [slot][component][thread], and every later product
// reads them there; only the neighbours' records come from L2.
template <int DOT, bool ONE_ROW, bool SMEM_A>
__global__ void __launch_bounds__(kMaxBlock) k_grid_cg_fused(const __grid_constant__ ClothDev c, GridBarrier* bar,
                                                             float4* rec0, float4* rec1)
{
    extern __shared__ float smem_a[];
    const uint32_t B = blockDim.x, tid = threadIdx.x;
    typedef DotT<DOT> D;
    typedef typename D::T T;
    StepScalars* sc = c.sc;
    const uint32_t n = c.n;
    const uint32_t nb = gridDim.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t first_row = blockIdx.x * blockDim.x + threadIdx.x;
    typedef FusedSums<DOT> F;
    typedef typename F::T FT;
    T* part_init = reinterpret_cast<T*>(c.partials);
    FT* part0 = reinterpret_cast<FT*>(c.partials);
    FT* part1 = part0 + nb;
    const uint32_t max_iter = sc->max_iter;
    uint32_t epoch = 0;

    const bool act = first_row < n;
    bool Si = false;
    RegRow rr;
    f3 x = zero3(), r = zero3(), s = zero3(), p = zero3(), sp = zero3();
    if (ONE_ROW && act) load_reg_row(c, first_row, rr);
    if (SMEM_A && act) stage_row_blocks(c, rr.base, rr.deg, smem_a, B, tid);

    // x0 = S m_x, r = S (b - A x0), b_delta, delta = r.S P^-1 r
    // (cloth_force_solver.cpp:90-100); record 0 holds r with s = p = 0.
    T v2[2] = {D::zero(), D::zero()};
    for (uint32_t row = first_row; row < n; row += stride) {
        const bool Sr = dyn(c, row);
        f3 ax = zero3();
        if (ONE_ROW) {
#pragma unroll
            for (int k = 0; k < kRegCols; ++k) {
                if ((uint32_t)k < rr.deg) {
                    const uint32_t col = rr.col[k];
                    const f3 xj = (c.cg_soft || dyn(c, col)) ? ld3(c.mx, n, col) : zero3();
                    const m3 a = block_at(c, rr.base + 32u * k);
                    ax = ax + a * xj;
                }
            }
        } else {
            const uint32_t base = rbase(c, row);
            const uint32_t deg = c.row_deg[row];
            for (uint32_t k = 0; k < deg; ++k) {
                const uint32_t idx = base + 32u * k;
                const uint32_t col = c.cols[idx];
                const f3 xj = (c.cg_soft || dyn(c, col)) ? ld3(c.mx, n, col) : zero3();
                ax = ax + block_at(c, idx) * xj;
            }
        }
        const f3 bi = ld3(c.b, n, row);
        const f3 pvr = ld3(c.pinv, n, row);
        const f3 rv = Sr ? bi - ax : zero3();
        const f3 spr = Sr ? pvr : zero3();
        const f3 zv = hadamard(rv, spr);
        const f3 bh = Sr ? bi : zero3();
        const f3 x0 = (c.cg_soft || Sr) ? ld3(c.mx, n, row) : zero3();
        st_rec(rec0, row, rv, zero3(), zero3(), spr);
        if (ONE_ROW) {
            Si = Sr, x = x0, r = rv, sp = spr;
        } else {
            st3(c.dv, n, row, x0);
        }
        const f3 w = c.cg_soft ? ld3(c.cg_diag, n, row) : pvr;
        v2[0] = D::add_term(v2[0], bh, mk(bh.x * w.x, bh.y * w.y, bh.z * w.z));
        v2[1] = D::add_term(v2[1], rv, zv);
        if (ONE_ROW) break;
    }
    if (!grid_total<DOT, 2>(v2, part_init, bar, nb, epoch)) goto timeout;
    {
        double b_delta = D::value(v2[0]), delta = D::value(v2[1]);
        if (DOT != 2) {
            b_delta = (double)(float)b_delta;
            delta = (double)(float)delta;
        }
        const double delta0 = delta;
        uint32_t status = (!isfinite(delta) || !isfinite(b_delta)) ? kStatusNumerical : 0u;
        uint32_t it = 0;
        float alpha = 0.0f, beta = 0.0f;
        bool pending = false;  // the last accepted pass's update of x is not applied yet
        bool cont = status == 0 && max_iter > 0 && !cg_stop(sc, delta, b_delta);
        while (cont) {
            const bool first = it == 0;
            const float4* rin = (it & 1u) ? rec1 : rec0;
            float4* rout = (it & 1u) ? rec0 : rec1;
            FT v4[1] = {F::zero()};
            if (ONE_ROW) {
                if (act) {
                    f3 z;
                    if (first) {
                        z = hadamard(r, sp);
                        p = z;
                    } else {
                        x = x + alpha * p;
                        r = r - alpha * s;
                        z = hadamard(r, sp);
                        p = z + beta * p;
                    }
                    // s = S A p; slot 0 is the row's own diagonal block
                    f3 acc = zero3() + (SMEM_A ? smem_block(smem_a, 0, B, tid) : block_at(c, rr.base)) * p;
#pragma unroll
                    for (int k = 1; k < kRegCols; ++k) {
                        if ((uint32_t)k < rr.deg) {
                            const m3 a = SMEM_A ? smem_block(smem_a, k, B, tid) : block_at(c, rr.base + 32u * k);
                            const Rec q = ld_rec(rin, rr.col[k]);
                            acc = acc + a * rec_direction(q, alpha, beta, first);
                        }
                    }
                    s = Si ? acc : zero3();
                    st_rec(rout, first_row, r, s, p, sp);
                    F::add(v4[0], p, s, z, r, sp);
                }
            } else {
                for (uint32_t row = first_row; row < n; row += stride) {
                    const Rec own = ld_rec(rin, row);
                    f3 rv = own.r, pv;
                    if (!first) {
                        st3(c.dv, n, row, ld3(c.dv, n, row) + alpha * own.p);
                        rv = own.r - alpha * own.s;
                    }
                    const f3 z = hadamard(rv, own.sp);
                    pv = first ? z : z + beta * own.p;
                    const uint32_t base = rbase(c, row);
                    const uint32_t deg = c.row_deg[row];
                    f3 acc = zero3() + block_at(c, base) * pv;
                    constexpr int W = 4;
                    for (uint32_t k0 = 1; k0 < deg; k0 += W) {
                        uint32_t cl[W];
#pragma unroll
                        for (int k = 0; k < W; ++k) cl[k] = (k0 + k < deg) ? c.cols[base + 32u * (k0 + k)] : 0u;
#pragma unroll
                        for (int k = 0; k < W; ++k) {
                            if (k0 + k < deg) {
                                const m3 a = block_at(c, base + 32u * (k0 + k));
                                const Rec q = ld_rec(rin, cl[k]);
                                acc = acc + a * rec_direction(q, alpha, beta, first);
                            }
                        }
                    }
                    const f3 sv = dyn(c, row) ? acc : zero3();
                    st_rec(rout, row, rv, sv, pv, own.sp);
                    F::add(v4[0], pv, sv, z, rv, own.sp);
                }
            }
            if (!grid_total_of<F, 1, kPrefetchFused>(v4, (it & 1u) ? part0 : part1, bar, nb, epoch)) goto timeout;
            double dn = 0.0, dt = 0.0;
            float a1 = 0.0f, b1 = 0.0f;
            const bool accept = fused_scalars<DOT>(sc, D::value(v4[0].ps), v4[0].sz, v4[0].sps, D::value(v4[0].rz),
                                                   F::rz_exact(v4[0]), b_delta, a1, b1, dn, dt);
            if (!accept) {
                // the iterate already meets the stop rule: the reference stops
                // before this pass; its x is the current one
                pending = false;
                delta = dt;
                break;
            }
            alpha = a1;
            beta = b1;
            pending = true;
            delta = dn;
            ++it;
            if (!isfinite(dn) || !isfinite(alpha) || !isfinite(beta)) status = kStatusNumerical;
            cont = status == 0 && it < max_iter && !cg_stop(sc, dn, b_delta);
        }
        // the last accepted update, x += alpha p
        if (ONE_ROW) {
            if (act) st3(c.dv, n, first_row, pending ? x + alpha * p : x);
        } else if (pending) {
            const float4* rl = (it & 1u) ? rec1 : rec0;
            for (uint32_t row = first_row; row < n; row += stride)
                st3(c.dv, n, row, ld3(c.dv, n, row) + alpha * ld_rec(rl, row).p);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            sc->b_delta = b_delta;
            sc->delta0 = delta0;
            sc->delta = delta;
            sc->iter = it;
            sc->status = status;
            sc->cont = 0;
        }
        return;
    }
timeout:
    if (threadIdx.x == 0) {
        sc->status = kStatusTimeout;
        sc->cont = 0;
    }
}

template <int DOT>
const void* fused_kernel(bool one_row, bool smem_a)
{
    if (!one_row) return (const void*)k_grid_cg_fused<DOT, false, false>;
    return smem_a ? (const void*)k_grid_cg_fused<DOT, true, true> : (const void*)k_grid_cg_fused<DOT, true, false>;
}

}  // namespace

GridCgShape grid_cg_shape(uint32_t n, int device, bool fused)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    GridCgShape g;
    const uint32_t rows_per_sm = (n + sms - 1) / (uint32_t)sms;
    if (rows_per_sm <= (uint32_t)kMaxBlock) {
        // one row per thread, at most one CTA per SM, rows spread evenly
        g.threads = (int)std::max<uint32_t>(32u, (rows_per_sm + 31u) & ~31u);
        g.blocks = (int)((n + g.threads - 1) / g.threads);
    } else {
        int per_sm = 1;
        const void* fn = fused ? (const void*)k_grid_cg_fused<2, false, false> : (const void*)k_grid_cg<2, false, false>;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kMaxBlock, 0) != cudaSuccess ||
            per_sm < 1) {
            cudaGetLastError();
            per_sm = 1;
        }
        g.threads = kMaxBlock;
        g.blocks = std::min(sms * per_sm, kMaxGridCgBlocks);
    }
    if (g.blocks < 1) g.blocks = 1;
    return g;
}

cudaError_t launch_grid_cg(const ClothDev& c, int dot, GridBarrier* bar, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const GridCgShape g = grid_cg_shape(c.n, dev, false);
    const bool one_row = (uint64_t)g.blocks * (uint64_t)g.threads >= c.n && c.max_deg <= (uint32_t)kRegCols;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g.blocks);
    cfg.blockDim = dim3(g.threads);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // the rows' blocks in shared memory when they fit beside the static
    // shared memory of the reductions
    const size_t smem = (size_t)c.max_deg * 9 * sizeof(float) * (size_t)g.threads;
    const bool smem_a = one_row && smem + 4096 <= kSmemLimit;
    const void* fn = dot == 2 ? grid_kernel<2>(one_row, smem_a)
                   : dot == 1 ? grid_kernel<1>(one_row, smem_a) : grid_kernel<0>(one_row, smem_a);
    if (smem_a) {
        cudaError_t ea = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (ea != cudaSuccess) return ea;
        cfg.dynamicSmemBytes = smem;
    }
    void* args[2] = {const_cast<ClothDev*>(&c), &bar};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
    count_launches(1);
    return e;
}

cudaError_t launch_grid_cg_fused(const ClothDev& c, int dot, GridBarrier* bar, float4* rec, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const GridCgShape g = grid_cg_shape(c.n, dev, true);
    const bool one_row = (uint64_t)g.blocks * (uint64_t)g.threads >= c.n && c.max_deg <= (uint32_t)kRegCols;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g.blocks);
    cfg.blockDim = dim3(g.threads);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // the rows' blocks in shared memory when they fit beside the static
    // shared memory of the reductions
    const size_t smem = (size_t)c.max_deg * 9 * sizeof(float) * (size_t)g.threads;
    const bool smem_a = one_row && smem + 4096 <= kSmemLimit;
    const void* fn = dot == 2 ? fused_kernel<2>(one_row, smem_a)
                   : dot == 1 ? fused_kernel<1>(one_row, smem_a) : fused_kernel<0>(one_row, smem_a);
    if (smem_a) {
        cudaError_t ea = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (ea != cudaSuccess) return ea;
        cfg.dynamicSmemBytes = smem;
    }
    float4* rec1 = rec + 3 * (size_t)c.n;
    void* args[4] = {const_cast<ClothDev*>(&c), &bar, &rec, &rec1};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
    count_launches(1);
    return e;
}

}  // namespace b3g
