// Persistent MPCG of one large cloth on the whole GPU.
//
// b3SolveMPCG (src/bounce/cloth/cloth_force_solver.cpp:61-136) as a single
// cooperative launch: every CTA stays resident, the phases of an iteration
// (SpMV + p.s, update + r.P^-1 r, new direction) are separated by a software
// grid barrier instead of kernel boundaries, and each reduction is summed by
// every CTA from the per-CTA partials in index order, so all CTAs agree on
// alpha and beta without another barrier and the result is deterministic.
// Every wait on the barrier is bounded: after kSpinLimit polls the CTA sets
// the cloth's status to B3G_ERR_TIMEOUT and leaves, and so do the others.
#include <cuda/atomic>

#include "cg_common.cuh"
#include "cloth_dev.cuh"
#include "grid_cg.cuh"
#include "sell_spmv.cuh"
#include "vec.cuh"

namespace b3g {

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr uint64_t kSpinLimit = 1ull << 26;
constexpr uint32_t kStatusTimeout = 7;

__device__ __forceinline__ uint32_t rbase(const ClothDev& c, uint32_t row)
{
    return c.slice_off[row >> 5] + (row & 31u);
}

__device__ __forceinline__ bool dyn(const ClothDev& c, uint32_t i) { return c.type[i] == 2; }

// p is rewritten by other CTAs inside the launch: read it around L1.
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

// Sense-counting grid barrier with a bounded wait.  Returns false (in every
// thread of the CTA) once any CTA has given up.
__device__ bool grid_sync(GridBarrier* b, uint32_t nblocks)
{
    __shared__ int ok;
    // every thread's writes of this phase become visible device-wide first
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> gen(b->gen);
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> count(b->count);
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> err(b->error);
        const uint32_t g = gen.load(cuda::memory_order_acquire);
        const uint64_t limit = b->spin_limit ? (uint64_t)b->spin_limit : kSpinLimit;
        int good = err.load(cuda::memory_order_relaxed) == 0;
        if (count.fetch_add(1u, cuda::memory_order_acq_rel) == nblocks - 1) {
            count.store(0u, cuda::memory_order_relaxed);
            gen.store(g + 1u, cuda::memory_order_release);
        } else {
            uint64_t spins = 0;
            while (gen.load(cuda::memory_order_acquire) == g) {
                if (err.load(cuda::memory_order_relaxed) != 0) {
                    good = 0;
                    break;
                }
                if (++spins > limit) {
                    err.store(1u, cuda::memory_order_relaxed);
                    good = 0;
                    break;
                }
                __nanosleep(20);
            }
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// CTA-level sum, then the grid total from all CTAs' partials (every CTA
// computes the same value from the same partials in the same order).
template <int DOT, int NV>
__device__ bool grid_total(typename DotT<DOT>::T (&v)[NV], typename DotT<DOT>::T* part, GridBarrier* bar,
                           uint32_t nblocks)
{
    typedef DotT<DOT> D;
    typedef typename D::T T;
    __shared__ T wsum[NV][kWarps];
    __shared__ T tot[NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
            for (int w = 1; w < kWarps; ++w) a = D::combine(a, wsum[k][w]);
            part[blockIdx.x * NV + k] = a;
        }
    }
    if (!grid_sync(bar, nblocks)) return false;
    // warp 0 sums the partials: lane l takes blocks l, l + 32, ... in order,
    // then the 32 lane sums combine in a fixed tree
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            T a = D::zero();
            for (uint32_t b = lane; b < nblocks; b += 32) a = D::combine(a, D::load(part + b * NV + k));
            for (int off = 16; off > 0; off >>= 1) a = D::combine(a, D::shfl(a, off));
            if (lane == 0) tot[k] = a;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = tot[k];
    return true;
}

template <int DOT>
__global__ void __launch_bounds__(kBlock) k_grid_cg(const __grid_constant__ ClothDev c, GridBarrier* bar)
{
    typedef DotT<DOT> D;
    typedef typename D::T T;
    StepScalars* sc = c.sc;
    const uint32_t n = c.n;
    const uint32_t nb = gridDim.x;
    const uint32_t stride = gridDim.x * kBlock;
    const uint32_t first = blockIdx.x * kBlock + threadIdx.x;
    // two alternating partial buffers: one is read while the next is written
    T* part0 = reinterpret_cast<T*>(c.partials);
    T* part1 = part0 + 2 * nb;
    const uint32_t max_iter = sc->max_iter;

    T v2[2] = {D::zero(), D::zero()};
    for (uint32_t row = first; row < n; row += stride) {
        const bool Si = dyn(c, row);
        const uint32_t base = rbase(c, row);
        const uint32_t deg = c.row_deg[row];
        f3 ax = zero3();
        for (uint32_t k = 0; k < deg; ++k) {
            const uint32_t idx = base + 32u * k;
            const uint32_t col = c.cols[idx];
            const f3 xj = dyn(c, col) ? ld3(c.mx, n, col) : zero3();
            ax = ax + block_at(c, idx) * xj;
        }
        const f3 bi = ld3(c.b, n, row);
        const f3 pv = ld3(c.pinv, n, row);
        const f3 r = Si ? bi - ax : zero3();
        const f3 p = Si ? mk(r.x * pv.x, r.y * pv.y, r.z * pv.z) : zero3();
        const f3 bh = Si ? bi : zero3();
        st3(c.dv, n, row, Si ? ld3(c.mx, n, row) : zero3());
        st3(c.r, n, row, r);
        st3(c.p, n, row, p);
        v2[0] = D::add_term(v2[0], bh, mk(bh.x * pv.x, bh.y * pv.y, bh.z * pv.z));
        v2[1] = D::add_term(v2[1], r, p);
    }
    if (!grid_total<DOT, 2>(v2, part0, bar, nb)) goto timeout;
    {
        double b_delta = D::value(v2[0]), delta = D::value(v2[1]);
        if (DOT != 2) {
            b_delta = (double)(float)b_delta;
            delta = (double)(float)delta;
        }
        const double delta0 = delta;
        uint32_t status = (!isfinite(delta) || !isfinite(b_delta)) ? kStatusNumerical : 0u;
        uint32_t it = 0;
        bool cont = status == 0 && max_iter > 0 && !cg_stop(sc, delta, b_delta);
        while (cont) {
            T v1[1] = {D::zero()};
            for (uint32_t row = first; row < n; row += stride) {
                const f3 ap = sell_row_times<true>(c, row, c.p);
                const f3 s = dyn(c, row) ? ap : zero3();
                st3(c.s, n, row, s);
                v1[0] = D::add_term(v1[0], ld3(c.p, n, row), s);
            }
            if (!grid_total<DOT, 1>(v1, part1, bar, nb)) goto timeout;
            const double pAp = D::value(v1[0]);
            const float alpha = DOT == 2 ? (float)(delta / pAp) : (float)delta / (float)pAp;
            T u1[1] = {D::zero()};
            for (uint32_t row = first; row < n; row += stride) {
                const f3 x = ld3(c.dv, n, row) + alpha * ld3(c.p, n, row);
                const f3 r = ld3(c.r, n, row) - alpha * ld3(c.s, n, row);
                const f3 pv = ld3(c.pinv, n, row);
                st3(c.dv, n, row, x);
                st3(c.r, n, row, r);
                u1[0] = D::add_term(u1[0], r, mk(r.x * pv.x, r.y * pv.y, r.z * pv.z));
            }
            if (!grid_total<DOT, 1>(u1, part0, bar, nb)) goto timeout;
            double dn = D::value(u1[0]);
            float beta;
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
            if (!cont) break;
            for (uint32_t row = first; row < n; row += stride) {
                const f3 r = ld3(c.r, n, row);
                const f3 pv = ld3(c.pinv, n, row);
                const f3 hv = mk(r.x * pv.x, r.y * pv.y, r.z * pv.z);
                st3(c.p, n, row, dyn(c, row) ? hv + beta * ld3(c.p, n, row) : zero3());
            }
            if (!grid_sync(bar, nb)) goto timeout;
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

}  // namespace

int grid_cg_blocks(int device)
{
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_cg<2>, kBlock, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return sms * per_sm;
}

cudaError_t launch_grid_cg(const ClothDev& c, int dot, GridBarrier* bar, int blocks, cudaStream_t st)
{
    // no more CTAs than row groups: idle CTAs would only add barrier arrivals
    const int need = (int)((c.n + kBlock - 1) / kBlock);
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kBlock);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    if (dot == 2) e = cudaLaunchKernelEx(&cfg, k_grid_cg<2>, c, bar);
    else if (dot == 1) e = cudaLaunchKernelEx(&cfg, k_grid_cg<1>, c, bar);
    else e = cudaLaunchKernelEx(&cfg, k_grid_cg<0>, c, bar);
    count_launches(1);
    return e;
}

}  // namespace b3g
