// Batched MPCG: many cloths of uneven sizes in one persistent launch.
//
// A team -- one CTA, or a thread-block cluster of TEAM CTAs for large cloths
// -- takes a cloth from a work queue (largest first), runs the whole
// S-filtered Jacobi-preconditioned CG of that cloth (b3SolveMPCG,
// src/bounce/cloth/cloth_force_solver.cpp:61-136) with team-local
// barriers and reductions, then takes the next cloth.  No grid-wide
// synchronisation.  Within a team the reduction tree is fixed (thread ->
// warp shuffle -> CTA -> cluster ranks in order), so a cloth's result does
// not depend on which other cloths share the launch.
#include <cooperative_groups.h>

#include "batch.cuh"
#include "cg_common.cuh"
#include "cloth_dev.cuh"
#include "sell_spmv.cuh"
#include "vec.cuh"

namespace cgx = cooperative_groups;

namespace b3g {

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;

__device__ __forceinline__ uint32_t rbase(const ClothDev& c, uint32_t row)
{
    return c.slice_off[row >> 5] + (row & 31u);
}

// With a cluster team, p rows are written by other SMs within the launch; the
// SpMV reads them around L1 (sell_row_times<true>).

__device__ __forceinline__ bool dyn(const ClothDev& c, uint32_t i) { return c.type[i] == 2; }

// Team = TEAM CTAs of one cluster (TEAM == 1: the CTA alone).
template <int TEAM>
struct Team {
    __device__ static uint32_t rank()
    {
        if (TEAM == 1) return 0;
        return cgx::this_cluster().block_rank();
    }
    __device__ static void sync()
    {
        if (TEAM == 1) {
            __syncthreads();
        } else {
            // barrier.cluster.arrive releases and barrier.cluster.wait
            // acquires at cluster scope: this phase's global writes are
            // visible to the cluster's other CTAs after it, with no
            // device-wide fence
            cgx::this_cluster().sync();
        }
    }
};

// Sum of NV values over the team, identical in every thread.  `slot` is
// this CTA's shared buffer of NV partials (TEAM ranks read each other's).
// Callers alternate between two slot buffers: a rank writes a buffer again
// only two reductions later, after the barrier of the reduction in between,
// which every rank passes only once it has read the buffer.  So one team
// barrier per reduction suffices.
template <int TEAM, int DOT, int NV>
__device__ void team_sum(typename DotT<DOT>::T (&v)[NV], typename DotT<DOT>::T* wsum, typename DotT<DOT>::T* slot)
{
    typedef DotT<DOT> D;
    typedef typename D::T T;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int off = 16; off > 0; off >>= 1) v[k] = D::combine(v[k], D::shfl(v[k], off));
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) wsum[k * kWarps + warp] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            T a = wsum[k * kWarps];
            for (int w = 1; w < kWarps; ++w) a = D::combine(a, wsum[k * kWarps + w]);
            slot[k] = a;
        }
    }
    Team<TEAM>::sync();
    if (TEAM == 1) {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] = slot[k];
    } else {
        cgx::cluster_group cl = cgx::this_cluster();
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            T a = *cl.map_shared_rank(slot + k, 0);
            for (int r = 1; r < TEAM; ++r) a = D::combine(a, *cl.map_shared_rank(slot + k, r));
            v[k] = a;
        }
    }
}

// Row `row` of s = A p with the direction p = z + beta p_old formed on the fly
// from the neighbours' z = S P^-1 r and previous direction (first iteration:
// p = z), the same float expression each row's owner evaluates for its own
// p.  With a cluster team the neighbours' values come from other SMs and are
// read around L1.
template <bool L2ONLY>
__device__ __forceinline__ f3 row_times_direction(const ClothDev& c, uint32_t row, const float* pold, float beta,
                                                  bool first)
{
    constexpr int W = 8;  // blocks whose loads are issued together (85 registers: 3 CTAs per SM)
    const uint32_t base = rbase(c, row);
    const uint32_t deg = c.row_deg[row];
    const uint32_t n = c.n, E = c.E;
    const float* v = c.vals;
    const float* z = c.z;
    f3 acc = zero3();
    for (uint32_t k0 = 0; k0 < deg; k0 += W) {
        uint32_t cl[W];
#pragma unroll
        for (int k = 0; k < W; ++k) cl[k] = (k0 + k < deg) ? c.cols[base + 32u * (k0 + k)] : 0u;
#pragma unroll
        for (int k = 0; k < W; ++k) {
            if (k0 + k < deg) {
                const uint32_t idx = base + 32u * (k0 + k);
                const m3 a{f3{v[idx], v[E + idx], v[2 * E + idx]}, f3{v[3 * E + idx], v[4 * E + idx], v[5 * E + idx]},
                           f3{v[6 * E + idx], v[7 * E + idx], v[8 * E + idx]}};
                const uint32_t j = cl[k];
                const f3 zj = L2ONLY ? f3{__ldcg(z + j), __ldcg(z + n + j), __ldcg(z + 2 * n + j)}
                                     : f3{z[j], z[n + j], z[2 * n + j]};
                f3 pj = zj;
                if (!first) {
                    const f3 qj = L2ONLY ? f3{__ldcg(pold + j), __ldcg(pold + n + j), __ldcg(pold + 2 * n + j)}
                                         : f3{pold[j], pold[n + j], pold[2 * n + j]};
                    pj = zj + beta * qj;
                }
                acc = acc + a * pj;
            }
        }
    }
    return acc;
}

// The CG of one cloth by one team.  Rows are split into TEAM contiguous
// chunks; thread t of a CTA takes rows chunk_begin + t, + kBlock, ...  An
// iteration is two phases, each ended by a team reduction:
//   A: p = z + beta p_old (own rows), s = S A p, p.s          -> alpha
//   B: x += alpha p, r -= alpha s, z = S P^-1 r, r.z         -> beta
// with p alternating between two buffers (cloth_force_solver.cpp:61-136).
template <int TEAM, int DOT>
__device__ void team_cg(const ClothDev& c, typename DotT<DOT>::T* wsum, typename DotT<DOT>::T* slots)
{
    typedef DotT<DOT> D;
    typedef typename D::T T;
    StepScalars* sc = c.sc;
    const uint32_t n = c.n;
    const uint32_t chunk = (n + TEAM - 1) / TEAM;
    const uint32_t r0 = Team<TEAM>::rank() * chunk;
    const uint32_t r1 = min(n, r0 + chunk);
    const uint32_t max_iter = sc->max_iter;
    T* slot0 = slots;
    T* slot1 = slots + 2;

    // x0 = S m_x, r = S (b - A x0), z = S P^-1 r (cloth_force_solver.cpp:90-100)
    T v2[2] = {D::zero(), D::zero()};
    for (uint32_t row = r0 + threadIdx.x; row < r1; row += kBlock) {
        const bool Si = dyn(c, row);
        const uint32_t base = rbase(c, row);
        const uint32_t deg = c.row_deg[row];
        f3 ax = zero3();
        for (uint32_t k = 0; k < deg; ++k) {
            const uint32_t idx = base + 32u * k;
            const uint32_t col = c.cols[idx];
            const f3 xj = dyn(c, col) ? ld3(c.mx, n, col) : zero3();
            const float* v = c.vals;
            const uint32_t E = c.E;
            const m3 a{f3{v[idx], v[E + idx], v[2 * E + idx]}, f3{v[3 * E + idx], v[4 * E + idx], v[5 * E + idx]},
                       f3{v[6 * E + idx], v[7 * E + idx], v[8 * E + idx]}};
            ax = ax + a * xj;
        }
        const f3 bi = ld3(c.b, n, row);
        const f3 pv = ld3(c.pinv, n, row);
        const f3 r = Si ? bi - ax : zero3();
        const f3 z = Si ? mk(r.x * pv.x, r.y * pv.y, r.z * pv.z) : zero3();
        const f3 bh = Si ? bi : zero3();
        st3(c.dv, n, row, Si ? ld3(c.mx, n, row) : zero3());
        st3(c.r, n, row, r);
        st3(c.z, n, row, z);
        v2[0] = D::add_term(v2[0], bh, mk(bh.x * pv.x, bh.y * pv.y, bh.z * pv.z));
        v2[1] = D::add_term(v2[1], r, z);
    }
    team_sum<TEAM, DOT, 2>(v2, wsum, slot0);  // also orders the z writes before the first SpMV
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
        // A: p = S (P^-1 r + beta p), s = S A p, alpha = delta / p.s
        T v1[1] = {D::zero()};
        for (uint32_t row = r0 + threadIdx.x; row < r1; row += kBlock) {
            const f3 zi = ld3(c.z, n, row);
            const f3 p = first ? zi : zi + beta * ld3(pold, n, row);
            const f3 ap = row_times_direction<(TEAM > 1)>(c, row, pold, beta, first);
            const f3 s = dyn(c, row) ? ap : zero3();
            st3(pnew, n, row, p);
            st3(c.s, n, row, s);
            v1[0] = D::add_term(v1[0], p, s);
        }
        team_sum<TEAM, DOT, 1>(v1, wsum, slot1);
        const double pAp = D::value(v1[0]);
        const float alpha = DOT == 2 ? (float)(delta / pAp) : (float)delta / (float)pAp;
        // B: x += alpha p, r -= alpha s, z = S P^-1 r, delta' = r.P^-1 r
        T u1[1] = {D::zero()};
        for (uint32_t row = r0 + threadIdx.x; row < r1; row += kBlock) {
            const f3 x = ld3(c.dv, n, row) + alpha * ld3(pnew, n, row);
            const f3 r = ld3(c.r, n, row) - alpha * ld3(c.s, n, row);
            const f3 pv = ld3(c.pinv, n, row);
            const f3 h = mk(r.x * pv.x, r.y * pv.y, r.z * pv.z);
            st3(c.dv, n, row, x);
            st3(c.r, n, row, r);
            st3(c.z, n, row, dyn(c, row) ? h : zero3());
            u1[0] = D::add_term(u1[0], r, h);
        }
        team_sum<TEAM, DOT, 1>(u1, wsum, slot0);
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
    if (Team<TEAM>::rank() == 0 && threadIdx.x == 0) {
        sc->b_delta = b_delta;
        sc->delta0 = delta0;
        sc->delta = delta;
        sc->iter = it;
        sc->status = status;
        sc->cont = 0;
    }
}

// The CG of cloth `c` by a team of TEAM CTAs in the dot precision DOTSEL,
// or in the cloth's own precision when DOTSEL < 0 (a batch that mixes them;
// the three inlined instances then share one register budget).
template <int TEAM, int DOTSEL>
__device__ __forceinline__ void run_cg(const ClothDev& c, double* wsum, double* slot)
{
    CompF* wc = reinterpret_cast<CompF*>(wsum);
    CompF* sc = reinterpret_cast<CompF*>(slot);
    float* wf = reinterpret_cast<float*>(wsum);
    float* sf = reinterpret_cast<float*>(slot);
    if constexpr (DOTSEL == 2) {
        team_cg<TEAM, 2>(c, wsum, slot);
    } else if constexpr (DOTSEL == 1) {
        team_cg<TEAM, 1>(c, wc, sc);
    } else if constexpr (DOTSEL == 0) {
        team_cg<TEAM, 0>(c, wf, sf);
    } else {
        const int dot = c.sc->dot;
        if (dot == 2) team_cg<TEAM, 2>(c, wsum, slot);
        else if (dot == 1) team_cg<TEAM, 1>(c, wc, sc);
        else team_cg<TEAM, 0>(c, wf, sf);
    }
}

// One persistent launch with clusters of T CTAs.  A task is either one
// large cloth split over the cluster's T CTAs (team_cg<T>) or up to T small
// cloths, one per CTA (team_cg<1>, block-per-instance).  The host orders the
// tasks largest first; clusters take them from a queue.
template <int T, int DOTSEL>
__global__ void __launch_bounds__(kBlock, 3) k_batch_cg(const __grid_constant__ BatchCgArgs a)
{
    __shared__ double wsum[2 * kWarps];
    __shared__ double slot[4];  // two alternating reduction buffers of 2 values
    __shared__ uint32_t item;
    for (;;) {
        if (threadIdx.x == 0 && Team<T>::rank() == 0) item = atomicAdd(a.next, 1u);
        Team<T>::sync();
        uint32_t k;
        if (T == 1) k = item;
        else k = *cgx::this_cluster().map_shared_rank(&item, 0);
        Team<T>::sync();
        if (k >= a.ntasks) break;
        const uint2 task = a.tasks[k];  // (first index into order, count); count 0 = split
        if (task.y == 0) {
            run_cg<T, DOTSEL>(a.descs[a.order[task.x]], wsum, slot);
        } else {
            const uint32_t r = Team<T>::rank();
            if (r < task.y) run_cg<1, DOTSEL>(a.descs[a.order[task.x + r]], wsum, slot);
        }
        Team<T>::sync();
    }
}

template <int T>
const void* batch_kernel(int dot)
{
    switch (dot) {
        case 0: return (const void*)k_batch_cg<T, 0>;
        case 1: return (const void*)k_batch_cg<T, 1>;
        case 2: return (const void*)k_batch_cg<T, 2>;
        default: return (const void*)k_batch_cg<T, -1>;
    }
}

const void* batch_kernel_for(int team, int dot)
{
    switch (team) {
        case 1: return batch_kernel<1>(dot);
        case 2: return batch_kernel<2>(dot);
        case 4: return batch_kernel<4>(dot);
        case 8: return batch_kernel<8>(dot);
        default: return nullptr;
    }
}

}  // namespace

int batch_team_max_blocks(int team, int dot)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void* fn = batch_kernel_for(team, dot);
    if (!fn) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return sms * per_sm;
}

cudaError_t launch_batch_cg(const BatchCgArgs& a, int team, int dot, int grid_blocks, cudaStream_t st)
{
    if (!a.ntasks) return cudaSuccess;
    const void* fn = batch_kernel_for(team, dot);
    if (!fn) return cudaErrorInvalidValue;
    int blocks = grid_blocks > 0 ? grid_blocks : batch_team_max_blocks(team, dot);
    blocks = (blocks / team) * team;
    const int teams_needed = (int)a.ntasks;
    if (blocks / team > teams_needed) blocks = teams_needed * team;
    if (blocks < team) blocks = team;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = team;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[1] = {const_cast<BatchCgArgs*>(&a)};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
    count_launches(1);
    return e;
}

}  // namespace b3g
