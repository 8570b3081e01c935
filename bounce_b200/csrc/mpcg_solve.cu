// Standalone MPCG on a caller-supplied block-CSR system in device memory:
// b3SolveMPCG (src/bounce/cloth/cloth_force_solver.cpp:61-136) -- Jacobi
// preconditioner from the diagonal blocks, S-filtered CG from x = S x0,
// stop at the iteration cap or at the stop rule.  Vectors are xyz per row
// (b3DenseVec3 layout); S holds one 1/0 per row.
#include <cstring>
#include <mutex>

#include "../../include/b3g.h"
#include "cg_common.cuh"
#include "cloth_dev.cuh"
#include "mpcg_solve.cuh"
#include "vec.cuh"

namespace b3g {

namespace {

__device__ __forceinline__ f3 ldv(const float* p, uint32_t i) { return f3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void stv(float* p, uint32_t i, f3 v)
{
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
__device__ __forceinline__ m3 ldm(const float* v, uint32_t k)
{
    const float* q = v + 9 * (size_t)k;
    return m3{f3{q[0], q[1], q[2]}, f3{q[3], q[4], q[5]}, f3{q[6], q[7], q[8]}};
}
__device__ __forceinline__ bool Sf(const CsrSystem& s, uint32_t i) { return s.S[i] != 0.0f; }

// P^-1 from the diagonal block, x = S x0, r = S (b - A x), p = S P^-1 r,
// b_delta and delta (cloth_force_solver.cpp:70-100).
template <int DOT>
__global__ void k_csr_init(CsrSystem s)
{
    typedef DotT<DOT> D;
    typename D::T v[2] = {D::zero(), D::zero()};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x) {
        const bool Si = Sf(s, i);
        f3 ax = zero3();
        m3 diag = mzero();
        for (uint32_t k = s.rowptr[i]; k < s.rowptr[i + 1]; ++k) {
            const uint32_t j = s.cols[k];
            const m3 a = ldm(s.vals, k);
            if (j == i) diag = a;
            const f3 xj = (s.softbody_mode || Sf(s, j)) ? ldv(s.x0, j) : zero3();
            ax = ax + a * xj;
        }
        const f3 pv = mk(1.0f / diag.x.x, 1.0f / diag.y.y, 1.0f / diag.z.z);
        const f3 bi = ldv(s.b, i);
        const f3 r = Si ? bi - ax : zero3();
        const f3 p = Si ? mk(r.x * pv.x, r.y * pv.y, r.z * pv.z) : zero3();
        const f3 bh = Si ? bi : zero3();
        stv(s.pinv, i, pv);
        stv(s.x, i, (s.softbody_mode || Si) ? ldv(s.x0, i) : zero3());
        stv(s.r, i, r);
        stv(s.p, i, p);
        const f3 w = s.softbody_mode ? mk(diag.x.x, diag.y.y, diag.z.z) : pv;
        v[0] = D::add_term(v[0], bh, mk(bh.x * w.x, bh.y * w.y, bh.z * w.z));
        v[1] = D::add_term(v[1], r, p);
    }
    if (grid_reduce<DOT, 2>(v, s.partials, &s.sc->ticket[0]) && threadIdx.x == 0) {
        StepScalars* sc = s.sc;
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
    }
}

// s = S A p and p.s, launched with four times the other kernels' threads
// per block (same grid, so the same reduction partials).  Four lanes share a
// row: lane g sums the row's blocks
// g, g + 4, ... (neighbouring lanes read neighbouring blocks, so the block
// loads coalesce), then the four partial sums combine as (0 + 1) + (2 + 3).
template <int DOT>
__global__ void __launch_bounds__(1024) k_csr_spmv(CsrSystem s)
{
    typedef DotT<DOT> D;
    if (s.sc->cont == 0u) return;
    typename D::T v[1] = {D::zero()};
    const uint32_t lane = threadIdx.x & 31u, g = lane & 3u;
    const unsigned mask = 0xFu << (lane & ~3u);
    const uint32_t stride = (gridDim.x * blockDim.x) >> 2;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 2; i < s.n; i += stride) {
        f3 ap = zero3();
        const uint32_t k1 = s.rowptr[i + 1];
        for (uint32_t k = s.rowptr[i] + g; k < k1; k += 4u) ap = ap + ldm(s.vals, k) * ldv(s.p, s.cols[k]);
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            ap.x += __shfl_xor_sync(mask, ap.x, o);
            ap.y += __shfl_xor_sync(mask, ap.y, o);
            ap.z += __shfl_xor_sync(mask, ap.z, o);
        }
        if (g == 0) {
            const f3 sv = Sf(s, i) ? ap : zero3();
            stv(s.s, i, sv);
            v[0] = D::add_term(v[0], ldv(s.p, i), sv);
        }
    }
    if (grid_reduce<DOT, 1>(v, s.partials, &s.sc->ticket[1]) && threadIdx.x == 0) {
        StepScalars* sc = s.sc;
        const double pAp = D::value(v[0]);
        sc->pAp = pAp;
        sc->alpha = DOT == 2 ? (float)(sc->delta / pAp) : (float)sc->delta / (float)pAp;
    }
}

template <int DOT>
__global__ void k_csr_update(CsrSystem s)
{
    typedef DotT<DOT> D;
    if (s.sc->cont == 0u) return;
    typename D::T v[1] = {D::zero()};
    const float alpha = s.sc->alpha;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x) {
        const f3 x = ldv(s.x, i) + alpha * ldv(s.p, i);
        const f3 r = ldv(s.r, i) - alpha * ldv(s.s, i);
        const f3 pv = ldv(s.pinv, i);
        stv(s.x, i, x);
        stv(s.r, i, r);
        v[0] = D::add_term(v[0], r, mk(r.x * pv.x, r.y * pv.y, r.z * pv.z));
    }
    if (grid_reduce<DOT, 1>(v, s.partials, &s.sc->ticket[2]) && threadIdx.x == 0) {
        StepScalars* sc = s.sc;
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
    }
}

__global__ void k_csr_direction(CsrSystem s)
{
    if (s.sc->cont == 0u) return;
    const float beta = s.sc->beta;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x) {
        const f3 r = ldv(s.r, i);
        const f3 pv = ldv(s.pinv, i);
        const f3 h = mk(r.x * pv.x, r.y * pv.y, r.z * pv.z);
        stv(s.p, i, Sf(s, i) ? h + beta * ldv(s.p, i) : zero3());
    }
}

template <int DOT>
cudaError_t launch_all(const CsrSystem& s, uint32_t max_iter, cudaStream_t st)
{
    k_csr_init<DOT><<<s.grid, s.block, 0, st>>>(s);
    for (uint32_t k = 0; k < max_iter; ++k) {
        k_csr_spmv<DOT><<<s.grid, 4 * s.block, 0, st>>>(s);  // four lanes per row, one partial per block
        k_csr_update<DOT><<<s.grid, s.block, 0, st>>>(s);
        k_csr_direction<<<s.grid, s.block, 0, st>>>(s);
    }
    count_launches(1 + 3ull * max_iter);
    return cudaGetLastError();
}

}  // namespace

size_t csr_scratch_bytes(uint32_t n, uint32_t grid)
{
    return csr_align(4 * 3 * (size_t)n * sizeof(float)) + csr_align((size_t)grid * 32) + csr_align(sizeof(StepScalars));
}

void csr_bind_scratch(CsrSystem* s, char* base)
{
    const size_t vec = 3 * (size_t)s->n;
    float* f = reinterpret_cast<float*>(base);
    s->pinv = f;
    s->r = f + vec;
    s->p = f + 2 * vec;
    s->s = f + 3 * vec;
    char* q = base + csr_align(4 * vec * sizeof(float));
    s->partials = q;
    q += csr_align((size_t)s->grid * 32);
    s->sc = reinterpret_cast<StepScalars*>(q);
}

uint32_t csr_grid(uint32_t n) { return std::min<uint32_t>((n + 255) / 256, 148 * 4) > 0 ? std::min<uint32_t>((n + 255) / 256, 148 * 4) : 1; }

b3g_status csr_validate(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals, const float* b,
                        const float* S, const float* x0, const b3g_solver_opts* o, float* x)
{
    if (n == 0 || !rowptr || !cols || !vals || !b || !S || !x0 || !o || !x) return B3G_ERR_INVALID_ARGUMENT;
    if (o->max_iterations < 1 || (o->stop_rule != B3G_STOP_REFERENCE && o->stop_rule != B3G_STOP_RELATIVE) ||
        (o->dot != B3G_DOT_F32 && o->dot != B3G_DOT_COMPENSATED && o->dot != B3G_DOT_F64))
        return B3G_ERR_INVALID_ARGUMENT;
    return B3G_OK;
}

// Runs the solve with scratch already bound; `host_sc` (pinned or pageable)
// receives the final scalars.  The scalar block is cleared first: scratch
// keeps whatever the previous user left in it.
b3g_status csr_run(CsrSystem& s, const b3g_solver_opts* o, cudaStream_t st, StepScalars* host_sc)
{
    StepScalars init;
    std::memset(&init, 0, sizeof(init));
    init.max_iter = o->max_iterations;
    init.stop_rule = (int)o->stop_rule;
    init.tol = o->tolerance;
    init.dot = (int)o->dot;
    cudaError_t e = cudaMemcpyAsync(s.sc, &init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if (o->dot == B3G_DOT_F32) e = launch_all<0>(s, o->max_iterations, st);
        else if (o->dot == B3G_DOT_COMPENSATED) e = launch_all<1>(s, o->max_iterations, st);
        else e = launch_all<2>(s, o->max_iterations, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_sc, s.sc, sizeof(StepScalars), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? B3G_ERR_OUT_OF_MEMORY : B3G_ERR_CUDA;
    }
    return B3G_OK;
}

void csr_report(const StepScalars& h, uint32_t* iterations, b3g_step_stats* stats)
{
    if (iterations) *iterations = h.iter;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->iterations = h.iter;
        stats->delta0 = h.delta0;
        stats->delta = h.delta;
        stats->b_delta = h.b_delta;
    }
}

}  // namespace b3g

using namespace b3g;

extern "C" b3g_status b3g_mpcg_solve(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals,
                                     const float* b, const float* S, const float* x0, const b3g_solver_opts* opts,
                                     float* x, uint32_t* iterations, b3g_step_stats* stats, void* stream)
{
    b3g_status v = csr_validate(n, rowptr, cols, vals, b, S, x0, opts, x);
    if (v != B3G_OK) return v;
    cudaStream_t st = (cudaStream_t)stream;
    CsrSystem s{};
    s.n = n;
    s.rowptr = rowptr;
    s.cols = cols;
    s.vals = vals;
    s.b = b;
    s.S = S;
    s.x0 = x0;
    s.x = x;
    s.block = 256;
    s.grid = csr_grid(n);
    char* scratch = nullptr;
    if (cudaMalloc(&scratch, csr_scratch_bytes(n, s.grid)) != cudaSuccess) {
        cudaGetLastError();
        return B3G_ERR_OUT_OF_MEMORY;
    }
    csr_bind_scratch(&s, scratch);
    StepScalars h;
    b3g_status r = csr_run(s, opts, st, &h);
    cudaFree(scratch);
    if (r != B3G_OK) return r;
    csr_report(h, iterations, stats);
    return h.status ? (b3g_status)h.status : B3G_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant
// ---------------------------------------------------------------------------
//
// Some callers cannot call cudaMalloc at solve time: a game or physics loop
// that reserves all of its device memory when a level loads and forbids
// allocation inside the frame (cudaMalloc can take milliseconds and
// synchronizes the device), a process whose device memory is already claimed
// up front by another framework's caching allocator, or code that runs the
// solver from inside its own allocator's callbacks.  For them the scratch
// (P^-1, r, p, s, the reduction partials and the CG scalars) lives in one
// file-scope device array, sized for systems of up to
// B3G_MPCG_NOALLOC_MAX_ROWS block rows, which every GPU that loads the library
// holds until the process exits.  The array's name is only a host-side
// stand-in in host code, so its device address is looked up once per device
// with cudaGetSymbolAddress, by the first call on that device, and kept for
// the life of the process: a cudaDeviceReset after that call is not
// supported, since the module and the array may then load at another address.

namespace b3g {
namespace {

constexpr uint32_t kNoAllocRows = B3G_MPCG_NOALLOC_MAX_ROWS;
constexpr uint32_t kNoAllocGrid = (kNoAllocRows + 255) / 256 < 148 * 4 ? (kNoAllocRows + 255) / 256 : 148 * 4;
constexpr size_t kNoAllocBytes = ((4ull * 3 * kNoAllocRows * sizeof(float) + 255) & ~size_t(255)) +
                                 ((kNoAllocGrid * 32ull + 255) & ~size_t(255)) +
                                 ((sizeof(StepScalars) + 255) & ~size_t(255));
constexpr int kNoAllocDevices = 64;

__device__ __align__(256) char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mutex;
char* g_noalloc_addr[kNoAllocDevices];

// Device address of the scratch array on the current device (looked up on
// first use of each device).
b3g_status noalloc_scratch(char** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return B3G_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= kNoAllocDevices) return B3G_ERR_CAPACITY;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? B3G_ERR_NO_DEVICE : B3G_ERR_CUDA;
        }
        g_noalloc_addr[dev] = static_cast<char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return B3G_OK;
}

}  // namespace
}  // namespace b3g

extern "C" b3g_status b3g_mpcg_solve_noalloc(uint32_t n, const uint32_t* rowptr, const uint32_t* cols,
                                             const float* vals, const float* b, const float* S, const float* x0,
                                             const b3g_solver_opts* opts, float* x, uint32_t* iterations,
                                             b3g_step_stats* stats, void* stream)
{
    b3g_status v = csr_validate(n, rowptr, cols, vals, b, S, x0, opts, x);
    if (v != B3G_OK) return v;
    if (n > kNoAllocRows) return B3G_ERR_CAPACITY;
    CsrSystem s{};
    s.n = n;
    s.rowptr = rowptr;
    s.cols = cols;
    s.vals = vals;
    s.b = b;
    s.S = S;
    s.x0 = x0;
    s.x = x;
    s.block = 256;
    s.grid = csr_grid(n);
    if (csr_scratch_bytes(n, s.grid) > kNoAllocBytes) return B3G_ERR_CAPACITY;
    char* scratch = nullptr;
    v = noalloc_scratch(&scratch);
    if (v != B3G_OK) return v;
    csr_bind_scratch(&s, scratch);
    // csr_run clears the CG scalars and reduction tickets before the first
    // kernel; every other scratch word is written before it is read.
    StepScalars h;
    b3g_status r = csr_run(s, opts, (cudaStream_t)stream, &h);
    if (r != B3G_OK) return r;
    csr_report(h, iterations, stats);
    return h.status ? (b3g_status)h.status : B3G_OK;
}
