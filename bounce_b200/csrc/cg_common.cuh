// Deterministic grid reductions for the CG inner products, in three
// precisions: FP32 (the reference accumulates b3Dot in float,
// include/bounce/sparse/dense_vec3.h:139-151), compensated FP32 (Neumaier
// per thread, TwoSum across threads) and FP64.  Every block writes one
// partial; the last block to take a ticket sums all partials in index order,
// so results do not depend on block scheduling.
#pragma once

#include <cfloat>
#include <cstdint>

#include "cloth_dev.cuh"
#include "vec.cuh"

namespace b3g {
namespace {

constexpr float kEps = FLT_EPSILON;  // B3_EPSILON (include/bounce/common/settings.h:42)
constexpr int kStatusNumerical = 6;

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------

// A partial sum in one of the three dot precisions.
struct CompF {
    float s, c;
};

template <int DOT> struct DotT;
template <> struct DotT<0> {
    typedef float T;
    static __device__ T zero() { return 0.0f; }
    static __device__ T add_term(T a, f3 x, f3 y) { return a + dot(x, y); }
    static __device__ T combine(T a, T b) { return a + b; }
    static __device__ double value(T a) { return (double)a; }
    static __device__ T shfl(T a, int off) { return __shfl_down_sync(0xffffffffu, a, off); }
    static __device__ T load(const T* p) { return __ldcg(p); }
};
template <> struct DotT<1> {
    typedef CompF T;
    static __device__ T zero() { return CompF{0.0f, 0.0f}; }
    // Neumaier step over the per-row terms
    static __device__ T add_term(T a, f3 x, f3 y)
    {
        float term = dot(x, y);
        float t = a.s + term;
        if (fabsf(a.s) >= fabsf(term)) a.c += (a.s - t) + term;
        else a.c += (term - t) + a.s;
        a.s = t;
        return a;
    }
    // TwoSum of the running sums, compensations added
    static __device__ T combine(T a, T b)
    {
        float s = a.s + b.s;
        float bp = s - a.s;
        float err = (a.s - (s - bp)) + (b.s - bp);
        return CompF{s, (a.c + b.c) + err};
    }
    static __device__ double value(T a) { return (double)(a.s + a.c); }
    static __device__ T shfl(T a, int off)
    {
        return CompF{__shfl_down_sync(0xffffffffu, a.s, off), __shfl_down_sync(0xffffffffu, a.c, off)};
    }
    static __device__ T load(const T* p) { return CompF{__ldcg(&p->s), __ldcg(&p->c)}; }
};
template <> struct DotT<2> {
    typedef double T;
    static __device__ T zero() { return 0.0; }
    static __device__ T add_term(T a, f3 x, f3 y)
    {
        return a + ((double)x.x * (double)y.x + (double)x.y * (double)y.y + (double)x.z * (double)y.z);
    }
    static __device__ T combine(T a, T b) { return a + b; }
    static __device__ double value(T a) { return a; }
    static __device__ T shfl(T a, int off) { return __shfl_down_sync(0xffffffffu, a, off); }
    static __device__ T load(const T* p) { return __ldcg(p); }
};

// Block-wide reduction of NV values; result valid in thread 0.
template <int DOT, int NV>
__device__ void block_reduce(typename DotT<DOT>::T (&v)[NV])
{
    typedef DotT<DOT> D;
    typedef typename D::T T;
    __shared__ T sh[NV][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int off = 16; off > 0; off >>= 1) v[k] = D::combine(v[k], D::shfl(v[k], off));
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            v[k] = lane < nwarps ? sh[k][lane] : D::zero();
            for (int off = 16; off > 0; off >>= 1) v[k] = D::combine(v[k], D::shfl(v[k], off));
        }
    }
    __syncthreads();
}

// Writes this block's partials; returns true (in every thread) in the last
// block to arrive, after which `v` holds the grid totals in thread 0.
template <int DOT, int NV>
__device__ bool grid_reduce(typename DotT<DOT>::T (&v)[NV], void* partials, uint32_t* ticket)
{
    typedef DotT<DOT> D;
    typedef typename D::T T;
    __shared__ bool last;
    block_reduce<DOT, NV>(v);
    T* part = reinterpret_cast<T*>(partials);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) part[blockIdx.x * NV + k] = v[k];
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    T acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = D::zero();
    for (uint32_t bi = threadIdx.x; bi < gridDim.x; bi += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] = D::combine(acc[k], D::load(part + bi * NV + k));
    block_reduce<DOT, NV>(acc);
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = acc[k];
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// CG stop rule (cloth_force_solver.cpp:105-113, or the relative tolerance)
__device__ bool cg_stop(const StepScalars* sc, double delta, double b_delta)
{
    if (sc->stop_rule == 0) {
        if (sc->dot == 2) return delta <= (double)(kEps * kEps) * b_delta;
        return (float)delta <= kEps * kEps * (float)b_delta;
    }
    return delta <= (double)sc->tol * (double)sc->tol * b_delta;
}

}  // namespace
}  // namespace b3g
