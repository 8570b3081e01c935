// Persistent whole-GPU MPCG of one cloth (grid_cg.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "cloth_dev.cuh"

namespace b3g {

// Software grid barrier state; zero before each launch.
struct GridBarrier {
    uint32_t count;       // CTA arrivals since the launch began
    uint32_t reserved;
    uint32_t error;
    uint32_t spin_limit;  // polls before a waiting CTA gives up; 0: the built-in limit
};

// Upper bound on the CTAs of one persistent CG launch; the cloth's partials
// buffer holds 8 values of the widest dot type (8 bytes) per CTA: two
// alternating sets of up to four sums.
constexpr int kMaxGridCgBlocks = 1024;
constexpr size_t kGridCgPartialBytes = (size_t)kMaxGridCgBlocks * 64;

struct GridCgShape {
    int blocks, threads;
};
GridCgShape grid_cg_shape(uint32_t n, int device, bool fused);
// Cooperative launch over the current device, shaped by grid_cg_shape():
// two grid reductions per iteration.
cudaError_t launch_grid_cg(const ClothDev& c, int dot, GridBarrier* bar, cudaStream_t st);
// The fused form, one grid reduction per iteration; slot 0 of every row must
// hold the row's diagonal block (it multiplies the row's own direction,
// formed in registers).  `rec`: device scratch
// of grid_cg_fused_rec_bytes(n) bytes, 16-byte aligned (the per-vertex
// records of two consecutive iterations).
cudaError_t launch_grid_cg_fused(const ClothDev& c, int dot, GridBarrier* bar, float4* rec, cudaStream_t st);
inline size_t grid_cg_fused_rec_bytes(uint32_t n) { return 2 * 3 * sizeof(float4) * (size_t)n; }


}  // namespace b3g
