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
// buffer holds 4 values of the widest dot type (8 bytes) per CTA.
constexpr int kMaxGridCgBlocks = 1024;
constexpr size_t kGridCgPartialBytes = (size_t)kMaxGridCgBlocks * 32;

struct GridCgShape {
    int blocks, threads;
};
GridCgShape grid_cg_shape(uint32_t n, int device);
// Cooperative launch over the current device, shaped by grid_cg_shape().
cudaError_t launch_grid_cg(const ClothDev& c, int dot, GridBarrier* bar, cudaStream_t st);

}  // namespace b3g
