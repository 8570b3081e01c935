// Persistent whole-GPU MPCG of one cloth (grid_cg.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "cloth_dev.cuh"

namespace b3g {

// Software grid barrier state; zero before each launch.
struct GridBarrier {
    uint32_t count;
    uint32_t gen;
    uint32_t error;
    uint32_t spin_limit;  // polls before a waiting CTA gives up; 0: the built-in limit
};

int grid_cg_blocks(int device);
// Cooperative launch of `blocks` CTAs (at most grid_cg_blocks()); the cloth's
// partials buffer must hold 4 * blocks values of the dot type.
cudaError_t launch_grid_cg(const ClothDev& c, int dot, GridBarrier* bar, int blocks, cudaStream_t st);

}  // namespace b3g
