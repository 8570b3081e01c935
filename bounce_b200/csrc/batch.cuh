// Batched stepping of many cloths (batch_cg.cu, batch_api.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "cloth_dev.cuh"

namespace b3g {

struct BatchCgArgs {
    const ClothDev* descs;   // cloth descriptors of the launch
    const uint32_t* order;   // cloth indices, task-grouped, largest first
    const uint2* tasks;      // (first index into order, count); count 0: one cloth split over the cluster
    uint32_t ntasks;
    uint32_t* next;          // work-queue counter, zero at launch
};

// Clusters of `team` CTAs (1, 2, 4 or 8); grid_blocks <= 0 fills the GPU.
// dot: the dot precision (0, 1, 2) every cloth of the launch uses, or -1 when
// they differ (each cloth's own setting is then read on the device).
cudaError_t launch_batch_cg(const BatchCgArgs& a, int team, int dot, int grid_blocks, cudaStream_t st);
int batch_team_max_blocks(int team, int dot);

}  // namespace b3g
