// Pieces of the standalone block-CSR MPCG shared by its entry points.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/b3g.h"
#include "cloth_dev.cuh"

namespace b3g {

struct CsrSystem {
    uint32_t n;
    const uint32_t* rowptr;
    const uint32_t* cols;
    const float* vals;   // 9 floats per block, column-major
    const float* b;      // xyz per row
    const float* S;      // 1 or 0 per row
    const float* x0;     // xyz per row
    float* x;            // xyz per row (output)
    // scratch
    float *pinv, *r, *p, *s;
    void* partials;
    StepScalars* sc;
    uint32_t grid, block;
    // 0: b3SolveMPCG of the cloth (cloth_force_solver.cpp:61-136): x = S x0,
    // b_delta = Sb . P^-1 Sb.  1: the soft body's (softbody_force_solver.cpp:
    // 93-164): x = x0 on every row, delta_0 = Sb . P Sb with P = diag(A).
    int softbody_mode;
};

inline size_t csr_align(size_t b) { return (b + 255) & ~size_t(255); }
size_t csr_scratch_bytes(uint32_t n, uint32_t grid);
void csr_bind_scratch(CsrSystem* s, char* base);
uint32_t csr_grid(uint32_t n);
b3g_status csr_validate(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const float* vals, const float* b,
                        const float* S, const float* x0, const b3g_solver_opts* o, float* x);
b3g_status csr_run(CsrSystem& s, const b3g_solver_opts* o, cudaStream_t st, StepScalars* host_sc);
void csr_report(const StepScalars& h, uint32_t* iterations, b3g_step_stats* stats);

}  // namespace b3g
