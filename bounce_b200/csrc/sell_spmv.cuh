// One row of y = A q for the SELL-32 block matrix of a cloth.
//
// The row's column indices are loaded first (up to W at a time), then all
// its blocks and the gathered q values, so a thread has the whole row's
// loads in flight together instead of one block's at a time.  Blocks are
// still summed in slot order, acc = acc + A_k q_k, with A q evaluated like
// b3Mat33 * b3Vec3 (include/bounce/common/math/mat33.h:129-132).
#pragma once

#include "cloth_dev.cuh"
#include "vec.cuh"

namespace b3g {

// L2ONLY: q is rewritten by other SMs during the same launch, so its loads
// go around L1 (ld.global.cg).  W: blocks whose loads are issued together
// (16 covers a whole row of a cloth with bending; 8 keeps kernels that must
// stay at 64 registers free of spills).
template <bool L2ONLY, int W = 16>
__device__ __forceinline__ f3 sell_row_times(const ClothDev& c, uint32_t row, const float* q)
{
    const uint32_t base = c.slice_off[row >> 5] + (row & 31u);
    const uint32_t deg = c.row_deg[row];
    const uint32_t n = c.n, E = c.E;
    const float* v = c.vals;
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
                const f3 qj = L2ONLY ? f3{__ldcg(q + j), __ldcg(q + n + j), __ldcg(q + 2 * n + j)}
                                     : f3{q[j], q[n + j], q[2 * n + j]};
                acc = acc + a * qj;
            }
        }
    }
    return acc;
}

}  // namespace b3g
