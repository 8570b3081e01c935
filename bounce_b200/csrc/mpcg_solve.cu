// Standalone MPCG on a caller-supplied block-CSR system (b3SolveMPCG,
// src/bounce/cloth/cloth_force_solver.cpp:61-136).
#include "../../include/b3g.h"

extern "C" b3g_status b3g_mpcg_solve(uint32_t, const uint32_t*, const uint32_t*, const float*, const float*,
                                     const float*, const float*, const b3g_solver_opts*, float*, uint32_t*,
                                     b3g_step_stats*, void*)
{
    return B3G_ERR_UNSUPPORTED;
}
