// Host-side preparation of one soft body: the reference constructor's data
// (src/bounce/softbody/softbody.cpp:436-553, ComputeMass :640-680) and the
// device layout (block rows in first-touch order, per-node incidence in
// element order).
#pragma once

#include <cstdint>
#include <vector>

namespace b3g {

struct SoftBodyPrep {
    uint32_t n = 0, t = 0;
    std::vector<float> mass;        // n
    // per element, in b3SoftBodyElement's arithmetic
    std::vector<float> Ke;          // 144: 16 blocks (block i + 4 j), 9 floats column-major
    std::vector<float> invE;        // 9
    std::vector<float> B;           // 72 (6 x 12, column-major)
    std::vector<float> P;           // 72 (12 x 6, column-major)
    // block rows: row i's columns in the order the element loop first
    // touches them (the reverse of the stiffness matrix's row list)
    std::vector<uint32_t> rowptr;   // n + 1
    std::vector<uint32_t> cols;
    std::vector<uint32_t> diag;     // n: index into cols of (i, i)
    uint32_t max_deg = 0;
    // incidence of node i: its elements in element order; meta = local index
    // of i (bits 0-1), then the row slots (relative to rowptr[i]) of the
    // element's 4 vertices, 7 bits each from bit 4
    std::vector<uint32_t> inc_ptr, inc_elem, inc_meta;
};

// Returns 0, or a b3g_status (a degenerate tetrahedron, a vertex id out of
// range, or a node with more than 127 neighbours).
int prepare_softbody(uint32_t n, const float* vertices, uint32_t t, const uint32_t* tets, float density, float E,
                     float nu, SoftBodyPrep* out);

}  // namespace b3g
