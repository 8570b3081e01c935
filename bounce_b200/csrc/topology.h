// Host-side preparation of one cloth: the reference constructor's data
// (lumped masses, rest-state triangle frames, bending and sewing springs,
// src/bounce/cloth/cloth.cpp:96-266, :388-427) and the device layout
// (SELL-32 block pattern, per-vertex incidence lists in force-list order).
#pragma once

#include <cstdint>
#include <vector>

namespace b3g {

struct ClothTopology {
    uint32_t n = 0, t = 0, ns = 0;
    // reference constructor data
    std::vector<float> mass;                 // n
    std::vector<float> rest;                 // 6 per triangle: du1, dv1, du2, dv2, inv_det, alpha
    std::vector<uint32_t> spring_pairs;      // 2 per spring, creation order (bending, then sewing)
    std::vector<float> spring_par;           // 3 per spring: L0, ks, kd
    // row pattern: slot 0 is the diagonal, then neighbours ascending
    std::vector<uint32_t> row_ptr;           // n + 1
    std::vector<uint32_t> row_cols;
    uint32_t max_deg = 0;
    // SELL-32
    uint32_t nslices = 0, E = 0;
    std::vector<uint32_t> slice_off;         // nslices + 1
    std::vector<uint8_t> row_deg;
    std::vector<uint32_t> sell_cols;         // E
    // incidence in force-list order
    std::vector<uint32_t> inc_ptr, inc_elem, inc_meta;
};

// Returns 0 on success, else a b3g_status (degenerate mesh, unsupported degree).
int build_topology(uint32_t n, const float* vertices, uint32_t t, const uint32_t* tris, uint32_t nsew,
                   const uint32_t* sewing, const float* def8, ClothTopology* out);

// Bending pairs of b3FindSharedEdges (cloth.cpp:40-94): for every triangle i,
// each edge (a -> b), every later triangle holding (b -> a); the pair is the
// two vertices not on the edge.  Same pairs, same order, O(T log T).
void bending_pairs(uint32_t t, const uint32_t* tris, std::vector<uint32_t>* pairs);

}  // namespace b3g
