// Host-side preparation of one cloth: the reference constructor's data
// (lumped masses, rest-state triangle frames, bending and sewing springs,
// src/bounce/cloth/cloth.cpp:96-266, :388-427) and the device layout
// (SELL-32 block pattern, per-vertex incidence lists in force-list order).
#pragma once

#include <cstdint>
#include <vector>

namespace b3g {

// A mouse force (include/bounce/cloth/forces/mouse_force.h:26-40): particle
// `particle` tied to the point w2 x(v1) + w3 x(v2) + w4 x(v3) of `triangle`.
struct MouseForceDesc {
    uint32_t particle, triangle;
    float w2, w3, w4, mouse, damping;
};

// Incidence element codes: a triangle id, or a spring id with kIncSpring set,
// or a mouse force id with kIncSpring | kIncMouse set.  A mouse entry's meta
// holds the row's role (0: the particle, 1-3: the triangle's vertices) in
// bits 0-1 and the slots of the force's four vertices, 7 bits each, from
// bit 4.
constexpr uint32_t kIncSpring = 0x80000000u;
constexpr uint32_t kIncMouse = 0x40000000u;

struct ClothTopology {
    uint32_t n = 0, t = 0, ns = 0;
    uint32_t n_mesh = 0;                     // particles of mesh vertices; created ones follow
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
    // Slot-major assembly: for every row and every slot of the row, the
    // element terms that add to that block, in the order the reference adds
    // them (the row's force-list order).  A term code holds the element kind
    // (bits 30-31: 0 triangle, 2 spring, 3 mouse force), the row's corner of
    // the element (bits 28-29), the corner of the slot's column (bits 26-27)
    // and the element id (bits 0-25).  The codes are laid out like the matrix:
    // term j of the block at SELL position slice_off[q] + 32 k + lane sits at
    // term_qk[slice_off[q] / 32 + k] + 32 j + lane, so a warp reading term j
    // of one slot of its 32 rows reads 32 consecutive words; term_slot holds
    // each block's term count.  Built only when every row has at most
    // kSlotMajorMaxDeg slots and every code fits (slot_terms).
    bool slot_terms = false;
    std::vector<uint32_t> term_qk;           // E / 32
    std::vector<uint32_t> term_slot;         // E
    std::vector<uint32_t> terms;
};

constexpr uint32_t kSlotMajorMaxDeg = 16;
constexpr uint32_t kTermKindSpring = 2u << 30, kTermKindMouse = 3u << 30;
constexpr uint32_t kTermIdBits = 26;

// Returns 0 on success, else a b3g_status (degenerate mesh, unsupported degree).
// n_extra created particles follow the n mesh vertices (masses left to the
// caller, 1 each here); `mice` holds the mouse forces in creation order.
// slot_terms: also build the slot-major assembly's term lists.
int build_topology(uint32_t n, const float* vertices, uint32_t t, const uint32_t* tris, uint32_t nsew,
                   const uint32_t* sewing, const float* def8, ClothTopology* out, uint32_t n_extra = 0,
                   const MouseForceDesc* mice = nullptr, uint32_t nmice = 0, bool slot_terms = true);

// Fills the slot-major term lists of a built topology (build_topology calls
// it); leaves slot_terms false when the layout does not fit them.
void build_slot_terms(ClothTopology* out);

// Bending pairs of b3FindSharedEdges (cloth.cpp:40-94): for every triangle i,
// each edge (a -> b), every later triangle holding (b -> a); the pair is the
// two vertices not on the edge.  Same pairs, same order, O(T log T).
void bending_pairs(uint32_t t, const uint32_t* tris, std::vector<uint32_t>* pairs);

}  // namespace b3g
