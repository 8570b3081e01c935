// Cloth self-collision on the GPU: particle-triangle contacts
// (b3ParticleTriangleContact) of one cloth whose thickness is above zero.
//
// The reference keeps these contacts in a linked list that its broadphase
// fills (src/bounce/cloth/cloth_contact_manager.cpp:43-48, 125-199) and its
// contact solver walks in list order (contacts/cloth_contact_solver.cpp).
// Here the list is an array in list order (head first), rebuilt each step by
// stream compaction and by prepending the new pairs; the sequential
// Gauss-Seidel sweeps run as dependency levels, so every particle sees its
// contacts' updates in list order and the result is the reference's bit for
// bit.  The broadphase move buffer is one flag per proxy.
#pragma once

#include <cstdint>

#include "cloth_dev.cuh"
#include "vec.cuh"

namespace b3g {

// One active particle-triangle contact as the solver sees it
// (b3ClothSolverTriangleContactVelocityConstraint and PositionConstraint,
// include/bounce/cloth/contacts/cloth_contact_solver.h).  Indices are vertex
// ids, masses the inverse masses (0 for static particles).
struct TriCon {
    uint32_t ia, ib, ic, id;
    float mA, mB, mC, mD;
    float wB, wC, wD, friction;
    float nx, ny, nz, normal_mass;
    float t1x, t1y, t1z, radius_a;
    float t2x, t2y, t2z, radius_t;
    float ni, ti1, ti2, pad;
};

// Device view of the self-collision state.
struct SelfDev {
    uint32_t n, t;
    uint32_t cap;                  // contacts each list buffer holds
    uint32_t hash_mask;            // hash slots - 1 (power of two, >= 2 cap)
    // the contact list, head first, in two buffers (current and scratch)
    uint2* key[2];                 // (particle, triangle)
    uint8_t* act[2];               // active flag
    float4* w[2];                  // barycentric weights w2, w3, w4 (valid while active)
    float4* imp[2];                // normal, tangent 1, tangent 2 impulses
    uint32_t* counts;              // see kCount* below
    uint32_t* pair_off;            // n + 1: new pairs per particle, then their offsets
    uint2* fresh;                  // this step's new pairs, ascending (particle, triangle)
    unsigned long long* table;     // keys of the current list (open addressing)
    uint32_t* active_idx;          // list index of each active contact, list order
    uint32_t* by_level;            // active contacts grouped by dependency level
    uint32_t* level_start;         // first entry of each level in by_level (cap + 2)
    TriCon* con;                   // constraints, by active-contact index
};

enum { kCountList = 0, kCountFresh = 1, kCountActive = 2, kCountLevels = 3, kCountStatus = 4, kCountWords = 8 };

// Largest cloth the self-collision path takes: the contact solve keeps one
// u32 level per particle in shared memory (160 KB at this size).
constexpr uint32_t kSelfMaxParticles = 40960;

__device__ __forceinline__ bool tri_contains(const float* lo, const float* hi, const float* tlo, const float* thi)
{
    // b3AABB3::Contains (include/bounce/collision/shapes/aabb3.h)
    bool in = true;
    for (int d = 0; d < 3; ++d) in = in && lo[d] <= tlo[d] && tlo[d] <= hi[d] && lo[d] <= thi[d] && thi[d] <= hi[d];
    return in;
}

// b3ClothTriangle::Synchronize (src/bounce/cloth/cloth_triangle.cpp:24-40)
// with b3BroadPhase::MoveProxy (src/bounce/collision/broad_phase.cpp:99-149):
// the triangle's AABB extended by the thickness; a new fat AABB (extended by
// 0.2, stretched by twice the displacement) when it left the old one.
__device__ __forceinline__ void tri_move_proxy_dev(const ClothDev& c, uint32_t k, f3 disp)
{
    const uint32_t n = c.n, t = c.t;
    const uint4 tv = c.tri[k];
    const f3 A = ld3(c.x, n, tv.x), B = ld3(c.x, n, tv.y), C = ld3(c.x, n, tv.z);
    const float r = c.thickness;
    // b3AABB3::Set(v1, v2, v3): lower = b3Min(v1, b3Min(v2, v3))
    const f3 mn = mk(B.x < C.x ? B.x : C.x, B.y < C.y ? B.y : C.y, B.z < C.z ? B.z : C.z);
    const f3 mx = mk(B.x > C.x ? B.x : C.x, B.y > C.y ? B.y : C.y, B.z > C.z ? B.z : C.z);
    float tlo[3] = {(A.x < mn.x ? A.x : mn.x) - r, (A.y < mn.y ? A.y : mn.y) - r, (A.z < mn.z ? A.z : mn.z) - r};
    float thi[3] = {(A.x > mx.x ? A.x : mx.x) + r, (A.y > mx.y ? A.y : mx.y) + r, (A.z > mx.z ? A.z : mx.z) + r};
    float lo[3] = {c.tri_lo[k], c.tri_lo[t + k], c.tri_lo[2 * t + k]};
    float hi[3] = {c.tri_hi[k], c.tri_hi[t + k], c.tri_hi[2 * t + k]};
    if (tri_contains(lo, hi, tlo, thi)) return;
    const float dd[3] = {2.0f * disp.x, 2.0f * disp.y, 2.0f * disp.z};  // B3_AABB_MULTIPLIER
    for (int d = 0; d < 3; ++d) {
        lo[d] = tlo[d] - 0.2f;  // B3_AABB_EXTENSION
        hi[d] = thi[d] + 0.2f;
        if (dd[d] < 0.0f) lo[d] += dd[d];
        else hi[d] += dd[d];
    }
    c.tri_lo[k] = lo[0]; c.tri_lo[t + k] = lo[1]; c.tri_lo[2 * t + k] = lo[2];
    c.tri_hi[k] = hi[0]; c.tri_hi[t + k] = hi[1]; c.tri_hi[2 * t + k] = hi[2];
    c.t_moved[k] = 1;
}

// b3Particle::SynchronizeTriangles (src/bounce/cloth/particle.cpp:66-82):
// every triangle of vertex i, with no displacement.  The vertex's incidence
// list names its triangles (entries without the spring / mouse bits).
__device__ __forceinline__ void sync_vertex_triangles_dev(const ClothDev& c, uint32_t i)
{
    for (uint32_t q = c.inc_ptr[i]; q < c.inc_ptr[i + 1]; ++q) {
        const uint32_t e = c.inc_elem[q];
        if ((e & 0x80000000u) == 0u) tri_move_proxy_dev(c, e, zero3());
    }
}

}  // namespace b3g
