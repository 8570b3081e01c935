// The cloth handle behind the C ABI, shared by cloth_api.cu and batch_api.cu.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "../../include/b3g.h"
#include "cloth_dev.cuh"
#include "topology.h"

namespace b3g {

struct SelfState;

// One device arena per cloth, carved into 256-byte aligned buffers.
struct Arena {
    char* base = nullptr;
    size_t size = 0, used = 0;
    template <class T> T* take(size_t count)
    {
        size_t off = (used + 255) & ~size_t(255);
        used = off + count * sizeof(T);
        return reinterpret_cast<T*>(base + off);
    }
};

// Host-side device images of a cloth between prepare_cloth and the end of
// its uploads.
struct HostImages {
    std::vector<uint4> tri;
    std::vector<float4> rest;
    std::vector<float2> rest2;
    std::vector<uint2> spr;
    std::vector<float4> sp;
    std::vector<float> x, lo, hi;
    std::vector<uint8_t> types;
    std::vector<float> radius, friction;
    std::vector<uint4> mouse_v;
    std::vector<float4> mouse_par;
};

}  // namespace b3g

namespace b3g {
// The body-contact solve of a cloth with body colliders (bodies.cu).
struct BodyScratch;
void body_scratch_free(BodyScratch* s);
cudaError_t launch_body_solve(const ClothDev& c, BodyScratch*& s, cudaStream_t st);
}  // namespace b3g

struct b3g_cloth {
    int device = 0;
    cudaStream_t stream = nullptr, body_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    b3g::Arena arena;
    b3g::ClothDev dev{};
    b3g::ClothTopology topo;
    float gravity[3] = {0.0f, 0.0f, 0.0f};
    b3g_solver_opts opts{B3G_STOP_REFERENCE, 0.0f, 20u, B3G_DOT_F32};
    uint32_t step_index = 0;
    int assemble_block = 0;  // threads per assembly block; 0: chosen at launch for occupancy
    bool row_assembly = false;  // the row-centric assembly even where the slot-major one applies
    bool lean_layout = false;   // laid out without the slot-major assembly's records (server cloths)

    // pinned staging
    b3g::StepScalars* h_sc = nullptr;
    b3g::ParticleOp* h_ops = nullptr;
    uint32_t ops_cap = 0;
    std::vector<b3g::ParticleOp> pending;
    b3g::ParticleOp* d_ops = nullptr;
    uint32_t d_ops_cap = 0;
    float* d_stage = nullptr;  // 3 n floats for array uploads
    uint8_t* d_stage_u8 = nullptr;

    // graph cache
    cudaGraphExec_t exec = nullptr;
    int graph_dot = -1;
    uint32_t graph_pos_iters = UINT32_MAX;
    uint32_t graph_nsph = UINT32_MAX;
    bool graph_ok = true;
    b3g_cg_strategy cg_strategy = B3G_CG_LAUNCHES;
    b3g_cg_strategy graph_strategy = B3G_CG_LAUNCHES;
    float4* cg_rec = nullptr;                 // fused persistent CG: per-vertex records of two iterations
    uint32_t cg_rec_n = 0;                    // vertices cg_rec was sized for

    b3g_step_stats last{};

    bool owns_arena = true;
    bool owns_stream = true;
    std::unique_ptr<b3g::HostImages> images;

    // creation inputs, kept to lay the cloth out again when particles or
    // forces are created or destroyed (cloth.cpp:307-364)
    std::vector<float> in_vertices;
    std::vector<uint32_t> in_tris, in_sewing;
    b3g_cloth_def in_def{};
    uint32_t n_extra = 0;                     // created particles, after the mesh vertices
    std::vector<b3g::MouseForceDesc> mice;    // mouse forces in creation order
    std::vector<uint32_t> mouse_ids;          // the id of each
    uint32_t next_force_id = 0;
    uint32_t layout_version = 0;              // bumped on every new layout (batches rebuild their graphs)

    b3g::SelfState* self = nullptr;           // particle-triangle contacts (thickness > 0)
    std::vector<void*> hull_bufs;             // device copies of the hull colliders' data
    void* ray_buf = nullptr;                  // ray cast scratch (key and result)
    void* body_buf = nullptr;                 // body colliders: the bodies, then the shapes' proxies
    b3g::BodyScratch* body_scratch = nullptr; // the body-contact solve's sort and constraint scratch
    bool report_fixed = false;                // collider ranks given by b3g_cloth_set_report_order
};


b3g_status flush_ops_on(b3g_cloth* c, cudaStream_t st);
void fill_step_scalars(b3g_cloth* c, float dt, uint32_t vel_iters, uint32_t pos_iters, b3g::StepScalars* h);
void record_stats(b3g_cloth* c, const b3g::StepScalars& h, float ms, bool solved);
// records = false lays the cloth out without the slot-major assembly's
// records and term lists (it then assembles row by row).
b3g_status prepare_cloth(const b3g_mesh_desc* mesh, const b3g_cloth_def* def, b3g_cloth** out,
                         bool records = true);
b3g_status layout_cloth(b3g_cloth* c);
// Page-locked staging for a cloth's uploads: each upload is copied into the
// staging buffer on the host and from there to the device asynchronously.
// When the buffer is full the upload stream is waited for and the buffer
// starts over; an upload larger than the buffer goes straight from its host
// array.
struct UploadStage {
    char* base = nullptr;
    size_t size = 0, used = 0;
};
b3g_status realize_cloth(b3g_cloth* c, int device, char* base, bool owns_arena, cudaStream_t st, bool own_stream,
                         UploadStage* stage = nullptr);
void finish_upload(b3g_cloth* c);
b3g_status destroy_cloth(b3g_cloth* c);

// Self-collision (self_collision.cu): set up for a cloth whose thickness is
// above zero, free, and the three phases of a step.
namespace b3g {
b3g_status self_attach(b3g_cloth* c);
void self_free(b3g_cloth* c);
b3g_status self_update(b3g_cloth* c, cudaStream_t st);
b3g_status self_solve(b3g_cloth* c, cudaStream_t st);
b3g_status self_find(b3g_cloth* c, cudaStream_t st);
b3g_status self_read(const b3g_cloth* c, uint32_t* count, uint32_t* pairs, uint8_t* active, float* weights,
                     float* impulses);
void self_stats(const b3g_cloth* c, uint32_t* contacts, uint32_t* active, uint32_t* levels);
}  // namespace b3g
b3g_status batch_step_impl(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, float dt, uint32_t vel_iters,
                           uint32_t pos_iters, b3g_step_stats* per_cloth, b3g_batch_stats* stats, bool use_graph);
// The same step without a graph in two halves: launch returns once the work
// is queued on the batch's stream, finish waits for it and collects the
// statistics.  The cloths must not change in between.
b3g_status batch_step_launch(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, float dt, uint32_t vel_iters,
                             uint32_t pos_iters);
b3g_status batch_step_finish(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, b3g_step_stats* per_cloth,
                             b3g_batch_stats* stats);
