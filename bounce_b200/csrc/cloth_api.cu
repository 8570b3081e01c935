// C ABI of libb3g.so (include/b3g.h): cloth handles, device memory, the
// per-step CUDA graph, particle edits and state transfers.
#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/b3g.h"
#include "cloth_dev.cuh"
#include "topology.h"
#include "cloth_internal.h"
#include "grid_cg.cuh"
#include "broadphase_order.h"

using namespace b3g;

namespace {

b3g_status from_cuda(cudaError_t e)
{
    if (e == cudaSuccess) return B3G_OK;
    if (e == cudaErrorMemoryAllocation) return B3G_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInvalidDevice)
        return B3G_ERR_NO_DEVICE;
    return B3G_ERR_CUDA;
}

#define B3G_TRY(expr)                               \
    do {                                            \
        cudaError_t e_ = (expr);                    \
        if (e_ != cudaSuccess) return from_cuda(e_); \
    } while (0)

}  // namespace

// Applies the queued particle edits on stream `st` (the cloth's own stream
// by default).
b3g_status flush_ops_on(b3g_cloth* c, cudaStream_t st)
{
    if (c->pending.empty()) return B3G_OK;
    uint32_t cnt = (uint32_t)c->pending.size();
    if (cnt > c->ops_cap) {
        if (c->h_ops) cudaFreeHost(c->h_ops);
        c->ops_cap = std::max<uint32_t>(cnt, 256);
        B3G_TRY(cudaMallocHost(&c->h_ops, c->ops_cap * sizeof(ParticleOp)));
    }
    if (cnt > c->d_ops_cap) {
        if (c->d_ops) cudaFree(c->d_ops);
        c->d_ops_cap = std::max<uint32_t>(cnt, 256);
        B3G_TRY(cudaMalloc(&c->d_ops, c->d_ops_cap * sizeof(ParticleOp)));
    }
    // The pinned buffer may still be read by an earlier copy.
    B3G_TRY(cudaStreamSynchronize(c->stream));
    if (st != c->stream) B3G_TRY(cudaStreamSynchronize(st));
    std::memcpy(c->h_ops, c->pending.data(), cnt * sizeof(ParticleOp));
    B3G_TRY(cudaMemcpyAsync(c->d_ops, c->h_ops, cnt * sizeof(ParticleOp), cudaMemcpyHostToDevice, st));
    B3G_TRY(launch_particle_ops(c->dev, c->d_ops, cnt, st));
    c->pending.clear();
    return B3G_OK;
}

// Step parameters of the next step of cloth c (b3Cloth::Step arguments,
// gravity, solver options); advances the cloth's step counter.
void fill_step_scalars(b3g_cloth* c, float dt, uint32_t vel_iters, uint32_t pos_iters, StepScalars* h)
{
    std::memset(h, 0, sizeof(StepScalars));
    h->dt = dt;
    h->vel_iters = vel_iters;
    h->pos_iters = pos_iters;
    h->step_index = ++c->step_index;
    h->max_iter = c->opts.max_iterations;
    h->stop_rule = (int)c->opts.stop_rule;
    h->tol = c->opts.tolerance;
    h->dot = (int)c->opts.dot;
    h->gx = c->gravity[0];
    h->gy = c->gravity[1];
    h->gz = c->gravity[2];
}

void record_stats(b3g_cloth* c, const StepScalars& h, float ms, bool solved)
{
    b3g_step_stats& L = c->last;
    L.iterations = solved ? h.iter : 0;
    L.delta0 = h.delta0;
    L.delta = h.delta;
    L.b_delta = h.b_delta;
    L.active_contacts = h.active_contacts;
    L.contacts = h.contacts;
    L.step_ms = ms;
}

namespace {

b3g_status flush_ops(b3g_cloth* c) { return flush_ops_on(c, c->stream); }

void destroy_graph(b3g_cloth* c)
{
    if (c->exec) cudaGraphExecDestroy(c->exec);
    c->exec = nullptr;
}

bool persistent_cg(const b3g_cloth* c) { return c->cg_strategy != B3G_CG_LAUNCHES; }

// The fused CG's record buffer, sized for the cloth's current vertex count
// (a new layout changes it; a captured graph holding the old one is dropped).
b3g_status ensure_cg_rec(b3g_cloth* c)
{
    if (c->cg_strategy != B3G_CG_PERSISTENT_FUSED || (c->cg_rec && c->cg_rec_n == c->dev.n)) return B3G_OK;
    destroy_graph(c);
    if (c->cg_rec) cudaFree(c->cg_rec);
    c->cg_rec = nullptr;
    c->cg_rec_n = 0;
    B3G_TRY(cudaMalloc(&c->cg_rec, grid_cg_fused_rec_bytes(c->dev.n)));
    c->cg_rec_n = c->dev.n;
    return B3G_OK;
}

// The persistent CG of the cloth's strategy: the barrier is cleared, then one
// cooperative launch (two grid reductions per iteration, or the fused form).
cudaError_t launch_persistent_cg(b3g_cloth* c, int dot, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(c->dev.bar, 0, sizeof(GridBarrier), st);
    if (e != cudaSuccess) return e;
    if (c->cg_strategy == B3G_CG_PERSISTENT_FUSED) return launch_grid_cg_fused(c->dev, dot, c->dev.bar, c->cg_rec, st);
    return launch_grid_cg(c->dev, dot, c->dev.bar, st);
}

// Captures one step: [contacts_update] assemble cg_init while{cg iteration}
// finalize [contact_position x (pos_iters - 1)] post.
b3g_status build_graph(b3g_cloth* c, uint32_t pos_iters)
{
    destroy_graph(c);
    const int dot = (int)c->opts.dot;
    cudaStream_t st = c->stream;
    cudaGraph_t graph = nullptr;
    // launches recorded while capturing are not executions
    const uint64_t launches_before = kernel_launches();
    B3G_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t err = cudaSuccess;
    do {
        if ((err = launch_contacts_update(c->dev, st)) != cudaSuccess) break;
        if ((err = launch_assemble(c->dev, c->assemble_block, st)) != cudaSuccess) break;
        if (persistent_cg(c)) {
            if ((err = launch_persistent_cg(c, dot, st)) != cudaSuccess) break;
        } else {
            cudaStreamCaptureStatus cs;
            cudaGraph_t cap;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            if ((err = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cap, &deps, &ndeps)) != cudaSuccess) break;
            cudaGraphConditionalHandle cond;
            if ((err = cudaGraphConditionalHandleCreate(&cond, cap, 0, 0)) != cudaSuccess) break;
            if ((err = launch_cg_init(c->dev, dot, cond, 1, st)) != cudaSuccess) break;
            if ((err = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cap, &deps, &ndeps)) != cudaSuccess) break;
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t wnode;
            if ((err = cudaGraphAddNode(&wnode, cap, deps, ndeps, &cp)) != cudaSuccess) break;
            if ((err = cudaStreamUpdateCaptureDependencies(st, &wnode, 1, cudaStreamSetCaptureDependencies)) !=
                cudaSuccess)
                break;
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            if ((err = cudaStreamBeginCaptureToGraph(c->body_stream, body, nullptr, nullptr, 0,
                                                     cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
                break;
            cudaError_t e2 = launch_cg_iteration(c->dev, dot, cond, 1, c->body_stream);
            cudaGraph_t body_out = nullptr;
            cudaError_t e3 = cudaStreamEndCapture(c->body_stream, &body_out);
            if (e2 != cudaSuccess) { err = e2; break; }
            if (e3 != cudaSuccess) { err = e3; break; }
        }
        if ((err = launch_finalize(c->dev, st)) != cudaSuccess) break;
        for (uint32_t k = 1; k < pos_iters && k < (uint32_t)kMaxPosIters; ++k)
            if ((err = launch_contact_position(c->dev, k, st)) != cudaSuccess) break;
        if (err != cudaSuccess) break;
        if ((err = launch_post(c->dev, st)) != cudaSuccess) break;
    } while (0);
    cudaError_t e_end = cudaStreamEndCapture(st, &graph);
    count_launches(launches_before - kernel_launches());
    if (err == cudaSuccess) err = e_end;
    if (err == cudaSuccess) err = cudaGraphInstantiate(&c->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (err != cudaSuccess) {
        cudaGetLastError();
        c->exec = nullptr;
        return from_cuda(err);
    }
    c->graph_dot = dot;
    c->graph_strategy = c->cg_strategy;
    c->graph_pos_iters = pos_iters;
    c->graph_nsph = c->dev.nsph;
    return B3G_OK;
}

// Same sequence without a graph: every CG iteration is launched and returns
// early on the device once the loop condition is cleared.
b3g_status launch_step_plain(b3g_cloth* c, uint32_t pos_iters)
{
    const int dot = (int)c->opts.dot;
    cudaStream_t st = c->stream;
    cudaGraphConditionalHandle none = 0;
    B3G_TRY(launch_contacts_update(c->dev, st));
    B3G_TRY(launch_assemble(c->dev, c->assemble_block, st));
    if (persistent_cg(c)) {
        B3G_TRY(launch_persistent_cg(c, dot, st));
    } else {
        B3G_TRY(launch_cg_init(c->dev, dot, none, 0, st));
        for (uint32_t k = 0; k < c->opts.max_iterations; ++k) B3G_TRY(launch_cg_iteration(c->dev, dot, none, 0, st));
    }
    B3G_TRY(launch_finalize(c->dev, st));
    for (uint32_t k = 1; k < pos_iters && k < (uint32_t)kMaxPosIters; ++k)
        B3G_TRY(launch_contact_position(c->dev, k, st));
    B3G_TRY(launch_post(c->dev, st));
    return B3G_OK;
}

// A step of a cloth with body colliders, launched without a graph: the
// contact update, assembly and CG as in any step, then the force solver's
// state update and the body-contact solve in list order on one block
// (bodies.cu), then the proxy sync and the new contacts.
b3g_status launch_step_bodies(b3g_cloth* c)
{
    const int dot = (int)c->opts.dot;
    cudaStream_t st = c->stream;
    cudaGraphConditionalHandle none = 0;
    B3G_TRY(launch_contacts_update(c->dev, st));
    B3G_TRY(launch_assemble(c->dev, c->assemble_block, st));
    if (persistent_cg(c)) {
        B3G_TRY(launch_persistent_cg(c, dot, st));
    } else {
        B3G_TRY(launch_cg_init(c->dev, dot, none, 0, st));
        for (uint32_t k = 0; k < c->opts.max_iterations; ++k) B3G_TRY(launch_cg_iteration(c->dev, dot, none, 0, st));
    }
    B3G_TRY(launch_body_solve(c->dev, c->body_scratch, st));
    B3G_TRY(launch_post(c->dev, st));
    return B3G_OK;
}

// A step of a cloth with self-collision, launched without a graph: the
// particle-triangle contact list is updated before the solve, the contact
// phase solves both contact kinds in list order, and the new pairs are found
// after the proxies moved (b3Cloth::Step, cloth.cpp:551-601).
b3g_status launch_step_self(b3g_cloth* c, float dt)
{
    const int dot = (int)c->opts.dot;
    cudaStream_t st = c->stream;
    cudaGraphConditionalHandle none = 0;
    b3g_status s = self_update(c, st);
    if (s != B3G_OK) return s;
    B3G_TRY(launch_contacts_update(c->dev, st));
    if (dt > 0.0f) {
        B3G_TRY(launch_assemble(c->dev, c->assemble_block, st));
        if (persistent_cg(c)) {
            B3G_TRY(launch_persistent_cg(c, dot, st));
        } else {
            B3G_TRY(launch_cg_init(c->dev, dot, none, 0, st));
            for (uint32_t k = 0; k < c->opts.max_iterations; ++k)
                B3G_TRY(launch_cg_iteration(c->dev, dot, none, 0, st));
        }
        if ((s = self_solve(c, st)) != B3G_OK) return s;
    }
    B3G_TRY(launch_post(c->dev, st));
    return self_find(c, st);
}

bool valid(const b3g_cloth* c) { return c != nullptr && c->dev.n > 0; }

}  // namespace

extern "C" {

const char* b3g_status_string(b3g_status s)
{
    switch (s) {
        case B3G_OK: return "ok";
        case B3G_ERR_INVALID_ARGUMENT: return "invalid argument";
        case B3G_ERR_DEGENERATE_MESH: return "degenerate mesh";
        case B3G_ERR_NO_DEVICE: return "no CUDA device";
        case B3G_ERR_OUT_OF_MEMORY: return "out of memory";
        case B3G_ERR_CUDA: return "CUDA error";
        case B3G_ERR_NUMERICAL: return "numerical breakdown in CG";
        case B3G_ERR_TIMEOUT: return "device wait timed out";
        case B3G_ERR_CAPACITY: return "capacity exceeded";
        case B3G_ERR_UNSUPPORTED: return "unsupported mesh";
    }
    return "unknown status";
}

uint64_t b3g_kernel_launch_count(void) { return kernel_launches(); }

}  // extern "C"

// Host half of cloth creation: validates the mesh, builds the topology and the
// device images, sizes the arena.  Touches no CUDA state; thread-safe.
b3g_status prepare_cloth(const b3g_mesh_desc* mesh, const b3g_cloth_def* def, b3g_cloth** out, bool records)
{
    if (!mesh || !def || !out || !mesh->vertices || !mesh->triangles || mesh->vertex_count == 0 ||
        mesh->triangle_count == 0 || (mesh->sewing_line_count && !mesh->sewing_lines))
        return B3G_ERR_INVALID_ARGUMENT;
    if (!(def->density > 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    b3g_cloth* c = new (std::nothrow) b3g_cloth();
    if (!c) return B3G_ERR_OUT_OF_MEMORY;
    c->in_vertices.assign(mesh->vertices, mesh->vertices + 3 * (size_t)mesh->vertex_count);
    c->in_tris.assign(mesh->triangles, mesh->triangles + 3 * (size_t)mesh->triangle_count);
    if (mesh->sewing_line_count)
        c->in_sewing.assign(mesh->sewing_lines, mesh->sewing_lines + 4 * (size_t)mesh->sewing_line_count);
    c->in_def = *def;
    c->lean_layout = !records;
    const b3g_status s = layout_cloth(c);
    if (s != B3G_OK) {
        delete c;
        return s;
    }
    *out = c;
    return B3G_OK;
}

// The topology, device scalars, arena size and host images of the cloth's
// current particles and forces: the mesh's, the created particles (after the
// mesh vertices) and the mouse forces.  Keeps the colliders.
b3g_status layout_cloth(b3g_cloth* c)
{
    const b3g_cloth_def* def = &c->in_def;
    const float d8[8] = {def->density, def->streching, def->shearing, def->bending,
                         def->sewing,  def->damping,   def->thickness, def->friction};
    const uint32_t n_mesh = (uint32_t)(c->in_vertices.size() / 3);
    ClothTopology topo;
    int rc = build_topology(n_mesh, c->in_vertices.data(), (uint32_t)(c->in_tris.size() / 3), c->in_tris.data(),
                            (uint32_t)(c->in_sewing.size() / 4), c->in_sewing.empty() ? nullptr : c->in_sewing.data(),
                            d8, &topo, c->n_extra, c->mice.data(), (uint32_t)c->mice.size(), !c->lean_layout);
    if (rc != 0) return (b3g_status)rc;
    c->topo = std::move(topo);
    const ClothTopology& T = c->topo;
    const uint32_t n = T.n, t = T.t, ns = T.ns;
    const uint32_t nmouse = (uint32_t)c->mice.size();
    ClothDev& d = c->dev;
    d.n = n;
    d.t = t;
    d.ns = ns;
    d.nmouse = nmouse;
    d.nslices = T.nslices;
    d.max_deg = T.max_deg;
    d.E = T.E;
    d.k_stretch = def->streching;
    d.k_shear = def->shearing;
    d.k_damp = def->damping;
    d.thickness = def->thickness;
    d.friction = def->friction;
    d.block = 256;
    d.grid = std::min<uint32_t>((n + 255) / 256, 148 * 8);

    const size_t vec = 3 * (size_t)n * sizeof(float);
    size_t bytes = 0;
    auto add = [&](size_t b) { bytes += ((b + 255) & ~size_t(255)) + 256; };
    add((T.nslices + 1) * 4); add(n); add((size_t)T.E * 4); add((size_t)T.E * 36);
    add((n + 1) * 4); add(T.inc_elem.size() * 4 + 4); add(T.inc_meta.size() * 4 + 4);
    add((size_t)t * 16); add((size_t)t * 16); add((size_t)t * 8); add((size_t)ns * 8 + 8); add((size_t)ns * 16 + 16);
    add((size_t)nmouse * 16 + 16); add((size_t)nmouse * 32 + 32);  // mouse forces
    for (int k = 0; k < 13; ++k) add(vec);  // x v fext y mx b dv r p s pinv z p2
    add((size_t)n * 4); add(n);             // mass, type
    add((size_t)n * 4); add((size_t)n * 4); // particle radius, friction
    add(vec); add(vec);                     // fat lo / hi
    const size_t nn = (size_t)kMaxSpheres * n;
    add(nn); add(nn); add(nn * 4); add(nn * 12); add(nn * 12); add(nn * 12); add(nn * 12); add(nn * 12);
    add(sizeof(StepScalars));
    add(sizeof(GridBarrier));
    add(std::max((size_t)d.grid * 32, kGridCgPartialBytes));
    add(vec); add(n);                       // staging
    add(T.E); add(n);                       // the assembly's first-touch order and its length
    if (T.slot_terms) {                     // slot-major assembly: term lists and element records
        add((size_t)T.E / 32 * 4 + 4); add((size_t)T.E * 4); add(T.terms.size() * 4 + 4);
        add((size_t)t * 240); add((size_t)ns * 48 + 48); add((size_t)nmouse * 80 + 80);
        add((size_t)T.E * 24);
    }
    d.slot_asm = T.slot_terms && !c->row_assembly ? 1u : 0u;
    c->arena.size = bytes + 256;

    HostImages* im = new (std::nothrow) HostImages();
    if (!im) return B3G_ERR_OUT_OF_MEMORY;
    const uint32_t* tris = c->in_tris.data();
    im->tri.resize(t);
    im->rest.resize(t);
    im->rest2.resize(t);
    for (uint32_t k = 0; k < t; ++k) {
        im->tri[k] = make_uint4(tris[3 * k], tris[3 * k + 1], tris[3 * k + 2], 0u);
        const float* r = &T.rest[6 * (size_t)k];
        im->rest[k] = make_float4(r[0], r[1], r[2], r[3]);
        im->rest2[k] = make_float2(r[4], r[5]);
    }
    im->spr.resize(ns + 1);
    im->sp.resize(ns + 1);
    for (uint32_t q = 0; q < ns; ++q) {
        im->spr[q] = make_uint2(T.spring_pairs[2 * q], T.spring_pairs[2 * q + 1]);
        im->sp[q] = make_float4(T.spring_par[3 * q], T.spring_par[3 * q + 1], T.spring_par[3 * q + 2], 0.0f);
    }
    im->mouse_v.resize(nmouse + 1);
    im->mouse_par.resize(2 * (size_t)nmouse + 2);
    for (uint32_t m = 0; m < nmouse; ++m) {
        const MouseForceDesc& f = c->mice[m];
        const uint32_t* tv = tris + 3 * (size_t)f.triangle;
        im->mouse_v[m] = make_uint4(f.particle, tv[0], tv[1], tv[2]);
        im->mouse_par[2 * m] = make_float4(f.w2, f.w3, f.w4, f.mouse);
        im->mouse_par[2 * m + 1] = make_float4(f.damping, 0.0f, 0.0f, 0.0f);
    }
    // mesh vertices at their creation positions; created particles are
    // written by the caller that created them
    im->x.assign(3 * (size_t)n, 0.0f);
    im->lo.assign(3 * (size_t)n, 0.0f);
    im->hi.assign(3 * (size_t)n, 0.0f);
    const float r = def->thickness;
    for (uint32_t i = 0; i < n_mesh; ++i)
        for (int q = 0; q < 3; ++q) {
            float x = c->in_vertices[3 * (size_t)i + q];
            im->x[(size_t)q * n + i] = x;
            // proxy at creation: [x - r, x + r] fattened by B3_AABB_EXTENSION (cloth.cpp:312-317)
            im->lo[(size_t)q * n + i] = (x - r) - 0.2f;
            im->hi[(size_t)q * n + i] = (x + r) + 0.2f;
        }
    im->types.assign(n, (uint8_t)B3G_DYNAMIC);
    // every particle starts with the cloth's thickness and friction (cloth.cpp:116-117)
    im->radius.assign(n, def->thickness);
    im->friction.assign(n, def->friction);
    c->images.reset(im);
    return B3G_OK;
}

// Device half: binds the arena `base` (c->arena.size bytes, caller-owned when
// owns_arena is false) and enqueues the uploads on `st`.  With own_stream the
// cloth gets its own stream and events and the call waits for the uploads;
// otherwise it uses `st` and the host images stay alive until
// finish_upload() after the caller has synchronised `st`.
b3g_status realize_cloth(b3g_cloth* c, int device, char* base, bool owns_arena, cudaStream_t st, bool own_stream,
                         UploadStage* stage)
{
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return from_cuda(e);
    c->device = device;
    c->owns_arena = owns_arena;
    c->arena.base = base;
    c->arena.used = 0;
    const ClothTopology& T = c->topo;
    const uint32_t n = T.n, t = T.t, ns = T.ns;
    ClothDev& d = c->dev;
    Arena& A = c->arena;
    const size_t nn = (size_t)kMaxSpheres * n;
    const size_t vec = 3 * (size_t)n * sizeof(float);
    uint32_t* slice_off = A.take<uint32_t>(T.nslices + 1);
    uint8_t* row_deg = A.take<uint8_t>(n);
    uint32_t* cols = A.take<uint32_t>(T.E);
    d.vals = A.take<float>((size_t)T.E * 9);
    uint32_t* inc_ptr = A.take<uint32_t>(n + 1);
    uint32_t* inc_elem = A.take<uint32_t>(T.inc_elem.size() + 1);
    uint32_t* inc_meta = A.take<uint32_t>(T.inc_meta.size() + 1);
    uint4* tri = A.take<uint4>(t);
    float4* tri_rest = A.take<float4>(t);
    float2* tri_rest2 = A.take<float2>(t);
    uint2* spr = A.take<uint2>(ns + 1);
    float4* spr_par = A.take<float4>(ns + 1);
    uint4* mouse_v = A.take<uint4>(d.nmouse + 1);
    float4* mouse_par = A.take<float4>(2 * (size_t)d.nmouse + 2);
    d.x = A.take<float>(3 * (size_t)n);
    d.v = A.take<float>(3 * (size_t)n);
    d.fext = A.take<float>(3 * (size_t)n);
    d.y = A.take<float>(3 * (size_t)n);
    d.mx = A.take<float>(3 * (size_t)n);
    d.b = A.take<float>(3 * (size_t)n);
    d.dv = A.take<float>(3 * (size_t)n);
    d.r = A.take<float>(3 * (size_t)n);
    d.p = A.take<float>(3 * (size_t)n);
    d.s = A.take<float>(3 * (size_t)n);
    d.pinv = A.take<float>(3 * (size_t)n);
    d.z = A.take<float>(3 * (size_t)n);
    d.p2 = A.take<float>(3 * (size_t)n);
    float* mass = A.take<float>(n);
    d.type = A.take<uint8_t>(n);
    d.p_radius = A.take<float>(n);
    d.p_friction = A.take<float>(n);
    d.fat_lo = A.take<float>(3 * (size_t)n);
    d.fat_hi = A.take<float>(3 * (size_t)n);
    d.c_exists = A.take<uint8_t>(nn);
    d.c_active = A.take<uint8_t>(nn);
    d.c_key = A.take<uint32_t>(nn);
    d.c_normal = A.take<float>(3 * nn);
    d.c_t1 = A.take<float>(3 * nn);
    d.c_t2 = A.take<float>(3 * nn);
    d.c_imp = A.take<float>(3 * nn);
    d.c_point = A.take<float>(3 * nn);
    d.sc = A.take<StepScalars>(1);
    d.bar = A.take<GridBarrier>(1);
    d.partials = A.take<char>(std::max((size_t)d.grid * 32, kGridCgPartialBytes));
    c->d_stage = A.take<float>(3 * (size_t)n);
    c->d_stage_u8 = A.take<uint8_t>(n);
    d.asm_touch = A.take<uint8_t>(T.E);
    d.asm_ntouch = A.take<uint8_t>(n);
    uint32_t *term_qk = nullptr, *term_slot = nullptr, *terms = nullptr;
    d.term_qk = d.term_slot = d.terms = nullptr;
    d.tri_rec = d.spr_rec = d.mouse_rec = nullptr;
    d.asm_kv = nullptr;
    if (T.slot_terms) {
        term_qk = A.take<uint32_t>(T.E / 32 + 1);
        term_slot = A.take<uint32_t>(T.E);
        terms = A.take<uint32_t>(T.terms.size() + 1);
        d.tri_rec = A.take<float4>((size_t)t * 15);
        d.spr_rec = A.take<float4>((size_t)ns * 3 + 3);
        d.mouse_rec = A.take<float4>((size_t)d.nmouse * 5 + 5);
        d.asm_kv = A.take<float>((size_t)T.E * 6);
        d.term_qk = term_qk;
        d.term_slot = term_slot;
        d.terms = terms;
    }
    if (A.used > A.size) return B3G_ERR_CUDA;  // sizing bug guard
    d.slice_off = slice_off;
    d.row_deg = row_deg;
    d.cols = cols;
    d.inc_ptr = inc_ptr;
    d.inc_elem = inc_elem;
    d.inc_meta = inc_meta;
    d.tri = tri;
    d.tri_rest = tri_rest;
    d.tri_rest2 = tri_rest2;
    d.spr = spr;
    d.spr_par = spr_par;
    d.mouse_v = mouse_v;
    d.mouse_par = mouse_par;
    d.mass = mass;

    if (own_stream) {
        if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&c->body_stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreate(&c->ev0)) != cudaSuccess || (e = cudaEventCreate(&c->ev1)) != cudaSuccess ||
            (e = cudaMallocHost(&c->h_sc, sizeof(StepScalars))) != cudaSuccess)
            return from_cuda(e);
        std::memset(c->h_sc, 0, sizeof(StepScalars));
        st = c->stream;
        c->owns_stream = true;
    } else {
        c->stream = st;
        c->owns_stream = false;
    }
    const HostImages& im = *c->images;
    auto up = [&](void* dst, const void* src, size_t b) {
        if (e != cudaSuccess || !b) return;
        if (stage && stage->used + b > stage->size && stage->used && b <= stage->size) {
            // the staging buffer is full: wait for the copies queued from it
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return;
            stage->used = 0;
        }
        if (stage && stage->used + b <= stage->size) {
            char* p = stage->base + stage->used;
            std::memcpy(p, src, b);
            stage->used += (b + 255) & ~size_t(255);
            e = cudaMemcpyAsync(dst, p, b, cudaMemcpyHostToDevice, st);
        } else {
            e = cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, st);
        }
    };
    e = cudaMemsetAsync(A.base, 0, A.size, st);
    up(slice_off, T.slice_off.data(), T.slice_off.size() * 4);
    up(row_deg, T.row_deg.data(), n);
    up(cols, T.sell_cols.data(), (size_t)T.E * 4);
    up(inc_ptr, T.inc_ptr.data(), (n + 1) * 4);
    up(inc_elem, T.inc_elem.data(), T.inc_elem.size() * 4);
    up(inc_meta, T.inc_meta.data(), T.inc_meta.size() * 4);
    if (T.slot_terms) {
        up(term_qk, T.term_qk.data(), T.term_qk.size() * 4);
        up(term_slot, T.term_slot.data(), (size_t)T.E * 4);
        up(terms, T.terms.data(), T.terms.size() * 4);
    }
    up(tri, im.tri.data(), (size_t)t * 16);
    up(tri_rest, im.rest.data(), (size_t)t * 16);
    up(tri_rest2, im.rest2.data(), (size_t)t * 8);
    up(spr, im.spr.data(), (size_t)ns * 8);
    up(spr_par, im.sp.data(), (size_t)ns * 16);
    up(mouse_v, im.mouse_v.data(), (size_t)d.nmouse * 16);
    up(mouse_par, im.mouse_par.data(), (size_t)d.nmouse * 32);
    up(d.x, im.x.data(), vec);
    up(mass, T.mass.data(), (size_t)n * 4);
    up(d.type, im.types.data(), n);
    up(d.p_radius, im.radius.data(), (size_t)n * 4);
    up(d.p_friction, im.friction.data(), (size_t)n * 4);
    up(d.fat_lo, im.lo.data(), vec);
    up(d.fat_hi, im.hi.data(), vec);
    if (e != cudaSuccess) return from_cuda(e);
    if (own_stream) {
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return from_cuda(e);
        c->images.reset();
    }
    return B3G_OK;
}

// Releases the host images once the uploads on the cloth's stream are done.
void finish_upload(b3g_cloth* c) { c->images.reset(); }

extern "C" {

b3g_status b3g_cloth_create(const b3g_mesh_desc* mesh, const b3g_cloth_def* def, int device, b3g_cloth** out)
{
    if (!out) return B3G_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        if (!mesh || !def) return B3G_ERR_INVALID_ARGUMENT;
        return B3G_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return B3G_ERR_INVALID_ARGUMENT;
    b3g_cloth* c = nullptr;
    b3g_status s = prepare_cloth(mesh, def, &c);
    if (s != B3G_OK) return s;
    cudaError_t e = cudaSetDevice(device);
    char* base = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&base, c->arena.size);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return e == cudaErrorMemoryAllocation ? B3G_ERR_OUT_OF_MEMORY : from_cuda(e);
    }
    s = realize_cloth(c, device, base, true, nullptr, true);
    if (s == B3G_OK && def->thickness > 0.0f) s = self_attach(c);
    if (s != B3G_OK) {
        b3g_cloth_destroy(c);
        return s;
    }
    *out = c;
    return B3G_OK;
}

b3g_status b3g_cloth_destroy(b3g_cloth* c)
{
    if (!c) return B3G_ERR_INVALID_ARGUMENT;
    if (!c->owns_stream && c->stream) return B3G_ERR_INVALID_ARGUMENT;  // owned by a server
    return destroy_cloth(c);
}

}  // extern "C"

b3g_status destroy_cloth(b3g_cloth* c)
{
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    self_free(c);
    for (void* p : c->hull_bufs) cudaFree(p);
    c->hull_bufs.clear();
    if (c->ray_buf) cudaFree(c->ray_buf);
    if (c->cg_rec) cudaFree(c->cg_rec);
    if (c->body_buf) cudaFree(c->body_buf);
    body_scratch_free(c->body_scratch);
    destroy_graph(c);
    if (c->arena.base && c->owns_arena) cudaFree(c->arena.base);
    if (c->d_ops) cudaFree(c->d_ops);
    if (c->h_ops) cudaFreeHost(c->h_ops);
    if (c->h_sc) cudaFreeHost(c->h_sc);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream && c->owns_stream) cudaStreamDestroy(c->stream);
    if (c->body_stream) cudaStreamDestroy(c->body_stream);
    delete c;
    return B3G_OK;
}

extern "C" {

b3g_status b3g_cloth_set_gravity(b3g_cloth* c, const float g[3])
{
    if (!valid(c) || !g) return B3G_ERR_INVALID_ARGUMENT;
    std::memcpy(c->gravity, g, sizeof(c->gravity));
    return B3G_OK;
}

b3g_status b3g_cloth_get_gravity(const b3g_cloth* c, float g[3])
{
    if (!valid(c) || !g) return B3G_ERR_INVALID_ARGUMENT;
    std::memcpy(g, c->gravity, sizeof(c->gravity));
    return B3G_OK;
}

b3g_status b3g_cloth_set_solver(b3g_cloth* c, const b3g_solver_opts* o)
{
    if (!valid(c) || !o) return B3G_ERR_INVALID_ARGUMENT;
    if (o->max_iterations < 1 || (o->stop_rule != B3G_STOP_REFERENCE && o->stop_rule != B3G_STOP_RELATIVE) ||
        (o->dot != B3G_DOT_F32 && o->dot != B3G_DOT_COMPENSATED && o->dot != B3G_DOT_F64) ||
        (o->stop_rule == B3G_STOP_RELATIVE && !(o->tolerance >= 0.0f)))
        return B3G_ERR_INVALID_ARGUMENT;
    c->opts = *o;
    return B3G_OK;
}

}  // extern "C"

namespace b3g {

void rank_colliders(SphereDev* sph, uint32_t count)
{
    float lo[kMaxSpheres][3], hi[kMaxSpheres][3];
    uint32_t rank[kMaxSpheres];
    for (uint32_t s = 0; s < count; ++s)
        for (int q = 0; q < 3; ++q) {
            lo[s][q] = sph[s].lo[q];
            hi[s][q] = sph[s].hi[q];
        }
    query_report_ranks(lo, hi, count, rank);
    for (uint32_t s = 0; s < count; ++s) sph[s].rank = rank[s];
}

}  // namespace b3g

extern "C" {

b3g_status b3g_cloth_add_static_sphere(b3g_cloth* c, const float center[3], float radius, float friction,
                                       uint32_t* shape_id)
{
    if (!valid(c) || !center || !(radius > 0.0f) || !(friction >= 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    if (c->dev.nsph >= (uint32_t)kMaxSpheres) return B3G_ERR_CAPACITY;
    SphereDev& s = c->dev.sph[c->dev.nsph];
    s = SphereDev{};
    s.kind = 0;
    s.cx = center[0];
    s.cy = center[1];
    s.cz = center[2];
    s.radius = radius;
    s.friction = friction;
    // sphere AABB (sphere_shape.cpp:53-59) fattened by B3_AABB_EXTENSION (broad_phase.cpp:78-82)
    for (int q = 0; q < 3; ++q) {
        s.lo[q] = (center[q] - radius) - 0.2f;
        s.hi[q] = (center[q] + radius) + 0.2f;
    }
    if (shape_id) *shape_id = c->dev.nsph;
    c->dev.nsph += 1;
    c->report_fixed = false;
    rank_colliders(c->dev.sph, c->dev.nsph);
    destroy_graph(c);
    return B3G_OK;
}

b3g_status b3g_cloth_add_static_capsule(b3g_cloth* c, const float a[3], const float b[3], float radius,
                                        float friction, uint32_t* shape_id)
{
    if (!valid(c) || !a || !b || !(radius > 0.0f) || !(friction >= 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    for (int q = 0; q < 3; ++q)
        if (!std::isfinite(a[q]) || !std::isfinite(b[q])) return B3G_ERR_INVALID_ARGUMENT;
    if (c->dev.nsph >= (uint32_t)kMaxSpheres) return B3G_ERR_CAPACITY;
    SphereDev& s = c->dev.sph[c->dev.nsph];
    s = SphereDev{};
    s.kind = 1;
    s.ax = a[0], s.ay = a[1], s.az = a[2];
    s.bx = b[0], s.by = b[1], s.bz = b[2];
    s.radius = radius;
    s.friction = friction;
    // b3CapsuleShape::ComputeAABB (capsule_shape.cpp:130-137) fattened by B3_AABB_EXTENSION
    for (int q = 0; q < 3; ++q) {
        s.lo[q] = (std::min(a[q], b[q]) - radius) - 0.2f;
        s.hi[q] = (std::max(a[q], b[q]) + radius) + 0.2f;
    }
    if (shape_id) *shape_id = c->dev.nsph;
    c->dev.nsph += 1;
    c->report_fixed = false;
    rank_colliders(c->dev.sph, c->dev.nsph);
    destroy_graph(c);
    return B3G_OK;
}

}  // extern "C"

namespace {

// Copies a hull's vertices and planes to the device (kept until the
// colliders are cleared).
b3g_status upload_hull(b3g_cloth* c, const float* vertices, uint32_t vertex_count, const float* planes,
                       uint32_t face_count, float** out)
{
    cudaSetDevice(c->device);
    const size_t nf = 3 * (size_t)vertex_count + 4 * (size_t)face_count;
    std::vector<float> img(nf);
    std::memcpy(img.data(), vertices, 3 * (size_t)vertex_count * sizeof(float));
    std::memcpy(img.data() + 3 * (size_t)vertex_count, planes, 4 * (size_t)face_count * sizeof(float));
    float* d = nullptr;
    B3G_TRY(cudaMalloc(&d, nf * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(d, img.data(), nf * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        cudaFree(d);
        return from_cuda(e);
    }
    c->hull_bufs.push_back(d);
    *out = d;
    return B3G_OK;
}

bool hull_args_ok(const float* vertices, uint32_t vertex_count, const float* planes, uint32_t face_count,
                  float friction)
{
    if (!vertices || !planes || vertex_count == 0 || face_count == 0 || vertex_count > 4096 || face_count > 4096 ||
        !(friction >= 0.0f))
        return false;
    for (uint32_t k = 0; k < 3 * vertex_count; ++k)
        if (!std::isfinite(vertices[k])) return false;
    for (uint32_t k = 0; k < 4 * face_count; ++k)
        if (!std::isfinite(planes[k])) return false;
    return true;
}

}  // namespace

extern "C" {

b3g_status b3g_cloth_add_static_hull(b3g_cloth* c, const float* vertices, uint32_t vertex_count,
                                     const float* planes, uint32_t face_count, float friction, uint32_t* shape_id)
{
    if (!valid(c) || !hull_args_ok(vertices, vertex_count, planes, face_count, friction))
        return B3G_ERR_INVALID_ARGUMENT;
    if (c->dev.nsph >= (uint32_t)kMaxSpheres) return B3G_ERR_CAPACITY;
    float* d = nullptr;
    const b3g_status us = upload_hull(c, vertices, vertex_count, planes, face_count, &d);
    if (us != B3G_OK) return us;
    SphereDev& s = c->dev.sph[c->dev.nsph];
    s = SphereDev{};
    s.kind = 2;
    s.radius = 0.0f;  // B3_HULL_RADIUS
    s.friction = friction;
    s.hull = d;
    s.nhv = vertex_count;
    s.nhf = face_count;
    // b3HullShape::ComputeAABB (hull_shape.cpp:162-166): the body-frame
    // vertices' bounds, extended by the hull radius, fattened by
    // B3_AABB_EXTENSION
    float lo[3], hi[3];
    for (uint32_t k = 0; k < vertex_count; ++k) {
        const float* v = vertices + 3 * k;
        // b3Mul(xf, v) with the identity rotation at the origin
        const float w[3] = {((v[0] * 1.0f + v[1] * 0.0f) + v[2] * 0.0f) + 0.0f,
                            ((v[0] * 0.0f + v[1] * 1.0f) + v[2] * 0.0f) + 0.0f,
                            ((v[0] * 0.0f + v[1] * 0.0f) + v[2] * 1.0f) + 0.0f};
        for (int q = 0; q < 3; ++q) {
            if (k == 0) {
                lo[q] = hi[q] = w[q];
            } else {
                lo[q] = lo[q] < w[q] ? lo[q] : w[q];
                hi[q] = hi[q] > w[q] ? hi[q] : w[q];
            }
        }
    }
    for (int q = 0; q < 3; ++q) {
        s.lo[q] = (lo[q] - s.radius) - 0.2f;
        s.hi[q] = (hi[q] + s.radius) + 0.2f;
    }
    if (shape_id) *shape_id = c->dev.nsph;
    c->dev.nsph += 1;
    c->report_fixed = false;
    rank_colliders(c->dev.sph, c->dev.nsph);
    destroy_graph(c);
    return B3G_OK;
}

static void free_hulls(b3g_cloth* c)
{
    for (void* p : c->hull_bufs) cudaFree(p);
    c->hull_bufs.clear();
}

b3g_status b3g_cloth_clear_colliders(b3g_cloth* c)
{
    if (!valid(c)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    B3G_TRY(launch_clear_contacts(c->dev, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    c->dev.nsph = 0;
    c->dev.nbody = 0;
    c->report_fixed = false;
    free_hulls(c);
    destroy_graph(c);
    return B3G_OK;
}

// ---------------------------------------------------------------------------
// colliders on bodies (b3Cloth::SetWorld with b3Body)
// ---------------------------------------------------------------------------

}  // extern "C"

namespace {

constexpr uint32_t kMaxBodies = kMaxSpheres;  // a body matters to the cloth only through a collider

bool body_ok(const b3g_body_state& b)
{
    if (b.type < 0 || b.type > 2) return false;
    const float* f = b.rotation;
    const size_t nf = (sizeof(b3g_body_state) - offsetof(b3g_body_state, rotation)) / sizeof(float);
    for (size_t k = 0; k < nf; ++k)
        if (!std::isfinite(f[k])) return false;
    return true;
}

// The bodies' and the body shapes' proxies' device buffer, made on first use.
b3g_status ensure_body_buf(b3g_cloth* c)
{
    if (c->body_buf) return B3G_OK;
    cudaSetDevice(c->device);
    const size_t bytes = kMaxBodies * sizeof(b3g_body_state) + 6 * kMaxSpheres * sizeof(float);
    B3G_TRY(cudaMalloc(&c->body_buf, bytes));
    B3G_TRY(cudaMemsetAsync(c->body_buf, 0, bytes, c->stream));
    c->dev.bodies = (b3g_body_state*)c->body_buf;
    c->dev.shape_fat = (float*)((char*)c->body_buf + kMaxBodies * sizeof(b3g_body_state));
    return B3G_OK;
}

// b3Mul(xf, v) on the host, in the device's float order
void xf_point(const float R[9], const float p[3], const float v[3], float out[3])
{
    for (int q = 0; q < 3; ++q) out[q] = ((v[0] * R[q] + v[1] * R[3 + q]) + v[2] * R[6 + q]) + p[q];
}

// b3Shape::ComputeAABB(m_xf) of a body shape, fattened by B3_AABB_EXTENSION
// (b3BroadPhase::CreateProxy, broad_phase.cpp:78-82).
void body_shape_proxy(const SphereDev& s, const float* hull_host, const b3g_body_state& b, float lo[3], float hi[3])
{
    float l[3], h[3];
    if (s.kind == 0) {
        const float ctr[3] = {s.cx, s.cy, s.cz};
        float w[3];
        xf_point(b.rotation, b.position, ctr, w);
        for (int q = 0; q < 3; ++q) l[q] = h[q] = w[q];
    } else if (s.kind == 1) {
        const float A[3] = {s.ax, s.ay, s.az}, B[3] = {s.bx, s.by, s.bz};
        float wa[3], wb[3];
        xf_point(b.rotation, b.position, A, wa);
        xf_point(b.rotation, b.position, B, wb);
        for (int q = 0; q < 3; ++q) {
            l[q] = wa[q] < wb[q] ? wa[q] : wb[q];
            h[q] = wa[q] > wb[q] ? wa[q] : wb[q];
        }
    } else {
        for (uint32_t k = 0; k < s.nhv; ++k) {
            float w[3];
            xf_point(b.rotation, b.position, hull_host + 3 * k, w);
            for (int q = 0; q < 3; ++q) {
                l[q] = k == 0 || w[q] < l[q] ? w[q] : l[q];
                h[q] = k == 0 || w[q] > h[q] ? w[q] : h[q];
            }
        }
    }
    for (int q = 0; q < 3; ++q) {
        lo[q] = (l[q] - s.radius) - 0.2f;
        hi[q] = (h[q] + s.radius) + 0.2f;
    }
}

b3g_status read_body(const b3g_cloth* c, uint32_t id, b3g_body_state* out)
{
    cudaSetDevice(c->device);
    B3G_TRY(cudaMemcpyAsync(out, c->dev.bodies + id, sizeof(b3g_body_state), cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

// Installs collider `s` on body `body_id`: its proxy from the body's
// current transform, host and device copies.
b3g_status add_body_shape(b3g_cloth* c, uint32_t body_id, SphereDev s, const float* hull_host, uint32_t* shape_id)
{
    b3g_body_state b;
    b3g_status st = read_body(c, body_id, &b);
    if (st != B3G_OK) return st;
    s.body1 = body_id + 1;
    body_shape_proxy(s, hull_host, b, s.lo, s.hi);
    const uint32_t id = c->dev.nsph;
    const float fat[6] = {s.lo[0], s.lo[1], s.lo[2], s.hi[0], s.hi[1], s.hi[2]};
    B3G_TRY(cudaMemcpyAsync(c->dev.shape_fat + 6 * id, fat, sizeof(fat), cudaMemcpyHostToDevice, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    c->dev.sph[id] = s;
    c->dev.nsph += 1;
    c->report_fixed = false;
    rank_colliders(c->dev.sph, c->dev.nsph);
    destroy_graph(c);
    if (shape_id) *shape_id = id;
    return B3G_OK;
}

bool body_target(const b3g_cloth* c, uint32_t body_id) { return valid(c) && body_id < c->dev.nbody; }

}  // namespace

extern "C" {

b3g_status b3g_cloth_add_body(b3g_cloth* c, const b3g_body_state* state, uint32_t* body_id)
{
    if (!valid(c) || !state || !body_ok(*state)) return B3G_ERR_INVALID_ARGUMENT;
    if (c->self || !c->owns_stream) return B3G_ERR_UNSUPPORTED;  // single cloths without self-collision
    if (c->dev.nbody >= kMaxBodies) return B3G_ERR_CAPACITY;
    b3g_status s = ensure_body_buf(c);
    if (s != B3G_OK) return s;
    B3G_TRY(cudaMemcpyAsync(c->dev.bodies + c->dev.nbody, state, sizeof(b3g_body_state), cudaMemcpyHostToDevice,
                            c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    if (body_id) *body_id = c->dev.nbody;
    c->dev.nbody += 1;
    destroy_graph(c);
    return B3G_OK;
}

b3g_status b3g_cloth_set_body(b3g_cloth* c, uint32_t body_id, const b3g_body_state* state)
{
    if (!valid(c) || !state || body_id >= c->dev.nbody || !body_ok(*state)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    B3G_TRY(cudaMemcpyAsync(c->dev.bodies + body_id, state, sizeof(b3g_body_state), cudaMemcpyHostToDevice,
                            c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

b3g_status b3g_cloth_get_body(const b3g_cloth* c, uint32_t body_id, b3g_body_state* state)
{
    if (!valid(c) || !state || body_id >= c->dev.nbody) return B3G_ERR_INVALID_ARGUMENT;
    return read_body(c, body_id, state);
}

b3g_status b3g_cloth_add_body_sphere(b3g_cloth* c, uint32_t body_id, const float center[3], float radius,
                                     float friction, uint32_t* shape_id)
{
    if (!body_target(c, body_id) || !center || !(radius > 0.0f) || !(friction >= 0.0f))
        return B3G_ERR_INVALID_ARGUMENT;
    for (int q = 0; q < 3; ++q)
        if (!std::isfinite(center[q])) return B3G_ERR_INVALID_ARGUMENT;
    if (c->dev.nsph >= (uint32_t)kMaxSpheres) return B3G_ERR_CAPACITY;
    SphereDev s{};
    s.kind = 0;
    s.cx = center[0], s.cy = center[1], s.cz = center[2];
    s.radius = radius;
    s.friction = friction;
    return add_body_shape(c, body_id, s, nullptr, shape_id);
}

b3g_status b3g_cloth_add_body_capsule(b3g_cloth* c, uint32_t body_id, const float a[3], const float b[3],
                                      float radius, float friction, uint32_t* shape_id)
{
    if (!body_target(c, body_id) || !a || !b || !(radius > 0.0f) || !(friction >= 0.0f))
        return B3G_ERR_INVALID_ARGUMENT;
    for (int q = 0; q < 3; ++q)
        if (!std::isfinite(a[q]) || !std::isfinite(b[q])) return B3G_ERR_INVALID_ARGUMENT;
    if (c->dev.nsph >= (uint32_t)kMaxSpheres) return B3G_ERR_CAPACITY;
    SphereDev s{};
    s.kind = 1;
    s.ax = a[0], s.ay = a[1], s.az = a[2];
    s.bx = b[0], s.by = b[1], s.bz = b[2];
    s.radius = radius;
    s.friction = friction;
    return add_body_shape(c, body_id, s, nullptr, shape_id);
}

b3g_status b3g_cloth_add_body_hull(b3g_cloth* c, uint32_t body_id, const float* vertices, uint32_t vertex_count,
                                   const float* planes, uint32_t face_count, float friction, uint32_t* shape_id)
{
    if (!body_target(c, body_id) || !hull_args_ok(vertices, vertex_count, planes, face_count, friction))
        return B3G_ERR_INVALID_ARGUMENT;
    if (c->dev.nsph >= (uint32_t)kMaxSpheres) return B3G_ERR_CAPACITY;
    float* d = nullptr;
    const b3g_status us = upload_hull(c, vertices, vertex_count, planes, face_count, &d);
    if (us != B3G_OK) return us;
    SphereDev s{};
    s.kind = 2;
    s.radius = 0.0f;  // B3_HULL_RADIUS
    s.friction = friction;
    s.hull = d;
    s.nhv = vertex_count;
    s.nhf = face_count;
    return add_body_shape(c, body_id, s, vertices, shape_id);
}

b3g_status b3g_cloth_set_shape_proxy(b3g_cloth* c, uint32_t shape_id, const float lo[3], const float hi[3])
{
    if (!valid(c) || !lo || !hi || shape_id >= c->dev.nsph || !c->dev.sph[shape_id].body1)
        return B3G_ERR_INVALID_ARGUMENT;
    for (int q = 0; q < 3; ++q)
        if (!std::isfinite(lo[q]) || !std::isfinite(hi[q]) || !(lo[q] <= hi[q])) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    const float fat[6] = {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]};
    B3G_TRY(cudaMemcpyAsync(c->dev.shape_fat + 6 * shape_id, fat, sizeof(fat), cudaMemcpyHostToDevice, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    SphereDev& s = c->dev.sph[shape_id];
    for (int q = 0; q < 3; ++q) {
        s.lo[q] = lo[q];
        s.hi[q] = hi[q];
    }
    return B3G_OK;
}

b3g_status b3g_cloth_get_shape_proxy(const b3g_cloth* c, uint32_t shape_id, float lo[3], float hi[3])
{
    if (!valid(c) || !lo || !hi || shape_id >= c->dev.nsph) return B3G_ERR_INVALID_ARGUMENT;
    const SphereDev& s = c->dev.sph[shape_id];
    if (!s.body1) {
        for (int q = 0; q < 3; ++q) {
            lo[q] = s.lo[q];
            hi[q] = s.hi[q];
        }
        return B3G_OK;
    }
    cudaSetDevice(c->device);
    float fat[6];
    B3G_TRY(cudaMemcpyAsync(fat, c->dev.shape_fat + 6 * shape_id, sizeof(fat), cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    for (int q = 0; q < 3; ++q) {
        lo[q] = fat[q];
        hi[q] = fat[3 + q];
    }
    return B3G_OK;
}

b3g_status b3g_cloth_set_report_order(b3g_cloth* c, const uint32_t* order, uint32_t count)
{
    if (!valid(c) || (count && !order)) return B3G_ERR_INVALID_ARGUMENT;
    const uint32_t m = c->dev.nsph;
    if (count == 0) {
        c->report_fixed = false;
        rank_colliders(c->dev.sph, m);
        return B3G_OK;
    }
    if (count != m) return B3G_ERR_INVALID_ARGUMENT;
    bool seen[kMaxSpheres] = {};
    for (uint32_t r = 0; r < count; ++r) {
        if (order[r] >= m || seen[order[r]]) return B3G_ERR_INVALID_ARGUMENT;
        seen[order[r]] = true;
    }
    for (uint32_t r = 0; r < count; ++r) c->dev.sph[order[r]].rank = r;
    c->report_fixed = true;
    destroy_graph(c);
    return B3G_OK;
}

// ---------------------------------------------------------------------------
// created particles and forces (cloth.cpp:307-364): the layout is rebuilt
// around the cloth's current state
// ---------------------------------------------------------------------------

namespace {

// Every per-particle device array of a cloth, on the host (SoA planes).
struct ParticleState {
    uint32_t n = 0, nsph = 0;
    std::vector<float> x, v, fext, y, mx, lo, hi, mass, radius, friction;
    std::vector<uint8_t> type, c_exists, c_active;
    std::vector<uint32_t> c_key;
    std::vector<float> c_normal, c_t1, c_t2, c_imp, c_point;
};

b3g_status download_state(b3g_cloth* c, ParticleState& s)
{
    const ClothDev& d = c->dev;
    cudaStream_t st = c->stream;
    s.n = d.n;
    s.nsph = d.nsph;
    const size_t n = s.n, nn = (size_t)s.nsph * n;
    auto get = [&](auto& dst, const void* src, size_t count) {
        dst.resize(count);
        return count ? cudaMemcpyAsync(dst.data(), src, count * sizeof(dst[0]), cudaMemcpyDeviceToHost, st)
                     : cudaSuccess;
    };
    B3G_TRY(get(s.x, d.x, 3 * n));
    B3G_TRY(get(s.v, d.v, 3 * n));
    B3G_TRY(get(s.fext, d.fext, 3 * n));
    B3G_TRY(get(s.y, d.y, 3 * n));
    B3G_TRY(get(s.mx, d.mx, 3 * n));
    B3G_TRY(get(s.lo, d.fat_lo, 3 * n));
    B3G_TRY(get(s.hi, d.fat_hi, 3 * n));
    B3G_TRY(get(s.mass, d.mass, n));
    B3G_TRY(get(s.type, d.type, n));
    B3G_TRY(get(s.radius, d.p_radius, n));
    B3G_TRY(get(s.friction, d.p_friction, n));
    B3G_TRY(get(s.c_exists, d.c_exists, nn));
    B3G_TRY(get(s.c_active, d.c_active, nn));
    B3G_TRY(get(s.c_key, d.c_key, nn));
    B3G_TRY(get(s.c_normal, d.c_normal, 3 * nn));
    B3G_TRY(get(s.c_t1, d.c_t1, 3 * nn));
    B3G_TRY(get(s.c_t2, d.c_t2, 3 * nn));
    B3G_TRY(get(s.c_imp, d.c_imp, 3 * nn));
    B3G_TRY(get(s.c_point, d.c_point, 3 * nn));
    B3G_TRY(cudaStreamSynchronize(st));
    return B3G_OK;
}

b3g_status upload_state(b3g_cloth* c, const ParticleState& s)
{
    const ClothDev& d = c->dev;
    cudaStream_t st = c->stream;
    const size_t n = s.n, nn = (size_t)s.nsph * n;
    auto put = [&](void* dst, const auto& src, size_t count) {
        return count ? cudaMemcpyAsync(dst, src.data(), count * sizeof(src[0]), cudaMemcpyHostToDevice, st)
                     : cudaSuccess;
    };
    B3G_TRY(put(d.x, s.x, 3 * n));
    B3G_TRY(put(d.v, s.v, 3 * n));
    B3G_TRY(put(d.fext, s.fext, 3 * n));
    B3G_TRY(put(d.y, s.y, 3 * n));
    B3G_TRY(put(d.mx, s.mx, 3 * n));
    B3G_TRY(put(d.fat_lo, s.lo, 3 * n));
    B3G_TRY(put(d.fat_hi, s.hi, 3 * n));
    B3G_TRY(put(const_cast<float*>(d.mass), s.mass, n));
    B3G_TRY(put(d.type, s.type, n));
    B3G_TRY(put(d.p_radius, s.radius, n));
    B3G_TRY(put(d.p_friction, s.friction, n));
    B3G_TRY(put(d.c_exists, s.c_exists, nn));
    B3G_TRY(put(d.c_active, s.c_active, nn));
    B3G_TRY(put(d.c_key, s.c_key, nn));
    B3G_TRY(put(d.c_normal, s.c_normal, 3 * nn));
    B3G_TRY(put(d.c_t1, s.c_t1, 3 * nn));
    B3G_TRY(put(d.c_t2, s.c_t2, 3 * nn));
    B3G_TRY(put(d.c_imp, s.c_imp, 3 * nn));
    B3G_TRY(put(d.c_point, s.c_point, 3 * nn));
    return B3G_OK;
}

// The state of a new particle set: particle k of the result is old particle
// keep[k], or a zeroed new one when keep[k] is kNone.
constexpr uint32_t kNone = 0xffffffffu;

ParticleState remap(const ParticleState& s, const std::vector<uint32_t>& keep)
{
    ParticleState r;
    r.n = (uint32_t)keep.size();
    r.nsph = s.nsph;
    const size_t n0 = s.n, n1 = r.n, nn0 = (size_t)s.nsph * n0, nn1 = (size_t)s.nsph * n1;
    auto planes = [&](const std::vector<float>& a, std::vector<float>& b, size_t stride0, size_t stride1,
                      uint32_t groups) {
        b.assign(stride1 * 3, 0.0f);
        for (int q = 0; q < 3; ++q)
            for (uint32_t g = 0; g < groups; ++g)
                for (size_t k = 0; k < n1; ++k)
                    if (keep[k] != kNone) b[q * stride1 + g * n1 + k] = a[q * stride0 + g * n0 + keep[k]];
    };
    auto column = [&](const auto& a, auto& b, uint32_t groups) {
        b.assign((size_t)groups * n1, {});
        for (uint32_t g = 0; g < groups; ++g)
            for (size_t k = 0; k < n1; ++k)
                if (keep[k] != kNone) b[g * n1 + k] = a[g * n0 + keep[k]];
    };
    planes(s.x, r.x, n0, n1, 1);
    planes(s.v, r.v, n0, n1, 1);
    planes(s.fext, r.fext, n0, n1, 1);
    planes(s.y, r.y, n0, n1, 1);
    planes(s.mx, r.mx, n0, n1, 1);
    planes(s.lo, r.lo, n0, n1, 1);
    planes(s.hi, r.hi, n0, n1, 1);
    column(s.mass, r.mass, 1);
    column(s.type, r.type, 1);
    column(s.radius, r.radius, 1);
    column(s.friction, r.friction, 1);
    column(s.c_exists, r.c_exists, s.nsph);
    column(s.c_active, r.c_active, s.nsph);
    column(s.c_key, r.c_key, s.nsph);
    planes(s.c_normal, r.c_normal, nn0, nn1, s.nsph);
    planes(s.c_t1, r.c_t1, nn0, nn1, s.nsph);
    planes(s.c_t2, r.c_t2, nn0, nn1, s.nsph);
    planes(s.c_imp, r.c_imp, nn0, nn1, s.nsph);
    planes(s.c_point, r.c_point, nn0, nn1, s.nsph);
    return r;
}

// Lays the cloth out again for its current particles and mouse forces
// (n_extra and mice already updated) into a new arena, installs `s` there,
// and frees the old arena.  On failure the previous layout is restored.
b3g_status relayout(b3g_cloth* c, const ParticleState& s, uint32_t old_extra, std::vector<MouseForceDesc> old_mice,
                    std::vector<uint32_t> old_ids)
{
    char* old_base = c->arena.base;
    const size_t old_size = c->arena.size;
    const ClothDev old_dev = c->dev;
    ClothTopology old_topo = c->topo;
    auto restore = [&]() {
        c->n_extra = old_extra;
        c->mice = std::move(old_mice);
        c->mouse_ids = std::move(old_ids);
        c->topo = std::move(old_topo);
        c->dev = old_dev;
        c->arena.base = old_base;
        c->arena.size = old_size;
        c->images.reset();
    };
    b3g_status st = layout_cloth(c);
    if (st != B3G_OK) {
        restore();
        return st;
    }
    c->dev.nsph = old_dev.nsph;
    std::memcpy(c->dev.sph, old_dev.sph, sizeof(old_dev.sph));
    c->dev.bodies = old_dev.bodies;
    c->dev.shape_fat = old_dev.shape_fat;
    c->dev.nbody = old_dev.nbody;
    // the host copy of the masses follows the state (created particles carry their own)
    for (uint32_t i = 0; i < s.n && i < c->topo.mass.size(); ++i) c->topo.mass[i] = s.mass[i];
    char* base = nullptr;
    if (cudaMalloc(&base, c->arena.size) != cudaSuccess) {
        cudaGetLastError();
        restore();
        return B3G_ERR_OUT_OF_MEMORY;
    }
    const bool owns_stream = c->owns_stream;
    st = realize_cloth(c, c->device, base, true, c->stream, false);
    c->owns_stream = owns_stream;
    if (st == B3G_OK) st = upload_state(c, s);
    if (st == B3G_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) st = B3G_ERR_CUDA;
    if (st != B3G_OK) {
        cudaStreamSynchronize(c->stream);
        cudaFree(base);
        cudaGetLastError();
        restore();
        return st;
    }
    finish_upload(c);
    destroy_graph(c);
    cudaFree(old_base);
    c->layout_version += 1;
    return B3G_OK;
}

bool editable(const b3g_cloth* c) { return valid(c) && c->owns_arena && c->owns_stream; }

}  // namespace

extern "C" {

b3g_status b3g_cloth_create_particle(b3g_cloth* c, const b3g_particle_def* def, uint32_t* index)
{
    if (c && c->self) return B3G_ERR_UNSUPPORTED;  // not with self-collision
    if (!editable(c) || !def || !index) return B3G_ERR_INVALID_ARGUMENT;
    for (int q = 0; q < 3; ++q)
        if (!std::isfinite(def->position[q]) || !std::isfinite(def->velocity[q]) || !std::isfinite(def->force[q]))
            return B3G_ERR_INVALID_ARGUMENT;
    if (!(def->mass >= 0.0f) || !std::isfinite(def->mass) || !(def->radius >= 0.0f) || !std::isfinite(def->radius) ||
        !(def->friction >= 0.0f) || !std::isfinite(def->friction))
        return B3G_ERR_INVALID_ARGUMENT;
    const bool dynamic = def->mass != 0.0f;
    cudaSetDevice(c->device);
    b3g_status st = flush_ops(c);
    if (st != B3G_OK) return st;
    ParticleState s;
    if ((st = download_state(c, s)) != B3G_OK) return st;
    std::vector<uint32_t> keep(s.n + 1);
    for (uint32_t k = 0; k < s.n; ++k) keep[k] = k;
    keep[s.n] = kNone;
    ParticleState r = remap(s, keep);
    // b3Particle::b3Particle (particle.cpp:24-51); proxy: its AABB fattened
    // by B3_AABB_EXTENSION (cloth.cpp:311-317)
    const uint32_t i = s.n, n1 = r.n;
    for (int q = 0; q < 3; ++q) {
        const float p = def->position[q];
        r.x[q * (size_t)n1 + i] = p;
        r.v[q * (size_t)n1 + i] = def->velocity[q];
        r.fext[q * (size_t)n1 + i] = def->force[q];
        r.lo[q * (size_t)n1 + i] = (p - def->radius) - 0.2f;
        r.hi[q * (size_t)n1 + i] = (p + def->radius) + 0.2f;
    }
    r.mass[i] = dynamic ? def->mass : 1.0f;
    r.radius[i] = def->radius;
    r.friction[i] = def->friction;
    r.type[i] = (uint8_t)(dynamic ? B3G_DYNAMIC : B3G_STATIC);
    const uint32_t old_extra = c->n_extra;
    c->n_extra += 1;
    if ((st = relayout(c, r, old_extra, c->mice, c->mouse_ids)) != B3G_OK) return st;
    *index = i;
    return B3G_OK;
}

b3g_status b3g_cloth_destroy_particle(b3g_cloth* c, uint32_t index)
{
    if (c && c->self) return B3G_ERR_UNSUPPORTED;  // not with self-collision
    if (!editable(c)) return B3G_ERR_INVALID_ARGUMENT;
    const uint32_t n_mesh = c->topo.n_mesh;
    if (index < n_mesh || index >= c->dev.n) return B3G_ERR_INVALID_ARGUMENT;  // only created particles
    cudaSetDevice(c->device);
    b3g_status st = flush_ops(c);
    if (st != B3G_OK) return st;
    ParticleState s;
    if ((st = download_state(c, s)) != B3G_OK) return st;
    std::vector<uint32_t> keep;
    for (uint32_t k = 0; k < s.n; ++k)
        if (k != index) keep.push_back(k);
    ParticleState r = remap(s, keep);
    const uint32_t old_extra = c->n_extra;
    std::vector<MouseForceDesc> old_mice = c->mice;
    std::vector<uint32_t> old_ids = c->mouse_ids;
    // its forces go with it (cloth.cpp:329-340); later particles move down one
    std::vector<MouseForceDesc> mice;
    std::vector<uint32_t> ids;
    for (size_t m = 0; m < c->mice.size(); ++m) {
        MouseForceDesc f = c->mice[m];
        if (f.particle == index) continue;
        if (f.particle > index) f.particle -= 1;
        mice.push_back(f);
        ids.push_back(c->mouse_ids[m]);
    }
    c->mice = mice;
    c->mouse_ids = ids;
    c->n_extra -= 1;
    return relayout(c, r, old_extra, old_mice, old_ids);
}

b3g_status b3g_cloth_create_mouse_force(b3g_cloth* c, const b3g_mouse_force_def* def, uint32_t* force_id)
{
    if (c && c->self) return B3G_ERR_UNSUPPORTED;  // not with self-collision
    if (!editable(c) || !def || !force_id) return B3G_ERR_INVALID_ARGUMENT;
    if (def->particle >= c->dev.n || def->triangle >= c->dev.t) return B3G_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(def->w2) || !std::isfinite(def->w3) || !std::isfinite(def->w4) ||
        !std::isfinite(def->mouse) || !std::isfinite(def->damping))
        return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status st = flush_ops(c);
    if (st != B3G_OK) return st;
    ParticleState s;
    if ((st = download_state(c, s)) != B3G_OK) return st;
    std::vector<MouseForceDesc> old_mice = c->mice;
    std::vector<uint32_t> old_ids = c->mouse_ids;
    c->mice.push_back(MouseForceDesc{def->particle, def->triangle, def->w2, def->w3, def->w4, def->mouse,
                                     def->damping});
    const uint32_t id = ++c->next_force_id;
    c->mouse_ids.push_back(id);
    if ((st = relayout(c, s, c->n_extra, old_mice, old_ids)) != B3G_OK) return st;
    *force_id = id;
    return B3G_OK;
}

b3g_status b3g_cloth_destroy_force(b3g_cloth* c, uint32_t force_id)
{
    if (c && c->self) return B3G_ERR_UNSUPPORTED;  // not with self-collision
    if (!editable(c)) return B3G_ERR_INVALID_ARGUMENT;
    size_t m = 0;
    while (m < c->mouse_ids.size() && c->mouse_ids[m] != force_id) ++m;
    if (m == c->mouse_ids.size()) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status st = flush_ops(c);
    if (st != B3G_OK) return st;
    ParticleState s;
    if ((st = download_state(c, s)) != B3G_OK) return st;
    std::vector<MouseForceDesc> old_mice = c->mice;
    std::vector<uint32_t> old_ids = c->mouse_ids;
    c->mice.erase(c->mice.begin() + m);
    c->mouse_ids.erase(c->mouse_ids.begin() + m);
    return relayout(c, s, c->n_extra, old_mice, old_ids);
}

}  // extern "C"

static b3g_status push_op(b3g_cloth* c, uint32_t vertex, uint32_t kind, const float* a)
{
    if (!valid(c) || vertex >= c->dev.n) return B3G_ERR_INVALID_ARGUMENT;
    ParticleOp op;
    op.vertex = vertex;
    op.kind = kind;
    op.a[0] = a ? a[0] : 0.0f;
    op.a[1] = a ? a[1] : 0.0f;
    op.a[2] = a ? a[2] : 0.0f;
    c->pending.push_back(op);
    return B3G_OK;
}

b3g_status b3g_particle_set_type(b3g_cloth* c, uint32_t vertex, b3g_particle_type type)
{
    if (type != B3G_STATIC && type != B3G_KINEMATIC && type != B3G_DYNAMIC) return B3G_ERR_INVALID_ARGUMENT;
    float a[3] = {(float)type, 0.0f, 0.0f};
    return push_op(c, vertex, OP_SET_TYPE, a);
}

b3g_status b3g_particle_set_position(b3g_cloth* c, uint32_t vertex, const float p[3])
{
    if (!p) return B3G_ERR_INVALID_ARGUMENT;
    return push_op(c, vertex, OP_SET_POSITION, p);
}

b3g_status b3g_particle_set_velocity(b3g_cloth* c, uint32_t vertex, const float v[3])
{
    if (!v) return B3G_ERR_INVALID_ARGUMENT;
    return push_op(c, vertex, OP_SET_VELOCITY, v);
}

b3g_status b3g_particle_apply_force(b3g_cloth* c, uint32_t vertex, const float f[3])
{
    if (!f) return B3G_ERR_INVALID_ARGUMENT;
    return push_op(c, vertex, OP_APPLY_FORCE, f);
}

b3g_status b3g_particle_apply_translation(b3g_cloth* c, uint32_t vertex, const float t[3])
{
    if (!t) return B3G_ERR_INVALID_ARGUMENT;
    return push_op(c, vertex, OP_APPLY_TRANSLATION, t);
}

b3g_status b3g_particle_set_radius(b3g_cloth* c, uint32_t vertex, float radius)
{
    if (!(radius >= 0.0f) || !std::isfinite(radius)) return B3G_ERR_INVALID_ARGUMENT;
    const float a[3] = {radius, 0.0f, 0.0f};
    return push_op(c, vertex, OP_SET_RADIUS, a);
}

b3g_status b3g_particle_set_friction(b3g_cloth* c, uint32_t vertex, float friction)
{
    if (!(friction >= 0.0f) || !std::isfinite(friction)) return B3G_ERR_INVALID_ARGUMENT;
    const float a[3] = {friction, 0.0f, 0.0f};
    return push_op(c, vertex, OP_SET_FRICTION, a);
}

// One float of a per-particle plane, after the queued edits.
static b3g_status read_scalar(const b3g_cloth* cc, uint32_t vertex, const float* plane, float* out)
{
    b3g_cloth* c = const_cast<b3g_cloth*>(cc);
    if (!valid(c) || vertex >= c->dev.n || !out) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    B3G_TRY(cudaMemcpyAsync(out, plane + vertex, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

b3g_status b3g_particle_get_radius(const b3g_cloth* c, uint32_t vertex, float* radius)
{
    return valid(c) ? read_scalar(c, vertex, c->dev.p_radius, radius) : B3G_ERR_INVALID_ARGUMENT;
}

b3g_status b3g_particle_get_friction(const b3g_cloth* c, uint32_t vertex, float* friction)
{
    return valid(c) ? read_scalar(c, vertex, c->dev.p_friction, friction) : B3G_ERR_INVALID_ARGUMENT;
}

static b3g_status read_vertex(const b3g_cloth* cc, uint32_t vertex, const float* planes, float out[3])
{
    b3g_cloth* c = const_cast<b3g_cloth*>(cc);
    if (!valid(c) || vertex >= c->dev.n || !out) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    const uint32_t n = c->dev.n;
    for (int q = 0; q < 3; ++q)
        B3G_TRY(cudaMemcpyAsync(out + q, planes + (size_t)q * n + vertex, 4, cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

b3g_status b3g_particle_get_position(const b3g_cloth* c, uint32_t vertex, float p[3])
{
    return c ? read_vertex(c, vertex, c->dev.x, p) : B3G_ERR_INVALID_ARGUMENT;
}

b3g_status b3g_particle_get_velocity(const b3g_cloth* c, uint32_t vertex, float v[3])
{
    return c ? read_vertex(c, vertex, c->dev.v, v) : B3G_ERR_INVALID_ARGUMENT;
}

b3g_status b3g_particle_get_mass(const b3g_cloth* c, uint32_t vertex, float* m)
{
    if (!valid(c) || vertex >= c->dev.n || !m) return B3G_ERR_INVALID_ARGUMENT;
    *m = c->topo.mass[vertex];
    return B3G_OK;
}

b3g_status b3g_particle_get_type(const b3g_cloth* cc, uint32_t vertex, b3g_particle_type* type)
{
    b3g_cloth* c = const_cast<b3g_cloth*>(cc);
    if (!valid(c) || vertex >= c->dev.n || !type) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    uint8_t t8 = 0;
    B3G_TRY(cudaMemcpyAsync(&t8, c->dev.type + vertex, 1, cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    *type = (b3g_particle_type)t8;
    return B3G_OK;
}

b3g_status b3g_cloth_set_types(b3g_cloth* c, const uint8_t* types)
{
    if (!valid(c) || !types) return B3G_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < c->dev.n; ++i)
        if (types[i] > 2) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    B3G_TRY(cudaMemcpyAsync(c->d_stage_u8, types, c->dev.n, cudaMemcpyHostToDevice, c->stream));
    // the caller's buffer is free on return, page-locked or not
    B3G_TRY(cudaStreamSynchronize(c->stream));
    B3G_TRY(launch_set_types(c->dev, c->d_stage_u8, c->stream));
    return B3G_OK;
}

static b3g_status add_array(b3g_cloth* c, float* dst, const float* src, int only_dynamic)
{
    if (!valid(c) || !src) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    B3G_TRY(cudaMemcpyAsync(c->d_stage, src, 3 * (size_t)c->dev.n * 4, cudaMemcpyHostToDevice, c->stream));
    // the caller's buffer is free on return: a copy from page-locked memory
    // runs asynchronously, one from pageable memory is only staged
    B3G_TRY(cudaStreamSynchronize(c->stream));
    B3G_TRY(launch_add_vectors(c->dev, dst, c->d_stage, only_dynamic, c->stream));
    return B3G_OK;
}

b3g_status b3g_cloth_apply_forces(b3g_cloth* c, const float* f)
{
    return c ? add_array(c, c->dev.fext, f, 1) : B3G_ERR_INVALID_ARGUMENT;
}

b3g_status b3g_cloth_apply_translations(b3g_cloth* c, const float* t)
{
    return c ? add_array(c, c->dev.y, t, 0) : B3G_ERR_INVALID_ARGUMENT;
}

b3g_status b3g_cloth_step(b3g_cloth* c, float dt, uint32_t vel_iters, uint32_t pos_iters, b3g_step_stats* stats)
{
    if (!valid(c) || !c->owns_stream) return B3G_ERR_INVALID_ARGUMENT;
    if (!(dt >= 0.0f) || pos_iters > (uint32_t)kMaxPosIters) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    cudaStream_t st = c->stream;
    // step parameters (the pinned buffer is free: the previous step was waited for)
    StepScalars* h = c->h_sc;
    std::memset(h, 0, sizeof(StepScalars));
    h->dt = dt;
    h->vel_iters = vel_iters;
    h->pos_iters = pos_iters;
    h->step_index = ++c->step_index;
    h->max_iter = c->opts.max_iterations;
    h->stop_rule = (int)c->opts.stop_rule;
    h->tol = c->opts.tolerance;
    h->dot = (int)c->opts.dot;
    h->gx = c->gravity[0];
    h->gy = c->gravity[1];
    h->gz = c->gravity[2];
    if ((s = ensure_cg_rec(c)) != B3G_OK) return s;
    B3G_TRY(cudaMemcpyAsync(c->dev.sc, h, sizeof(StepScalars), cudaMemcpyHostToDevice, st));
    B3G_TRY(cudaEventRecord(c->ev0, st));
    if (c->self) {
        if ((s = launch_step_self(c, dt)) != B3G_OK) return s;
    } else if (dt > 0.0f && c->dev.nbody) {
        if ((s = launch_step_bodies(c)) != B3G_OK) return s;
    } else if (dt > 0.0f) {
        if (c->graph_ok && (!c->exec || c->graph_dot != (int)c->opts.dot || c->graph_pos_iters != pos_iters ||
                            c->graph_nsph != c->dev.nsph || c->graph_strategy != c->cg_strategy)) {
            if (build_graph(c, pos_iters) != B3G_OK) c->graph_ok = false;
        }
        if (c->graph_ok && c->exec) {
            B3G_TRY(cudaGraphLaunch(c->exec, st));
        } else {
            if ((s = launch_step_plain(c, pos_iters)) != B3G_OK) return s;
        }
    } else {
        // Step with dt = 0: contacts update, no solve, clear and AABB sync
        B3G_TRY(launch_contacts_update(c->dev, st));
        B3G_TRY(launch_post(c->dev, st));
    }
    B3G_TRY(cudaEventRecord(c->ev1, st));
    B3G_TRY(cudaMemcpyAsync(h, c->dev.sc, sizeof(StepScalars), cudaMemcpyDeviceToHost, st));
    B3G_TRY(cudaStreamSynchronize(st));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    b3g_step_stats& L = c->last;
    L.iterations = dt > 0.0f ? h->iter : 0;
    L.delta0 = h->delta0;
    L.delta = h->delta;
    L.b_delta = h->b_delta;
    L.active_contacts = h->active_contacts;
    L.contacts = h->contacts;
    L.step_ms = ms;
    if (dt > 0.0f && !c->self && !c->dev.nbody && c->graph_ok && c->exec) {
        // kernel nodes the graph ran: [contacts_update, hull contacts update]
        // assemble (two passes), cg_init, 3 per CG iteration (or the one
        // persistent CG), finalize, [contact_position x (pos_iters - 1)], post
        const uint64_t ns = c->dev.nsph ? 1 : 0;
        uint64_t hulls = 0;
        for (uint32_t q = 0; q < c->dev.nsph; ++q) hulls |= c->dev.sph[q].kind == 2 ? 1u : 0u;
        const uint64_t cg = persistent_cg(c) ? 1 : 1 + 3ull * L.iterations;
        count_launches(ns + hulls + 2 + cg + 1 + (ns && pos_iters > 1 ? pos_iters - 1 : 0) + 1);
    }
    if (stats) *stats = L;
    if (dt > 0.0f && h->status != 0) return (b3g_status)h->status;
    return B3G_OK;
}

b3g_status b3g_cloth_assemble(b3g_cloth* c, float dt)
{
    if (!valid(c) || !c->owns_stream || !(dt > 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    StepScalars* h = c->h_sc;
    B3G_TRY(cudaStreamSynchronize(c->stream));
    std::memset(h, 0, sizeof(StepScalars));
    h->dt = dt;
    h->gx = c->gravity[0];
    h->gy = c->gravity[1];
    h->gz = c->gravity[2];
    B3G_TRY(cudaMemcpyAsync(c->dev.sc, h, sizeof(StepScalars), cudaMemcpyHostToDevice, c->stream));
    B3G_TRY(launch_assemble(c->dev, c->assemble_block, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

b3g_status b3g_cloth_step_profiled(b3g_cloth* c, float dt, uint32_t vel_iters, uint32_t pos_iters,
                                   b3g_phase_times* times, b3g_step_stats* stats)
{
    if (c && c->self) return B3G_ERR_UNSUPPORTED;
    if (!valid(c) || !c->owns_stream || !times || !(dt > 0.0f) || pos_iters > (uint32_t)kMaxPosIters)
        return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    cudaStream_t st = c->stream;
    B3G_TRY(cudaStreamSynchronize(st));
    StepScalars* h = c->h_sc;
    std::memset(h, 0, sizeof(StepScalars));
    h->dt = dt;
    h->vel_iters = vel_iters;
    h->pos_iters = pos_iters;
    h->step_index = ++c->step_index;
    h->max_iter = c->opts.max_iterations;
    h->stop_rule = (int)c->opts.stop_rule;
    h->tol = c->opts.tolerance;
    h->dot = (int)c->opts.dot;
    h->gx = c->gravity[0];
    h->gy = c->gravity[1];
    h->gz = c->gravity[2];
    if ((s = ensure_cg_rec(c)) != B3G_OK) return s;
    B3G_TRY(cudaMemcpyAsync(c->dev.sc, h, sizeof(StepScalars), cudaMemcpyHostToDevice, st));
    std::memset(times, 0, sizeof(*times));
    const int dot = (int)c->opts.dot;
    float ms = 0.0f;
    auto timed = [&](float* acc, auto&& fn) -> b3g_status {
        B3G_TRY(cudaEventRecord(c->ev0, st));
        B3G_TRY(fn());
        B3G_TRY(cudaEventRecord(c->ev1, st));
        B3G_TRY(cudaEventSynchronize(c->ev1));
        B3G_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        *acc += ms;
        return B3G_OK;
    };
    cudaGraphConditionalHandle none = 0;
    if (c->dev.nsph && (s = timed(&times->contacts_update_ms, [&] { return launch_contacts_update(c->dev, st); })))
        return s;
    if ((s = timed(&times->assemble_ms, [&] { return launch_assemble(c->dev, c->assemble_block, st); }))) return s;
    StepScalars probe;
    if (persistent_cg(c)) {
        if ((s = timed(&times->cg_spmv_ms, [&] { return launch_persistent_cg(c, dot, st); }))) return s;
        B3G_TRY(cudaMemcpy(&probe, c->dev.sc, sizeof(StepScalars), cudaMemcpyDeviceToHost));
        times->cg_iterations = probe.iter;
    } else if ((s = timed(&times->cg_init_ms, [&] { return launch_cg_init(c->dev, dot, none, 0, st); }))) {
        return s;
    }
    for (; !persistent_cg(c);) {
        B3G_TRY(cudaMemcpy(&probe, c->dev.sc, sizeof(StepScalars), cudaMemcpyDeviceToHost));
        if (!probe.cont) break;
        if ((s = timed(&times->cg_spmv_ms, [&] { return launch_cg_part(c->dev, dot, 0, st); }))) return s;
        if ((s = timed(&times->cg_update_ms, [&] { return launch_cg_part(c->dev, dot, 1, st); }))) return s;
        if ((s = timed(&times->cg_direction_ms, [&] { return launch_cg_part(c->dev, dot, 2, st); }))) return s;
        times->cg_iterations += 1;
    }
    if ((s = timed(&times->finalize_ms, [&] { return launch_finalize(c->dev, st); }))) return s;
    for (uint32_t k = 1; c->dev.nsph && k < pos_iters && k < (uint32_t)kMaxPosIters; ++k) {
        if ((s = timed(&times->contact_position_ms, [&] { return launch_contact_position(c->dev, k, st); })))
            return s;
        times->contact_position_launches += 1;
    }
    if ((s = timed(&times->post_ms, [&] { return launch_post(c->dev, st); }))) return s;
    B3G_TRY(cudaMemcpyAsync(h, c->dev.sc, sizeof(StepScalars), cudaMemcpyDeviceToHost, st));
    B3G_TRY(cudaStreamSynchronize(st));
    b3g_step_stats& L = c->last;
    L.iterations = h->iter;
    L.delta0 = h->delta0;
    L.delta = h->delta;
    L.b_delta = h->b_delta;
    L.active_contacts = h->active_contacts;
    L.contacts = h->contacts;
    L.step_ms = times->contacts_update_ms + times->assemble_ms + times->cg_init_ms + times->cg_spmv_ms +
                times->cg_update_ms + times->cg_direction_ms + times->finalize_ms + times->contact_position_ms +
                times->post_ms;
    if (stats) *stats = L;
    if (h->status != 0) return (b3g_status)h->status;
    return B3G_OK;
}

b3g_status b3g_debug_cg_barrier_timeout(b3g_cloth* c, uint32_t spin_limit, b3g_status* result)
{
    if (!valid(c) || !c->owns_stream || !result || spin_limit == 0) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    cudaStream_t st = c->stream;
    // a barrier that cannot complete: the arrival counter starts half its
    // range away from every target, so every CTA waits until its limit
    GridBarrier bar = {0x80000000u, 0u, 0u, spin_limit};
    StepScalars* h = c->h_sc;
    B3G_TRY(cudaStreamSynchronize(st));
    fill_step_scalars(c, 1.0f / 60.0f, 8, 2, h);
    c->step_index -= 1;
    B3G_TRY(cudaMemcpyAsync(c->dev.sc, h, sizeof(StepScalars), cudaMemcpyHostToDevice, st));
    B3G_TRY(cudaMemcpyAsync(c->dev.bar, &bar, sizeof(bar), cudaMemcpyHostToDevice, st));
    B3G_TRY(launch_assemble(c->dev, c->assemble_block, st));
    if (c->cg_strategy == B3G_CG_PERSISTENT_FUSED) {
        b3g_status s = ensure_cg_rec(c);
        if (s != B3G_OK) return s;
        B3G_TRY(launch_grid_cg_fused(c->dev, (int)c->opts.dot, c->dev.bar, c->cg_rec, st));
    } else {
        B3G_TRY(launch_grid_cg(c->dev, (int)c->opts.dot, c->dev.bar, st));
    }
    B3G_TRY(cudaMemcpyAsync(h, c->dev.sc, sizeof(StepScalars), cudaMemcpyDeviceToHost, st));
    B3G_TRY(cudaStreamSynchronize(st));
    *result = (b3g_status)h->status;
    return B3G_OK;
}

b3g_status b3g_cloth_set_cg_strategy(b3g_cloth* c, b3g_cg_strategy s)
{
    if (!valid(c) || (s != B3G_CG_LAUNCHES && s != B3G_CG_PERSISTENT && s != B3G_CG_PERSISTENT_FUSED))
        return B3G_ERR_INVALID_ARGUMENT;
    c->cg_strategy = s;
    if (!c->owns_stream) return B3G_OK;  // batch and server cloths run their own CG
    cudaSetDevice(c->device);
    return ensure_cg_rec(c);
}

b3g_status b3g_cloth_set_assembly(b3g_cloth* c, b3g_assembly form)
{
    if (!valid(c) || (form != B3G_ASSEMBLY_ELEMENT_RECORDS && form != B3G_ASSEMBLY_ROWS))
        return B3G_ERR_INVALID_ARGUMENT;
    c->row_assembly = form == B3G_ASSEMBLY_ROWS;
    c->dev.slot_asm = c->topo.slot_terms && !c->row_assembly ? 1u : 0u;
    cudaSetDevice(c->device);
    destroy_graph(c);
    c->layout_version += 1;  // batches holding the cloth capture their step again
    return B3G_OK;
}

b3g_assembly b3g_cloth_get_assembly(const b3g_cloth* c)
{
    return valid(c) && c->dev.slot_asm ? B3G_ASSEMBLY_ELEMENT_RECORDS : B3G_ASSEMBLY_ROWS;
}

b3g_status b3g_cloth_get_info(const b3g_cloth* c, b3g_cloth_info* info)
{
    if (!valid(c) || !info) return B3G_ERR_INVALID_ARGUMENT;
    info->vertices = c->topo.n;
    info->triangles = c->topo.t;
    info->springs = c->topo.ns;
    info->blocks = (uint32_t)c->topo.row_cols.size();
    info->sell_entries = c->topo.E;
    info->max_degree = c->topo.max_deg;
    return B3G_OK;
}

uint32_t b3g_cloth_vertex_count(const b3g_cloth* c) { return valid(c) ? c->dev.n : 0u; }

// Planes to the caller's xyz buffer: transposed on the device into the
// staging buffer, then one copy.
static b3g_status read_planes(b3g_cloth* c, const float* planes, float* out)
{
    const uint32_t n = c->dev.n;
    B3G_TRY(launch_planes_to_xyz(planes, c->d_stage, n, c->stream));
    B3G_TRY(cudaMemcpyAsync(out, c->d_stage, 3 * (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

b3g_status b3g_cloth_read_state(const b3g_cloth* cc, float* x, float* v, float* mx)
{
    b3g_cloth* c = const_cast<b3g_cloth*>(cc);
    if (!valid(c)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    if (x && (s = read_planes(c, c->dev.x, x)) != B3G_OK) return s;
    if (v && (s = read_planes(c, c->dev.v, v)) != B3G_OK) return s;
    if (mx && (s = read_planes(c, c->dev.mx, mx)) != B3G_OK) return s;
    return B3G_OK;
}

b3g_status b3g_cloth_write_state(b3g_cloth* c, const float* x, const float* v, const float* mx)
{
    if (!valid(c)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    const uint32_t n = c->dev.n;
    const float* srcs[3] = {x, v, mx};
    float* dsts[3] = {c->dev.x, c->dev.v, c->dev.mx};
    for (int k = 0; k < 3; ++k) {
        if (!srcs[k]) continue;
        B3G_TRY(cudaMemcpyAsync(c->d_stage, srcs[k], 3 * (size_t)n * 4, cudaMemcpyHostToDevice, c->stream));
        B3G_TRY(launch_xyz_to_planes(c->d_stage, dsts[k], n, c->stream));
    }
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

b3g_status b3g_cloth_read_masses(const b3g_cloth* c, float* m)
{
    if (!valid(c) || !m) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    // the device copy: created particles carry their own masses
    B3G_TRY(cudaMemcpyAsync(m, c->dev.mass, (size_t)c->dev.n * 4, cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

b3g_status b3g_cloth_get_energy(const b3g_cloth* cc, float* energy)
{
    b3g_cloth* c = const_cast<b3g_cloth*>(cc);
    if (!valid(c) || !energy) return B3G_ERR_INVALID_ARGUMENT;
    const uint32_t n = c->dev.n;
    std::vector<float> v(3 * (size_t)n);
    b3g_status s = b3g_cloth_read_state(c, nullptr, v.data(), nullptr);
    if (s != B3G_OK) return s;
    // summed in particle-list order (newest particle first), cloth.cpp:366-374
    float E = 0.0f;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t i = n - 1 - k;
        E += c->topo.mass[i] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    }
    *energy = 0.5f * E;
    return B3G_OK;
}

b3g_status b3g_cloth_read_proxies(const b3g_cloth* cc, float* lo, float* hi)
{
    b3g_cloth* c = const_cast<b3g_cloth*>(cc);
    if (!valid(c) || (!lo && !hi)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    if (lo && (s = read_planes(c, c->dev.fat_lo, lo)) != B3G_OK) return s;
    if (hi && (s = read_planes(c, c->dev.fat_hi, hi)) != B3G_OK) return s;
    return B3G_OK;
}

b3g_status b3g_cloth_read_contacts(const b3g_cloth* cc, uint8_t* exists, uint8_t* active, float* impulses)
{
    b3g_cloth* c = const_cast<b3g_cloth*>(cc);
    if (!valid(c)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    const size_t nn = (size_t)c->dev.nsph * c->dev.n;
    if (!nn) return B3G_OK;
    const size_t nall = (size_t)kMaxSpheres * c->dev.n;
    if (exists) B3G_TRY(cudaMemcpyAsync(exists, c->dev.c_exists, nn, cudaMemcpyDeviceToHost, c->stream));
    if (active) B3G_TRY(cudaMemcpyAsync(active, c->dev.c_active, nn, cudaMemcpyDeviceToHost, c->stream));
    if (impulses) {
        std::vector<float> tmp(3 * nall);
        B3G_TRY(cudaMemcpyAsync(tmp.data(), c->dev.c_imp, 3 * nall * 4, cudaMemcpyDeviceToHost, c->stream));
        B3G_TRY(cudaStreamSynchronize(c->stream));
        // c_imp planes have stride nsph * n
        for (size_t q = 0; q < nn; ++q)
            for (int k = 0; k < 3; ++k) impulses[3 * q + k] = tmp[k * nn + q];
    }
    B3G_TRY(cudaStreamSynchronize(c->stream));
    return B3G_OK;
}

// One ray query: `triangle` < 0 casts against every triangle
// (RayCastSingle), otherwise against that triangle alone (RayCast).
static b3g_status ray_query(b3g_cloth* c, const float p1[3], const float p2[3], float max_fraction, int64_t triangle,
                            uint32_t* tri_out, float* fraction, float normal[3], int* hit)
{
    if (!valid(c) || !p1 || !p2 || !hit || !(max_fraction >= 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    if (triangle >= (int64_t)c->dev.t) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b3g_status s = flush_ops(c);
    if (s != B3G_OK) return s;
    if (!c->ray_buf) B3G_TRY(cudaMalloc(&c->ray_buf, 64));
    RayQuery q{};
    for (int k = 0; k < 3; ++k) {
        q.p1[k] = p1[k];
        q.p2[k] = p2[k];
    }
    q.max_fraction = max_fraction;
    q.best = static_cast<unsigned long long*>(c->ray_buf);
    q.out = reinterpret_cast<RayHit*>(static_cast<char*>(c->ray_buf) + 16);
    if (triangle < 0) {
        B3G_TRY(launch_ray_cast(c->dev, q, c->stream));
    } else {
        const unsigned long long key = (unsigned long long)triangle;
        B3G_TRY(cudaMemcpyAsync(q.best, &key, sizeof(key), cudaMemcpyHostToDevice, c->stream));
        B3G_TRY(launch_ray_result(c->dev, q, c->stream));
    }
    RayHit h{};
    B3G_TRY(cudaMemcpyAsync(&h, q.out, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    *hit = (int)h.hit;
    if (h.hit) {
        if (tri_out) *tri_out = h.triangle;
        if (fraction) *fraction = h.fraction;
        if (normal)
            for (int k = 0; k < 3; ++k) normal[k] = h.normal[k];
    }
    return B3G_OK;
}

b3g_status b3g_cloth_ray_cast_single(b3g_cloth* c, const float p1[3], const float p2[3], uint32_t* triangle,
                                     float* fraction, float normal[3], int* hit)
{
    return ray_query(c, p1, p2, 1.0f, -1, triangle, fraction, normal, hit);
}

b3g_status b3g_cloth_ray_cast(b3g_cloth* c, const float p1[3], const float p2[3], float max_fraction,
                              uint32_t triangle, float* fraction, float normal[3], int* hit)
{
    return ray_query(c, p1, p2, max_fraction, (int64_t)triangle, nullptr, fraction, normal, hit);
}

b3g_status b3g_cloth_read_tri_contacts(const b3g_cloth* c, uint32_t* count, uint32_t* pairs, uint8_t* active,
                                       float* weights, float* impulses)
{
    if (!valid(c) || !count) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    return self_read(c, count, pairs, active, weights, impulses);
}

b3g_status b3g_cloth_get_self_stats(const b3g_cloth* c, uint32_t* contacts, uint32_t* active, uint32_t* levels)
{
    if (!valid(c) || !contacts || !active || !levels) return B3G_ERR_INVALID_ARGUMENT;
    self_stats(c, contacts, active, levels);
    return B3G_OK;
}

b3g_status b3g_cloth_last_stats(const b3g_cloth* c, b3g_step_stats* stats)
{
    if (!valid(c) || !stats) return B3G_ERR_INVALID_ARGUMENT;
    *stats = c->last;
    return B3G_OK;
}

b3g_status b3g_cloth_read_system(const b3g_cloth* cc, uint32_t* nnz, uint32_t* rowptr, uint32_t* cols, float* vals,
                                 float* b, float* S, float* x0)
{
    b3g_cloth* c = const_cast<b3g_cloth*>(cc);
    if (!valid(c) || !nnz) return B3G_ERR_INVALID_ARGUMENT;
    const ClothTopology& T = c->topo;
    const uint32_t n = T.n;
    *nnz = (uint32_t)T.row_cols.size();
    if (!vals) return B3G_OK;
    if (!rowptr || !cols) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    std::vector<float> sv(9 * (size_t)T.E);
    B3G_TRY(cudaMemcpyAsync(sv.data(), c->dev.vals, 9 * (size_t)T.E * 4, cudaMemcpyDeviceToHost, c->stream));
    B3G_TRY(cudaStreamSynchronize(c->stream));
    std::memcpy(rowptr, T.row_ptr.data(), (n + 1) * 4);
    std::memcpy(cols, T.row_cols.data(), T.row_cols.size() * 4);
    for (uint32_t r = 0; r < n; ++r) {
        uint32_t q = r / 32, lane = r % 32;
        for (uint32_t k = 0; k < T.row_deg[r]; ++k) {
            size_t idx = T.slice_off[q] + 32 * k + lane;
            for (int m = 0; m < 9; ++m) vals[9 * (size_t)(T.row_ptr[r] + k) + m] = sv[(size_t)m * T.E + idx];
        }
    }
    b3g_status s;
    if (b && (s = read_planes(c, c->dev.b, b)) != B3G_OK) return s;
    if (S || x0) {
        std::vector<uint8_t> ty(n);
        std::vector<float> mx(3 * (size_t)n);
        B3G_TRY(cudaMemcpyAsync(ty.data(), c->dev.type, n, cudaMemcpyDeviceToHost, c->stream));
        if ((s = read_planes(c, c->dev.mx, mx.data())) != B3G_OK) return s;
        // the system's warm start is the m_x the step began with: after a
        // step, m_x already holds the new solution; report S and m_x as stored
        for (uint32_t i = 0; i < n; ++i) {
            if (S) S[i] = ty[i] == B3G_DYNAMIC ? 1.0f : 0.0f;
            if (x0)
                for (int q = 0; q < 3; ++q) x0[3 * i + q] = mx[3 * i + q];
        }
    }
    return B3G_OK;
}

}  // extern "C"
