// Batched stepping: one b3g_batch_step advances many cloths of uneven sizes
// with a fixed number of launches, captured once into a CUDA graph:
//   H2D step parameters -> scatter -> contacts update -> assembly ->
//   persistent batched CG -> finalize -> position iterations -> post ->
//   gather -> D2H results.
// The per-row kernels cover every row of every cloth in one launch; the CG
// runs one cloth per CTA (block-per-instance) or one cloth per cluster
// (split-instance), chosen per size class by b3g_batch_autotune.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/b3g.h"
#include "batch.cuh"
#include "cloth_dev.cuh"
#include "cloth_internal.h"

using namespace b3g;

namespace {

b3g_status from_cuda(cudaError_t e)
{
    if (e == cudaSuccess) return B3G_OK;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return B3G_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return B3G_ERR_NO_DEVICE;
    return B3G_ERR_CUDA;
}

#define B3G_TRY(expr)                                 \
    do {                                              \
        cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return from_cuda(e_);  \
    } while (0)

__global__ void k_scatter_scalars(const ClothDev* descs, const StepScalars* stage, uint32_t count)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) *descs[k].sc = stage[k];
}

__global__ void k_gather_scalars(const ClothDev* descs, StepScalars* stage, uint32_t count)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) stage[k] = *descs[k].sc;
}

int size_class(uint32_t rows)
{
    int c = 0;
    while ((1u << (c + 1)) <= rows && c < 31) ++c;
    return c;
}

}  // namespace

struct b3g_batch {
    int device = 0;
    uint32_t cap = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_cg0 = nullptr, ev_cg1 = nullptr;
    // device
    ClothDev* d_descs = nullptr;
    StepScalars* d_stage = nullptr;
    uint32_t* d_prefix = nullptr;  // row prefix sums (count + 1), then element prefix sums (count + 1)
    uint32_t* d_order = nullptr;
    uint2* d_tasks = nullptr;
    uint32_t* d_next = nullptr;
    // pinned host
    ClothDev* h_descs = nullptr;
    StepScalars* h_stage = nullptr;
    uint32_t* h_prefix = nullptr;
    uint32_t* h_order = nullptr;
    uint2* h_tasks = nullptr;
    // schedule
    b3g_batch_schedule sched{};
    uint32_t sched_version = 1;
    // graph cache
    cudaGraphExec_t exec = nullptr;
    std::vector<b3g_cloth*> graph_list;
    std::vector<uint32_t> graph_layouts;  // each listed cloth's layout version when the graph was built
    uint32_t graph_pi = UINT32_MAX, graph_sched = 0;
    uint32_t graph_hulls = 0;  // whether the graph holds the hull contact kernel
    uint32_t graph_kernels = 0;
    uint32_t ntasks = 0, total_rows = 0, max_deg = 0;
    uint32_t total_elems = 0;  // triangles, springs and mouse forces of every cloth
    uint32_t hulls = 0;  // some cloth of the batch has a hull collider
    uint32_t slot_asm = 0;  // every cloth of the batch has the slot-major assembly
    int assemble_block = 0;
    int dot = -1;  // dot precision shared by every planned cloth, -1 if mixed
};

namespace {

constexpr uint64_t kBatchRecordBytes = 64ull << 20;

void destroy_graph(b3g_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->graph_list.clear();
    b->graph_layouts.clear();
}

// Host-side launch plan of a cloth list: row prefix sums, the CG task list
// (split cloths first, then groups of `cluster` small cloths, largest first).
void plan(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count)
{
    uint32_t total = 0, max_deg = 1, hulls = 0, slot_asm = 1, elems = 0;
    uint64_t record_bytes = 0;
    int dot = count ? (int)cloths[0]->opts.dot : -1;
    for (uint32_t k = 0; k < count; ++k) {
        if ((int)cloths[k]->opts.dot != dot) dot = -1;
        b->h_descs[k] = cloths[k]->dev;
        b->h_prefix[k] = total;
        total += cloths[k]->dev.n;
        b->h_prefix[count + 1 + k] = elems;
        elems += cloths[k]->dev.t + cloths[k]->dev.ns + cloths[k]->dev.nmouse;
        record_bytes += 240ull * cloths[k]->dev.t + 48ull * cloths[k]->dev.ns + 80ull * cloths[k]->dev.nmouse;
        max_deg = std::max(max_deg, cloths[k]->dev.max_deg);
        slot_asm &= cloths[k]->dev.slot_asm ? 1u : 0u;
        for (uint32_t q = 0; q < cloths[k]->dev.nsph; ++q) hulls |= cloths[k]->dev.sph[q].kind == 2 ? 1u : 0u;
    }
    b->h_prefix[count] = total;
    b->h_prefix[2 * count + 1] = elems;
    b->total_elems = elems;
    b->dot = dot;
    b->total_rows = total;
    b->max_deg = max_deg;
    b->hulls = hulls;
    // The element records are written by one launch and read by the next
    // two; that pays while they stay in L2.  A batch whose records exceed
    // half of it assembles row by row (512 cloths of 16^2..128^2, 1.5 GB of
    // records: 13.7 ms a step row by row against 14.6 with the records).
    b->slot_asm = slot_asm && record_bytes <= kBatchRecordBytes ? 1u : 0u;
    std::vector<uint32_t> idx(count);
    for (uint32_t k = 0; k < count; ++k) idx[k] = k;
    // work estimate: stored blocks
    auto work = [&](uint32_t k) { return (uint64_t)cloths[k]->topo.row_cols.size(); };
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t c) { return work(a) > work(c); });
    const uint32_t T = b->sched.cluster;
    uint32_t w = 0, nt = 0;
    std::vector<uint32_t> small;
    for (uint32_t k : idx) {
        const bool split = T > 1 && b->sched.split_class[size_class(cloths[k]->dev.n)] != 0;
        if (split) {
            b->h_order[w] = k;
            b->h_tasks[nt++] = make_uint2(w, 0u);
            ++w;
        } else {
            small.push_back(k);
        }
    }
    for (size_t q = 0; q < small.size(); q += T) {
        const uint32_t cnt = (uint32_t)std::min<size_t>(T, small.size() - q);
        b->h_tasks[nt++] = make_uint2(w, cnt);
        for (uint32_t r = 0; r < cnt; ++r) b->h_order[w++] = small[q + r];
    }
    b->ntasks = nt;
    b->assemble_block = 0;  // chosen at launch for occupancy
}

b3g_status enqueue(b3g_batch* b, uint32_t count, uint32_t pi, cudaStream_t st, uint32_t* kernels)
{
    RowSpan sp{b->d_descs, b->d_prefix, count, b->total_rows, b->max_deg, b->hulls, b->slot_asm,
                       b->d_prefix + count + 1, b->total_elems};
    BatchCgArgs a{b->d_descs, b->d_order, b->d_tasks, b->ntasks, b->d_next};
    uint32_t k = 0;
    B3G_TRY(cudaMemcpyAsync(b->d_descs, b->h_descs, count * sizeof(ClothDev), cudaMemcpyHostToDevice, st));
    B3G_TRY(cudaMemcpyAsync(b->d_stage, b->h_stage, count * sizeof(StepScalars), cudaMemcpyHostToDevice, st));
    B3G_TRY(cudaMemcpyAsync(b->d_prefix, b->h_prefix, 2 * (count + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            st));
    B3G_TRY(cudaMemcpyAsync(b->d_order, b->h_order, count * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    B3G_TRY(cudaMemcpyAsync(b->d_tasks, b->h_tasks, b->ntasks * sizeof(uint2), cudaMemcpyHostToDevice, st));
    k_scatter_scalars<<<(count + 127) / 128, 128, 0, st>>>(b->d_descs, b->d_stage, count);
    ++k;
    B3G_TRY(cudaGetLastError());
    B3G_TRY(launch_span_contacts_update(sp, st));
    B3G_TRY(launch_span_assemble(sp, b->assemble_block, st));
    B3G_TRY(cudaMemsetAsync(b->d_next, 0, sizeof(uint32_t), st));
    // under stream capture the records must be external to become event
    // nodes, so that the CG launch is timed on every replay of the graph
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    B3G_TRY(cudaStreamIsCapturing(st, &cap));
    const unsigned rec_flags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
    B3G_TRY(cudaEventRecordWithFlags(b->ev_cg0, st, rec_flags));
    B3G_TRY(launch_batch_cg(a, (int)b->sched.cluster, b->dot, 0, st));
    B3G_TRY(cudaEventRecordWithFlags(b->ev_cg1, st, rec_flags));
    B3G_TRY(launch_span_finalize(sp, st));
    k += 4;
    for (uint32_t it = 1; it < pi && it < (uint32_t)kMaxPosIters; ++it) {
        B3G_TRY(launch_span_contact_position(sp, it, st));
        ++k;
    }
    B3G_TRY(launch_span_post(sp, st));
    k_gather_scalars<<<(count + 127) / 128, 128, 0, st>>>(b->d_descs, b->d_stage, count);
    k += 2;
    B3G_TRY(cudaGetLastError());
    B3G_TRY(cudaMemcpyAsync(b->h_stage, b->d_stage, count * sizeof(StepScalars), cudaMemcpyDeviceToHost, st));
    if (kernels) *kernels = k;
    return B3G_OK;
}

b3g_status check_list(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count)
{
    if (!b || !cloths || count == 0) return B3G_ERR_INVALID_ARGUMENT;
    if (count > b->cap) return B3G_ERR_CAPACITY;
    for (uint32_t k = 0; k < count; ++k)
        if (!cloths[k] || cloths[k]->dev.n == 0 || cloths[k]->device != b->device) return B3G_ERR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < count; ++k)
        // self-collision and body colliders run on single cloths only
        if (cloths[k]->self || cloths[k]->dev.nbody) return B3G_ERR_UNSUPPORTED;
    return B3G_OK;
}

}  // namespace

extern "C" {

b3g_status b3g_batch_create(int device, uint32_t capacity, b3g_batch** out)
{
    if (!out || capacity == 0) return B3G_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return B3G_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return B3G_ERR_INVALID_ARGUMENT;
    b3g_batch* b = new (std::nothrow) b3g_batch();
    if (!b) return B3G_ERR_OUT_OF_MEMORY;
    b->device = device;
    b->cap = capacity;
    b->sched.cluster = 1;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev_cg0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev_cg1);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_descs, capacity * sizeof(ClothDev));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_stage, capacity * sizeof(StepScalars));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_prefix, 2 * (capacity + 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_order, capacity * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tasks, capacity * sizeof(uint2));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_next, 256);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_descs, capacity * sizeof(ClothDev));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_stage, capacity * sizeof(StepScalars));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_prefix, 2 * (capacity + 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_order, capacity * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_tasks, capacity * sizeof(uint2));
    if (e != cudaSuccess) {
        b3g_batch_destroy(b);
        return from_cuda(e);
    }
    *out = b;
    return B3G_OK;
}

b3g_status b3g_batch_destroy(b3g_batch* b)
{
    if (!b) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    destroy_graph(b);
    cudaFree(b->d_descs);
    cudaFree(b->d_stage);
    cudaFree(b->d_prefix);
    cudaFree(b->d_order);
    cudaFree(b->d_tasks);
    cudaFree(b->d_next);
    cudaFreeHost(b->h_descs);
    cudaFreeHost(b->h_stage);
    cudaFreeHost(b->h_prefix);
    cudaFreeHost(b->h_order);
    cudaFreeHost(b->h_tasks);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->ev_cg0) cudaEventDestroy(b->ev_cg0);
    if (b->ev_cg1) cudaEventDestroy(b->ev_cg1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return B3G_OK;
}

b3g_status b3g_batch_set_schedule(b3g_batch* b, const b3g_batch_schedule* s)
{
    if (!b || !s) return B3G_ERR_INVALID_ARGUMENT;
    if (s->cluster != 1 && s->cluster != 2 && s->cluster != 4 && s->cluster != 8) return B3G_ERR_INVALID_ARGUMENT;
    b->sched = *s;
    b->sched_version += 1;
    return B3G_OK;
}

b3g_status b3g_batch_get_schedule(const b3g_batch* b, b3g_batch_schedule* s)
{
    if (!b || !s) return B3G_ERR_INVALID_ARGUMENT;
    *s = b->sched;
    return B3G_OK;
}

}  // extern "C"

// Waits for the cloths' queued edits and earlier work: the edits go first,
// on the batch's stream; earlier work on the cloths' own streams is waited
// for once per distinct stream (a server's cloths share one).
static b3g_status sync_inputs(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, cudaStream_t st)
{
    b3g_status s;
    std::vector<cudaStream_t> waited;
    for (uint32_t k = 0; k < count; ++k) {
        if (!cloths[k]->pending.empty() && (s = flush_ops_on(cloths[k], st)) != B3G_OK) return s;
        cudaStream_t cs = cloths[k]->stream;
        if (cs && cs != st && std::find(waited.begin(), waited.end(), cs) == waited.end()) {
            B3G_TRY(cudaStreamSynchronize(cs));
            waited.push_back(cs);
        }
    }
    B3G_TRY(cudaStreamSynchronize(st));
    return B3G_OK;
}

// One step of the cloths, launched without a graph; returns once the work
// is queued.  batch_step_finish waits for it and collects the statistics.
b3g_status batch_step_launch(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, float dt, uint32_t vel_iters,
                             uint32_t pos_iters)
{
    b3g_status s = check_list(b, cloths, count);
    if (s != B3G_OK) return s;
    if (!(dt > 0.0f) || pos_iters > (uint32_t)kMaxPosIters) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    cudaStream_t st = b->stream;
    if ((s = sync_inputs(b, cloths, count, st)) != B3G_OK) return s;
    destroy_graph(b);
    plan(b, cloths, count);
    for (uint32_t k = 0; k < count; ++k) fill_step_scalars(cloths[k], dt, vel_iters, pos_iters, b->h_stage + k);
    B3G_TRY(cudaEventRecord(b->ev0, st));
    uint32_t kern = 0;
    if ((s = enqueue(b, count, pos_iters, st, &kern)) != B3G_OK) return s;
    B3G_TRY(cudaEventRecord(b->ev1, st));
    return B3G_OK;
}

// The statistics of the step just run, per cloth and for the batch.
static b3g_status collect(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, b3g_step_stats* per_cloth,
                          b3g_batch_stats* stats)
{
    float ms = 0.0f, cg_ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    if (cudaEventElapsedTime(&cg_ms, b->ev_cg0, b->ev_cg1) != cudaSuccess) {
        cudaGetLastError();
        cg_ms = 0.0f;
    }
    uint32_t it_total = 0, it_max = 0, status = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const StepScalars& h = b->h_stage[k];
        record_stats(cloths[k], h, ms, true);
        if (per_cloth) per_cloth[k] = cloths[k]->last;
        it_total += h.iter;
        it_max = std::max(it_max, h.iter);
        if (h.status) status = h.status;
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->count = count;
        stats->rows = b->total_rows;
        stats->step_ms = ms;
        stats->cg_ms = cg_ms;
        stats->cg_iterations_total = it_total;
        stats->cg_iterations_max = it_max;
        stats->tasks = b->ntasks;
    }
    return status ? (b3g_status)status : B3G_OK;
}

b3g_status batch_step_finish(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, b3g_step_stats* per_cloth,
                             b3g_batch_stats* stats)
{
    cudaSetDevice(b->device);
    B3G_TRY(cudaStreamSynchronize(b->stream));
    return collect(b, cloths, count, per_cloth, stats);
}

b3g_status batch_step_impl(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, float dt, uint32_t vel_iters,
                           uint32_t pos_iters, b3g_step_stats* per_cloth, b3g_batch_stats* stats, bool use_graph)
{
    if (!use_graph) {
        b3g_status s = batch_step_launch(b, cloths, count, dt, vel_iters, pos_iters);
        if (s != B3G_OK) return s;
        return batch_step_finish(b, cloths, count, per_cloth, stats);
    }
    b3g_status s = check_list(b, cloths, count);
    if (s != B3G_OK) return s;
    if (!(dt > 0.0f) || pos_iters > (uint32_t)kMaxPosIters) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    cudaStream_t st = b->stream;
    if ((s = sync_inputs(b, cloths, count, st)) != B3G_OK) return s;
    uint32_t hulls_now = 0;
    for (uint32_t k = 0; k < count; ++k)
        for (uint32_t q = 0; q < cloths[k]->dev.nsph; ++q) hulls_now |= cloths[k]->dev.sph[q].kind == 2 ? 1u : 0u;
    bool same = (b->exec && b->graph_pi == pos_iters && b->graph_sched == b->sched_version &&
                b->graph_hulls == hulls_now &&
                b->graph_list.size() == count && std::equal(b->graph_list.begin(), b->graph_list.end(), cloths));
    // a cloth laid out again (particles or forces created) has new sizes and buffers
    for (uint32_t k = 0; same && k < count; ++k) same = b->graph_layouts[k] == cloths[k]->layout_version;
    if (!same) {
        destroy_graph(b);
        plan(b, cloths, count);
        const uint64_t before = kernel_launches();
        cudaGraph_t g = nullptr;
        B3G_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        uint32_t kern = 0;
        b3g_status es = enqueue(b, count, pos_iters, st, &kern);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        count_launches(before - kernel_launches());
        if (es != B3G_OK) {
            if (g) cudaGraphDestroy(g);
            return es;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            return from_cuda(e);
        }
        b->graph_list.assign(cloths, cloths + count);
        b->graph_layouts.resize(count);
        for (uint32_t k = 0; k < count; ++k) b->graph_layouts[k] = cloths[k]->layout_version;
        b->graph_pi = pos_iters;
        b->graph_sched = b->sched_version;
        b->graph_hulls = hulls_now;
        b->graph_kernels = kern;
    } else {
        // descriptors may have changed (colliders added): refresh the pinned copy the graph uploads
        for (uint32_t k = 0; k < count; ++k) b->h_descs[k] = cloths[k]->dev;
    }
    for (uint32_t k = 0; k < count; ++k) fill_step_scalars(cloths[k], dt, vel_iters, pos_iters, b->h_stage + k);
    B3G_TRY(cudaEventRecord(b->ev0, st));
    B3G_TRY(cudaGraphLaunch(b->exec, st));
    B3G_TRY(cudaEventRecord(b->ev1, st));
    B3G_TRY(cudaStreamSynchronize(st));
    count_launches(b->graph_kernels);
    return collect(b, cloths, count, per_cloth, stats);
}

extern "C" {

b3g_status b3g_batch_step(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, float dt, uint32_t vel_iters,
                          uint32_t pos_iters, b3g_step_stats* per_cloth, b3g_batch_stats* stats)
{
    return batch_step_impl(b, cloths, count, dt, vel_iters, pos_iters, per_cloth, stats, true);
}

// Times the batched CG alone on the systems assembled from the cloths'
// current state (no state changes: the CG writes only its own vectors and
// the solution, which the next step recomputes) and picks, per size class,
// block-per-instance or split-instance, and the cluster size.
b3g_status b3g_batch_autotune(b3g_batch* b, b3g_cloth* const* cloths, uint32_t count, float dt,
                              b3g_batch_schedule* out)
{
    b3g_status s = check_list(b, cloths, count);
    if (s != B3G_OK) return s;
    if (!(dt > 0.0f)) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    cudaStream_t st = b->stream;
    for (uint32_t k = 0; k < count; ++k) {
        if ((s = flush_ops_on(cloths[k], st)) != B3G_OK) return s;
        B3G_TRY(cudaStreamSynchronize(cloths[k]->stream));
    }
    destroy_graph(b);
    // step parameters without advancing the step counters
    for (uint32_t k = 0; k < count; ++k) {
        fill_step_scalars(cloths[k], dt, 8, 2, b->h_stage + k);
        cloths[k]->step_index -= 1;
    }
    bool present[32] = {false};
    for (uint32_t k = 0; k < count; ++k) present[size_class(cloths[k]->dev.n)] = true;
    b3g_batch_schedule best = b->sched;
    float best_ms = 1e30f;
    const uint32_t clusters[4] = {1, 2, 4, 8};
    const char* env = std::getenv("B3G_TRACE_AUTOTUNE");  // every timed candidate to stderr
    const bool trace_on = env && env[0] && env[0] != '0';
    for (uint32_t ci = 0; ci < 4; ++ci) {
        b3g_batch_schedule cand{};
        cand.cluster = clusters[ci];
        auto time_cg = [&](const b3g_batch_schedule& sc, float* ms_out) -> b3g_status {
            b->sched = sc;
            plan(b, cloths, count);
            RowSpan sp{b->d_descs, b->d_prefix, count, b->total_rows, b->max_deg, b->hulls, b->slot_asm,
                       b->d_prefix + count + 1, b->total_elems};
            BatchCgArgs a{b->d_descs, b->d_order, b->d_tasks, b->ntasks, b->d_next};
            B3G_TRY(cudaMemcpyAsync(b->d_descs, b->h_descs, count * sizeof(ClothDev), cudaMemcpyHostToDevice, st));
            B3G_TRY(cudaMemcpyAsync(b->d_stage, b->h_stage, count * sizeof(StepScalars), cudaMemcpyHostToDevice, st));
            B3G_TRY(cudaMemcpyAsync(b->d_prefix, b->h_prefix, 2 * (count + 1) * 4, cudaMemcpyHostToDevice, st));
            B3G_TRY(cudaMemcpyAsync(b->d_order, b->h_order, count * 4, cudaMemcpyHostToDevice, st));
            B3G_TRY(cudaMemcpyAsync(b->d_tasks, b->h_tasks, b->ntasks * sizeof(uint2), cudaMemcpyHostToDevice, st));
            k_scatter_scalars<<<(count + 127) / 128, 128, 0, st>>>(b->d_descs, b->d_stage, count);
            B3G_TRY(cudaGetLastError());
            B3G_TRY(launch_span_assemble(sp, b->assemble_block, st));
            float bestrun = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                B3G_TRY(cudaMemsetAsync(b->d_next, 0, 4, st));
                B3G_TRY(cudaEventRecord(b->ev0, st));
                B3G_TRY(launch_batch_cg(a, (int)sc.cluster, b->dot, 0, st));
                B3G_TRY(cudaEventRecord(b->ev1, st));
                B3G_TRY(cudaEventSynchronize(b->ev1));
                float ms = 0.0f;
                B3G_TRY(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
                bestrun = std::min(bestrun, ms);
            }
            *ms_out = bestrun;
            return B3G_OK;
        };
        auto trace = [&](const b3g_batch_schedule& sc, float ms) {
            if (!trace_on) return;
            std::fprintf(stderr, "b3g autotune: cluster %u split", sc.cluster);
            for (int cls = 0; cls < 32; ++cls)
                if (sc.split_class[cls]) std::fprintf(stderr, " %d", cls);
            std::fprintf(stderr, ": CG %.3f ms\n", ms);
        };
        float cur = 0.0f;
        if ((s = time_cg(cand, &cur)) != B3G_OK) return s;
        trace(cand, cur);
        if (cand.cluster > 1) {
            // split every class at or above a threshold, for each threshold from
            // the largest class down: larger cloths gain the most from a whole
            // cluster, so the useful split sets are these prefixes
            b3g_batch_schedule trial = cand;
            for (int cls = 31; cls >= 0; --cls) {
                if (!present[cls]) continue;
                trial.split_class[cls] = 1;
                float t = 0.0f;
                if ((s = time_cg(trial, &t)) != B3G_OK) return s;
                trace(trial, t);
                if (t < cur) {
                    cur = t;
                    cand = trial;
                }
            }
        }
        if (cur < best_ms) {
            best_ms = cur;
            best = cand;
        }
    }
    best.tuned_cg_ms = best_ms;
    b->sched = best;
    b->sched_version += 1;
    if (out) *out = best;
    return B3G_OK;
}

}  // extern "C"
