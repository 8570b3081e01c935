// Cloth-step serving with continuous batching.
//
// Requests (a cloth plus a number of steps) are prepared on host worker
// threads (topology: prepare_cloth), admitted in arrival order while the
// HBM budget and the active-slot limit allow, and then live on the device:
// their state stays resident between steps.  Every tick advances all
// active cloths by one step in one batched launch sequence (batch_api.cu),
// so requests that arrive while others are mid-flight join the next tick and
// their work overlaps on the GPU.  Finished requests are copied out and their
// memory goes back to a stream-ordered pool.  The batch schedule is fixed per
// server, so a request's result does not depend on which others share its
// ticks.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/b3g.h"
#include "cloth_dev.cuh"
#include "cloth_internal.h"

using namespace b3g;

namespace {

enum ReqState { R_QUEUED = 0, R_READY = 1, R_ACTIVE = 2, R_DONE = 3, R_FAILED = 4 };

struct Request {
    uint64_t id = 0;
    double arrival = 0.0, admitted = 0.0, finished = 0.0;
    uint32_t steps_total = 0, steps_done = 0;
    int state = R_QUEUED;
    b3g_status status = B3G_OK;
    // inputs (copied at submit)
    std::vector<float> verts;
    std::vector<uint32_t> tris;
    b3g_cloth_def def{};
    std::vector<uint8_t> types;
    std::vector<float> spheres;  // 5 per sphere: center xyz, radius, friction
    float gravity[3] = {0.0f, -9.8f, 0.0f};
    // prepared / resident
    b3g_cloth* cloth = nullptr;
    char* arena = nullptr;
    size_t bytes = 0;
    std::vector<float> result;  // positions at completion
};

b3g_status from_cuda(cudaError_t e)
{
    if (e == cudaSuccess) return B3G_OK;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return B3G_ERR_OUT_OF_MEMORY;
    return B3G_ERR_CUDA;
}

}  // namespace

struct b3g_server {
    int device = 0;
    b3g_server_config cfg{};
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    b3g_batch* batch = nullptr;
    uint8_t* d_types = nullptr;
    uint32_t d_types_cap = 0;

    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request*> prep;
    std::vector<std::thread> workers;
    bool stop = false;

    std::map<uint64_t, Request*> ready;      // prepared, awaiting admission (arrival order)
    // Workers prepare ahead only while fewer than this many requests wait
    // prepared: the free slots plus a margin, set by each tick.  Preparing
    // further ahead than admission can follow only takes cores from the tick.
    size_t prep_limit = 0;
    UploadStage stage;                       // page-locked staging of the activations' uploads
    std::vector<Request*> active;
    std::unordered_map<uint64_t, Request*> all;
    uint64_t next_id = 1;
    size_t used = 0;

    // statistics
    std::vector<std::pair<float, uint32_t>> tick_samples;  // (tick ms, active cloths stepped)
    uint64_t vertex_steps = 0, steps = 0, ticks = 0, admitted = 0, completed = 0, rejected = 0;
    double busy_ms = 0.0;
    uint32_t peak_active = 0;
    size_t peak_used = 0;
};

namespace {

// Requests prepared beyond the free slots, so that the next ticks' admissions
// do not wait for the topology workers.
constexpr size_t kPrepMargin = 512;
// Page-locked staging of the admitted cloths' uploads (reused every tick).
constexpr size_t kStageBytes = 256ull << 20;

void worker_main(b3g_server* s)
{
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [&] { return s->stop || (!s->prep.empty() && s->ready.size() < s->prep_limit); });
            if (s->stop && s->prep.empty()) return;
            r = s->prep.front();
            s->prep.pop_front();
        }
        b3g_mesh_desc m{(uint32_t)(r->verts.size() / 3), r->verts.data(), (uint32_t)(r->tris.size() / 3),
                        r->tris.data(), 0, nullptr};
        b3g_cloth* c = nullptr;
        // the server's batches assemble row by row (their records would not
        // stay in L2), so its cloths are laid out without the records: the
        // HBM budget then admits more of them
        b3g_status st = prepare_cloth(&m, &r->def, &c, false);
        std::lock_guard<std::mutex> lk(s->mu);
        if (st != B3G_OK) {
            r->status = st;
            r->state = R_FAILED;
        } else {
            r->cloth = c;
            r->bytes = c->arena.size;
            r->state = R_READY;
            if (r->bytes > s->cfg.hbm_budget_bytes) {
                r->status = B3G_ERR_CAPACITY;
                r->state = R_FAILED;
                s->rejected += 1;
                destroy_cloth(c);
                r->cloth = nullptr;
            } else {
                s->ready[r->id] = r;
            }
        }
        // the mesh copy is no longer needed
        std::vector<float>().swap(r->verts);
        std::vector<uint32_t>().swap(r->tris);
    }
}

// Brings a prepared request onto the device: arena from the pool, uploads,
// pins, colliders, solver options.  Runs on the server stream.
b3g_status activate(b3g_server* s, Request* r)
{
    b3g_cloth* c = r->cloth;
    cudaError_t e = cudaMallocFromPoolAsync((void**)&r->arena, r->bytes, s->pool, s->stream);
    if (e != cudaSuccess) return from_cuda(e);
    b3g_status st = realize_cloth(c, s->device, r->arena, false, s->stream, false, &s->stage);
    if (st != B3G_OK) return st;
    c->opts = s->cfg.solver;
    std::memcpy(c->gravity, r->gravity, sizeof(c->gravity));
    if (!r->types.empty()) {
        const void* src = r->types.data();
        if (s->stage.used + c->dev.n <= s->stage.size) {
            char* p = s->stage.base + s->stage.used;
            std::memcpy(p, src, c->dev.n);
            s->stage.used += ((size_t)c->dev.n + 255) & ~size_t(255);
            src = p;
        }
        e = cudaMemcpyAsync(c->d_stage_u8, src, c->dev.n, cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) e = launch_set_types(c->dev, c->d_stage_u8, s->stream);
        if (e != cudaSuccess) return from_cuda(e);
    }
    for (size_t k = 0; k + 5 <= r->spheres.size() && c->dev.nsph < (uint32_t)kMaxSpheres; k += 5) {
        SphereDev& sp = c->dev.sph[c->dev.nsph++];
        sp = SphereDev{};
        sp.cx = r->spheres[k];
        sp.cy = r->spheres[k + 1];
        sp.cz = r->spheres[k + 2];
        sp.radius = r->spheres[k + 3];
        sp.friction = r->spheres[k + 4];
        const float ctr[3] = {sp.cx, sp.cy, sp.cz};
        for (int q = 0; q < 3; ++q) {
            sp.lo[q] = (ctr[q] - sp.radius) - 0.2f;
            sp.hi[q] = (ctr[q] + sp.radius) + 0.2f;
        }
    }
    rank_colliders(c->dev.sph, c->dev.nsph);
    return B3G_OK;
}

// Finished requests: every cloth's positions are transposed on the device
// and copied out on the server's stream, one wait for all of them, then the
// arenas go back to the pool.
void retire(b3g_server* s, const std::vector<Request*>& done, double now)
{
    if (done.empty()) return;
    for (Request* r : done) {
        b3g_cloth* c = r->cloth;
        const uint32_t n = c->dev.n;
        r->result.resize(3 * (size_t)n);
        launch_planes_to_xyz(c->dev.x, c->d_stage, n, s->stream);
        cudaMemcpyAsync(r->result.data(), c->d_stage, 3 * (size_t)n * 4, cudaMemcpyDeviceToHost, s->stream);
    }
    cudaStreamSynchronize(s->stream);
    for (Request* r : done) {
        cudaFreeAsync(r->arena, s->stream);
        r->arena = nullptr;
        r->cloth->stream = nullptr;  // the server's stream, waited for above
        destroy_cloth(r->cloth);
        r->cloth = nullptr;
        s->used -= r->bytes;
        r->finished = now;
        r->state = R_DONE;
        s->completed += 1;
    }
}

}  // namespace

extern "C" {

b3g_status b3g_server_create(int device, const b3g_server_config* cfg, b3g_server** out)
{
    if (!cfg || !out || cfg->max_active == 0 || !(cfg->dt > 0.0f) ||
        cfg->position_iterations > (uint32_t)kMaxPosIters)
        return B3G_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return B3G_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return B3G_ERR_INVALID_ARGUMENT;
    b3g_server* s = new (std::nothrow) b3g_server();
    if (!s) return B3G_ERR_OUT_OF_MEMORY;
    s->device = device;
    s->cfg = *cfg;
    if (s->cfg.solver.max_iterations == 0) s->cfg.solver = b3g_solver_opts{B3G_STOP_RELATIVE, 1e-4f, 200, B3G_DOT_F64};
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (e == cudaSuccess) e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) {
        uint64_t keep = UINT64_MAX;  // keep freed blocks for reuse instead of returning them to the driver
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess && cfg->hbm_budget_bytes) {
        // reserve the budget in the pool up front: a block freed to the pool
        // stays with it, and later arenas are carved from it instead of each
        // growing the pool while requests wait
        void* all = nullptr;
        if (cudaMallocFromPoolAsync(&all, cfg->hbm_budget_bytes, s->pool, s->stream) == cudaSuccess) {
            cudaFreeAsync(all, s->stream);
            cudaStreamSynchronize(s->stream);
        }
        cudaGetLastError();  // a budget above the free memory leaves the pool to grow on demand
    }
    if (e == cudaSuccess) {
        s->stage.size = kStageBytes;
        e = cudaMallocHost(&s->stage.base, s->stage.size);
        if (e != cudaSuccess) s->stage = UploadStage{};
    }
    if (e != cudaSuccess) {
        b3g_server_destroy(s);
        return from_cuda(e);
    }
    b3g_status st = b3g_batch_create(device, cfg->max_active, &s->batch);
    if (st != B3G_OK) {
        b3g_server_destroy(s);
        return st;
    }
    b3g_batch_schedule sched = cfg->schedule;
    if (sched.cluster == 0) sched.cluster = 1;
    if ((st = b3g_batch_set_schedule(s->batch, &sched)) != B3G_OK) {
        b3g_server_destroy(s);
        return st;
    }
    // one core stays with the thread that ticks
    const uint32_t hw = std::thread::hardware_concurrency();
    const uint32_t nw = cfg->host_threads ? cfg->host_threads : std::max(1u, hw > 1 ? hw - 1 : 1u);
    s->prep_limit = (size_t)cfg->max_active + kPrepMargin;
    for (uint32_t k = 0; k < nw; ++k) s->workers.emplace_back(worker_main, s);
    *out = s;
    return B3G_OK;
}

b3g_status b3g_server_destroy(b3g_server* s)
{
    if (!s) return B3G_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto& t : s->workers) t.join();
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& kv : s->all) {
        Request* r = kv.second;
        if (r->cloth) destroy_cloth(r->cloth);
        if (r->arena) cudaFreeAsync(r->arena, s->stream);
        delete r;
    }
    for (Request* r : s->prep) (void)r;  // owned through `all`
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->batch) b3g_batch_destroy(s->batch);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->stage.base) cudaFreeHost(s->stage.base);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return B3G_OK;
}

b3g_status b3g_server_submit(b3g_server* s, const b3g_mesh_desc* mesh, const b3g_cloth_def* def,
                             const uint8_t* types, const float* spheres, uint32_t sphere_count, uint32_t steps,
                             double arrival, uint64_t* id)
{
    if (!s || !mesh || !def || !mesh->vertices || !mesh->triangles || mesh->vertex_count == 0 ||
        mesh->triangle_count == 0 || steps == 0 || (sphere_count && !spheres) || sphere_count > kMaxSpheres)
        return B3G_ERR_INVALID_ARGUMENT;
    if (def->thickness > 0.0f) return B3G_ERR_UNSUPPORTED;  // self-collision runs on single cloths only
    Request* r = new (std::nothrow) Request();
    if (!r) return B3G_ERR_OUT_OF_MEMORY;
    r->verts.assign(mesh->vertices, mesh->vertices + 3 * (size_t)mesh->vertex_count);
    r->tris.assign(mesh->triangles, mesh->triangles + 3 * (size_t)mesh->triangle_count);
    r->def = *def;
    if (types) r->types.assign(types, types + mesh->vertex_count);
    if (sphere_count) r->spheres.assign(spheres, spheres + 5 * (size_t)sphere_count);
    r->steps_total = steps;
    r->arrival = arrival;
    std::memcpy(r->gravity, s->cfg.gravity, sizeof(r->gravity));
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        s->all[r->id] = r;
        s->prep.push_back(r);
    }
    s->cv.notify_one();
    if (id) *id = r->id;
    return B3G_OK;
}

b3g_status b3g_server_tick(b3g_server* s, double now, b3g_server_tick_info* info)
{
    if (!s) return B3G_ERR_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    // B3G_TRACE_SERVER=1: each tick's host phases to stderr
    static const bool trace = std::getenv("B3G_TRACE_SERVER") != nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    auto ms_since = [](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    };
    double t_activate = 0.0, t_wait = 0.0, t_retire = 0.0;
    b3g_server_tick_info ti{};
    // The active cloths' step goes to the device first; requests admitted
    // meanwhile are brought onto the device while it runs and join from the
    // next tick on.  A request's steps are the same whichever tick it joins.
    std::vector<b3g_cloth*> cl(s->active.size());
    uint64_t rows = 0;
    for (size_t k = 0; k < cl.size(); ++k) {
        cl[k] = s->active[k]->cloth;
        rows += cl[k]->dev.n;
    }
    if (!cl.empty()) {
        const b3g_status st = batch_step_launch(s->batch, cl.data(), (uint32_t)cl.size(), s->cfg.dt,
                                                s->cfg.velocity_iterations, s->cfg.position_iterations);
        if (st != B3G_OK) return st;
    }
    // the last tick's uploads are done (the launch above waited for the
    // server stream); the staging buffer starts over
    if (s->stage.used) {
        cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) return from_cuda(e);
        s->stage.used = 0;
    }
    // admission in arrival order while memory and slots allow
    std::vector<Request*> newly;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        // the slot limit counts the cloths admitted in this tick too
        while (!s->ready.empty() && s->active.size() + newly.size() < s->cfg.max_active) {
            Request* r = s->ready.begin()->second;
            if (s->used + r->bytes > s->cfg.hbm_budget_bytes) break;
            s->ready.erase(s->ready.begin());
            s->used += r->bytes;
            newly.push_back(r);
        }
        ti.queued = (uint32_t)(s->prep.size() + s->ready.size());
    }
    const auto ta = std::chrono::steady_clock::now();
    std::vector<Request*> joined;
    for (Request* r : newly) {
        b3g_status st = activate(s, r);
        if (st != B3G_OK) {
            r->status = st;
            r->state = R_FAILED;
            if (r->arena) cudaFreeAsync(r->arena, s->stream);
            r->arena = nullptr;
            if (r->cloth) {
                r->cloth->stream = nullptr;
                destroy_cloth(r->cloth);
                r->cloth = nullptr;
            }
            s->used -= r->bytes;
            continue;
        }
        r->state = R_ACTIVE;
        r->admitted = now;
        joined.push_back(r);
        s->admitted += 1;
        ti.admitted += 1;
    }
    t_activate = ms_since(ta);
    s->peak_used = std::max(s->peak_used, s->used);
    if (!cl.empty()) {
        b3g_batch_stats bs{};
        const auto tw = std::chrono::steady_clock::now();
        const b3g_status st = batch_step_finish(s->batch, cl.data(), (uint32_t)cl.size(), nullptr, &bs);
        t_wait = ms_since(tw);
        if (st != B3G_OK && st != B3G_ERR_NUMERICAL) return st;
        ti.stepped = (uint32_t)cl.size();
        ti.rows = (uint32_t)rows;
        ti.tick_ms = bs.step_ms;
        s->tick_samples.emplace_back(bs.step_ms, (uint32_t)cl.size());
        s->vertex_steps += rows;
        s->steps += cl.size();
        s->busy_ms += bs.step_ms;
        s->ticks += 1;
        std::vector<Request*> still, done;
        for (Request* r : s->active) {
            r->steps_done += 1;
            if (r->steps_done >= r->steps_total) {
                done.push_back(r);
                ti.completed += 1;
            } else {
                still.push_back(r);
            }
        }
        const auto tr = std::chrono::steady_clock::now();
        retire(s, done, now);  // waits for the server stream, so the new cloths' uploads are done too
        t_retire = ms_since(tr);
        s->active.swap(still);
    }
    if (!joined.empty()) {
        cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) return from_cuda(e);
        for (Request* r : joined) {
            finish_upload(r->cloth);
            s->active.push_back(r);
        }
    }
    s->peak_active = std::max<uint32_t>(s->peak_active, (uint32_t)s->active.size());
    if (trace)
        std::fprintf(stderr, "tick %llu: stepped %zu admitted %zu | activate %.1f ms, wait %.1f ms (device %.1f), "
                             "retire %.1f ms, total %.1f ms\n",
                     (unsigned long long)s->ticks, cl.size(), joined.size(), t_activate, t_wait, ti.tick_ms, t_retire,
                     ms_since(t0));
    ti.active = (uint32_t)s->active.size();
    ti.bytes_used = s->used;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->prep_limit = (s->cfg.max_active - std::min<size_t>(s->active.size(), s->cfg.max_active)) + kPrepMargin;
    }
    s->cv.notify_all();
    if (info) *info = ti;
    return B3G_OK;
}

b3g_status b3g_server_poll(b3g_server* s, uint64_t id, b3g_request_info* info)
{
    if (!s || !info) return B3G_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return B3G_ERR_INVALID_ARGUMENT;
    const Request* r = it->second;
    info->state = (uint32_t)r->state;
    info->status = r->status;
    info->steps_done = r->steps_done;
    info->steps_total = r->steps_total;
    info->vertex_count = r->state == R_DONE ? (uint32_t)(r->result.size() / 3)
                                            : (r->cloth ? r->cloth->dev.n : (uint32_t)(r->verts.size() / 3));
    info->arrival = r->arrival;
    info->admitted = r->admitted;
    info->finished = r->finished;
    info->bytes = r->bytes;
    return B3G_OK;
}

b3g_status b3g_server_result(b3g_server* s, uint64_t id, float* positions)
{
    if (!s || !positions) return B3G_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end() || it->second->state != R_DONE) return B3G_ERR_INVALID_ARGUMENT;
    std::memcpy(positions, it->second->result.data(), it->second->result.size() * sizeof(float));
    return B3G_OK;
}

b3g_status b3g_server_release(b3g_server* s, uint64_t id)
{
    if (!s) return B3G_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return B3G_ERR_INVALID_ARGUMENT;
    Request* r = it->second;
    if (r->state != R_DONE && r->state != R_FAILED) return B3G_ERR_INVALID_ARGUMENT;
    delete r;
    s->all.erase(it);
    return B3G_OK;
}

b3g_status b3g_server_stats(const b3g_server* cs, b3g_server_statistics* out)
{
    b3g_server* s = const_cast<b3g_server*>(cs);
    if (!s || !out) return B3G_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->ticks = s->ticks;
    out->steps = s->steps;
    out->vertex_steps = s->vertex_steps;
    out->busy_ms = s->busy_ms;
    out->admitted = s->admitted;
    out->completed = s->completed;
    out->rejected = s->rejected;
    out->active = (uint32_t)s->active.size();
    out->queued = (uint32_t)(s->prep.size() + s->ready.size());
    out->peak_active = s->peak_active;
    out->peak_bytes = s->peak_used;
    // step latency percentiles: every cloth stepped in a tick waited that tick
    std::vector<std::pair<float, uint32_t>> v = s->tick_samples;
    std::sort(v.begin(), v.end());
    uint64_t total = 0;
    for (auto& p : v) total += p.second;
    auto pct = [&](double q) -> float {
        if (!total) return 0.0f;
        const uint64_t target = (uint64_t)(q * (double)(total - 1));
        uint64_t acc = 0;
        for (auto& p : v) {
            acc += p.second;
            if (acc > target) return p.first;
        }
        return v.back().first;
    };
    out->p50_step_ms = pct(0.50);
    out->p99_step_ms = pct(0.99);
    out->max_step_ms = v.empty() ? 0.0f : v.back().first;
    return B3G_OK;
}

}  // extern "C"
