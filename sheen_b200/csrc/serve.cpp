// serve.cpp -- the request loop behind sheen_server_* (continuous batching).
//
// The reference renders one frame per C-API call and rebuilds and re-uploads
// the scene every time (api/sheen_c_api.cu:187-361).  Here scenes are added
// once and stay resident; render requests of any resolution and sample
// count are queued as they arrive and admitted onto the GPU as soon as a
// slot (one CUDA stream) is free and their device footprint fits in the HBM
// budget, so requests that arrive while others run overlap with them on the
// device.
//
// Layout of one admitted request:
//   * one device block from the server's stream-ordered memory pool, freed
//     in stream order after the request's last copy:
//       [ wavefront queues for one tile | tile output (float4) | 8 tallies ]
//   * the image is rendered in bands of whole rows ("tiles", at most
//     tile_samples samples each, rows a multiple of 16 except the last); each
//     band is copied into the slot's pinned staging image, and the staging
//     image into the caller's host buffer when the stream reaches the end.
// Results do not depend on the tiling or on what else runs: every sample's
// random numbers are a function of its pixel, sample index and bounce only.
//
// Threads: the caller's threads (submit / wait / add_scene), one worker that
// admits and launches, and CUDA's host-callback thread, which copies a
// finished request into the caller's buffer and frees its slot.  The worker
// never holds the server lock across a CUDA call that could wait for a
// callback.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace sheen {
namespace {

constexpr int kDefaultInflight = 4;
constexpr long long kDefaultTileSamples = 1ll << 22;
constexpr int kMaxBypass = 16;   // later requests admitted past a blocked head before it gets priority

struct Server;

struct Request {
    unsigned long long id = 0;
    int scene_id = -1;
    DeviceScene* scene = nullptr;
    int W = 0, H = 0, aa = 1;
    float* out_host = nullptr;
    int status = SHEEN_REQ_PENDING;
    std::string error;
    double t_submit = 0, t_start = 0, t_done = 0;
    unsigned long long rays = 0;
    size_t device_bytes = 0;    // block from the pool
    size_t scratch_bytes = 0;   // wavefront queues inside the block
    int rows_per_tile = 0, tiles = 0;
    int bypassed = 0;
};

struct Slot {
    Server* server = nullptr;
    int index = 0;
    cudaStream_t stream = nullptr;
    float4* staging = nullptr;          // pinned, grow-only
    size_t staging_bytes = 0;
    unsigned long long* h_tally = nullptr;   // pinned, 8 counters
    Request* req = nullptr;
};

struct SceneEntry {
    DeviceScene* scene = nullptr;
    size_t bytes = 0;
    int refs = 0;              // pending + in-flight requests
    bool removed = false;      // freed when refs drops to 0
};

struct Server {
    std::mutex mu;
    std::condition_variable cv_work;   // worker: new request, slot freed, stop
    std::condition_variable cv_done;   // waiters: a request finished
    std::thread worker;
    bool stop = false;
    int device = 0;
    int form = SHEEN_FORM_WAVEFRONT;
    long long tile_samples = kDefaultTileSamples;
    size_t budget = 0, used = 0, peak = 0, scene_bytes = 0;
    cudaMemPool_t pool = nullptr;
    std::vector<Slot*> slots;
    std::vector<Slot*> free_slots;
    std::deque<Request*> pending;
    std::unordered_map<unsigned long long, Request*> requests;   // until waited for
    std::map<int, SceneEntry> scenes;
    int next_scene = 0;
    unsigned long long next_request = 1;
    // statistics
    unsigned long long submitted = 0, completed = 0, failed = 0, rays = 0;
    std::vector<double> latencies;
    double first_submit = -1, last_done = -1;
    int inflight = 0, inflight_peak = 0;
};

std::mutex g_servers_mu;
std::set<Server*> g_servers;

void release_scene_ref(Server& sv, int scene_id) {
    auto it = sv.scenes.find(scene_id);
    if (it == sv.scenes.end()) return;
    if (--it->second.refs == 0 && it->second.removed) {
        sv.used -= it->second.bytes;
        sv.scene_bytes -= it->second.bytes;
        scene_release(it->second.scene);
        sv.scenes.erase(it);
    }
}

// Marks `r` finished (lock held).
void finish_locked(Server& sv, Request* r, int status, const char* err) {
    r->status = status;
    if (err) r->error = err;
    r->t_done = now_ms();
    if (status == SHEEN_REQ_DONE) {
        sv.completed++;
        sv.rays += r->rays;
        sv.latencies.push_back(r->t_done - r->t_submit);
    } else {
        sv.failed++;
    }
    sv.last_done = std::max(sv.last_done, r->t_done);
    release_scene_ref(sv, r->scene_id);
    r->scene = nullptr;
    sv.cv_done.notify_all();
}

// Stream callback: the request's last copy has landed in the slot's staging
// image.  Runs on CUDA's callback thread: no CUDA calls here.
void CUDART_CB on_request_done(void* p) {
    Slot* slot = static_cast<Slot*>(p);
    Server& sv = *slot->server;
    Request* r = slot->req;
    std::memcpy(r->out_host, slot->staging, (size_t)r->W * r->H * sizeof(float4));
    r->rays = slot->h_tally[0] + slot->h_tally[1] + slot->h_tally[2];
    std::lock_guard<std::mutex> lk(sv.mu);
    sv.used -= r->device_bytes;
    sv.inflight--;
    slot->req = nullptr;
    sv.free_slots.push_back(slot);
    finish_locked(sv, r, r->error.empty() ? SHEEN_REQ_DONE : SHEEN_REQ_FAILED, nullptr);
    sv.cv_work.notify_all();
}

// Plans the bands of `r` and its device footprint.
void plan_request(const Server& sv, Request& r) {
    const int ns = std::min(std::max(r.aa, 1), 64);
    // queue scratch for a band padded to any of the wavefront sample order's
    // tile shapes (8x16, 16x8, 32x4: widths up to 32, heights up to 16)
    const long long wpad = (long long)((r.W + 31) / 32) * 32;
    long long rows = sv.tile_samples / (wpad * ns);
    rows = std::max<long long>(16, rows / 16 * 16);
    if (rows >= r.H) rows = r.H;
    r.rows_per_tile = (int)rows;
    r.tiles = (int)((r.H + rows - 1) / rows);
    const long long tile_samples = wpad * ((rows + 15) / 16 * 16) * ns;
    const bool queues = sv.form == SHEEN_FORM_WAVEFRONT && wave_pipeline_used(*r.scene);
    r.scratch_bytes = queues ? wave_scratch_bytes(r.scene->view.num_lights, tile_samples) : 0;
    const size_t tile_out = ((size_t)r.W * rows * sizeof(float4) + 255) & ~(size_t)255;
    r.device_bytes = r.scratch_bytes + tile_out + 8 * sizeof(unsigned long long);
}

// Enqueues every launch and copy of `r` on the slot's stream.  Returns false
// (with r->error set) when nothing was enqueued.
bool launch_request(Server& sv, Slot* slot, Request* r) {
    const cudaStream_t st = slot->stream;
    const size_t image_bytes = (size_t)r->W * r->H * sizeof(float4);
    if (slot->staging_bytes < image_bytes) {
        if (slot->staging) cudaFreeHost(slot->staging);
        slot->staging = nullptr;
        slot->staging_bytes = 0;
        if (cudaHostAlloc((void**)&slot->staging, image_bytes, cudaHostAllocDefault) != cudaSuccess) {
            slot->staging = nullptr;
            r->error = "pinned staging allocation failed";
            return false;
        }
        slot->staging_bytes = image_bytes;
    }
    void* block = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&block, r->device_bytes, sv.pool, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        r->error = std::string("device allocation failed: ") + cudaGetErrorString(e);
        return false;
    }
    char* base = static_cast<char*>(block);
    float4* tile_out = reinterpret_cast<float4*>(base + r->scratch_bytes);
    const size_t tile_out_bytes = ((size_t)r->W * r->rows_per_tile * sizeof(float4) + 255) & ~(size_t)255;
    auto* tally = reinterpret_cast<unsigned long long*>(base + r->scratch_bytes + tile_out_bytes);
    e = cudaMemsetAsync(tally, 0, 8 * sizeof(unsigned long long), st);
    for (int t = 0; t < r->tiles && e == cudaSuccess; t++) {
        const int y0 = t * r->rows_per_tile, y1 = std::min(r->H, y0 + r->rows_per_tile);
        const Region rg{0, y0, r->W, y1};
        // The kernels index the output as a whole image (y * W + x); the
        // band's rows land at the start of tile_out.
        float4* out = tile_out - (ptrdiff_t)y0 * r->W;
        if (sv.form == SHEEN_FORM_PLAIN)
            e = launch_plain(*r->scene, r->W, r->H, r->aa, rg, out, st, false, tally);
        else
            e = launch_wavefront_scratch(*r->scene, block, r->scratch_bytes, r->W, r->H, r->aa, rg, out, st, tally);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(slot->staging + (size_t)y0 * r->W, tile_out, (size_t)(y1 - y0) * r->W * sizeof(float4),
                                cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(slot->h_tally, tally, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) r->error = std::string("launch failed: ") + cudaGetErrorString(e);
    // The block goes back to the pool and the callback runs even after a
    // failed launch, so the slot and the accounting are always released.
    cudaFreeAsync(block, st);
    slot->req = r;
    if (cudaLaunchHostFunc(st, on_request_done, slot) != cudaSuccess) {
        cudaStreamSynchronize(st);
        slot->req = nullptr;
        if (r->error.empty()) r->error = "host callback failed";
        return false;
    }
    return true;
}

void worker_main(Server* svp) {
    Server& sv = *svp;
    cudaSetDevice(sv.device);
    std::unique_lock<std::mutex> lk(sv.mu);
    for (;;) {
        if (sv.stop && sv.pending.empty() && sv.inflight == 0) break;
        // Admission: walk the queue in arrival order; a request is admitted
        // when a slot is free and its footprint fits.  Requests behind a
        // blocked one may go first until it has been passed kMaxBypass
        // times; from then on nothing is admitted ahead of it.
        std::vector<std::pair<Slot*, Request*>> admitted;
        Request* blocked = nullptr;   // first request that did not fit
        for (auto it = sv.pending.begin(); it != sv.pending.end() && !sv.free_slots.empty();) {
            Request* r = *it;
            if (sv.used + r->device_bytes <= sv.budget) {
                if (blocked) blocked->bypassed++;
                Slot* slot = sv.free_slots.back();
                sv.free_slots.pop_back();
                sv.used += r->device_bytes;
                sv.peak = std::max(sv.peak, sv.used);
                sv.inflight++;
                sv.inflight_peak = std::max(sv.inflight_peak, sv.inflight);
                r->status = SHEEN_REQ_RUNNING;
                r->t_start = now_ms();
                admitted.emplace_back(slot, r);
                it = sv.pending.erase(it);
                continue;
            }
            if (!blocked) blocked = r;
            if (blocked->bypassed >= kMaxBypass) break;
            ++it;
        }
        if (admitted.empty()) {
            if (sv.stop && sv.inflight == 0) {
                // Pending requests that can never be admitted end here.
                while (!sv.pending.empty()) {
                    finish_locked(sv, sv.pending.front(), SHEEN_REQ_FAILED, "server destroyed");
                    sv.pending.pop_front();
                }
                continue;
            }
            sv.cv_work.wait(lk);
            continue;
        }
        lk.unlock();
        for (auto& a : admitted) {
            if (!launch_request(sv, a.first, a.second)) {
                std::lock_guard<std::mutex> g(sv.mu);
                sv.used -= a.second->device_bytes;
                sv.inflight--;
                sv.free_slots.push_back(a.first);
                finish_locked(sv, a.second, SHEEN_REQ_FAILED, nullptr);
            }
        }
        lk.lock();
    }
}

void server_destroy(Server* sv) {
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        // Pending requests are cancelled; in-flight ones finish.
        while (!sv->pending.empty()) {
            finish_locked(*sv, sv->pending.front(), SHEEN_REQ_FAILED, "server destroyed");
            sv->pending.pop_front();
        }
        sv->cv_work.notify_all();
    }
    if (sv->worker.joinable()) sv->worker.join();
    cudaSetDevice(sv->device);
    for (Slot* s : sv->slots) {
        if (s->stream) {
            cudaStreamSynchronize(s->stream);
            cudaStreamDestroy(s->stream);
        }
        if (s->staging) cudaFreeHost(s->staging);
        if (s->h_tally) cudaFreeHost(s->h_tally);
        delete s;
    }
    for (auto& kv : sv->scenes) scene_release(kv.second.scene);
    for (auto& kv : sv->requests) delete kv.second;
    if (sv->pool) cudaMemPoolDestroy(sv->pool);
    delete sv;
}

Server* lookup(SheenServer h) {
    auto* sv = reinterpret_cast<Server*>(h);
    std::lock_guard<std::mutex> lk(g_servers_mu);
    return g_servers.count(sv) ? sv : nullptr;
}

void fill_info(const Request& r, SheenRequestInfo* info) {
    if (!info) return;
    std::memset(info, 0, sizeof(*info));
    info->status = r.status;
    info->scene_id = r.scene_id;
    info->width = r.W;
    info->height = r.H;
    info->aa_samples = r.aa;
    info->tiles = r.tiles;
    info->rays = r.rays;
    info->hbm_bytes = r.device_bytes;
    const double now = now_ms();
    const double start = r.t_start > 0 ? r.t_start : now;
    const double done = r.t_done > 0 ? r.t_done : now;
    info->queue_ms = start - r.t_submit;
    info->run_ms = r.t_start > 0 ? done - r.t_start : 0.0;
    info->latency_ms = done - r.t_submit;
    std::snprintf(info->error, sizeof(info->error), "%s", r.error.c_str());
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    // Nearest-rank percentile.
    size_t k = (size_t)std::ceil(q * v.size());
    k = std::min(std::max<size_t>(k, 1), v.size());
    return v[k - 1];
}

}  // namespace

void release_all_servers() {
    std::vector<Server*> all;
    {
        std::lock_guard<std::mutex> lk(g_servers_mu);
        all.assign(g_servers.begin(), g_servers.end());
        g_servers.clear();
    }
    for (Server* s : all) server_destroy(s);
}

}  // namespace sheen

using namespace sheen;

extern "C" int sheen_server_create(const SheenServerConfig* cfg, SheenServer* out) {
    if (!out) { set_error("null output handle"); return -1; }
    *out = nullptr;
    SheenServerConfig c{};
    c.form = SHEEN_FORM_WAVEFRONT;
    if (cfg) c = *cfg;
    if (c.form != SHEEN_FORM_PLAIN && c.form != SHEEN_FORM_WAVEFRONT) { set_error("unknown renderer form"); return -1; }
    if (c.max_inflight > 64) { set_error("max_inflight above 64"); return -1; }
    auto* sv = new Server();
    cudaGetDevice(&sv->device);
    sv->form = c.form;
    sv->tile_samples = c.tile_samples > 0 ? c.tile_samples : kDefaultTileSamples;
    size_t free_b = 0, total_b = 0;
    trim_pool();   // blocks the library keeps for reuse count as free
    cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) {
        delete sv;
        set_error(cudaGetErrorString(e));
        return -1;
    }
    sv->budget = c.hbm_budget ? (size_t)c.hbm_budget : (size_t)(0.9 * (double)free_b);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = sv->device;
    if ((e = cudaMemPoolCreate(&sv->pool, &props)) != cudaSuccess) {
        delete sv;
        set_error(cudaGetErrorString(e));
        return -1;
    }
    // Keep freed blocks in the pool (no trips to the driver between requests).
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    const int n = c.max_inflight > 0 ? c.max_inflight : kDefaultInflight;
    for (int i = 0; i < n; i++) {
        Slot* s = new Slot();
        s->server = sv;
        s->index = i;
        sv->slots.push_back(s);
        sv->free_slots.push_back(s);
        if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaHostAlloc((void**)&s->h_tally, 8 * sizeof(unsigned long long), cudaHostAllocDefault)) !=
                cudaSuccess) {
            server_destroy(sv);
            set_error(cudaGetErrorString(e));
            return -1;
        }
    }
    std::reverse(sv->free_slots.begin(), sv->free_slots.end());
    sv->worker = std::thread(worker_main, sv);
    {
        std::lock_guard<std::mutex> lk(g_servers_mu);
        g_servers.insert(sv);
    }
    *out = reinterpret_cast<SheenServer>(sv);
    return 0;
}

extern "C" void sheen_server_destroy(SheenServer h) {
    auto* sv = reinterpret_cast<Server*>(h);
    {
        std::lock_guard<std::mutex> lk(g_servers_mu);
        if (!g_servers.erase(sv)) return;
    }
    server_destroy(sv);
}

extern "C" int sheen_server_add_scene(SheenServer h, const SheenScene* scene, int* scene_id) {
    Server* sv = lookup(h);
    if (!sv) { set_error("unknown server handle"); return -1; }
    if (!scene || !scene_id) { set_error("null scene or scene_id"); return -1; }
    // Build and upload outside the server lock: requests keep flowing.
    DeviceScene* ds = nullptr;
    cudaSetDevice(sv->device);
    if (scene_upload(scene, sv->form, &ds) != 0) return -1;
    const size_t bytes = ds->arena_bytes + ds->extra_bytes;
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->used + bytes > sv->budget) {
        scene_release(ds);
        set_error("scene does not fit in the server's HBM budget");
        return -1;
    }
    sv->used += bytes;
    sv->peak = std::max(sv->peak, sv->used);
    sv->scene_bytes += bytes;
    const int id = sv->next_scene++;
    sv->scenes[id] = SceneEntry{ds, bytes, 0, false};
    *scene_id = id;
    return 0;
}

extern "C" int sheen_server_remove_scene(SheenServer h, int scene_id) {
    Server* sv = lookup(h);
    if (!sv) { set_error("unknown server handle"); return -1; }
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->scenes.find(scene_id);
    if (it == sv->scenes.end() || it->second.removed) { set_error("unknown scene id"); return -1; }
    it->second.removed = true;
    if (it->second.refs == 0) {
        it->second.refs = 1;
        release_scene_ref(*sv, scene_id);
    }
    return 0;
}

extern "C" int sheen_server_submit(SheenServer h, int scene_id, int width, int height, int aa_samples,
                                   float* out_rgba_host, unsigned long long* request_id) {
    Server* sv = lookup(h);
    if (!sv) { set_error("unknown server handle"); return -1; }
    if (width <= 0 || height <= 0) { set_error("Invalid image dimensions"); return -1; }
    if (aa_samples < 1 || aa_samples > 64) { set_error("AA samples must be between 1 and 64"); return -1; }
    if (!out_rgba_host || !request_id) { set_error("null output buffer or request_id"); return -1; }
    if ((long long)width * height > (1ll << 28)) { set_error("image too large"); return -1; }
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) { set_error("server is shutting down"); return -1; }
    auto it = sv->scenes.find(scene_id);
    if (it == sv->scenes.end() || it->second.removed) { set_error("unknown scene id"); return -1; }
    auto* r = new Request();
    r->id = sv->next_request++;
    r->scene_id = scene_id;
    r->scene = it->second.scene;
    r->W = width;
    r->H = height;
    r->aa = aa_samples;
    r->out_host = out_rgba_host;
    plan_request(*sv, *r);
    // A request whose footprint can never fit beside the resident scenes is
    // refused now rather than left waiting.
    if (sv->scene_bytes + r->device_bytes > sv->budget) {
        delete r;
        set_error("request footprint exceeds the server's HBM budget");
        return -1;
    }
    it->second.refs++;
    r->t_submit = now_ms();
    if (sv->first_submit < 0) sv->first_submit = r->t_submit;
    sv->submitted++;
    sv->requests[r->id] = r;
    sv->pending.push_back(r);
    sv->cv_work.notify_all();
    *request_id = r->id;
    return 0;
}

extern "C" int sheen_server_poll(SheenServer h, unsigned long long request_id) {
    Server* sv = lookup(h);
    if (!sv) { set_error("unknown server handle"); return -1; }
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->requests.find(request_id);
    if (it == sv->requests.end()) { set_error("unknown request id"); return -1; }
    return it->second->status;
}

extern "C" int sheen_server_wait(SheenServer h, unsigned long long request_id, double timeout_ms,
                                 SheenRequestInfo* info) {
    Server* sv = lookup(h);
    if (!sv) { set_error("unknown server handle"); return -1; }
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->requests.find(request_id);
    if (it == sv->requests.end()) { set_error("unknown request id"); return -1; }
    Request* r = it->second;
    auto finished = [r] { return r->status == SHEEN_REQ_DONE || r->status == SHEEN_REQ_FAILED; };
    if (timeout_ms < 0) {
        sv->cv_done.wait(lk, finished);
    } else if (!sv->cv_done.wait_for(lk, std::chrono::microseconds((long long)(timeout_ms * 1000.0)), finished)) {
        fill_info(*r, info);
        return 0;
    }
    fill_info(*r, info);
    sv->requests.erase(request_id);
    delete r;
    return 1;
}

extern "C" int sheen_server_stats(SheenServer h, SheenServerStats* out) {
    Server* sv = lookup(h);
    if (!sv) { set_error("unknown server handle"); return -1; }
    if (!out) { set_error("null stats"); return -1; }
    std::lock_guard<std::mutex> lk(sv->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = sv->submitted;
    out->completed = sv->completed;
    out->failed = sv->failed;
    out->rays = sv->rays;
    out->p50_ms = percentile(sv->latencies, 0.50);
    out->p99_ms = percentile(sv->latencies, 0.99);
    double sum = 0, mx = 0;
    for (double v : sv->latencies) { sum += v; mx = std::max(mx, v); }
    out->mean_ms = sv->latencies.empty() ? 0.0 : sum / sv->latencies.size();
    out->max_ms = mx;
    out->busy_ms = (sv->first_submit >= 0 && sv->last_done >= 0) ? sv->last_done - sv->first_submit : 0.0;
    out->hbm_budget = sv->budget;
    out->hbm_used = sv->used;
    out->hbm_peak = sv->peak;
    out->scene_bytes = sv->scene_bytes;
    out->inflight_peak = sv->inflight_peak;
    out->pending = (int)sv->pending.size();
    out->inflight = sv->inflight;
    return 0;
}
