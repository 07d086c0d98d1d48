// tuning.cpp -- launch parameters of the wavefront form, settable by name.
//
// The autotuner (sheen_autotune) times candidate settings on a caller's
// scene and frame and keeps the fastest; callers may also set them
// directly.  Every change bumps a generation number so that captured frame
// graphs built under older settings are re-captured.
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

#include "engine.h"

namespace sheen {
namespace {

std::mutex g_tune_mu;
Tuning g_tuning;
std::atomic<int> g_generation{1};

struct Key {
    const char* name;
    int Tuning::*field;
    int lo, hi;
};

const Key kKeys[] = {
    {"wave.shadow_kernel", &Tuning::shadow_kernel, 0, 1},
    {"wave.refill_min", &Tuning::refill_min, 1, 32},
    {"wave.inner_min", &Tuning::inner_min, 0, 32},
    {"build.node_cost", &Tuning::node_cost, 1, 64},
    {"wave.shadow_blocks_per_sm", &Tuning::shadow_blocks_per_sm, 0, 16},
    {"wave.shadow_stack", &Tuning::shadow_stack, 0, 1},
    {"build.device", &Tuning::build_device, 0, 1},
    {"build.concurrent", &Tuning::build_concurrent, 0, 1},
    {"mem.pool_keep_mb", &Tuning::pool_keep_mb, 0, 1 << 20},
    {"mem.prewarm_mb", &Tuning::prewarm_mb, 0, 1 << 20},
    {"trace.watertight", &Tuning::watertight, 0, 1},
    {"camera.centered", &Tuning::aa_centered, 0, 1},
    {"trace.se_polish", &Tuning::se_polish, 0, 1},
    {"caustic.knn", &Tuning::caustic_knn, 0, 64},
    {"wave.mega_samples", &Tuning::mega_samples, 0, 1 << 30},
    {"wave.tile_w", &Tuning::tile_w, 8, 32},
};

}  // namespace

Tuning tuning() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return g_tuning;
}

int tuning_generation() { return g_generation.load(); }

int tuning_set(const char* name, int value) {
    if (!name) { set_error("null tuning key"); return -1; }
    for (const Key& k : kKeys) {
        if (std::strcmp(k.name, name) != 0) continue;
        if (value < k.lo || value > k.hi) { set_errorf("tuning value out of range for %s", name); return -1; }
        if (k.field == &Tuning::tile_w && value != 8 && value != 16 && value != 32) {
            set_errorf("%s must be 8, 16 or 32", name);
            return -1;
        }
        std::lock_guard<std::mutex> lk(g_tune_mu);
        if (g_tuning.*(k.field) != value) {
            g_tuning.*(k.field) = value;
            g_generation++;
        }
        return 0;
    }
    set_errorf("unknown tuning key %s", name);
    return -1;
}

int tuning_get(const char* name, int* value) {
    if (!name || !value) { set_error("null tuning key or value"); return -1; }
    for (const Key& k : kKeys) {
        if (std::strcmp(k.name, name) != 0) continue;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        *value = g_tuning.*(k.field);
        return 0;
    }
    set_errorf("unknown tuning key %s", name);
    return -1;
}

}  // namespace sheen

extern "C" int sheen_tune_set(const char* key, int value) { return sheen::tuning_set(key, value); }
extern "C" int sheen_tune_get(const char* key, int* value) { return sheen::tuning_get(key, value); }

// ---------------------------------------------------------------------
// Autotuner: times the candidate settings on the caller's scene and frame
// shape, keeps the fastest.
// ---------------------------------------------------------------------
namespace sheen {
namespace {

struct Candidate {
    int shadow_kernel, refill_min, shadow_blocks_per_sm, shadow_stack, inner_min, tile_w, mega_samples;
};

void apply(const Candidate& c) {
    tuning_set("wave.shadow_kernel", c.shadow_kernel);
    tuning_set("wave.refill_min", c.refill_min);
    tuning_set("wave.shadow_blocks_per_sm", c.shadow_blocks_per_sm);
    tuning_set("wave.shadow_stack", c.shadow_stack);
    tuning_set("wave.inner_min", c.inner_min);
    tuning_set("wave.tile_w", c.tile_w);
    tuning_set("wave.mega_samples", c.mega_samples);
}

}  // namespace
}  // namespace sheen

extern "C" int sheen_autotune(SheenDeviceScene h, int W, int H, int aa, int reps, SheenTuneResult* out) {
    using namespace sheen;
    auto* s = reinterpret_cast<DeviceScene*>(h);
    if (!s || !out) { set_error("null scene or result"); return -1; }
    if (W <= 0 || H <= 0 || aa < 1 || aa > 64) { set_error("bad render params"); return -1; }
    if (s->form != SHEEN_FORM_WAVEFRONT) { set_error("autotuning applies to SHEEN_FORM_WAVEFRONT scenes"); return -1; }
    if (reps < 1) reps = 3;
    const Tuning t0 = tuning();
    const Candidate start{t0.shadow_kernel, t0.refill_min, t0.shadow_blocks_per_sm, t0.shadow_stack, t0.inner_min,
                          t0.tile_w, t0.mega_samples};
    std::vector<Candidate> cands;
    cands.push_back(start);
    cands.push_back({0, t0.refill_min, 0, 0, 0, t0.tile_w, t0.mega_samples});
    for (int st : {0, 1})
        for (int r : {8, 16, 24})
            for (int im : {0, 6, 10, 14}) cands.push_back({1, r, 0, st, im, t0.tile_w, t0.mega_samples});
    cands.push_back({1, 16, 4, 0, 10, t0.tile_w, t0.mega_samples});
    float4* buf = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = dmalloc(&buf, (size_t)W * H * sizeof(float4));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    double best = 1e30, first = 0.0;
    int best_i = 0;
    const Region rg{0, 0, W, H};
    auto time_from = [&](size_t from) {
        for (size_t i = from; i < cands.size() && e == cudaSuccess; i++) {
            apply(cands[i]);
            if ((e = launch_wavefront(*s, W, H, aa, rg, buf, st, false)) != cudaSuccess) break;   // warm-up + capture
            cudaEventRecord(e0, st);
            for (int k = 0; k < reps && e == cudaSuccess; k++) e = launch_wavefront(*s, W, H, aa, rg, buf, st, false);
            cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double per = ms / reps;
            if (i == 0) first = per;
            if (per < best) { best = per; best_i = (int)i; }
        }
    };
    // 1. the shadow stage's parameters
    time_from(0);
    // 2. the pixel tile of the sample order, with the best shadow setting
    if (e == cudaSuccess) {
        const size_t from = cands.size();
        for (int tw : {8, 16, 32}) {
            if (tw == cands[(size_t)best_i].tile_w) continue;
            Candidate c = cands[(size_t)best_i];
            c.tile_w = tw;
            cands.push_back(c);
        }
        time_from(from);
    }
    // 3. the small-frame switch: queue stages or the megakernel for this frame
    if (e == cudaSuccess) {
        const size_t from = cands.size();
        for (int m : {0, 1 << 30}) {
            Candidate c = cands[(size_t)best_i];
            c.mega_samples = m;
            cands.push_back(c);
        }
        time_from(from);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    dfree(buf);
    if (e != cudaSuccess) {
        apply(start);
        set_error(cudaGetErrorString(e));
        return -1;
    }
    apply(cands[best_i]);
    out->shadow_kernel = cands[best_i].shadow_kernel;
    out->refill_min = cands[best_i].refill_min;
    out->shadow_blocks_per_sm = cands[best_i].shadow_blocks_per_sm;
    out->shadow_stack = cands[best_i].shadow_stack;
    out->inner_min = cands[best_i].inner_min;
    out->tile_w = cands[best_i].tile_w;
    out->mega_samples = cands[best_i].mega_samples;
    out->candidates = (int)cands.size();
    out->best_ms = best;
    out->default_ms = first;
    return 0;
}
