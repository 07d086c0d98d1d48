// tuning.cpp -- launch parameters of the wavefront form, settable by name.
//
// The autotuner (sheen_autotune) times candidate settings on a caller's
// scene and frame and keeps the fastest; callers may also set them
// directly.  Every change bumps a generation number so that captured frame
// graphs built under older settings are re-captured.
#include <atomic>
#include <cstring>
#include <mutex>

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
    {"wave.shadow_blocks_per_sm", &Tuning::shadow_blocks_per_sm, 0, 16},
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
