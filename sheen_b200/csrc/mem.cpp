// mem.cpp -- device memory of the library: one stream-ordered pool per
// device that keeps freed blocks for reuse.
//
// Plain cudaMalloc / cudaFree of blocks of hundreds of MB map and unmap
// memory in the driver every time; on the B200 boxes this was measured at
// 1-2 ms usually but up to 0.1 s (allocation) and 0.7 s (free) at random,
// which dominated a host-arrays-in, image-out render call (scene arena,
// BVH build scratch, wavefront queues, output).  Blocks returned to the
// pool stay mapped (up to the pool's release threshold, "mem.pool_keep_mb",
// default 16 GB) and are handed out again without a driver call.
// sheen_cleanup destroys the pools.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "engine.h"

namespace sheen {
namespace {

constexpr int kMaxDevices = 64;

struct DevPool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;   // allocations are ordered on this otherwise idle stream
    uint64_t keep = 0;
};
std::mutex g_mu;
DevPool g_pools[kMaxDevices];

cudaError_t pool_of(int dev, DevPool*& out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    DevPool& p = g_pools[dev];
    if (!p.pool) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaError_t e = cudaMemPoolCreate(&p.pool, &props);
        if (e != cudaSuccess) { p.pool = nullptr; return e; }
        e = cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(p.pool);
            p.pool = nullptr;
            p.stream = nullptr;
            return e;
        }
    }
    const uint64_t keep = (uint64_t)tuning().pool_keep_mb << 20;
    if (keep != p.keep) {
        uint64_t v = keep;
        cudaMemPoolSetAttribute(p.pool, cudaMemPoolAttrReleaseThreshold, &v);
        p.keep = keep;
    }
    out = &p;
    return cudaSuccess;
}

}  // namespace

// An allocation that fails for lack of memory is retried once after the
// pool has returned every unused block to the device.
static cudaError_t pool_alloc(void** ptr, size_t bytes, cudaStream_t stream, bool sync) {
    *ptr = nullptr;
    if (bytes == 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    DevPool* p = nullptr;
    if ((e = pool_of(dev, p)) != cudaSuccess) return e;
    cudaStream_t st = sync ? p->stream : stream;
    e = cudaMallocFromPoolAsync(ptr, bytes, p->pool, st);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        release_parked_waves();
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(p->pool, 0);
        e = cudaMallocFromPoolAsync(ptr, bytes, p->pool, st);
    }
    if (e == cudaSuccess && sync) e = cudaStreamSynchronize(st);
    return e;
}

cudaError_t dmalloc(void** ptr, size_t bytes) { return pool_alloc(ptr, bytes, nullptr, true); }

cudaError_t dmalloc_async(void** ptr, size_t bytes, cudaStream_t stream) {
    return pool_alloc(ptr, bytes, stream, false);
}

// Returns the unused blocks of the current device's pool to the device
// (before a caller sizes itself by cudaMemGetInfo).
void trim_pool() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    DevPool* p = nullptr;
    if (pool_of(dev, p) != cudaSuccess) return;
    release_parked_waves();
    cudaDeviceSynchronize();
    cudaMemPoolTrimTo(p->pool, 0);
}

void dfree(void* ptr) {
    if (!ptr) return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    DevPool* p = nullptr;
    if (pool_of(dev, p) != cudaSuccess) return;
    cudaDeviceSynchronize();   // like cudaFree: no kernel may still use the block
    cudaFreeAsync(ptr, p->stream);
    cudaStreamSynchronize(p->stream);   // the free has happened: any stream may reuse the block
}

void dfree_async(void* ptr, cudaStream_t stream) {
    if (ptr) cudaFreeAsync(ptr, stream);
}

void release_pools() {
    std::lock_guard<std::mutex> lk(g_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (int d = 0; d < kMaxDevices; d++) {
        DevPool& p = g_pools[d];
        if (!p.pool) continue;
        cudaSetDevice(d);
        cudaStreamSynchronize(p.stream);
        cudaStreamDestroy(p.stream);
        cudaMemPoolDestroy(p.pool);
        p = DevPool();
    }
    cudaSetDevice(cur);
}

}  // namespace sheen
