// png_pack.cu -- the PNG path's sRGB8 conversion on the device.
//
// sheen_render_scene packs the rendered float4 image into PNG raw rows (a
// filter byte 0, then RGB8 per pixel) on the device and reads back 3 bytes a
// pixel instead of 16.  Each channel's byte is the number of the host
// conversion's step thresholds (srgb_thresholds, png.cpp: the smallest
// linear value of every byte 1..255 under png_color.h:11-20) at or below the
// value, found by binary search -- the same bytes as the host conversion,
// with no pow evaluated on the device.
#include <mutex>

#include "engine.h"

namespace sheen {

const float* srgb_thresholds();

namespace dev {

__constant__ float c_srgb_thr[255];

__global__ void srgb_pack_rows(const float4* __restrict__ img, int W, int H, unsigned char* __restrict__ rows) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)W * H) return;
    const int y = (int)(i / W), x = (int)(i - (long long)y * W);
    const float4 p = img[i];
    unsigned char* row = rows + (size_t)y * (1 + 3 * (size_t)W);
    if (x == 0) row[0] = 0;
    const float c[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        int lo = 0;
        if (c[k] > 0.0f) {   // zero, negative and NaN give byte 0
            int hi = 255;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (c_srgb_thr[mid] <= c[k]) lo = mid + 1;
                else hi = mid;
            }
        }
        row[1 + 3 * x + k] = (unsigned char)lo;
    }
}

}  // namespace dev

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
bool g_ready[kMaxDevices] = {false};
}  // namespace

// sheen_cleanup resets the device, which clears the constant table: the next
// pack on each device uploads it again.
void release_srgb_tables() {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto& r : g_ready) r = false;
}

cudaError_t pack_srgb_rows(const float4* img, int W, int H, unsigned char* rows, cudaStream_t stream) {
    int dev_id = 0;
    cudaError_t e = cudaGetDevice(&dev_id);
    if (e != cudaSuccess) return e;
    if (dev_id < 0 || dev_id >= kMaxDevices) return cudaErrorInvalidDevice;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_ready[dev_id]) {
            e = cudaMemcpyToSymbol(dev::c_srgb_thr, srgb_thresholds(), 255 * sizeof(float));
            if (e != cudaSuccess) return e;
            g_ready[dev_id] = true;
        }
    }
    const long long n = (long long)W * H;
    dev::srgb_pack_rows<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(img, W, H, rows);
    return cudaGetLastError();
}

}  // namespace sheen
