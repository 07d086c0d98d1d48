// temporary stubs (replaced by the wavefront implementation)
#include "engine.h"
namespace sheen {
void build_qbvh4(const Triangle*, int, QBvh&) {}
cudaError_t launch_mega_bvh4(const DeviceScene& s, int W, int H, int aa, Region rg, float4* out, cudaStream_t st) {
    return launch_plain(s, W, H, aa, rg, out, st, false);
}
cudaError_t launch_wavefront(DeviceScene& s, int W, int H, int aa, Region rg, float4* out, cudaStream_t st) {
    return launch_plain(s, W, H, aa, rg, out, st, false);
}
void wave_release(DeviceScene&) {}
cudaError_t launch_primary_hits_bvh4(const DeviceScene& s, int W, int H, int ns, int* obj, int* mat, float* t,
                                     cudaStream_t stream) {
    return launch_primary_hits_plain(s, W, H, ns, obj, mat, t, stream);
}
}
