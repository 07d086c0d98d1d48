// api.cu -- the C-ABI of libsheen_c_api.so (include/sheen_c_api.h).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <set>
#include <vector>

#include "engine.h"

namespace sheen {
void release_all_servers();
}

namespace {

std::mutex g_mu;
std::set<sheen::DeviceScene*> g_scenes;

int fail_cuda(cudaError_t e) {
    sheen::set_error(cudaGetErrorString(e));
    return -1;
}

// Parameter rules of sheen_render_scene (api/sheen_c_api.cu:189-193).
int check_params(const SheenScene* s, int w, int h, int aa) {
    if (!s) { sheen::set_error("null scene"); return -1; }
    if (w <= 0 || h <= 0 || aa < 1 || aa > 64) { sheen::set_error("bad render params"); return -1; }
    if (!s->num_materials) { sheen::set_error("no materials"); return -1; }
    return 0;
}

void fill_stats(const sheen::DeviceScene& s, const unsigned long long* t, double render_ms, SheenRenderStats* st) {
    if (!st) return;
    std::memset(st, 0, sizeof(*st));
    if (t) {
        st->primary_rays = t[0];
        st->shadow_rays = t[1];
        st->secondary_rays = t[2];
        st->node_visits = t[3];
        st->prim_tests = t[4];
        st->shadow_node_visits = t[5];
        st->shadow_prim_tests = t[6];
        st->total_rays = t[0] + t[1] + t[2];
    }
    st->build_ms = s.build_ms;
    st->upload_ms = s.upload_ms;
    st->photon_ms = s.photon_ms;
    st->render_ms = render_ms;
    st->device_bytes = s.arena_bytes + s.extra_bytes;
    st->upload_bytes = s.arena_bytes;
}

// Launch one frame of `s` into device buffer `out`; optionally count rays
// and time it with events on `stream`.
int render_device(sheen::DeviceScene& s, int W, int H, int aa, sheen::Region rg, float4* out, cudaStream_t stream,
                  int flags, SheenRenderStats* stats) {
    if (rg.x0 < 0 || rg.y0 < 0 || rg.x1 > W || rg.y1 > H || rg.x0 >= rg.x1 || rg.y0 >= rg.y1) {
        sheen::set_error("bad render region");
        return -1;
    }
    const bool want_stats = stats != nullptr || (flags & (SHEEN_RENDER_COUNT_RAYS | SHEEN_RENDER_COUNT_NODES));
    cudaError_t e;
    if (want_stats) {
        e = cudaMemsetAsync(s.d_tally, 0, 8 * sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return fail_cuda(e);
    }
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (want_stats) {
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, stream);
    }
    if (s.form == SHEEN_FORM_PLAIN)
        e = sheen::launch_plain(s, W, H, aa, rg, out, stream, (flags & SHEEN_RENDER_COUNT_NODES) != 0);
    else
        e = sheen::launch_wavefront(s, W, H, aa, rg, out, stream, (flags & SHEEN_RENDER_COUNT_NODES) != 0);
    if (e != cudaSuccess) return fail_cuda(e);
    if (want_stats) {
        cudaEventRecord(ev1, stream);
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return fail_cuda(e);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        unsigned long long t[8] = {0};
        e = cudaMemcpy(t, s.d_tally, sizeof(t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return fail_cuda(e);
        fill_stats(s, t, ms, stats);
    }
    return 0;
}

}  // namespace

extern "C" {

int sheen_init(int device_id, int cuda_arch) {
    (void)cuda_arch;
    cudaError_t e = cudaSetDevice(device_id);
    if (e != cudaSuccess) return fail_cuda(e);
    e = cudaFree(0);
    if (e != cudaSuccess) return fail_cuda(e);
    e = sheen::prewarm_device(sheen::tuning().prewarm_mb);
    if (e != cudaSuccess) return fail_cuda(e);
    return 0;
}

void sheen_cleanup(void) {
    sheen::release_all_servers();
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (auto* s : g_scenes) sheen::scene_release(s);
        g_scenes.clear();
    }
    cudaDeviceSynchronize();
    sheen::release_parked_waves();
    sheen::release_upload_rings();
    sheen::release_build_streams();
    sheen::release_noalloc_scratch();
    sheen::release_srgb_tables();
    sheen::release_pools();
    cudaDeviceReset();
}

int sheen_scene_create(const SheenScene* scene, int form, SheenDeviceScene* out) {
    return sheen_scene_create_ext(scene, nullptr, form, out);
}

int sheen_scene_create_ext(const SheenScene* scene, const SheenSceneExt* ext, int form, SheenDeviceScene* out) {
    if (!out) { sheen::set_error("null output handle"); return -1; }
    *out = nullptr;
    if (!scene) { sheen::set_error("null scene"); return -1; }
    if (!scene->num_materials) { sheen::set_error("no materials"); return -1; }
    sheen::DeviceScene* s = nullptr;
    if (sheen::scene_upload_ext(scene, ext, form, &s) != 0) return -1;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_scenes.insert(s);
    }
    *out = reinterpret_cast<SheenDeviceScene>(s);
    return 0;
}

void sheen_scene_destroy(SheenDeviceScene h) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scenes.erase(s)) return;
    }
    cudaDeviceSynchronize();
    sheen::scene_release(s);
}

unsigned long long sheen_scene_device_bytes(SheenDeviceScene h) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    return s ? (unsigned long long)(s->arena_bytes + s->extra_bytes) : 0ull;
}

int sheen_scene_form(SheenDeviceScene h) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    return s ? s->form : -1;
}

int sheen_scene_frame_path(SheenDeviceScene h, int W, int H, int aa) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    if (!s) { sheen::set_error("null scene handle"); return -1; }
    if (W <= 0 || H <= 0 || aa < 1 || aa > 64) { sheen::set_error("bad render params"); return -1; }
    return sheen::frame_path(*s, W, H, aa);
}

int sheen_scene_render_device(SheenDeviceScene h, int W, int H, int aa, float* out, void* stream, int flags,
                              SheenRenderStats* stats) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    if (!s) { sheen::set_error("null scene handle"); return -1; }
    if (W <= 0 || H <= 0 || aa < 1 || aa > 64 || !out) { sheen::set_error("bad render params"); return -1; }
    return render_device(*s, W, H, aa, sheen::Region{0, 0, W, H}, reinterpret_cast<float4*>(out),
                         (cudaStream_t)stream, flags, stats);
}

int sheen_scene_render_region(SheenDeviceScene h, int W, int H, int aa, int x0, int y0, int x1, int y1, float* out,
                              void* stream, int flags, SheenRenderStats* stats) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    if (!s) { sheen::set_error("null scene handle"); return -1; }
    if (W <= 0 || H <= 0 || aa < 1 || aa > 64 || !out) { sheen::set_error("bad render params"); return -1; }
    return render_device(*s, W, H, aa, sheen::Region{x0, y0, x1, y1}, reinterpret_cast<float4*>(out),
                         (cudaStream_t)stream, flags, stats);
}

int sheen_scene_render_host(SheenDeviceScene h, int W, int H, int aa, float* out_host, int flags,
                            SheenRenderStats* stats) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    if (!s) { sheen::set_error("null scene handle"); return -1; }
    if (W <= 0 || H <= 0 || aa < 1 || aa > 64 || !out_host) { sheen::set_error("bad render params"); return -1; }
    float4* d = nullptr;
    cudaError_t e = sheen::dmalloc(&d, (size_t)W * H * sizeof(float4));
    if (e != cudaSuccess) return fail_cuda(e);
    int rc = render_device(*s, W, H, aa, sheen::Region{0, 0, W, H}, d, 0, flags, stats);
    if (rc == 0) {
        // a pinned destination takes the copy directly; a pageable one of
        // more than a few MB goes through the pinned ring
        const size_t bytes = (size_t)W * H * sizeof(float4);
        cudaPointerAttributes pa{};
        const bool pinned = cudaPointerGetAttributes(&pa, out_host) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (pinned || bytes < ((size_t)8 << 20)) {
            e = cudaMemcpy(out_host, d, bytes, cudaMemcpyDeviceToHost);
        } else {
            e = cudaStreamSynchronize(0);
            if (e == cudaSuccess) e = sheen::download_to_host(out_host, d, bytes);
        }
        if (e != cudaSuccess) rc = fail_cuda(e);
    }
    sheen::dfree(d);
    return rc;
}

int sheen_render_batch(const SheenBatchJob* jobs, int num_jobs, void* stream, SheenRenderStats* stats) {
    if (num_jobs < 0 || (num_jobs > 0 && !jobs)) { sheen::set_error("bad job list"); return -1; }
    const cudaStream_t st = (cudaStream_t)stream;
    std::vector<sheen::BatchItem> batch;
    std::vector<std::pair<sheen::DeviceScene*, int>> single;   // (scene, job index)
    for (int j = 0; j < num_jobs; j++) {
        const SheenBatchJob& b = jobs[j];
        auto* s = reinterpret_cast<sheen::DeviceScene*>(b.scene);
        if (!s) { sheen::set_error("null scene handle in batch"); return -1; }
        if (b.width <= 0 || b.height <= 0 || b.aa_samples < 1 || b.aa_samples > 64 || !b.out_rgba_device) {
            sheen::set_error("bad render params in batch");
            return -1;
        }
        sheen::Region rg{b.x0, b.y0, b.x1, b.y1};
        if (rg.x1 <= rg.x0 || rg.y1 <= rg.y0) rg = sheen::Region{0, 0, b.width, b.height};
        if (rg.x0 < 0 || rg.y0 < 0 || rg.x1 > b.width || rg.y1 > b.height) {
            sheen::set_error("bad render region in batch");
            return -1;
        }
        if (s->form == SHEEN_FORM_WAVEFRONT && sheen::wave_pipeline_used(*s))
            batch.push_back({s, b.width, b.height, b.aa_samples, rg, reinterpret_cast<float4*>(b.out_rgba_device)});
        else
            single.push_back({s, j});
    }
    unsigned long long* d_tally = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaError_t e = cudaSuccess;
    if (stats) {
        e = sheen::dmalloc(&d_tally, 8 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemsetAsync(d_tally, 0, 8 * sizeof(unsigned long long), st);
        if (e == cudaSuccess) e = cudaEventCreate(&ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&ev1);
        if (e == cudaSuccess) e = cudaEventRecord(ev0, st);
    }
    for (size_t k = 0; k < single.size() && e == cudaSuccess; k++) {
        const SheenBatchJob& b = jobs[single[k].second];
        sheen::DeviceScene& s = *single[k].first;
        sheen::Region rg{b.x0, b.y0, b.x1, b.y1};
        if (rg.x1 <= rg.x0 || rg.y1 <= rg.y0) rg = sheen::Region{0, 0, b.width, b.height};
        float4* out = reinterpret_cast<float4*>(b.out_rgba_device);
        if (s.form == SHEEN_FORM_PLAIN)
            e = sheen::launch_plain(s, b.width, b.height, b.aa_samples, rg, out, st, false, d_tally);
        else
            e = sheen::launch_mega_bvh4(s, b.width, b.height, b.aa_samples, rg, out, st, false, d_tally);
    }
    if (e == cudaSuccess) e = sheen::launch_wavefront_batch(batch, st, d_tally);
    if (e == cudaSuccess && stats) {
        e = cudaEventRecord(ev1, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        unsigned long long t[8] = {0};
        if (e == cudaSuccess) e = cudaMemcpy(t, d_tally, sizeof(t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            std::memset(stats, 0, sizeof(*stats));
            stats->primary_rays = t[0];
            stats->shadow_rays = t[1];
            stats->secondary_rays = t[2];
            stats->total_rays = t[0] + t[1] + t[2];
            stats->render_ms = ms;
        }
    }
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (d_tally) sheen::dfree(d_tally);
    if (e != cudaSuccess) return fail_cuda(e);
    return 0;
}

int sheen_scene_profile_stages(SheenDeviceScene h, int W, int H, int aa, float* out_device, void* stream,
                               SheenStageProfile* prof) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    if (!s || !prof) { sheen::set_error("null scene handle or profile"); return -1; }
    if (W <= 0 || H <= 0 || aa < 1 || aa > 64 || !out_device) { sheen::set_error("bad render params"); return -1; }
    if (s->form != SHEEN_FORM_WAVEFRONT) { sheen::set_error("stage profiles apply to SHEEN_FORM_WAVEFRONT scenes"); return -1; }
    std::memset(prof, 0, sizeof(*prof));
    const cudaError_t e = sheen::profile_wavefront(*s, W, H, aa, reinterpret_cast<float4*>(out_device),
                                                   (cudaStream_t)stream, prof);
    if (e == cudaErrorNotSupported) {
        sheen::set_error("this scene's frames run on the megakernel: no queue stages");
        return -1;
    }
    if (e != cudaSuccess) return fail_cuda(e);
    return 0;
}

int sheen_scene_trace(SheenDeviceScene h, const float* rays_host, int n, int* obj, int* mat, float* t) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    if (!s) { sheen::set_error("null scene handle"); return -1; }
    if (n < 0 || (n > 0 && (!rays_host || !obj || !mat || !t))) { sheen::set_error("bad ray query"); return -1; }
    if (n == 0) return 0;
    float4* drays = nullptr;
    int *dobj = nullptr, *dmat = nullptr;
    float* dt = nullptr;
    const size_t N = (size_t)n;
    cudaError_t e = sheen::dmalloc(&drays, N * 2 * sizeof(float4));
    if (e == cudaSuccess) e = sheen::dmalloc(&dobj, N * sizeof(int));
    if (e == cudaSuccess) e = sheen::dmalloc(&dmat, N * sizeof(int));
    if (e == cudaSuccess) e = sheen::dmalloc(&dt, N * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(drays, rays_host, N * 2 * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = sheen::launch_trace_rays(*s, drays, n, dobj, dmat, dt, 0);
    if (e == cudaSuccess) e = cudaMemcpy(obj, dobj, N * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(mat, dmat, N * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(t, dt, N * sizeof(float), cudaMemcpyDeviceToHost);
    sheen::dfree(drays);
    sheen::dfree(dobj);
    sheen::dfree(dmat);
    sheen::dfree(dt);
    if (e != cudaSuccess) return fail_cuda(e);
    return 0;
}

int sheen_scene_primary_hits(SheenDeviceScene h, int W, int H, int aa, int* obj, int* mat, float* t) {
    auto* s = reinterpret_cast<sheen::DeviceScene*>(h);
    if (!s) { sheen::set_error("null scene handle"); return -1; }
    if (W <= 0 || H <= 0 || !obj || !mat || !t) { sheen::set_error("bad render params"); return -1; }
    const int ns = aa < 1 ? 1 : (aa > 64 ? 64 : aa);
    const size_t n = (size_t)W * H * ns;
    int *dobj = nullptr, *dmat = nullptr;
    float* dt = nullptr;
    cudaError_t e = sheen::dmalloc(&dobj, n * sizeof(int));
    if (e == cudaSuccess) e = sheen::dmalloc(&dmat, n * sizeof(int));
    if (e == cudaSuccess) e = sheen::dmalloc(&dt, n * sizeof(float));
    if (e == cudaSuccess)
        e = s->form == SHEEN_FORM_PLAIN ? sheen::launch_primary_hits_plain(*s, W, H, ns, dobj, dmat, dt, 0)
                                        : sheen::launch_primary_hits_bvh4(*s, W, H, ns, dobj, dmat, dt, 0);
    if (e == cudaSuccess) e = cudaMemcpy(obj, dobj, n * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(mat, dmat, n * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(t, dt, n * sizeof(float), cudaMemcpyDeviceToHost);
    sheen::dfree(dobj);
    sheen::dfree(dmat);
    sheen::dfree(dt);
    return e == cudaSuccess ? 0 : fail_cuda(e);
}

int sheen_render_scene_rgba(const SheenScene* scene, int W, int H, int aa, int form, float* out_host,
                            SheenRenderStats* stats) {
    if (check_params(scene, W, H, aa) != 0) return -1;
    if (!out_host) { sheen::set_error("null output buffer"); return -1; }
    sheen::DeviceScene* s = nullptr;
    if (sheen::scene_upload(scene, form, &s) != 0) return -1;
    int rc = sheen_scene_render_host(reinterpret_cast<SheenDeviceScene>(s), W, H, aa, out_host, 0, stats);
    sheen::scene_release(s);
    return rc;
}

// The drop-in call: plain form, 8-bit sRGB PNG.  The image is converted on
// the device (the host conversion's exact bytes) and read back as PNG rows,
// 3 bytes a pixel instead of the float4 image.
int sheen_render_scene(const SheenScene* scene, int W, int H, int aa, const char* path) {
    if (check_params(scene, W, H, aa) != 0) return -1;
    if (!path) { sheen::set_error("bad render params"); return -1; }
    sheen::DeviceScene* s = nullptr;
    if (sheen::scene_upload(scene, SHEEN_FORM_PLAIN, &s) != 0) return -1;
    float4* img = nullptr;
    unsigned char* rows = nullptr;
    const size_t row_bytes = (size_t)H * (1 + 3 * (size_t)W);
    std::vector<unsigned char> host_rows(row_bytes);
    cudaError_t e = sheen::dmalloc(&img, (size_t)W * H * sizeof(float4));
    if (e == cudaSuccess) e = sheen::dmalloc(&rows, row_bytes);
    int rc = e == cudaSuccess ? 0 : fail_cuda(e);
    if (rc == 0) rc = render_device(*s, W, H, aa, sheen::Region{0, 0, W, H}, img, 0, 0, nullptr);
    if (rc == 0) {
        e = sheen::pack_srgb_rows(img, W, H, rows, 0);
        if (e == cudaSuccess) e = cudaMemcpy(host_rows.data(), rows, row_bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail_cuda(e);
    }
    sheen::dfree(img);
    sheen::dfree(rows);
    sheen::scene_release(s);
    if (rc != 0) return rc;
    return sheen::write_png_rows(path, host_rows.data(), W, H);
}

}  // extern "C"
