// photon.cu -- photon pass on the device: emission/tracing, then the hash
// grid, with no host round trip.
//
// Emission restates photon_kernel (render_kernel.cu:820-926): seed
// 0x5eed1234, spot/area/point emitters (sun lights emit nothing), up to 4
// bounces through glass (transmission > 0.5, eta = 1/ior on every face) and
// mirrors (reflect > 0.5), the first diffuse hit is stored.
//
// The reference appends with atomicAdd (arbitrary order) and builds the grid
// with a count kernel, a host prefix sum over 2^18 cells with two 1 MB
// copies, and an atomic scatter (render_kernel.cu:992-1045).  Here each
// emission index owns its slot, survivors are compacted in emission order
// (flag scan), capped at the C-API's 4M, and ordered by cell with a stable
// radix sort, so the photons inside a cell keep emission order: the gather's
// "first 128 found" is deterministic and run-to-run identical.
#include <cub/cub.cuh>

#include "dev/integrator.cuh"
#include "dev/trace_bvh4.cuh"
#include "engine.h"

namespace sheen {
namespace dev {

// T: the scene's query policy (the plain form's reference-order walks, or
// the wavefront form's BVH4s: same closest hits except exact ties).
template <class T>
__global__ void photon_emit_kernel(const __grid_constant__ DevScene S, int per_light, int total, float4* pos, float4* nrm, float4* flux,
                                   int* valid) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    valid[idx] = 0;
    const Light& l = S.lights[idx / per_light];
    if (l.type == 0) return;
    const uint32_t sd = hash32(0x5eed1234u + (uint32_t)idx * 2654435761u);
    const float u1 = rand01(sd), u2 = rand01(sd ^ 0x9e3779b9u), u3 = rand01(sd ^ 0x85ebca6bu);
    float3 p0 = f3(l.position), dir;
    if (l.type == 3) {
        const float ch = cosf(l.angle);
        const float ct = ch + (1.0f - ch) * u1;
        const float st = sqrtf(fmaxf(1.0f - ct * ct, 0.0f));
        const float phi = 6.2831853f * u2;
        const float3 ax = f3(l.direction);
        const float3 t1 = normalize(cross(ax, up_for(ax)));
        const float3 t2 = cross(ax, t1);
        dir = normalize(ax * ct + t1 * (cosf(phi) * st) + t2 * (sinf(phi) * st));
    } else if (l.type == 2) {
        p0 = f3(l.position) + f3(l.u_axis) * (u1 * 2.0f - 1.0f) + f3(l.v_axis) * (u2 * 2.0f - 1.0f);
        const float3 n = normalize(cross(f3(l.u_axis), f3(l.v_axis)));
        const float3 t1 = normalize(cross(n, up_for(n)));
        const float3 t2 = cross(n, t1);
        const float cz = sqrtf(fmaxf(1.0f - u3, 0.0f)), r = sqrtf(u3);
        const float phi = 6.2831853f * rand01(sd ^ 0xc2b2ae35u);
        dir = normalize(n * cz + t1 * (cosf(phi) * r) + t2 * (sinf(phi) * r));
    } else {
        const float cz = 2.0f * u1 - 1.0f;
        const float st = sqrtf(fmaxf(1.0f - cz * cz, 0.0f));
        const float phi = 6.2831853f * u2;
        dir = f3(st * cosf(phi), cz, st * sinf(phi));
    }
    float3 fl = f3(l.color) * (l.intensity / (float)per_light);
    Ray ray;
    ray.o = p0; ray.d = dir; ray.tmin = 0.001f; ray.tmax = 1.0e10f;
    Counters c;
    for (int b = 0; b < 4; b++) {
        Hit h;
        if (!T::closest(S, ray, h, c)) return;
        const Material& m = S.materials[h.mat];
        if (m.transmission > 0.5f) {
            const float3 n = h.n;
            const float eta = 1.0f / fmaxf(m.ior, 1.0f);
            const float cosi = fmaxf(-dot(ray.d, n), 1.0e-4f);
            const float k = 1.0f - eta * eta * (1.0f - cosi * cosi);
            const float3 td = k < 0.0f ? normalize(ray.d + 2.0f * cosi * n)
                                       : normalize(eta * ray.d + (eta * cosi - sqrtf(k)) * n);
            fl = fl * m.transmission;
            ray.o = h.p + td * 0.002f;
            ray.d = td;
            continue;
        }
        if (m.reflect > 0.5f) {
            const float3 rd = ray.d - h.n * (2.0f * dot(ray.d, h.n));
            ray.o = h.p + h.n * 0.002f;
            ray.d = normalize(rd);
            continue;
        }
        pos[idx] = make_float4(h.p.x, h.p.y, h.p.z, 0.0f);
        nrm[idx] = make_float4(h.n.x, h.n.y, h.n.z, 0.0f);
        flux[idx] = make_float4(fl.x, fl.y, fl.z, 0.0f);
        valid[idx] = 1;
        return;
    }
}

// Stream compaction in emission order, capped at `cap` survivors; also
// computes the hash cell of every survivor (render_kernel.cu:963-966).
__global__ void photon_compact_kernel(int total, const int* valid, const int* rank, int cap, float cell, int num_cells,
                                      const float4* pos, int* keys, int* src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total || !valid[i]) return;
    const int r = rank[i];
    if (r >= cap) return;
    const float4 p = pos[i];
    keys[r] = photon_cell((int)floorf(p.x / cell), (int)floorf(p.y / cell), (int)floorf(p.z / cell), num_cells);
    src[r] = i;
}

__global__ void photon_count_cells(int n, const int* keys, int* count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(&count[keys[i]], 1);
}

__global__ void photon_gather_sorted(int n, const int* order, const float4* pos, const float4* nrm, const float4* flux,
                                     float4* opos, float4* onrm, float4* oflux) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = order[i];
    opos[i] = pos[s];
    onrm[i] = nrm[s];
    oflux[i] = flux[s];
}

}  // namespace dev

int build_photon_map_device(DeviceScene& s, int per_light, float cell) {
    const long long total64 = (long long)per_light * s.view.num_lights;
    if (total64 <= 0) return 0;
    if (total64 > (1ll << 30)) { set_error("photon count too large"); return -1; }
    const int total = (int)total64;
    const int cap = 4000000;   // api/sheen_c_api.cu:276-278
    const int num_cells = 1 << 18;

    float4 *pos = nullptr, *nrm = nullptr, *flux = nullptr;
    int *valid = nullptr, *rank = nullptr, *keys = nullptr, *src = nullptr, *keys_sorted = nullptr, *order = nullptr;
    int* counter = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    cudaError_t e = cudaSuccess;
#define CK(x) do { e = (x); if (e != cudaSuccess) goto fail; } while (0)
    CK(dmalloc(&pos, (size_t)total * sizeof(float4)));
    CK(dmalloc(&nrm, (size_t)total * sizeof(float4)));
    CK(dmalloc(&flux, (size_t)total * sizeof(float4)));
    CK(dmalloc(&valid, (size_t)total * sizeof(int)));
    CK(dmalloc(&rank, (size_t)total * sizeof(int)));
    if (s.form == SHEEN_FORM_PLAIN)
        dev::photon_emit_kernel<dev::RefTracer<false>><<<(total + 127) / 128, 128>>>(s.view, per_light, total, pos, nrm,
                                                                                   flux, valid);
    else
        dev::photon_emit_kernel<dev::FastTracer<false>><<<(total + 127) / 128, 128>>>(s.view, per_light, total, pos,
                                                                                    nrm, flux, valid);
    CK(cudaGetLastError());
    {
        size_t b1 = 0, b2 = 0;
        CK(cub::DeviceScan::ExclusiveSum(nullptr, b1, valid, rank, total));
        CK(cub::DeviceRadixSort::SortPairs(nullptr, b2, keys, keys_sorted, src, order, cap, 0, 18));
        cub_bytes = b1 > b2 ? b1 : b2;
        CK(dmalloc(&cub_tmp, cub_bytes));
        CK(cub::DeviceScan::ExclusiveSum(cub_tmp, b1, valid, rank, total));
        int last_rank = 0, last_valid = 0;
        CK(cudaMemcpy(&last_rank, rank + total - 1, sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&last_valid, valid + total - 1, sizeof(int), cudaMemcpyDeviceToHost));
        int n = last_rank + last_valid;
        if (n > cap) n = cap;
        s.photons_stored = n;
        if (n == 0) goto done;
        CK(dmalloc(&keys, (size_t)n * sizeof(int)));
        CK(dmalloc(&src, (size_t)n * sizeof(int)));
        CK(dmalloc(&keys_sorted, (size_t)n * sizeof(int)));
        CK(dmalloc(&order, (size_t)n * sizeof(int)));
        dev::photon_compact_kernel<<<(total + 127) / 128, 128>>>(total, valid, rank, n, cell, num_cells, pos, keys, src);
        CK(cudaGetLastError());
        size_t b3 = cub_bytes;
        CK(cub::DeviceRadixSort::SortPairs(cub_tmp, b3, keys, keys_sorted, src, order, n, 0, 18));

        // Resident map: sorted photons + cell_count + cell_start.
        float4 *mpos = nullptr, *mnrm = nullptr, *mflux = nullptr;
        int *cstart = nullptr, *ccount = nullptr;
        CK(dmalloc(&mpos, (size_t)n * sizeof(float4)));
        s.extra.push_back(mpos);
        CK(dmalloc(&mnrm, (size_t)n * sizeof(float4)));
        s.extra.push_back(mnrm);
        CK(dmalloc(&mflux, (size_t)n * sizeof(float4)));
        s.extra.push_back(mflux);
        CK(dmalloc(&ccount, (size_t)num_cells * sizeof(int)));
        s.extra.push_back(ccount);
        CK(dmalloc(&cstart, (size_t)(num_cells + 1) * sizeof(int)));
        s.extra.push_back(cstart);
        s.extra_bytes = (size_t)n * 3 * sizeof(float4) + (size_t)(2 * num_cells + 1) * sizeof(int);
        CK(cudaMemset(ccount, 0, (size_t)num_cells * sizeof(int)));
        dev::photon_count_cells<<<(n + 127) / 128, 128>>>(n, keys, ccount);
        CK(cudaGetLastError());
        size_t b4 = 0;
        CK(cub::DeviceScan::ExclusiveSum(nullptr, b4, ccount, cstart, num_cells));
        if (b4 > cub_bytes) {
            dfree(cub_tmp);
            cub_tmp = nullptr;
            CK(dmalloc(&cub_tmp, b4));
            cub_bytes = b4;
        }
        CK(cub::DeviceScan::ExclusiveSum(cub_tmp, b4, ccount, cstart, num_cells));
        CK(cudaMemcpy(cstart + num_cells, &n, sizeof(int), cudaMemcpyHostToDevice));
        dev::photon_gather_sorted<<<(n + 127) / 128, 128>>>(n, order, pos, nrm, flux, mpos, mnrm, mflux);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        s.view.pmap.pos = mpos;
        s.view.pmap.nrm = mnrm;
        s.view.pmap.flux = mflux;
        s.view.pmap.cell_start = cstart;
        s.view.pmap.cell_count = ccount;
        s.view.pmap.num_cells = num_cells;
        s.view.pmap.cell_size = cell;
    }
done:
    dfree(pos); dfree(nrm); dfree(flux); dfree(valid); dfree(rank);
    dfree(keys); dfree(src); dfree(keys_sorted); dfree(order); dfree(cub_tmp); dfree(counter);
    return 0;
fail:
    set_error(cudaGetErrorString(e));
    dfree(pos); dfree(nrm); dfree(flux); dfree(valid); dfree(rank);
    dfree(keys); dfree(src); dfree(keys_sorted); dfree(order); dfree(cub_tmp); dfree(counter);
    return -1;
#undef CK
}

}  // namespace sheen
