// png.cpp -- 8-bit sRGB PNG output of sheen_render_scene.
//
// Conversion per channel as png_color.h:11-20 (clamp, sRGB curve, +0.5,
// truncate); the file is a plain RGB8 PNG (IHDR, one zlib IDAT, IEND) with
// filter 0 rows.  The conversion is a non-decreasing step function of the
// linear value, so it is also given as the 255 thresholds at which the byte
// steps up (srgb_thresholds): the device packs pixels by searching them
// (png_pack.cu), which yields exactly the bytes of this host conversion
// without evaluating pow on the device.
#include <zlib.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "sheen_c_api.h"

namespace sheen {
void set_error(const char* msg);

static unsigned char srgb_byte(float c) {
    float e;
    if (!(c > 0.0f)) e = 0.0f;
    else {
        if (c > 1.0f) c = 1.0f;
        e = (c <= 0.0031308f) ? c * 12.92f : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f;
    }
    float v = e * 255.0f + 0.5f;
    return (unsigned char)(v > 255.0f ? 255.0f : v);
}

// thr[b - 1] = the smallest non-negative float whose byte is >= b, for
// b = 1..255 (found by bisection over the ordered bit patterns of [0, 1]).
const float* srgb_thresholds() {
    static float thr[255];
    static bool ready = [] {
        for (int b = 1; b <= 255; b++) {
            uint32_t lo = 0, hi = 0x3f800000u;   // srgb_byte(1.0f) == 255 >= b
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo) / 2;
                float f;
                std::memcpy(&f, &mid, 4);
                if (srgb_byte(f) >= b) hi = mid;
                else lo = mid + 1;
            }
            std::memcpy(&thr[b - 1], &lo, 4);
        }
        return true;
    }();
    (void)ready;
    return thr;
}

static void put32(std::vector<unsigned char>& b, uint32_t v) {
    b.push_back((unsigned char)(v >> 24)); b.push_back((unsigned char)(v >> 16));
    b.push_back((unsigned char)(v >> 8)); b.push_back((unsigned char)v);
}

static void chunk(std::vector<unsigned char>& out, const char* tag, const unsigned char* data, size_t n) {
    put32(out, (uint32_t)n);
    size_t start = out.size();
    out.insert(out.end(), tag, tag + 4);
    if (n) out.insert(out.end(), data, data + n);
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, out.data() + start, (uInt)(out.size() - start));
    put32(out, (uint32_t)crc);
}

// Writes a PNG from raw filter-0 rows (h rows of 1 + 3w bytes).
int write_png_rows(const char* path, const unsigned char* rows, int w, int h) {
    std::vector<unsigned char> raw(rows, rows + (size_t)h * (1 + (size_t)w * 3));
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<unsigned char> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) { set_error("png deflate failed"); return -1; }
    std::vector<unsigned char> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    unsigned char ihdr[13];
    ihdr[0] = (unsigned char)(w >> 24); ihdr[1] = (unsigned char)(w >> 16); ihdr[2] = (unsigned char)(w >> 8); ihdr[3] = (unsigned char)w;
    ihdr[4] = (unsigned char)(h >> 24); ihdr[5] = (unsigned char)(h >> 16); ihdr[6] = (unsigned char)(h >> 8); ihdr[7] = (unsigned char)h;
    ihdr[8] = 8; ihdr[9] = 2; ihdr[10] = 0; ihdr[11] = 0; ihdr[12] = 0;
    chunk(out, "IHDR", ihdr, 13);
    chunk(out, "IDAT", z.data(), zlen);
    chunk(out, "IEND", nullptr, 0);
    FILE* f = std::fopen(path, "wb");
    if (!f) { set_error("stbi_write_png failed"); return -1; }
    size_t wr = std::fwrite(out.data(), 1, out.size(), f);
    std::fclose(f);
    if (wr != out.size()) { set_error("stbi_write_png failed"); return -1; }
    return 0;
}

}  // namespace sheen

extern "C" void sheen_srgb_thresholds(float* out) {
    if (!out) return;
    const float* t = sheen::srgb_thresholds();
    for (int i = 0; i < 255; i++) out[i] = t[i];
}

extern "C" int sheen_write_png_srgb(const char* path, const float* rgba, int w, int h) {
    using namespace sheen;
    if (!path || !rgba || w <= 0 || h <= 0) { set_error("bad png params"); return -1; }
    std::vector<unsigned char> raw((size_t)h * (1 + (size_t)w * 3));
    for (int y = 0; y < h; y++) {
        unsigned char* row = raw.data() + (size_t)y * (1 + (size_t)w * 3);
        row[0] = 0;
        for (int x = 0; x < w; x++)
            for (int c = 0; c < 3; c++) row[1 + 3 * x + c] = srgb_byte(rgba[4 * ((size_t)y * w + x) + c]);
    }
    return write_png_rows(path, raw.data(), w, h);
}
