// Result encoders: PFM (Photon's save_pfm format, src/scene/image.cpp:88-96) and PNG (RGBA8, as
// Photon's save_png writes the display buffer, image.cpp:84-86), to memory or to a file. These are the
// wire formats of rendered results; they run on the host over images already downloaded.
#include <zlib.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "image_io.h"
#include "photon_wavefront.h"

namespace {

void put_u32be(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back(uint8_t(x >> 24));
    v.push_back(uint8_t(x >> 16));
    v.push_back(uint8_t(x >> 8));
    v.push_back(uint8_t(x));
}

void put_chunk(std::vector<uint8_t>& out, const char type[4], const uint8_t* data, size_t n) {
    put_u32be(out, uint32_t(n));
    size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    if (n) out.insert(out.end(), data, data + n);
    uLong crc = crc32(0L, out.data() + start, uInt(4 + n));
    put_u32be(out, uint32_t(crc));
}

}  // namespace

namespace ptw {

// PFM: "PF\n<w> <h>\n-1.0\n" then float rgb rows, bottom row first, little endian.
std::vector<uint8_t> encode_pfm(const float* rgb, int w, int h) {
    char head[64];
    int hn = std::snprintf(head, sizeof(head), "PF\n%d %d\n-1.0\n", w, h);
    std::vector<uint8_t> out(size_t(hn) + size_t(w) * size_t(h) * 12);
    std::memcpy(out.data(), head, size_t(hn));
    uint8_t* p = out.data() + hn;
    const size_t row = size_t(w) * 12;
    for (int y = h - 1; y >= 0; y--, p += row) std::memcpy(p, reinterpret_cast<const uint8_t*>(rgb) + size_t(y) * row, row);
    return out;
}

// PNG, 8-bit RGBA, top row first; each pixel's bytes in memory order (R, G, B, A) of the uint32.
bool encode_png(const uint32_t* rgba, int w, int h, int level, std::vector<uint8_t>& out) {
    const size_t stride = size_t(w) * 4;
    std::vector<uint8_t> raw((stride + 1) * size_t(h));
    for (int y = 0; y < h; y++) {
        raw[size_t(y) * (stride + 1)] = 0;  // filter: none
        std::memcpy(raw.data() + size_t(y) * (stride + 1) + 1, reinterpret_cast<const uint8_t*>(rgba) + size_t(y) * stride, stride);
    }
    uLongf zn = compressBound(uLong(raw.size()));
    std::vector<uint8_t> z(zn);
    if (compress2(z.data(), &zn, raw.data(), uLong(raw.size()), level) != Z_OK) return false;
    out.clear();
    const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    out.insert(out.end(), sig, sig + 8);
    std::vector<uint8_t> ihdr;
    put_u32be(ihdr, uint32_t(w));
    put_u32be(ihdr, uint32_t(h));
    ihdr.push_back(8);  // bit depth
    ihdr.push_back(6);  // colour type: RGBA
    ihdr.push_back(0);  // compression
    ihdr.push_back(0);  // filter method
    ihdr.push_back(0);  // no interlace
    put_chunk(out, "IHDR", ihdr.data(), ihdr.size());
    put_chunk(out, "IDAT", z.data(), size_t(zn));
    put_chunk(out, "IEND", nullptr, 0);
    return true;
}

}  // namespace ptw

namespace {

int32_t copy_out(const std::vector<uint8_t>& v, uint8_t* out, size_t cap, size_t* len) {
    if (len) *len = v.size();
    if (!out) return PT_OK;  // size query
    if (cap < v.size()) return PT_ERR_INVALID;
    std::memcpy(out, v.data(), v.size());
    return PT_OK;
}

int32_t write_file(const char* path, const std::vector<uint8_t>& v) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return PT_ERR_INVALID;
    size_t n = std::fwrite(v.data(), 1, v.size(), f);
    int rc = std::fclose(f);
    return (n == v.size() && rc == 0) ? PT_OK : PT_ERR_INVALID;
}

}  // namespace

using ptw::encode_pfm;
using ptw::encode_png;

extern "C" {

int32_t pt_encode_pfm(const float* rgb, int32_t width, int32_t height, uint8_t* out, size_t capacity, size_t* length) {
    if (!rgb || width <= 0 || height <= 0) return PT_ERR_INVALID;
    return copy_out(encode_pfm(rgb, width, height), out, capacity, length);
}

int32_t pt_encode_png(const uint32_t* rgba, int32_t width, int32_t height, int32_t level, uint8_t* out, size_t capacity, size_t* length) {
    if (!rgba || width <= 0 || height <= 0 || level < 0 || level > 9) return PT_ERR_INVALID;
    std::vector<uint8_t> v;
    if (!encode_png(rgba, width, height, level, v)) return PT_ERR_ALLOC;
    return copy_out(v, out, capacity, length);
}

int32_t pt_write_pfm(const char* path, int32_t width, int32_t height, const float* rgb) {
    if (!path || !rgb || width <= 0 || height <= 0) return PT_ERR_INVALID;
    return write_file(path, encode_pfm(rgb, width, height));
}

int32_t pt_write_png(const char* path, int32_t width, int32_t height, const uint32_t* rgba) {
    if (!path || !rgba || width <= 0 || height <= 0) return PT_ERR_INVALID;
    std::vector<uint8_t> v;
    if (!encode_png(rgba, width, height, 6, v)) return PT_ERR_ALLOC;
    return write_file(path, v);
}

}  // extern "C"
