// The result encoders (image_io.cpp), for the server's encoded fetch.
#pragma once

#include <cstdint>
#include <vector>

namespace ptw {

// PFM in the format of Photon's save_pfm (src/scene/image.cpp:88-96): float rgb, bottom row first.
std::vector<uint8_t> encode_pfm(const float* rgb, int w, int h);
// PNG, 8-bit RGBA (each uint32's bytes in memory order are R, G, B, A), zlib `level`; false if zlib fails.
bool encode_png(const uint32_t* rgba, int w, int h, int level, std::vector<uint8_t>& out);

}  // namespace ptw
