// What an engine samples, as it ships: crates/lightbaker/src/encode.rs. BC4/BC5 blocks, RGB9E5, and a
// one-level KTX2 container (zstd supercompressed) with its data format descriptor.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace lb {

enum Format { FORMAT_BC5, FORMAT_RGB9E5 };

std::array<uint8_t, 8> bc4_block(const uint8_t v[16]);                 // encode.rs:7-35
std::vector<uint8_t> bc5(const uint8_t *rg, size_t w, size_t h);       // :37-51 (rg interleaved)
uint32_t rgb9e5(const float c[3]);                                     // :53-70
void rgb9e5_decode(uint32_t p, float out[3]);                          // :72-75
std::vector<uint8_t> ktx2(Format f, uint32_t w, uint32_t h, const std::vector<uint8_t> &data);  // :100-126

}  // namespace lb
