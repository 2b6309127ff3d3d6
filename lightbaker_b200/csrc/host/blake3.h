// BLAKE3 (O'Connor, Aumasson, Neves, Wilcox-O'Hearn, 2020), the hash the reference keys its cache
// with (blake3 1.8 in its Cargo.lock): 32-byte digests, incremental. Written from the published
// specification; portable, one block at a time.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

namespace lb {

class Blake3 {
  public:
    Blake3();
    void update(const void *data, size_t len);
    void finalize(uint8_t out[32]) const;
    std::string hex() const;

  private:
    uint32_t cv_[8];
    uint8_t block_[64];
    size_t block_len_ = 0;
    uint64_t chunk_counter_ = 0;
    size_t blocks_compressed_ = 0;
    uint32_t stack_[54][8];
    size_t stack_len_ = 0;
    void compress_chunk_block(bool last, uint32_t out_cv[8]);
    void push_chunk_cv(const uint32_t cv[8], uint64_t total_chunks);
};

void blake3_hash(const void *data, size_t len, uint8_t out[32]);
std::string to_hex(const uint8_t *h, size_t n);

}  // namespace lb
