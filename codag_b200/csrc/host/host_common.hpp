// Shared declarations of the host-side format producers (encoders, layout writers and
// synthetic column generators).  These run on the CPU; the decompressors are in ../kernels.
#pragma once
#include <cstdint>
#include <vector>

#include "../../../include/codag_format.h"

namespace codag_host {

// byte sink of the shared RLE writers (../rle_writers.h) over a growing vector
struct VectorSink {
  std::vector<uint8_t>& v;
  void put(uint8_t b) { v.push_back(b); }
  uint64_t size() const { return v.size(); }
  void set(uint64_t i, uint8_t b) { v[i] = b; }
};

// --- per-chunk encoders -------------------------------------------------------------
// Each appends one compressed stream for `chunk_bytes` bytes of input to `out`.
int rlev1_encode_chunk(const uint8_t* chunk, uint64_t chunk_bytes, int elem_bytes,
                       std::vector<uint8_t>& out);
int rlev2_encode_chunk(const uint8_t* chunk, uint64_t chunk_bytes, int elem_bytes,
                       std::vector<uint8_t>& out);
// zlib-wrapped (wrapper=1, RFC 1950) or raw (wrapper=0) Deflate of one chunk.
// `types` receives a bitmask of the block types in the stream (1 stored, 2 fixed, 4 dynamic).
int deflate_encode_chunk(const uint8_t* chunk, uint64_t chunk_bytes, int level, int wrapper,
                         int strategy, std::vector<uint8_t>& out, uint32_t* types);
uint32_t deflate_block_types(const uint8_t* stream, uint64_t len, int header_bytes);

// --- deterministic random numbers (splitmix64 seeding xoshiro256**) -------------------
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed);
  uint64_t next();
  uint64_t below(uint64_t n);                     // uniform in [0, n)
  int64_t range(int64_t lo, int64_t hi);           // uniform in [lo, hi]
  double uniform();                                // [0, 1)
};
uint64_t derive_seed(uint64_t base, uint64_t stream);

}  // namespace codag_host
