// ORC RLE v1 chunk encoder (host): the shared writer of ../rle_writers.h over a growing byte
// vector.  File layout (include/rlev1/rlev1.h:103-192) is written by capi_host.cpp:
//   n_chunks_pad = ceil(bytes / (chunk*32)) * 32, input zero padded to n_chunks_pad*chunk;
//   blob = [u64 original_bytes][stream_0 ...]; stream i starts at 8 + blk_off[i];
//   blk_off[0] = 0, blk_off[i+1] = blk_off[i] + round_up4(col_len[i]).
#include <cstdint>
#include <cstring>
#include <vector>

#include "../rle_writers.h"
#include "host_common.hpp"

namespace codag_host {
namespace {

template <typename T>
void encode_chunk_t(const uint8_t* chunk, uint64_t chunk_bytes, std::vector<uint8_t>& out) {
  const uint64_t n = chunk_bytes / sizeof(T);
  std::vector<T> vals(n);
  std::memcpy(vals.data(), chunk, n * sizeof(T));
  VectorSink sink{out};
  codag_fmt::RleV1Writer<T, VectorSink> w(sink);
  w.encode([&](uint64_t i) { return vals[i]; }, n);
}

}  // namespace

int rlev1_encode_chunk(const uint8_t* chunk, uint64_t chunk_bytes, int elem_bytes,
                       std::vector<uint8_t>& out) {
  if (chunk_bytes % elem_bytes || chunk_bytes / elem_bytes < 2) return CODAG_EINVAL;
  switch (elem_bytes) {
    case 1: encode_chunk_t<uint8_t>(chunk, chunk_bytes, out); break;
    case 2: encode_chunk_t<uint16_t>(chunk, chunk_bytes, out); break;
    case 4: encode_chunk_t<uint32_t>(chunk, chunk_bytes, out); break;
    case 8: encode_chunk_t<uint64_t>(chunk, chunk_bytes, out); break;
    default: return CODAG_EINVAL;
  }
  return CODAG_OK;
}

}  // namespace codag_host
