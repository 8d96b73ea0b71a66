// ORC RLE v2 chunk encoder (host, unsigned values): the shared writer of ../rle_writers.h over
// a growing byte vector.  The layout (include/rlev2/encoder_trans.h:482-564) is written by
// capi_host.cpp.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../rle_writers.h"
#include "host_common.hpp"

namespace codag_host {

int rlev2_encode_chunk(const uint8_t* chunk, uint64_t chunk_bytes, int elem_bytes,
                       std::vector<uint8_t>& out) {
  if (!(elem_bytes == 1 || elem_bytes == 2 || elem_bytes == 4 || elem_bytes == 8) ||
      chunk_bytes % elem_bytes)
    return CODAG_EINVAL;
  const uint64_t n = chunk_bytes / elem_bytes;
  VectorSink sink{out};
  codag_fmt::RleV2Writer<VectorSink> w(sink);
  w.encode([&](uint64_t i) {
    uint64_t v = 0;
    std::memcpy(&v, chunk + i * elem_bytes, elem_bytes);  // little-endian zero extension
    return v;
  }, n);
  return CODAG_OK;
}

}  // namespace codag_host
