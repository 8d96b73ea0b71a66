// Deflate chunk compressor (host, system zlib) and a block-type scanner.
//
// CODAG's chunk compressor (deflate_compressor.py:44-125) calls zlib.compress(chunk, level),
// i.e. compress2 -> deflateInit2(level, Z_DEFLATED, 15, 8, Z_DEFAULT_STRATEGY), and stores
// the zlib-wrapped (RFC 1950) stream.  deflate_encode_chunk makes the same call, so with the
// same zlib and level the bytes are identical.  CODAG's decoder silently skips stored
// blocks (include/zlib/zlib.h:840-842); deflate_block_types lets the generators prove that a
// file contains none before it is handed to that decoder.
#include <zlib.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "host_common.hpp"

namespace codag_host {

int deflate_encode_chunk(const uint8_t* chunk, uint64_t chunk_bytes, int level, int wrapper,
                         int strategy, std::vector<uint8_t>& out, uint32_t* types) {
  z_stream zs;
  std::memset(&zs, 0, sizeof(zs));
  if (deflateInit2(&zs, level, Z_DEFLATED, wrapper ? 15 : -15, 8, strategy) != Z_OK)
    return CODAG_EINVAL;
  const uint64_t bound = deflateBound(&zs, static_cast<uLong>(chunk_bytes));
  const size_t base = out.size();
  out.resize(base + bound);
  zs.next_in = const_cast<Bytef*>(chunk);
  zs.avail_in = static_cast<uInt>(chunk_bytes);
  zs.next_out = out.data() + base;
  zs.avail_out = static_cast<uInt>(bound);
  const int rc = deflate(&zs, Z_FINISH);
  const uint64_t produced = zs.total_out;
  deflateEnd(&zs);
  if (rc != Z_STREAM_END) {
    out.resize(base);
    return CODAG_EINVAL;
  }
  out.resize(base + produced);
  if (types) *types = deflate_block_types(out.data() + base, produced, wrapper ? 2 : 0);
  return CODAG_OK;
}

// Walks the block boundaries with inflate(Z_BLOCK) and reads each block's 3 header bits.
// Returns a bitmask: 1 stored, 2 fixed, 4 dynamic, 0x80000000 when the stream is invalid.
uint32_t deflate_block_types(const uint8_t* stream, uint64_t len, int header_bytes) {
  if (static_cast<uint64_t>(header_bytes) > len) return 0x80000000u;
  const uint8_t* raw = stream + header_bytes;
  const uint64_t raw_len = len - header_bytes;
  z_stream zs;
  std::memset(&zs, 0, sizeof(zs));
  if (inflateInit2(&zs, -15) != Z_OK) return 0x80000000u;
  std::vector<uint8_t> sink(1 << 16);
  zs.next_in = const_cast<Bytef*>(raw);
  zs.avail_in = static_cast<uInt>(raw_len);
  uint32_t seen = 0;
  // bit position of the next block header, counted from raw[0]
  uint64_t header_bit = 0;
  for (;;) {
    // read BTYPE of the block starting at header_bit
    const uint64_t byte = header_bit >> 3;
    const unsigned shift = header_bit & 7;
    if (byte >= raw_len) { seen |= 0x80000000u; break; }
    unsigned bits = raw[byte] >> shift;
    if (shift > 5 && byte + 1 < raw_len) bits |= static_cast<unsigned>(raw[byte + 1]) << (8 - shift);
    const unsigned btype = (bits >> 1) & 3;
    seen |= btype == 0 ? 1u : btype == 1 ? 2u : btype == 2 ? 4u : 0x80000000u;
    if (btype == 3) break;
    // inflate to the end of this block
    int rc;
    do {
      zs.next_out = sink.data();
      zs.avail_out = static_cast<uInt>(sink.size());
      rc = inflate(&zs, Z_BLOCK);
    } while (rc == Z_OK && !(zs.data_type & 128) && zs.avail_out == 0);
    if (rc == Z_STREAM_END) break;
    if (rc != Z_OK || !(zs.data_type & 128)) { seen |= 0x80000000u; break; }
    if (zs.data_type & 64) break;  // the block that just ended was the final one
    const uint64_t consumed = raw_len - zs.avail_in;
    header_bit = consumed * 8 - (zs.data_type & 7);
  }
  inflateEnd(&zs);
  return seen;
}

}  // namespace codag_host
