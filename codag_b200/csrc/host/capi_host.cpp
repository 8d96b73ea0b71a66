// extern "C" host entry points of the format producers: file-level layouts in CODAG's
// on-disk format, built from the per-chunk encoders (OpenMP over chunks).
#include <zlib.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../rle_writers.h"
#include "host_common.hpp"

using namespace codag_host;

namespace {

bool to_hbuf(const void* src, uint64_t bytes, codag_hbuf* dst) {
  dst->data = static_cast<uint8_t*>(std::malloc(bytes ? bytes : 1));
  dst->bytes = bytes;
  if (!dst->data) return false;
  if (bytes) std::memcpy(dst->data, src, bytes);
  return true;
}

inline uint64_t round_up(uint64_t v, uint64_t m) { return (v + m - 1) / m * m; }

bool valid_elem(int e) { return e == 1 || e == 2 || e == 4 || e == 8; }

// Encodes n_chunks chunks of `padded` with `enc`; returns per-chunk streams.
template <typename F>
int encode_chunks(const std::vector<uint8_t>& padded, uint64_t n_chunks, uint64_t chunk_bytes,
                  std::vector<std::vector<uint8_t>>& streams, F enc) {
  streams.assign(n_chunks, {});
  int failed = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(| : failed)
  for (int64_t i = 0; i < static_cast<int64_t>(n_chunks); i++)
    failed |= enc(padded.data() + i * chunk_bytes, chunk_bytes, streams[i]);
  return failed ? CODAG_EINVAL : CODAG_OK;
}

}  // namespace

extern "C" void codag_hbuf_free(codag_hbuf* b) {
  if (!b) return;
  std::free(b->data);
  b->data = nullptr;
  b->bytes = 0;
}

extern "C" codag_status codag_encode_rlev1(const uint8_t* in, uint64_t in_bytes, uint64_t chunk_bytes,
                                           int elem_bytes, codag_hbuf* blob, codag_hbuf* blk_off,
                                           codag_hbuf* col_len) {
  if (!in || !blob || !blk_off || !col_len || !valid_elem(elem_bytes) || chunk_bytes == 0 ||
      chunk_bytes % elem_bytes || chunk_bytes / elem_bytes < 2 || in_bytes == 0)
    return CODAG_EINVAL;
  const uint64_t n = (in_bytes + chunk_bytes * 32 - 1) / (chunk_bytes * 32) * 32;  // rlev1.h:111-112
  std::vector<uint8_t> padded(n * chunk_bytes, 0);
  std::memcpy(padded.data(), in, in_bytes);
  std::vector<std::vector<uint8_t>> streams;
  if (encode_chunks(padded, n, chunk_bytes, streams, [&](const uint8_t* c, uint64_t b, std::vector<uint8_t>& o) {
        return rlev1_encode_chunk(c, b, elem_bytes, o);
      }))
    return CODAG_EINVAL;
  std::vector<uint64_t> off(n + 1, 0), len(n, 0);
  for (uint64_t i = 0; i < n; i++) {
    len[i] = streams[i].size();
    off[i + 1] = off[i] + round_up(len[i], 4);  // encoder.h:780-783
  }
  std::vector<uint8_t> out(8 + off[n], 0);
  std::memcpy(out.data(), &in_bytes, 8);
  for (uint64_t i = 0; i < n; i++) std::memcpy(out.data() + 8 + off[i], streams[i].data(), len[i]);
  if (!to_hbuf(out.data(), out.size(), blob) || !to_hbuf(off.data(), off.size() * 8, blk_off) ||
      !to_hbuf(len.data(), len.size() * 8, col_len))
    return CODAG_ENOMEM;
  return CODAG_OK;
}

extern "C" codag_status codag_encode_rlev2(const uint8_t* in, uint64_t in_bytes, uint64_t chunk_bytes,
                                           int elem_bytes, codag_hbuf* comp, codag_hbuf* blk_off,
                                           codag_hbuf* col_len) {
  if (!in || !comp || !blk_off || !col_len || !valid_elem(elem_bytes) || chunk_bytes == 0 ||
      chunk_bytes % elem_bytes || in_bytes == 0)
    return CODAG_EINVAL;
  const uint64_t n = (in_bytes + chunk_bytes * 32 - 1) / (chunk_bytes * 32) * 32;  // encoder_trans.h:490
  std::vector<uint8_t> padded(n * chunk_bytes, 0);
  std::memcpy(padded.data(), in, in_bytes);
  std::vector<std::vector<uint8_t>> streams;
  if (encode_chunks(padded, n, chunk_bytes, streams, [&](const uint8_t* c, uint64_t b, std::vector<uint8_t>& o) {
        return rlev2_encode_chunk(c, b, elem_bytes, o);
      }))
    return CODAG_EINVAL;
  std::vector<uint64_t> off(n + 1, 0), len(n, 0);
  for (uint64_t i = 0; i < n; i++) {
    len[i] = streams[i].size();
    off[i + 1] = off[i] + round_up(len[i], 128);  // encoder_trans.h:352
  }
  std::vector<uint8_t> out(off[n], 0);
  for (uint64_t i = 0; i < n; i++) std::memcpy(out.data() + off[i], streams[i].data(), len[i]);
  off[n] = in_bytes;  // encoder_trans.h:545: last entry carries the original size
  if (!to_hbuf(out.data(), out.size(), comp) || !to_hbuf(off.data(), off.size() * 8, blk_off) ||
      !to_hbuf(len.data(), len.size() * 8, col_len))
    return CODAG_ENOMEM;
  return CODAG_OK;
}

extern "C" codag_status codag_encode_deflate(const uint8_t* in, uint64_t in_bytes, uint64_t chunk_bytes,
                                             int level, int zlib_wrapper, int require_no_stored,
                                             codag_hbuf* comp, codag_hbuf* blk_offset, codag_hbuf* col_len) {
  if (!in || !comp || !blk_offset || !col_len || chunk_bytes == 0 || in_bytes == 0 || level < 0 || level > 9)
    return CODAG_EINVAL;
  const uint64_t n = (in_bytes + chunk_bytes - 1) / chunk_bytes;  // deflate_compressor.py:62-66
  std::vector<uint8_t> padded(n * chunk_bytes, 0);
  std::memcpy(padded.data(), in, in_bytes);
  std::vector<std::vector<uint8_t>> streams;
  int stored = 0;
  if (encode_chunks(padded, n, chunk_bytes, streams, [&](const uint8_t* c, uint64_t b, std::vector<uint8_t>& o) {
        uint32_t types = 0;
        int rc = deflate_encode_chunk(c, b, level, zlib_wrapper, Z_DEFAULT_STRATEGY, o, &types);
        if (rc == CODAG_OK && (types & 0x80000001u) && require_no_stored) rc = CODAG_EINVAL;
        o.resize(round_up(o.size(), 8), 0);  // deflate_compressor.py:104-112
        return rc;
      }))
    return CODAG_EINVAL;
  (void)stored;
  std::vector<uint64_t> off(n + 2, 0), len(n, 0);
  off[0] = in_bytes;
  off[1] = 0;
  uint64_t total = 0;
  for (uint64_t i = 0; i < n; i++) {
    len[i] = streams[i].size();
    total += len[i];
    off[i + 2] = total;
  }
  std::vector<uint8_t> out(total);
  uint64_t pos = 0;
  for (uint64_t i = 0; i < n; i++) {
    std::memcpy(out.data() + pos, streams[i].data(), len[i]);
    pos += len[i];
  }
  if (!to_hbuf(out.data(), out.size(), comp) || !to_hbuf(off.data(), off.size() * 8, blk_offset) ||
      !to_hbuf(len.data(), len.size() * 8, col_len))
    return CODAG_ENOMEM;
  return CODAG_OK;
}

// CODAG's transposed RLE v2 layout (rlev2::compress_gpu_transpose, include/rlev2/encoder_trans.h:
// 8-182 block_encode and 359-391 tranpose_col_len_single).  Chunk c of the input (zero padded to
// a multiple of chunk_bytes; no padding of the chunk count) is split into 32 substreams:
// substream t holds the values t*ru + k*32*ru + j (0 <= j < ru), each encoded on its own.  The
// chunk's region starts at blk_off[c] and interleaves the substreams in 4-byte words: for
// w = 0, 1, ... every substream still longer than 4w contributes its bytes [4w, 4w+4), in
// substream order.  The bytes of such a word past a substream's end are the bytes that follow
// it when all substreams of all chunks are laid end to end (zero past the last one), which is
// what CODAG's copy reads.  A region is round_up(sum of round_up4(length), 128) bytes (zero
// filled), blk_off[n] holds the original size, col_len the 32 exact lengths per chunk.
extern "C" codag_status codag_encode_rlev2_transposed(const uint8_t* in, uint64_t in_bytes, uint64_t chunk_bytes,
                                                      int elem_bytes, int read_unit, codag_hbuf* comp,
                                                      codag_hbuf* blk_off, codag_hbuf* col_len) {
  if (!in || !comp || !blk_off || !col_len || !valid_elem(elem_bytes) || chunk_bytes == 0 || in_bytes == 0 ||
      read_unit <= 0 || chunk_bytes % (static_cast<uint64_t>(elem_bytes) * 32u * static_cast<uint64_t>(read_unit)))
    return CODAG_EINVAL;
  const uint64_t n = (in_bytes + chunk_bytes - 1) / chunk_bytes;
  std::vector<uint8_t> padded(n * chunk_bytes, 0);
  std::memcpy(padded.data(), in, in_bytes);
  const uint64_t per = chunk_bytes / elem_bytes / 32, ru = static_cast<uint64_t>(read_unit);
  std::vector<std::vector<uint8_t>> subs(n * 32);
#pragma omp parallel for schedule(dynamic, 32)
  for (int64_t f = 0; f < static_cast<int64_t>(n * 32); f++) {
    const uint64_t c = f / 32, t = f % 32;
    const uint8_t* base = padded.data() + c * chunk_bytes;
    VectorSink sink{subs[f]};
    codag_fmt::RleV2Writer<VectorSink> w(sink);
    w.encode([&](uint64_t j) {
      const uint64_t e = t * ru + (j / ru) * 32 * ru + j % ru;
      uint64_t v = 0;
      std::memcpy(&v, base + e * elem_bytes, elem_bytes);
      return v;
    }, per);
  }
  // all substreams end to end (the source of the interleaved words)
  std::vector<uint64_t> acc(n * 32 + 1, 0);
  for (uint64_t f = 0; f < n * 32; f++) acc[f + 1] = acc[f] + subs[f].size();
  std::vector<uint8_t> packed(acc[n * 32] + 4, 0);
  for (uint64_t f = 0; f < n * 32; f++) std::memcpy(packed.data() + acc[f], subs[f].data(), subs[f].size());
  std::vector<uint64_t> off(n + 1, 0), len(n * 32, 0);
  for (uint64_t c = 0; c < n; c++) {
    uint64_t words = 0;
    for (uint64_t t = 0; t < 32; t++) {
      len[c * 32 + t] = subs[c * 32 + t].size();
      words += (len[c * 32 + t] + 3) / 4;
    }
    off[c + 1] = off[c] + round_up(4 * words, 128);
  }
  std::vector<uint8_t> out(off[n], 0);
  for (uint64_t c = 0; c < n; c++) {
    uint64_t o = off[c];
    for (uint64_t w = 0;; w++) {
      bool any = false;
      for (uint64_t t = 0; t < 32; t++) {
        const uint64_t f = c * 32 + t;
        if (len[f] > 4 * w) {
          std::memcpy(out.data() + o, packed.data() + acc[f] + 4 * w, 4);
          o += 4;
          any = true;
        }
      }
      if (!any) break;
    }
  }
  off[n] = in_bytes;  // the last entry carries the original size (encoder_trans.h:460)
  if (!to_hbuf(out.data(), out.size(), comp) || !to_hbuf(off.data(), off.size() * 8, blk_off) ||
      !to_hbuf(len.data(), len.size() * 8, col_len))
    return CODAG_ENOMEM;
  return CODAG_OK;
}

// The layout CODAG's cuDF comparison reads (rapids_compressor.py:222-275 writes it,
// include/base_deflate.h:20-130 decodes it): [u64 chunk_bytes][u64 n][u64 size_i x n] followed
// by the n zlib streams back to back, no padding; chunk i holds bytes [i*chunk, (i+1)*chunk)
// of the input zero padded to a multiple of chunk_bytes.
extern "C" codag_status codag_encode_cudf_deflate(const uint8_t* in, uint64_t in_bytes, uint64_t chunk_bytes, int level,
                                                  codag_hbuf* file) {
  if (!in || !file || chunk_bytes == 0 || in_bytes == 0 || level < 0 || level > 9) return CODAG_EINVAL;
  const uint64_t n = (in_bytes + chunk_bytes - 1) / chunk_bytes;
  std::vector<uint8_t> padded(n * chunk_bytes, 0);
  std::memcpy(padded.data(), in, in_bytes);
  std::vector<std::vector<uint8_t>> streams;
  if (encode_chunks(padded, n, chunk_bytes, streams, [&](const uint8_t* c, uint64_t b, std::vector<uint8_t>& o) {
        return deflate_encode_chunk(c, b, level, 1, Z_DEFAULT_STRATEGY, o, nullptr);
      }))
    return CODAG_EINVAL;
  uint64_t total = 16 + 8 * n;
  for (const auto& st : streams) total += st.size();
  std::vector<uint8_t> out(total);
  uint64_t* head = reinterpret_cast<uint64_t*>(out.data());
  head[0] = chunk_bytes;
  head[1] = n;
  uint64_t pos = 16 + 8 * n;
  for (uint64_t i = 0; i < n; i++) {
    head[2 + i] = streams[i].size();
    std::memcpy(out.data() + pos, streams[i].data(), streams[i].size());
    pos += streams[i].size();
  }
  return to_hbuf(out.data(), out.size(), file) ? CODAG_OK : CODAG_ENOMEM;
}

extern "C" codag_status codag_cudf_deflate_layout(const uint8_t* file, uint64_t file_bytes, uint64_t* chunk_bytes,
                                                  uint64_t* n_chunks, uint64_t* data_offset, uint64_t* blk_off) {
  if (!file || !chunk_bytes || !n_chunks || !data_offset || file_bytes < 16) return CODAG_EINVAL;
  uint64_t head[2];
  std::memcpy(head, file, 16);
  const uint64_t n = head[1];
  if (head[0] == 0 || head[0] >= (1ull << 31) || n > (file_bytes - 16) / 8) return CODAG_EINVAL;
  const uint64_t data = 16 + 8 * n;
  uint64_t cum = 0;
  for (uint64_t i = 0; i < n; i++) {
    uint64_t sz;
    std::memcpy(&sz, file + 16 + 8 * i, 8);
    if (sz > file_bytes - data - cum) return CODAG_EINVAL;  // stream i must lie inside the file
    if (blk_off) blk_off[i] = cum;
    cum += sz;
  }
  if (blk_off) blk_off[n] = cum;
  *chunk_bytes = head[0];
  *n_chunks = n;
  *data_offset = data;
  return CODAG_OK;
}

extern "C" codag_status codag_encode_one(int codec, const uint8_t* in, uint64_t in_bytes, int elem_bytes,
                                         int level, codag_hbuf* stream) {
  if (!in || !stream || in_bytes == 0) return CODAG_EINVAL;
  std::vector<uint8_t> out;
  int rc;
  switch (codec) {
    case CODAG_CODEC_RLEV1: rc = rlev1_encode_chunk(in, in_bytes, elem_bytes, out); break;
    case CODAG_CODEC_RLEV2: rc = rlev2_encode_chunk(in, in_bytes, elem_bytes, out); break;
    case CODAG_CODEC_DEFLATE: {
      uint32_t types = 0;
      rc = deflate_encode_chunk(in, in_bytes, level, 1, Z_DEFAULT_STRATEGY, out, &types);
      if (rc == CODAG_OK && (types & 0x80000001u)) rc = CODAG_EINVAL;
    } break;
    default: rc = CODAG_EINVAL;
  }
  if (rc != CODAG_OK) return static_cast<codag_status>(rc);
  return to_hbuf(out.data(), out.size(), stream) ? CODAG_OK : CODAG_ENOMEM;
}

extern "C" codag_status codag_encode_set(const uint8_t* in, const uint64_t* in_off, const uint64_t* in_len,
                                         const uint8_t* codecs, const uint8_t* elem_bytes, uint64_t n, int level,
                                         codag_chunk_desc* descs, codag_hbuf* comp, uint64_t* out_bytes) {
  if (!in || !in_off || !in_len || !codecs || !elem_bytes || !descs || !comp || !out_bytes || n == 0 || level < 0 ||
      level > 9)
    return CODAG_EINVAL;
  for (uint64_t i = 0; i < n; i++) {
    if (in_len[i] == 0 || in_len[i] > 0xffffffffull || codecs[i] > CODAG_CODEC_DEFLATE) return CODAG_EINVAL;
    if (codecs[i] != CODAG_CODEC_DEFLATE && (!valid_elem(elem_bytes[i]) || in_len[i] % elem_bytes[i]))
      return CODAG_EINVAL;
  }
  std::vector<std::vector<uint8_t>> streams(n);
  int failed = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(| : failed)
  for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
    const uint8_t* src = in + in_off[i];
    int rc;
    if (codecs[i] == CODAG_CODEC_RLEV1) {
      rc = rlev1_encode_chunk(src, in_len[i], elem_bytes[i], streams[i]);
    } else if (codecs[i] == CODAG_CODEC_RLEV2) {
      rc = rlev2_encode_chunk(src, in_len[i], elem_bytes[i], streams[i]);
    } else {
      uint32_t types = 0;
      rc = deflate_encode_chunk(src, in_len[i], level, 1, Z_DEFAULT_STRATEGY, streams[i], &types);
    }
    failed |= rc != CODAG_OK || streams[i].size() > 0xffffffffull;
  }
  if (failed) return CODAG_EINVAL;
  uint64_t c = 0, o = 0;
  for (uint64_t i = 0; i < n; i++) {
    codag_chunk_desc& d = descs[i];
    std::memset(&d, 0, sizeof(d));
    d.comp_off = c;
    d.comp_len = static_cast<uint32_t>(streams[i].size());
    d.out_off = o;
    d.out_len = static_cast<uint32_t>(in_len[i]);
    d.codec = codecs[i];
    d.elem_bytes = codecs[i] == CODAG_CODEC_DEFLATE ? 1 : elem_bytes[i];
    d.wrapper_bytes = codecs[i] == CODAG_CODEC_DEFLATE ? 2 : 0;
    c += round_up(streams[i].size(), 16);
    o += round_up(in_len[i], 256);
  }
  comp->data = static_cast<uint8_t*>(std::calloc(c ? c : 1, 1));
  comp->bytes = c;
  if (!comp->data) return CODAG_ENOMEM;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < static_cast<int64_t>(n); i++)
    if (!streams[i].empty()) std::memcpy(comp->data + descs[i].comp_off, streams[i].data(), streams[i].size());
  *out_bytes = o;
  return CODAG_OK;
}
