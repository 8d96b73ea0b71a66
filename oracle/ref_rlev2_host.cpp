// Reference harness: CODAG's own RLE v2 encoder, run on the host.
// TEST INFRASTRUCTURE ONLY: it produces the golden RLE v2 files that pin the oracle and the
// CUDA decoder to CODAG (tests/golden/make_ref_rlev2.py); nothing in the library calls it.
//
//   ref_rlev2_host encode <elem 1|2|4|8> <column.bin> <prefix>
//       writes <prefix>_comp.bin, <prefix>_blk_off.bin (n+1 u64, the last entry the input
//       size) and <prefix>_col_len.bin (n u64), the arrays CODAG's rlev2 tool builds
//   ref_rlev2_host transposed <elem 1|2|4|8> <read_unit 1|2|4|8> <column.bin> <prefix>
//       the same files for CODAG's transposed layout (rlev2::compress_gpu_transpose,
//       encoder_trans.h:411-480): block_encode<false/true, READ_UNIT> (encoder_trans.h:8-182)
//       and tranpose_col_len_single (:359-391) run the same way; col_len has 32 entries per
//       chunk.  Bytes CODAG reads from uninitialised memory (past the last substream, and
//       between a region's data and its 128-byte end) are zero here.
//   ref_rlev2_host tables <out.bin>
//       writes CODAG's width tables: decode map (32 bytes), encode map, closest-width map
//       and closest-aligned map (65 bytes each), in that order (include/rlev2/utils.h:28-59)
//
// The encode command follows the steps of rlev2::compress_gpu_orig
// (include/rlev2/encoder_trans.h:482-564) with host buffers: CODAG's kernels
// block_encode_orig<false> (sizing pass) and block_encode_orig<true> (writing pass),
// compiled for the host through oracle/ref_shim_host/codag_host_shim.h, run one block of
// 32 emulated threads per 32 chunks; the scans are done here; the final copy of each
// stream to its 128-byte aligned offset (orig_col_len_single, encoder_trans.h:393-409) is
// CODAG's kernel run the same way.  Bytes between streams are zero here (CODAG leaves them
// uninitialised).
#include "codag_host_shim.h"

#include <common.h>
#include <rlev2/encoder_trans.h>

#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

namespace {

std::vector<uint8_t> slurp(const char* p) {
  std::vector<uint8_t> v;
  FILE* f = std::fopen(p, "rb");
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", p);
    std::exit(2);
  }
  std::fseek(f, 0, SEEK_END);
  v.resize(static_cast<size_t>(std::ftell(f)));
  std::fseek(f, 0, SEEK_SET);
  if (!v.empty() && std::fread(v.data(), 1, v.size(), f) != v.size()) std::exit(2);
  std::fclose(f);
  return v;
}

void spill(const std::string& p, const void* d, size_t n) {
  FILE* f = std::fopen(p.c_str(), "wb");
  if (!f || (n && std::fwrite(d, 1, n, f) != n)) std::exit(2);
  std::fclose(f);
}

template <class COMP>
int encode(const std::vector<uint8_t>& col, const std::string& prefix) {
  const uint64_t CH = 1024 * 128;  // the tool's CHUNK_SIZE (src/rlev2/rlev2.cu)
  const uint64_t in_bytes = col.size();
  const uint64_t n = (in_bytes + CH * 32 - 1) / (CH * 32) * 32;  // chunk count, a multiple of 32
  const uint64_t padded = n * CH;
  const uint64_t out_chunk = static_cast<uint64_t>(1.5 * CH);
  std::vector<uint8_t> in(padded, 0);
  std::memcpy(in.data(), col.data(), in_bytes);
  std::vector<uint8_t> scratch(n * out_chunk + 4 * out_chunk, 0);
  std::vector<col_len_t> col_len(n * BLK_SIZE, 0), acc(n * BLK_SIZE, 0);
  std::vector<blk_off_t> blk_off(n + 1, 0);
  INPUT_T* d_in = reinterpret_cast<INPUT_T*>(in.data());

  // sizing pass: writes col_len (through its acc_col_len argument) and blk_off[i+1]
  shim_launch(static_cast<unsigned>(n / 32), BLK_SIZE, [&] {
    rlev2::block_encode_orig<false, COMP>(d_in, padded, scratch.data(), col_len.data(), blk_off.data(), CH * 32,
                                          CH / sizeof(COMP));
  });
  for (uint64_t i = 1; i <= n; i++) blk_off[i] += blk_off[i - 1];
  acc[0] = col_len[0];
  for (uint64_t i = 1; i < n * BLK_SIZE; i++) acc[i] = acc[i - 1] + col_len[i];
  // writing pass: streams packed back to back at the scanned lengths
  std::fill(scratch.begin(), scratch.end(), 0);
  shim_launch(static_cast<unsigned>(n / 32), BLK_SIZE, [&] {
    rlev2::block_encode_orig<true, COMP>(d_in, padded, scratch.data(), acc.data(), blk_off.data(), CH * 32,
                                         CH / sizeof(COMP));
  });
  const uint64_t out_bytes = blk_off[n];
  std::vector<uint8_t> out(out_bytes, 0);
  shim_launch(static_cast<unsigned>(n), 1, [&] {
    rlev2::orig_col_len_single(scratch.data(), acc.data(), col_len.data(), blk_off.data(), out.data());
  });
  blk_off[n] = in_bytes;  // the last entry carries the original size (encoder_trans.h:545)
  spill(prefix + "_comp.bin", out.data(), out.size());
  spill(prefix + "_blk_off.bin", blk_off.data(), blk_off.size() * sizeof(blk_off_t));
  spill(prefix + "_col_len.bin", col_len.data(), n * sizeof(col_len_t));
  std::printf("%llu chunks, %llu bytes\n", static_cast<unsigned long long>(n), static_cast<unsigned long long>(out_bytes));
  return 0;
}

template <class COMP, int RU>
int encode_transposed(const std::vector<uint8_t>& col, const std::string& prefix) {
  const uint64_t CH = 1024 * 128;
  const uint64_t in_bytes = col.size();
  const uint64_t n = (in_bytes + CH - 1) / CH;  // encoder_trans.h:416-417: no padding of the chunk count
  const uint64_t padded = n * CH;
  const uint64_t out_chunk = static_cast<uint64_t>(1.5 * CH);
  std::vector<uint8_t> in(padded, 0);
  std::memcpy(in.data(), col.data(), in_bytes);
  std::vector<uint8_t> scratch(n * out_chunk + 4 * out_chunk, 0);
  std::vector<col_len_t> col_len(n * BLK_SIZE, 0), acc(n * BLK_SIZE, 0);
  std::vector<blk_off_t> blk_off(n + 1, 0);
  INPUT_T* d_in = reinterpret_cast<INPUT_T*>(in.data());
  shim_launch(static_cast<unsigned>(n), BLK_SIZE, [&] {
    rlev2::block_encode<false, RU, COMP>(d_in, padded, scratch.data(), col_len.data(), blk_off.data(), CH);
  });
  for (uint64_t i = 1; i <= n; i++) blk_off[i] += blk_off[i - 1];
  acc[0] = col_len[0];
  for (uint64_t i = 1; i < n * BLK_SIZE; i++) acc[i] = acc[i - 1] + col_len[i];
  std::fill(scratch.begin(), scratch.end(), 0);
  shim_launch(static_cast<unsigned>(n), BLK_SIZE, [&] {
    rlev2::block_encode<true, RU, COMP>(d_in, padded, scratch.data(), acc.data(), blk_off.data(), CH);
  });
  const uint64_t out_bytes = blk_off[n];
  std::vector<uint8_t> out(out_bytes, 0);
  shim_launch(static_cast<unsigned>(n), 1, [&] {
    rlev2::tranpose_col_len_single(scratch.data(), acc.data(), col_len.data(), blk_off.data(), out.data());
  });
  blk_off[n] = in_bytes;
  spill(prefix + "_comp.bin", out.data(), out.size());
  spill(prefix + "_blk_off.bin", blk_off.data(), blk_off.size() * sizeof(blk_off_t));
  spill(prefix + "_col_len.bin", col_len.data(), col_len.size() * sizeof(col_len_t));
  std::printf("%llu chunks, %llu bytes\n", static_cast<unsigned long long>(n), static_cast<unsigned long long>(out_bytes));
  return 0;
}

template <class COMP>
int encode_transposed_ru(int ru, const std::vector<uint8_t>& col, const std::string& prefix) {
  switch (ru) {
    case 1: return encode_transposed<COMP, 1>(col, prefix);
    case 2: return encode_transposed<COMP, 2>(col, prefix);
    case 4: return encode_transposed<COMP, 4>(col, prefix);
    case 8: return encode_transposed<COMP, 8>(col, prefix);
    default: return 1;
  }
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 6 && std::string(argv[1]) == "transposed") {
    const int elem = std::atoi(argv[2]), ru = std::atoi(argv[3]);
    const std::vector<uint8_t> col = slurp(argv[4]);
    if (col.empty()) return 1;
    switch (elem) {
      case 8: return encode_transposed_ru<uint64_t>(ru, col, argv[5]);
      case 4: return encode_transposed_ru<uint32_t>(ru, col, argv[5]);
      case 2: return encode_transposed_ru<uint16_t>(ru, col, argv[5]);
      case 1: return encode_transposed_ru<uint8_t>(ru, col, argv[5]);
      default: return 1;
    }
  }
  if (argc == 3 && std::string(argv[1]) == "tables") {
    std::vector<uint8_t> t;
    t.insert(t.end(), __BIT_WIDTH_DECODE_MAP, __BIT_WIDTH_DECODE_MAP + 32);
    t.insert(t.end(), __BIT_WIDTH_ENCODE_MAP, __BIT_WIDTH_ENCODE_MAP + 65);
    t.insert(t.end(), __CLOSEST_FIXED_BIT_MAP, __CLOSEST_FIXED_BIT_MAP + 65);
    t.insert(t.end(), __CLOSEST_ALIGNED_FIXED_BIT_MAP, __CLOSEST_ALIGNED_FIXED_BIT_MAP + 65);
    spill(argv[2], t.data(), t.size());
    return 0;
  }
  if (argc != 5 || std::string(argv[1]) != "encode") {
    std::fprintf(stderr, "usage: ref_rlev2_host encode <elem 1|2|4|8> <column.bin> <prefix>\n"
                         "       ref_rlev2_host tables <out.bin>\n");
    return 1;
  }
  const int elem = std::atoi(argv[2]);
  const std::vector<uint8_t> col = slurp(argv[3]);
  if (col.empty() || col.size() % static_cast<size_t>(elem ? elem : 1)) return 1;
  switch (elem) {
    case 8: return encode<uint64_t>(col, argv[4]);
    case 4: return encode<uint32_t>(col, argv[4]);
    case 2: return encode<uint16_t>(col, argv[4]);
    case 1: return encode<uint8_t>(col, argv[4]);
    default: return 1;
  }
}
