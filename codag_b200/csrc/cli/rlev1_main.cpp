// rlev1 -f <raw column> -t <1|2|4|8> [-n <warps per CTA>]
//
// The command line and output of CODAG's rlev1 tool (src/rlev1/rlev1.cu:46-280): encode the
// column in CODAG's RLE v1 layout, write ./input_data/rle_v1_col_len.bin and
// ./input_data/rle_v1_blk_offset.bin (rlev1.h:178-186), read them back as the decoder does
// (rlev1.h:436-469), decode on the GPU through codag_decompress_rlev1 and print
//   NUM WARP: <n>
//   <compressed bytes>\t<metadata bytes>\t<compressed/original>\t<seconds>
// followed by "File Differ at <i>" when the output differs from the column.
#include <getopt.h>

#include <cstdlib>
#include <iostream>

#include "cli_common.hpp"

using namespace codag_cli;

int main(int argc, char** argv) {
  std::string file;
  int elem = 8, warps = 1;
  static struct option opts[] = {{"file", required_argument, nullptr, 'f'},
                                 {"type", required_argument, nullptr, 't'},
                                 {"num_warp", required_argument, nullptr, 'n'},
                                 {nullptr, 0, nullptr, 0}};
  int c;
  while ((c = getopt_long(argc, argv, "f:t:n:", opts, nullptr)) != -1) {
    if (c == 'f') file = optarg;
    else if (c == 't') elem = std::atoi(optarg);
    else if (c == 'n') warps = std::atoi(optarg);
    else {
      std::cerr << "usage: rlev1 -f <column file> -t <1|2|4|8> [-n <warps>]\n";
      return 1;
    }
  }
  if (file.empty() || (elem != 1 && elem != 2 && elem != 4 && elem != 8) || warps < 1 || warps > 8) {
    std::cerr << "usage: rlev1 -f <column file> -t <1|2|4|8> [-n <warps>]\n";
    return 1;
  }
  std::vector<uint8_t> in;
  if (!read_file(file, in) || in.empty()) {
    std::printf("Fatal Error: INPUT File open error\n");
    return -1;
  }
  if (in.size() % elem) {
    std::cerr << "read bytes should be multiple of input bytes \n";
    return 1;
  }
  const uint64_t chunk = 131072;
  std::cout << "CHUNK_SIZE" << "\t" << "COLUMN WIDTH\t BUFFER SIZE \t COMPRESSED SIZE \t META DATA SIZE \t DECOMPRESSION TIME\n";

  codag_hbuf blob{}, off{}, len{};
  if (codag_encode_rlev1(in.data(), in.size(), chunk, elem, &blob, &off, &len) != CODAG_OK) {
    std::printf("Fatal Error: encode failed\n");
    return -1;
  }
  const uint64_t n_pad = len.bytes / 8;
  // CODAG's files hold 32x the entries the decoder uses (rlev1.h:117, 149, 180, 185);
  // the extra entries are written as zeros here
  std::vector<uint64_t> off_file(n_pad * 32 + 1, 0), len_file(n_pad * 32 * 32, 0);
  std::memcpy(off_file.data(), off.data, off.bytes);
  std::memcpy(len_file.data(), len.data, len.bytes);
  if (!ensure_dir("./input_data") ||
      !write_file("./input_data/rle_v1_col_len.bin", len_file.data(), len_file.size() * 8) ||
      !write_file("./input_data/rle_v1_blk_offset.bin", off_file.data(), off_file.size() * 8)) {
    std::printf("Fatal Error: metadata write error\n");
    return -1;
  }
  codag_hbuf_free(&off);
  codag_hbuf_free(&len);

  // decoder side: the metadata comes back from the files
  std::vector<uint8_t> col_f, blk_f;
  if (!read_file("./input_data/rle_v1_col_len.bin", col_f)) {
    std::printf("Fatal Error: Col Len read error\n");
    return -1;
  }
  if (!read_file("./input_data/rle_v1_blk_offset.bin", blk_f)) {
    std::printf("Fatal Error: Block off read error\n");
    return -1;
  }
  const uint64_t n = (blk_f.size() / 8 - 1) / 32;  // rlev1.h:469
  uint64_t real_out = 0;
  std::memcpy(&real_out, blob.data, 8);
  const uint64_t meta_bytes = col_f.size() + blk_f.size();
  DevBuf d_in, d_off, d_len, d_out, d_st;
  if (!d_in.alloc(blob.bytes) || !d_off.alloc(n * 8) || !d_len.alloc(n * 8) || !d_out.alloc(n * chunk) ||
      !d_st.alloc(n * 4) || !d_in.upload(blob.data, blob.bytes) || !d_off.upload(blk_f.data(), n * 8) ||
      !d_len.upload(col_f.data(), n * 8)) {
    std::printf("Fatal Error: device buffers\n");
    return -1;
  }
  codag_tune t;
  codag_get_tune(CODAG_CODEC_RLEV1, &t);
  t.warps_per_cta = warps;
  codag_set_tune(CODAG_CODEC_RLEV1, &t);
  std::printf("NUM WARP: %i\n", warps);
  std::fflush(stdout);
  cudaDeviceSynchronize();
  const double t0 = now_s();
  const codag_status s = codag_decompress_rlev1(d_in.as<uint8_t>() + 8, blob.bytes - 8, d_off.as<uint64_t>(),
                                                d_len.as<uint64_t>(), n, chunk, elem, d_out.as<uint8_t>(), real_out,
                                                d_st.as<int32_t>(), nullptr, 0, nullptr);
  cudaDeviceSynchronize();
  const double secs = now_s() - t0;
  if (s != CODAG_OK) {
    std::printf("Fatal Error: codag_decompress_rlev1 returned %d\n", static_cast<int>(s));
    return -1;
  }
  const float ratio = (1.0f * blob.bytes) / (real_out * 1.0f);
  std::cout << blob.bytes << "\t" << meta_bytes << "\t" << ratio << "\t" << secs << "\n";
  std::vector<uint8_t> out(real_out);
  cudaMemcpy(out.data(), d_out.p, real_out, cudaMemcpyDeviceToHost);
  const uint64_t bad = bad_chunks(d_st, n);
  const long long diff = first_diff(in.data(), out.data(), std::min<uint64_t>(in.size(), real_out));
  if (diff >= 0) std::cout << "File Differ at " << diff << std::endl;
  codag_hbuf_free(&blob);
  if (bad) std::cerr << bad << " chunk(s) reported a decode error\n";
  return (diff >= 0 || bad || real_out != in.size()) ? 1 : 0;
}
