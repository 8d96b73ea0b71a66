// rlev2 <raw column> <1|2|4|8>      (also: rlev2 -f <raw column> -t <1|2|4|8>)
//
// The command line and output of CODAG's rlev2 tool (src/rlev2/rlev2.cu:44-199): encode the
// column in CODAG's RLE v2 layout (128-byte aligned streams, blk_off[n] = original size),
// save the layout as ./input_data/<column>_{comp,blk_offset,col_len}.bin, then decode it on
// the GPU several times through codag_decompress_rlev2, printing
//   CHUNK_SIZE\t BUFFER SIZE \t COMPRESSED SIZE \t META DATA SIZE \t DECOMPRESSION TIME
//   131072 \t48\t<compressed bytes>\t<metadata bytes>\t<seconds> secs     (one line per run)
// and "fail at <i> <want>(<got>)" for the first differing byte of a run.
#include <getopt.h>

#include <cstdlib>
#include <iostream>

#include "cli_common.hpp"

using namespace codag_cli;

int main(int argc, char** argv) {
  std::string file;
  int elem = 0;
  int c;
  while ((c = getopt(argc, argv, "f:t:")) != -1) {
    if (c == 'f') file = optarg;
    else if (c == 't') elem = std::atoi(optarg);
    else {
      std::cerr << "please provide arguments INPUT_FILE SIZE_OF_DATATYPE\n";
      return 1;
    }
  }
  if (file.empty() && optind + 2 <= argc) {
    file = argv[optind];
    elem = std::atoi(argv[optind + 1]);
  }
  if (file.empty() || (elem != 1 && elem != 2 && elem != 4 && elem != 8)) {
    std::cerr << "please provide arguments INPUT_FILE SIZE_OF_DATATYPE\n";
    return 1;
  }
  std::vector<uint8_t> in;
  if (!read_file(file, in) || in.empty()) {
    std::printf("fatal error: input file open error\n");
    return -1;
  }
  const uint64_t chunk = 131072;
  std::cout << "CHUNK_SIZE" << "\t" << " BUFFER SIZE \t COMPRESSED SIZE \t META DATA SIZE \t DECOMPRESSION TIME\n";
  codag_hbuf comp{}, off{}, len{};
  if (codag_encode_rlev2(in.data(), in.size() - in.size() % elem, chunk, elem, &comp, &off, &len) != CODAG_OK) {
    std::printf("fatal error: encode failed\n");
    return -1;
  }
  const uint64_t n = len.bytes / 8;
  const uint64_t size = reinterpret_cast<const uint64_t*>(off.data)[n];
  const uint64_t meta_bytes = 8 * n * 32 + 8 * (n + 1);  // encoder_trans.h:502
  const std::string stem = "./input_data/" + base_name(file);
  if (!ensure_dir("./input_data") || !write_file(stem + "_comp.bin", comp.data, comp.bytes) ||
      !write_file(stem + "_blk_offset.bin", off.data, off.bytes) ||
      !write_file(stem + "_col_len.bin", len.data, len.bytes)) {
    std::printf("fatal error: output write error\n");
    return -1;
  }
  DevBuf d_in, d_off, d_len, d_out, d_st;
  if (!d_in.alloc(comp.bytes) || !d_off.alloc(n * 8) || !d_len.alloc(n * 8) || !d_out.alloc(n * chunk) ||
      !d_st.alloc(n * 4) || !d_in.upload(comp.data, comp.bytes) || !d_off.upload(off.data, n * 8) ||
      !d_len.upload(len.data, n * 8)) {
    std::printf("fatal error: device buffers\n");
    return -1;
  }
  std::vector<uint8_t> out(size);
  int rc = 0;
  const int shapes[2][5] = {{2, 2, 4, 8, 8}, {1, 1, 2, 4, 8}};
  codag_tune t;
  codag_get_tune(CODAG_CODEC_RLEV2, &t);
  for (int line = 0; line < 2; line++) {
    std::cout << chunk << " \t" << 48 << "\t" << comp.bytes << "\t" << meta_bytes << "\t";
    for (int run = 0; run < 5; run++) {
      t.warps_per_cta = shapes[line][run];
      codag_set_tune(CODAG_CODEC_RLEV2, &t);
      cudaMemset(d_out.p, 0, n * chunk);
      cudaDeviceSynchronize();
      const double t0 = now_s();
      const codag_status s = codag_decompress_rlev2(d_in.as<uint8_t>(), comp.bytes, d_off.as<uint64_t>(),
                                                    d_len.as<uint64_t>(), n, chunk, elem, d_out.as<uint8_t>(), size,
                                                    d_st.as<int32_t>(), nullptr, 0, nullptr);
      cudaDeviceSynchronize();
      const double secs = now_s() - t0;
      if (s != CODAG_OK) {
        std::printf("fatal error: codag_decompress_rlev2 returned %d\n", static_cast<int>(s));
        return -1;
      }
      std::cout << secs << " secs\n";
      cudaMemcpy(out.data(), d_out.p, size, cudaMemcpyDeviceToHost);
      const long long d = first_diff(in.data(), out.data(), size);
      if (d >= 0) {
        std::printf("fail at %llu %lx(%lx)\n", static_cast<unsigned long long>(d),
                    static_cast<unsigned long>(in[d]), static_cast<unsigned long>(out[d]));
        rc = 1;
      }
      if (bad_chunks(d_st, n)) rc = 1;
    }
  }
  codag_hbuf_free(&comp);
  codag_hbuf_free(&off);
  codag_hbuf_free(&len);
  return rc;
}
