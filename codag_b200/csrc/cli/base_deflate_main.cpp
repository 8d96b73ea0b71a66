// base_deflate SOURCE_FILE DESTINATION_FILE
//
// The command line of CODAG's cuDF-comparison tool (src/util/base_deflate.cu,
// include/base_deflate.h:20-130): decode a file in the layout rapids_compressor.py writes
// ([u64 chunk size][u64 n][u64 sizes x n][zlib streams]) on the GPU and write the decoded
// bytes (n x chunk size, the last chunk included in full, as CODAG's tool does for its padded
// inputs).  CODAG's tool hands each stream to cuDF's inflate kernel; here the layout is parsed
// by codag_cudf_deflate_layout and the streams go to codag_decompress_deflate.  Every chunk's
// status is checked; the tool exits non-zero on a bad chunk.
#include <cstdlib>
#include <iostream>

#include "cli_common.hpp"

using namespace codag_cli;

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "Usage: " << argv[0] << " SOURCE_FILE DESTINATION_FILE" << std::endl;
    return 1;
  }
  std::vector<uint8_t> file;
  if (!read_file(argv[1], file)) {
    std::cerr << "Couldn't open input file: " << argv[1] << std::endl;
    return 1;
  }
  uint64_t chunk = 0, n = 0, data = 0;
  if (codag_cudf_deflate_layout(file.data(), file.size(), &chunk, &n, &data, nullptr) != CODAG_OK) {
    std::cerr << "not a chunked zlib file: " << argv[1] << std::endl;
    return 1;
  }
  std::vector<uint64_t> off(n + 1);
  codag_cudf_deflate_layout(file.data(), file.size(), &chunk, &n, &data, off.data());
  std::printf("chunk size: %llu num chunks: %llu\n", static_cast<unsigned long long>(chunk),
              static_cast<unsigned long long>(n));
  const uint64_t data_size = file.size() - data;
  std::printf("data size: %llu\n", static_cast<unsigned long long>(data_size));
  DevBuf d_in, d_off, d_out, d_st;
  if (!d_in.alloc(data_size) || !d_off.alloc((n + 1) * 8) || !d_out.alloc(n * chunk) || !d_st.alloc(n * 4) ||
      !d_in.upload(file.data() + data, data_size) || !d_off.upload(off.data(), (n + 1) * 8)) {
    std::cerr << "device buffers" << std::endl;
    return 1;
  }
  cudaDeviceSynchronize();
  const double t0 = now_s();
  const codag_status s = codag_decompress_deflate(d_in.as<uint8_t>(), data_size, d_off.as<uint64_t>(), n, chunk, 2,
                                                  d_out.as<uint8_t>(), n * chunk, d_st.as<int32_t>(), nullptr);
  cudaDeviceSynchronize();
  const double secs = now_s() - t0;
  if (s != CODAG_OK) {
    std::cerr << "codag_decompress_deflate returned " << static_cast<int>(s) << std::endl;
    return 1;
  }
  std::cout << "kernel time: " << secs << " secs\n";
  const uint64_t bad = bad_chunks(d_st, n);
  std::printf("status %u\n", bad ? 1u : 0u);
  const uint64_t out_size = n * chunk;
  std::printf("out size: %llu\n", static_cast<unsigned long long>(out_size));
  std::vector<uint8_t> out(out_size);
  cudaMemcpy(out.data(), d_out.p, out_size, cudaMemcpyDeviceToHost);
  if (!write_file(argv[2], out.data(), out.size())) {
    std::cerr << "Couldn't open output file: " << argv[2] << std::endl;
    return 1;
  }
  if (bad) {
    std::cerr << bad << " chunk(s) reported a decode error\n";
    return 1;
  }
  return 0;
}
