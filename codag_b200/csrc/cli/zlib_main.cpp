// zlib <name>_comp.bin <output> <name>_blk_offset.bin <chunk_size>
//
// The command line and output of CODAG's zlib tool (src/zlib/zlib.cu:25-132): decode the
// chunked Deflate file written by CODAG's compressor (zlib-wrapped streams padded to 8
// bytes; blk_offset = [original size, 0, end of chunk 1, ...]) on the GPU through
// codag_decompress_deflate, print "\t<seconds>" and write the original bytes to <output>.
// Unlike CODAG's tool it checks every chunk's status and exits non-zero on a bad chunk.
#include <cstdlib>
#include <iostream>

#include "cli_common.hpp"

using namespace codag_cli;

int main(int argc, char** argv) {
  if (argc < 5) {
    std::cerr << "Please provide arguments  input output blk_offset chunk_size\n";
    return 1;
  }
  const std::string input = argv[1], output = argv[2], blk = argv[3];
  const uint64_t chunk = std::strtoull(argv[4], nullptr, 10);
  std::vector<uint8_t> comp, blk_f;
  if (!read_file(input, comp)) {
    std::printf("Fatal Error: INPUT File open error\n");
    return -1;
  }
  if (!read_file(blk, blk_f) || blk_f.size() < 24 || blk_f.size() % 8) {
    std::printf("Fatal Error: BLK_OFFSET File open error\n");
    return -1;
  }
  if (chunk == 0) {
    std::cerr << "chunk_size must be positive\n";
    return 1;
  }
  const uint64_t* bo = reinterpret_cast<const uint64_t*>(blk_f.data());
  const uint64_t n = blk_f.size() / 8 - 2;  // zlib.h:1589
  const uint64_t size = bo[0];
  DevBuf d_in, d_off, d_out, d_st;
  if (!d_in.alloc(comp.size()) || !d_off.alloc((n + 1) * 8) || !d_out.alloc(n * chunk) || !d_st.alloc(n * 4) ||
      !d_in.upload(comp.data(), comp.size()) || !d_off.upload(bo + 1, (n + 1) * 8)) {
    std::printf("Fatal Error: device buffers\n");
    return -1;
  }
  cudaDeviceSynchronize();
  const double t0 = now_s();
  const codag_status s = codag_decompress_deflate(d_in.as<uint8_t>(), comp.size(), d_off.as<uint64_t>(), n, chunk, 2,
                                                  d_out.as<uint8_t>(), size, d_st.as<int32_t>(), nullptr);
  cudaDeviceSynchronize();
  const double secs = now_s() - t0;
  if (s != CODAG_OK) {
    std::printf("Fatal Error: codag_decompress_deflate returned %d\n", static_cast<int>(s));
    return -1;
  }
  std::cout << "\t" << secs << std::endl;
  std::vector<uint8_t> out(size);
  cudaMemcpy(out.data(), d_out.p, size, cudaMemcpyDeviceToHost);
  const uint64_t bad = bad_chunks(d_st, n);
  if (!write_file(output, out.data(), out.size())) {
    std::printf("Fatal Error: OUTPUT File open error\n");
    return -1;
  }
  if (bad) {
    std::cerr << bad << " chunk(s) reported a decode error\n";
    return 1;
  }
  return 0;
}
