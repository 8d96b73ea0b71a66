// Reference harness: runs CODAG's own RLE v1 GPU decoder, compiled from CODAG's headers, on
// chunks written by this project's producer, and writes its output.
// TEST INFRASTRUCTURE ONLY: it produces the golden digests that pin the oracle
// (tests/golden/make_ref_golden.py); nothing in the library calls it.
//
//   ref_rlev1 rlev1 <elem 4|8> <streams.bin> <blk_off.bin> <col_len.bin> <n_chunks> <out.bin>
//
// It launches the one-warp-per-chunk kernel CODAG's rlev1 tool launches (inflate_orig_rdw
// with one chunk per block, include/rlev1/rlev1.h:513-516) directly, so that none of
// CODAG's host code (./input_data, cudaSetDevice(1)) is involved.  CODAG's input reader
// reads up to four times a stream's length past its start (include/common_warp.h:874), so
// the device input is padded with zeros by four times the largest stream plus 4 KiB, and
// the output buffer has one spare chunk.
//
// CODAG's RLE v2 and Deflate decoders are not built here: the RLE v2 kernel did not finish
// within 600 s on six well-formed chunks, and the Deflate kernel reads through the same
// input stream class.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <rlev1/rlev1.h>

namespace {

std::vector<uint8_t> slurp(const char* p) {
  std::vector<uint8_t> v;
  FILE* f = std::fopen(p, "rb");
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", p);
    std::exit(2);
  }
  std::fseek(f, 0, SEEK_END);
  v.resize(std::ftell(f));
  std::fseek(f, 0, SEEK_SET);
  if (!v.empty() && std::fread(v.data(), 1, v.size(), f) != v.size()) std::exit(2);
  std::fclose(f);
  return v;
}

void spill(const char* p, const void* d, size_t n) {
  FILE* f = std::fopen(p, "wb");
  if (!f || std::fwrite(d, 1, n, f) != n) std::exit(2);
  std::fclose(f);
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    std::exit(3);
  }
}

template <class T>
T* to_device(const void* h, size_t n, size_t alloc) {
  void* d = nullptr;
  check(cudaMalloc(&d, alloc), "cudaMalloc");
  check(cudaMemset(d, 0, alloc), "cudaMemset");
  if (n) check(cudaMemcpy(d, h, n, cudaMemcpyHostToDevice), "cudaMemcpy");
  return static_cast<T*>(d);
}

template <class DT>
void run_rlev1(const std::vector<uint8_t>& s, const std::vector<uint64_t>& off, const std::vector<uint64_t>& len,
               uint64_t n, uint8_t* d_out) {
  uint64_t maxlen = 0;
  for (uint64_t i = 0; i < n; i++) maxlen = len[i] > maxlen ? len[i] : maxlen;
  uint8_t* d_in = to_device<uint8_t>(s.data(), s.size(), s.size() + 4 * maxlen + 4096);
  uint64_t* d_off = to_device<uint64_t>(off.data(), n * 8, n * 8);
  uint64_t* d_len = to_device<uint64_t>(len.data(), n * 8, n * 8);
  inflate_orig_rdw<uint32_t, DT, uint32_t, 1, 64, 32, 32><<<n, dim3(32, 1, 1)>>>(d_in, d_out, d_len, d_off, 131072, 8, n);
  check(cudaDeviceSynchronize(), "rlev1 kernel");
  cudaFree(d_in);
  cudaFree(d_off);
  cudaFree(d_len);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 8 || std::string(argv[1]) != "rlev1") {
    std::fprintf(stderr, "usage: ref_rlev1 rlev1 <elem 4|8> <streams> <blk_off> <col_len> <n_chunks> <out>\n");
    return 1;
  }
  const int elem = std::atoi(argv[2]);
  const std::vector<uint8_t> s = slurp(argv[3]);
  const std::vector<uint8_t> ob = slurp(argv[4]), lb = slurp(argv[5]);
  const uint64_t n = std::strtoull(argv[6], nullptr, 10);
  if (n == 0 || ob.size() < n * 8 || lb.size() < n * 8) return 1;
  std::vector<uint64_t> off(n), len(n);
  std::memcpy(off.data(), ob.data(), n * 8);
  std::memcpy(len.data(), lb.data(), n * 8);
  for (uint64_t i = 0; i < n; i++)
    if (off[i] > s.size() || len[i] > s.size() - off[i]) return 1;
  uint8_t* d_out = nullptr;
  check(cudaMalloc(&d_out, (n + 1) * 131072), "cudaMalloc out");
  check(cudaMemset(d_out, 0, (n + 1) * 131072), "cudaMemset out");
  if (elem == 8) run_rlev1<uint64_t>(s, off, len, n, d_out);
  else if (elem == 4) run_rlev1<uint32_t>(s, off, len, n, d_out);
  else return 1;
  std::vector<uint8_t> h(n * 131072);
  check(cudaMemcpy(h.data(), d_out, h.size(), cudaMemcpyDeviceToHost), "copy out");
  spill(argv[7], h.data(), h.size());
  return 0;
}
