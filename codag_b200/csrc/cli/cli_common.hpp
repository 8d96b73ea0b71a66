// Shared pieces of the command-line tools that keep CODAG's executables' command lines
// (src/rlev1/rlev1.cu, src/rlev2/rlev2.cu, src/zlib/zlib.cu): whole-file I/O, device
// buffers and wall-clock timing around a synchronised decode.
#pragma once
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "codag_format.h"

namespace codag_cli {

inline bool read_file(const std::string& path, std::vector<uint8_t>& out) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  out.resize(n > 0 ? static_cast<size_t>(n) : 0);
  const size_t got = n > 0 ? std::fread(out.data(), 1, out.size(), f) : 0;
  std::fclose(f);
  return got == out.size();
}

inline bool write_file(const std::string& path, const void* data, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const size_t put = n ? std::fwrite(data, 1, n, f) : 0;
  return std::fclose(f) == 0 && put == n;
}

inline bool ensure_dir(const std::string& d) {
  struct stat st;
  if (stat(d.c_str(), &st) == 0) return S_ISDIR(st.st_mode);
  return mkdir(d.c_str(), 0755) == 0;
}

inline std::string base_name(const std::string& p) {
  const size_t k = p.find_last_of('/');
  return k == std::string::npos ? p : p.substr(k + 1);
}

// device buffer owned by the tool
struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  bool alloc(size_t bytes) {
    n = bytes;
    return cudaMalloc(&p, bytes ? bytes : 16) == cudaSuccess;
  }
  bool upload(const void* h, size_t bytes) { return cudaMemcpy(p, h, bytes, cudaMemcpyHostToDevice) == cudaSuccess; }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

inline double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// first differing byte of two buffers, or -1
inline long long first_diff(const uint8_t* a, const uint8_t* b, uint64_t n) {
  for (uint64_t i = 0; i < n; i++)
    if (a[i] != b[i]) return static_cast<long long>(i);
  return -1;
}

// number of chunks whose status is not CODAG_OK
inline uint64_t bad_chunks(const DevBuf& st, uint64_t n) {
  std::vector<int32_t> h(n);
  if (cudaMemcpy(h.data(), st.p, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return n;
  uint64_t bad = 0;
  for (int32_t v : h) bad += v != CODAG_OK;
  return bad;
}

}  // namespace codag_cli
