// Host execution of CODAG's encoder kernels (TEST INFRASTRUCTURE ONLY).
//
// CODAG's RLE v2 encoder is a pair of __global__ kernels (include/rlev2/encoder_trans.h:8-357)
// whose bodies are plain sequential C++ per thread, plus one __syncthreads() and one
// atomicAdd on a __shared__ counter.  This header lets the host compiler build those
// bodies as ordinary functions: the CUDA execution-space keywords become empty, __shared__
// variables become function statics (shared by the emulated threads of a block), threadIdx is
// thread-local, and launch() runs a grid block by block with one std::thread per CUDA
// thread and a std::barrier standing in for __syncthreads().  The kernel launch syntax in
// CODAG's host functions (which are compiled but never called) is removed by the build
// recipe (oracle/build_ref.sh) before compilation.
#pragma once
#include <cuda_runtime_api.h>

#include <atomic>
#include <barrier>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

#undef __global__
#undef __host__
#undef __device__
#undef __shared__
#undef __constant__
#undef __forceinline__
#define __global__
#define __host__
#define __device__
#define __shared__ static
#define __constant__
#define __forceinline__ inline

struct shim_dim3 {
  unsigned x = 0, y = 0, z = 0;
};
inline thread_local shim_dim3 threadIdx;
inline shim_dim3 blockIdx, blockDim, gridDim;
inline std::barrier<>* shim_block_barrier = nullptr;

inline void __syncthreads() { shim_block_barrier->arrive_and_wait(); }

template <class T>
inline T atomicAdd(T* p, T v) {
  return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}

// Runs fn() for every (block, thread) of a 1-D grid, blocks one after the other.
inline void shim_launch(unsigned grid, unsigned block, const std::function<void()>& fn) {
  gridDim.x = grid;
  blockDim.x = block;
  for (unsigned b = 0; b < grid; b++) {
    blockIdx.x = b;
    std::barrier<> bar(static_cast<std::ptrdiff_t>(block));
    shim_block_barrier = &bar;
    std::vector<std::thread> ts;
    ts.reserve(block);
    for (unsigned t = 0; t < block; t++)
      ts.emplace_back([t, &fn] {
        threadIdx.x = t;
        fn();
      });
    for (auto& th : ts) th.join();
    shim_block_barrier = nullptr;
  }
}
