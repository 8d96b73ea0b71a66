// GPU encoders: ORC RLE v1 and RLE v2 files in CODAG's layouts (include/codag.h,
// codag_compress_rlev1/_rlev2).
//
// CODAG encodes on the GPU with one thread per chunk (rlev1/encoder.h:1728-1847 setup_deflate_orig
// / deflate_orig, rlev2/encoder_trans.h:184-357 block_encode_orig driven by compress_gpu_orig
// :482-564), then scans the stream lengths and moves every stream to its aligned offset.  The
// same three steps run here as three kernels on the caller's stream:
//   k_encode_rlev1_warp  RLE v1: one warp per chunk runs the shared writer of ../rle_writers.h (the
//                    code the host producers run, so the bytes are the same) into its own slot of
//                    the caller's workspace, literal streams and runs 32 values at a time;
//   k_encode_rlev2_warp  RLE v2: one warp per chunk runs the same writer, its group operations
//                    split over the lanes (see below);
//   k_scan_offsets   one CTA turns the stream lengths into the aligned offsets (blk_off);
//   k_gather         one warp per chunk copies its stream to its offset with the alignment
//                    padding zeroed, and fills col_len.
// Nothing is allocated; a stream that overruns its workspace slot, or a file larger than the
// caller's output capacity, is reported in *d_status.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../../include/codag.h"
#include "../rle_writers.h"

namespace {

constexpr uint64_t kOverflow = ~0ull;


// element j of one chunk of the input zero padded past in_bytes (d_in is element aligned)
template <typename T>
struct PaddedChunk {
  const uint8_t* in;
  uint64_t in_bytes;
  uint64_t base;
  __device__ T operator()(uint64_t j) const {
    const uint64_t o = base + j * sizeof(T);
    if (o + sizeof(T) <= in_bytes) return __ldg(reinterpret_cast<const T*>(in + o));
    T v = 0;
    for (uint32_t k = 0; k < sizeof(T); k++)
      if (o + k < in_bytes) v = static_cast<T>(v | (static_cast<T>(in[o + k]) << (8 * k)));
    return v;
  }
};

// Same integer types as the host producer reads the values with.
template <typename T>
struct Wide;
template <>
struct Wide<uint8_t> { using T = unsigned char; };
template <>
struct Wide<uint16_t> { using T = unsigned short; };
template <>
struct Wide<uint32_t> { using T = unsigned int; };
template <>
struct Wide<uint64_t> { using T = unsigned long long; };


// ---------------------------------------------------------------------------------------
// RLE v2, one warp per chunk.  With one thread per chunk the 32 threads of a warp take
// different paths through the writer's decisions (a warp ran them largely one after another,
// 6.4 GB/s on 1 GiB).  Here every lane of a warp runs the writer on the same chunk (same values,
// same branches, the pending values and the patch list in shared memory, every lane storing the
// same value to the same place), and WarpGroups splits each group operation over the lanes.
// The writer's decisions are the ones the host producers run, so the bytes are the same.
// ---------------------------------------------------------------------------------------
constexpr uint32_t FULL_MASK = 0xffffffffu;

// output of one warp: lane 0 writes the writer's single bytes, all lanes write packed bodies
struct WarpSink {
  uint8_t* p;
  uint64_t cap;
  uint64_t n;  // the same on every lane
  uint32_t lane;
  __device__ void put(uint8_t b) {
    if (lane == 0 && n < cap) p[n] = b;
    n++;
  }
  __device__ void put_at(uint64_t k, uint8_t b) {
    if (n + k < cap) p[n + k] = b;
  }
  __device__ void advance(uint64_t k) { n += k; }
  __device__ uint64_t size() const { return n; }
  __device__ void set(uint64_t i, uint8_t b) {
    if (lane == 0 && i < cap) p[i] = b;
  }
};

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__device__ __forceinline__ uint64_t umax64(uint64_t a, uint64_t b) { return a > b ? a : b; }

// codag_fmt::SerialGroups' operations, split over the 32 lanes; each starts and ends with the warp
// converged, so what one lane writes the others read afterwards and no lane overwrites what
// another still reads
struct WarpGroups {
  uint64_t* lit;   // kMaxLiterals pending values (shared memory)
  uint64_t* list;  // kMaxLiterals patch entries (shared memory)
  uint32_t* hs;    // 32 histogram counters (shared memory)
  uint32_t lane;
  using Scan = codag_fmt::SerialGroups::Scan;
  static constexpr bool kBulk = true;
  __device__ uint64_t* lits() { return lit; }

  // Up to min(32, lim) values i, i+1, ... that extend a variable run: lane k takes value i+k and
  // its step from the value before; the run stops before the first value whose step and the
  // step before it are both zero (the writer's fixed-run test) and at the end of the input.
  // Appends the values taken to l[nl..], leaves the last step taken in prev_delta, and returns
  // the count (0: the writer's per-value steps take value i).
  template <class Get>
  __device__ uint32_t append_run(const Get& get, uint64_t i, uint64_t n, uint64_t* l, uint32_t nl,
                                 uint64_t& prev_delta, uint32_t lim) const {
    __syncwarp();
    const uint64_t j = i + lane;
    const bool in = j < n;
    const uint64_t v = in ? static_cast<uint64_t>(get(j)) : 0ull;
    uint64_t before = __shfl_up_sync(FULL_MASK, v, 1);
    if (lane == 0) before = l[nl - 1];
    const uint64_t d = v - before;
    const uint32_t zero = __ballot_sync(FULL_MASK, in && d == 0);
    const uint32_t zero_before = (zero << 1) | (prev_delta == 0 ? 1u : 0u);
    const uint32_t stop = (zero & zero_before) | __ballot_sync(FULL_MASK, !in);
    uint32_t take = stop ? static_cast<uint32_t>(__ffs(stop)) - 1u : 32u;
    if (take > lim) take = lim;
    if (lane < take) l[nl + lane] = v;
    if (take) prev_delta = __shfl_sync(FULL_MASK, d, static_cast<int>(take - 1));
    __syncwarp();
    return take;
  }

  // Up to min(32, lim) values i, i+1, ... equal to the last pending value (a fixed run going on),
  // appended to l[nl..]; returns the count
  template <class Get>
  __device__ uint32_t append_equal(const Get& get, uint64_t i, uint64_t n, uint64_t* l, uint32_t nl,
                                   uint32_t lim) const {
    __syncwarp();
    const uint64_t last = l[nl - 1];
    const uint64_t j = i + lane;
    const bool eq = j < n && static_cast<uint64_t>(get(j)) == last;
    const uint32_t stop = __ballot_sync(FULL_MASK, !eq);
    uint32_t take = stop ? static_cast<uint32_t>(__ffs(stop)) - 1u : 32u;
    if (take > lim) take = lim;
    if (lane < take) l[nl + lane] = last;
    __syncwarp();
    return take;
  }
  __device__ uint64_t* lists() { return list; }

  __device__ Scan scan(const uint64_t* l, uint32_t n) const {
    __syncwarp();
    const uint64_t initial = l[1] - l[0];
    uint64_t lmin = l[0], lmax = l[0], md = 0;
    bool inc = true, dec = true, fix = true;
    for (uint32_t i = 1 + lane; i < n; i += 32) {
      const uint64_t l1 = l[i], l0 = l[i - 1], d = l1 - l0;
      lmin = umin64(lmin, l1);
      lmax = umax64(lmax, l1);
      inc &= l0 <= l1;
      dec &= l0 >= l1;
      fix &= d == initial;
      md = umax64(md, d);
    }
    for (int o = 16; o; o >>= 1) {
      lmin = umin64(lmin, __shfl_xor_sync(FULL_MASK, lmin, o));
      lmax = umax64(lmax, __shfl_xor_sync(FULL_MASK, lmax, o));
      md = umax64(md, __shfl_xor_sync(FULL_MASK, md, o));
    }
    Scan r{lmin, lmax, md, __all_sync(FULL_MASK, inc) != 0, __all_sync(FULL_MASK, dec) != 0,
           __all_sync(FULL_MASK, fix) != 0};
    return r;
  }

  template <class D>
  __device__ void hist(const D& d, uint32_t n, uint8_t* h) const {
    __syncwarp();
    hs[lane] = 0;
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32) atomicAdd(&hs[v2_code(codag_fmt::closest_width(d(i)))], 1u);
    __syncwarp();
    for (int k = 0; k < 32; k++) h[k] = static_cast<uint8_t>(hs[k]);
    __syncwarp();
  }

  // output byte k of the aligned packing, computed by lane k mod 32
  template <class S, class D>
  __device__ void pack_aligned(S& out, const D& d, uint32_t n, uint8_t bits) const {
    __syncwarp();
    uint64_t total;
    if (bits < 8) {
      const uint32_t per = 8u / bits;
      const uint32_t mask = (1u << bits) - 1u;
      total = (n + per - 1) / per;
      for (uint64_t k = lane; k < total; k += 32) {
        uint32_t b = 0;
        for (uint32_t j = 0; j < per; j++) {
          const uint64_t i = k * per + j;
          if (i < n) b |= (static_cast<uint32_t>(d(static_cast<uint32_t>(i))) & mask) << (8u - (j + 1u) * bits);
        }
        out.put_at(k, static_cast<uint8_t>(b));
      }
    } else {
      const uint32_t bytes = bits / 8u;
      total = static_cast<uint64_t>(n) * bytes;
      for (uint64_t k = lane; k < total; k += 32) {
        const uint32_t i = static_cast<uint32_t>(k / bytes);
        const uint32_t j = bytes - 1u - static_cast<uint32_t>(k % bytes);
        out.put_at(k, static_cast<uint8_t>(d(i) >> (8u * j)));
      }
    }
    out.advance(total);
    __syncwarp();
  }

  // output byte k of the MSB-first packing: the bits of every value that overlaps it
  template <class S, class D>
  __device__ void pack_unaligned(S& out, const D& d, uint32_t n, uint8_t bits) const {
    __syncwarp();
    const uint64_t tb = static_cast<uint64_t>(n) * bits, total = (tb + 7) / 8;
    for (uint64_t k = lane; k < total; k += 32) {
      const uint64_t s = 8 * k, e = s + 8 < tb ? s + 8 : tb;
      uint32_t byte = 0;
      for (uint64_t i = s / bits; i * bits < e; i++) {
        const uint64_t vs = i * bits, ve = vs + bits;
        const uint64_t a = vs > s ? vs : s, b = ve < e ? ve : e;
        const uint64_t field = (d(static_cast<uint32_t>(i)) >> (ve - b)) & ((1ull << (b - a)) - 1ull);
        byte |= static_cast<uint32_t>(field << (s + 8 - b));
      }
      out.put_at(k, static_cast<uint8_t>(byte));
    }
    out.advance(total);
    __syncwarp();
  }

  __device__ uint32_t patches(const uint64_t* l, uint32_t n, uint64_t lmin, uint64_t mask, uint32_t b95,
                              uint32_t pwidth, uint64_t* out, uint64_t* max_gap) const {
    static_assert(codag_fmt::kMaxLiterals == 128, "four rounds of 32 values");
    __syncwarp();
    uint32_t before = 0;
    int32_t prev_pos = -1;  // last patched position of the earlier rounds
    uint64_t mg = 0;
#pragma unroll
    for (uint32_t q = 0; q < 4; q++) {
      const uint32_t i = q * 32 + lane;
      const uint64_t r = i < n ? l[i] - lmin : 0ull;
      const bool hit = i < n && r > mask;
      const uint32_t bq = __ballot_sync(FULL_MASK, hit);
      if (hit) {
        const uint32_t below = bq & ((1u << lane) - 1u);
        const uint32_t prev = below ? q * 32 + 31 - __clz(below) : (prev_pos >= 0 ? static_cast<uint32_t>(prev_pos) : 0u);
        const uint64_t gap = i - prev;
        out[before + __popc(below)] = (gap << pwidth) | (r >> b95);
        mg = umax64(mg, gap);
      }
      if (bq) prev_pos = static_cast<int32_t>(q * 32 + 31 - __clz(bq));
      before += __popc(bq);
    }
    for (int o = 16; o; o >>= 1) mg = umax64(mg, __shfl_xor_sync(FULL_MASK, mg, o));
    *max_gap = mg;
    __syncwarp();
    return before;
  }
};

constexpr uint32_t kEncWarps = 4;

// codag_fmt::RleV1Writer's bulk steps for a warp whose lanes all run the writer on one chunk
struct WarpV1 {
  static constexpr bool kBulk = true;
  uint32_t lane_;
  __device__ uint32_t lane() const { return lane_; }
  __device__ uint32_t ballot(bool p) const { return __ballot_sync(FULL_MASK, p); }
  __device__ uint32_t ffs(uint32_t m) const { return static_cast<uint32_t>(__ffs(m)); }
  __device__ void sync() const { __syncwarp(); }
  template <typename V>
  __device__ V shfl(V v, int src) const {
    if constexpr (sizeof(V) == 8) return static_cast<V>(__shfl_sync(FULL_MASK, static_cast<unsigned long long>(v), src));
    else return static_cast<V>(__shfl_sync(FULL_MASK, static_cast<uint32_t>(v), src));
  }
  // the value of the lane below (lane 0 gets its own)
  template <typename V>
  __device__ V shfl_up(V v) const {
    if constexpr (sizeof(V) == 8) return static_cast<V>(__shfl_up_sync(FULL_MASK, static_cast<unsigned long long>(v), 1));
    else return static_cast<V>(__shfl_up_sync(FULL_MASK, static_cast<uint32_t>(v), 1));
  }
  // sum of v over the lanes below
  __device__ uint32_t excl_sum(uint32_t v) const {
    uint32_t s = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(FULL_MASK, s, d);
      if (lane_ >= static_cast<uint32_t>(d)) s += o;
    }
    return s - v;
  }
};

// RLE v1, one warp per chunk: every lane runs the writer on the same values (lane 0 writes its
// single bytes); literal streams and runs going on are taken 32 values at a time (WarpV1)
template <typename T>
__global__ void __launch_bounds__(32 * kEncWarps) k_encode_rlev1_warp(const uint8_t* __restrict__ in, uint64_t in_bytes,
                                                                     uint64_t chunk_bytes, uint64_t n,
                                                                     uint8_t* __restrict__ scratch, uint64_t slot,
                                                                     uint64_t* __restrict__ lens) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kEncWarps + (threadIdx.x >> 5);
  if (i >= n) return;  // the whole warp
  WarpSink s{scratch + i * slot, slot, 0, lane};
  using W = typename Wide<T>::T;
  const PaddedChunk<W> get{in, in_bytes, i * chunk_bytes};
  codag_fmt::RleV1Writer<T, WarpSink, WarpV1> w(s, WarpV1{lane});
  w.encode([&](uint64_t j) { return static_cast<T>(get(j)); }, chunk_bytes / sizeof(T));
  if (lane == 0) lens[i] = s.n > slot ? kOverflow : s.n;
}

template <typename T>
__global__ void __launch_bounds__(32 * kEncWarps) k_encode_rlev2_warp(const uint8_t* __restrict__ in, uint64_t in_bytes,
                                                                     uint64_t chunk_bytes, uint64_t n,
                                                                     uint8_t* __restrict__ scratch, uint64_t slot,
                                                                     uint64_t* __restrict__ lens) {
  __shared__ uint64_t s_lit[kEncWarps][codag_fmt::kMaxLiterals];
  __shared__ uint64_t s_list[kEncWarps][codag_fmt::kMaxLiterals];
  __shared__ uint32_t s_h[kEncWarps][32];
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kEncWarps + w;
  if (i >= n) return;  // the whole warp
  WarpSink s{scratch + i * slot, slot, 0, lane};
  const WarpGroups g{s_lit[w], s_list[w], s_h[w], lane};
  using W = typename Wide<T>::T;
  const PaddedChunk<W> get{in, in_bytes, i * chunk_bytes};
  codag_fmt::RleV2Writer<WarpSink, WarpGroups> wr(s, g);
  wr.encode([&](uint64_t j) { return static_cast<uint64_t>(get(j)); }, chunk_bytes / sizeof(T));
  if (lane == 0) lens[i] = s.n > slot ? kOverflow : s.n;
}

// blk_off[i] = sum of round_up(lens[k], ALIGN) for k < i, blk_off[n] = the total; one CTA of
// 1024 threads, each summing a contiguous range.
template <uint64_t ALIGN>
__global__ void __launch_bounds__(1024) k_scan_offsets(const uint64_t* __restrict__ lens, uint64_t n,
                                                       uint64_t* __restrict__ blk_off, int32_t* __restrict__ status) {
  __shared__ uint64_t part[1024];
  __shared__ int bad;
  const uint32_t t = threadIdx.x;
  if (t == 0) bad = 0;
  const uint64_t per = (n + 1023) / 1024, a = t * per, b = a + per < n ? a + per : n;
  uint64_t s = 0;
  for (uint64_t i = a; i < b; i++) {
    const uint64_t l = lens[i];
    if (l == kOverflow) bad = 1;
    s += (l + ALIGN - 1) / ALIGN * ALIGN;
  }
  part[t] = s;
  __syncthreads();
  for (uint32_t d = 1; d < 1024; d <<= 1) {  // inclusive scan of the partial sums
    const uint64_t o = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += o;
    __syncthreads();
  }
  uint64_t run = part[t] - s;
  for (uint64_t i = a; i < b; i++) {
    blk_off[i] = run;
    run += (lens[i] + ALIGN - 1) / ALIGN * ALIGN;
  }
  if (t == 1023) blk_off[n] = part[1023];
  if (t == 0 && bad && status) *status = CODAG_ECORRUPT;
}

// One warp per chunk: stream i goes to out + head + blk_off[i] and is zero padded to ALIGN
// bytes.  RLE v1 (head 8): the blob starts with the original size.  RLE v2: blk_off[n] is
// overwritten with the original size.  The file is out_bytes = head + blk_off[n] long.
template <uint64_t ALIGN, uint32_t HEAD>
__global__ void __launch_bounds__(256) k_gather(const uint8_t* __restrict__ scratch, uint64_t slot,
                                                const uint64_t* __restrict__ lens, uint64_t n, uint8_t* __restrict__ out,
                                                uint64_t capacity, uint64_t* __restrict__ blk_off,
                                                uint64_t* __restrict__ col_len, uint64_t in_bytes,
                                                uint64_t* __restrict__ out_bytes, int32_t* __restrict__ status) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  const uint64_t total = HEAD + blk_off[n];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (out_bytes) *out_bytes = total;
    if (total > capacity && status) *status = CODAG_ELIMIT;
    if (HEAD == 8 && capacity >= 8) *reinterpret_cast<uint64_t*>(out) = in_bytes;
  }
  if (total > capacity) return;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const uint64_t len = lens[i], off = HEAD + blk_off[i];
    if (lane == 0) col_len[i] = len;
    if (len == kOverflow) continue;
    const uint64_t padded = (len + ALIGN - 1) / ALIGN * ALIGN;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(scratch + i * slot);
    uint32_t* dst = reinterpret_cast<uint32_t*>(out + off);  // 4-byte aligned: HEAD, ALIGN multiples of 4
    for (uint64_t w = lane; w < padded / 4; w += 32) {
      uint32_t v = 0;
      const uint64_t b0 = 4 * w;
      if (b0 + 4 <= len) {
        v = src[w];
      } else if (b0 < len) {
        v = src[w] & ((1u << (8 * (len - b0))) - 1u);  // keep the stream's bytes, zero the padding
      }
      dst[w] = v;
    }
  }
}

__global__ void k_set_last_offset(uint64_t* blk_off, uint64_t n, uint64_t in_bytes) { blk_off[n] = in_bytes; }

bool valid_elem(int e) { return e == 1 || e == 2 || e == 4 || e == 8; }

uint64_t chunks_of(uint64_t in_bytes, uint64_t chunk_bytes) {
  return (in_bytes + chunk_bytes * 32 - 1) / (chunk_bytes * 32) * 32;  // rlev1.h:111-112, encoder_trans.h:490
}

// Workspace slot per chunk: the longest stream a chunk can give, 16-byte aligned.  RLE v1: every
// value a varint of ceil(8E/7) bytes plus a header per 127 literals; RLE v2: at most 1.25x the
// input for 64-bit values, taken as 2x plus a margin for every width.
uint64_t slot_of(int codec, uint64_t chunk_bytes, int e) {
  const uint64_t cnt = chunk_bytes / static_cast<uint64_t>(e);
  const uint64_t b = codec == CODAG_CODEC_RLEV1 ? cnt * ((8u * e + 6u) / 7u) + cnt / 127u + 64u : 2u * chunk_bytes + 4096u;
  return (b + 15u) / 16u * 16u;
}

template <int CODEC, typename T>
void launch_encode(const uint8_t* in, uint64_t in_bytes, uint64_t chunk, uint64_t n, uint8_t* scratch, uint64_t slot,
                   uint64_t* lens, cudaStream_t s) {
  if constexpr (CODEC == CODAG_CODEC_RLEV2) {
    k_encode_rlev2_warp<T><<<static_cast<unsigned>((n + kEncWarps - 1) / kEncWarps), 32 * kEncWarps, 0, s>>>(
        in, in_bytes, chunk, n, scratch, slot, lens);
  } else {
    k_encode_rlev1_warp<T><<<static_cast<unsigned>((n + kEncWarps - 1) / kEncWarps), 32 * kEncWarps, 0, s>>>(
        in, in_bytes, chunk, n, scratch, slot, lens);
  }
}

template <int CODEC>
codag_status compress(const uint8_t* d_in, uint64_t in_bytes, uint64_t chunk, int e, uint8_t* d_out, uint64_t capacity,
                      uint64_t* d_blk_off, uint64_t* d_col_len, uint64_t* d_out_bytes, int32_t* d_status, void* ws,
                      uint64_t ws_bytes, cudaStream_t s) {
  if (!d_in || !d_out || !d_blk_off || !d_col_len || !valid_elem(e) || chunk == 0 || chunk % e || in_bytes == 0 ||
      chunk >= (1ull << 31) || (reinterpret_cast<uintptr_t>(d_in) % e) || (reinterpret_cast<uintptr_t>(d_out) & 15u))
    return CODAG_EINVAL;
  if (CODEC == CODAG_CODEC_RLEV1 && chunk / e < 2) return CODAG_EINVAL;
  const uint64_t n = chunks_of(in_bytes, chunk), slot = slot_of(CODEC, chunk, e);
  if (!ws || ws_bytes < codag_compress_workspace_bytes(CODEC, in_bytes, chunk, e) ||
      (reinterpret_cast<uintptr_t>(ws) & 255u))
    return CODAG_EINVAL;
  (void)cudaGetLastError();  // an error earlier work left pending is not this call's
  uint8_t* scratch = static_cast<uint8_t*>(ws);
  uint64_t* lens = reinterpret_cast<uint64_t*>(scratch + n * slot);
  if (d_status && cudaMemsetAsync(d_status, 0, sizeof(int32_t), s) != cudaSuccess) return CODAG_ECUDA;
  switch (e) {
    case 8: launch_encode<CODEC, uint64_t>(d_in, in_bytes, chunk, n, scratch, slot, lens, s); break;
    case 4: launch_encode<CODEC, uint32_t>(d_in, in_bytes, chunk, n, scratch, slot, lens, s); break;
    case 2: launch_encode<CODEC, uint16_t>(d_in, in_bytes, chunk, n, scratch, slot, lens, s); break;
    default: launch_encode<CODEC, uint8_t>(d_in, in_bytes, chunk, n, scratch, slot, lens, s); break;
  }
  constexpr uint64_t A = CODEC == CODAG_CODEC_RLEV1 ? 4 : 128;  // encoder.h:780-783 / encoder_trans.h:352
  constexpr uint32_t H = CODEC == CODAG_CODEC_RLEV1 ? 8 : 0;    // rlev1.h:103-192: [u64 size][streams]
  k_scan_offsets<A><<<1, 1024, 0, s>>>(lens, n, d_blk_off, d_status);
  const uint64_t blocks = (n + 7) / 8;
  k_gather<A, H><<<static_cast<unsigned>(blocks < 4096 ? blocks : 4096), 256, 0, s>>>(
      scratch, slot, lens, n, d_out, capacity, d_blk_off, d_col_len, in_bytes, d_out_bytes, d_status);
  if (CODEC == CODAG_CODEC_RLEV2) k_set_last_offset<<<1, 1, 0, s>>>(d_blk_off, n, in_bytes);  // encoder_trans.h:545
  return cudaGetLastError() == cudaSuccess ? CODAG_OK : CODAG_ECUDA;
}

}  // namespace

extern "C" uint64_t codag_compress_chunks(uint64_t in_bytes, uint64_t chunk_bytes) {
  return chunk_bytes ? chunks_of(in_bytes, chunk_bytes) : 0;
}

extern "C" uint64_t codag_compress_workspace_bytes(int codec, uint64_t in_bytes, uint64_t chunk_bytes, int elem_bytes) {
  if ((codec != CODAG_CODEC_RLEV1 && codec != CODAG_CODEC_RLEV2) || !valid_elem(elem_bytes) || !chunk_bytes) return 0;
  const uint64_t n = chunks_of(in_bytes, chunk_bytes);
  return n * slot_of(codec, chunk_bytes, elem_bytes) + n * 8;
}

extern "C" uint64_t codag_compress_bound(int codec, uint64_t in_bytes, uint64_t chunk_bytes, int elem_bytes) {
  if ((codec != CODAG_CODEC_RLEV1 && codec != CODAG_CODEC_RLEV2) || !valid_elem(elem_bytes) || !chunk_bytes) return 0;
  const uint64_t n = chunks_of(in_bytes, chunk_bytes), slot = slot_of(codec, chunk_bytes, elem_bytes);
  return codec == CODAG_CODEC_RLEV1 ? 8 + n * ((slot + 3) / 4 * 4) : n * ((slot + 127) / 128 * 128);
}

extern "C" codag_status codag_compress_rlev1(const uint8_t* d_in, uint64_t in_bytes, uint64_t chunk_bytes,
                                             int elem_bytes, uint8_t* d_blob, uint64_t blob_capacity,
                                             uint64_t* d_blk_off, uint64_t* d_col_len, uint64_t* d_blob_bytes,
                                             int32_t* d_status, void* d_workspace, uint64_t workspace_bytes,
                                             codag_stream_t stream) {
  return compress<CODAG_CODEC_RLEV1>(d_in, in_bytes, chunk_bytes, elem_bytes, d_blob, blob_capacity, d_blk_off,
                                     d_col_len, d_blob_bytes, d_status, d_workspace, workspace_bytes,
                                     reinterpret_cast<cudaStream_t>(stream));
}

extern "C" codag_status codag_compress_rlev2(const uint8_t* d_in, uint64_t in_bytes, uint64_t chunk_bytes,
                                             int elem_bytes, uint8_t* d_comp, uint64_t comp_capacity,
                                             uint64_t* d_blk_off, uint64_t* d_col_len, uint64_t* d_comp_bytes,
                                             int32_t* d_status, void* d_workspace, uint64_t workspace_bytes,
                                             codag_stream_t stream) {
  return compress<CODAG_CODEC_RLEV2>(d_in, in_bytes, chunk_bytes, elem_bytes, d_comp, comp_capacity, d_blk_off,
                                     d_col_len, d_comp_bytes, d_status, d_workspace, workspace_bytes,
                                     reinterpret_cast<cudaStream_t>(stream));
}
