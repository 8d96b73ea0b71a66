// Kernels and extern "C" entry points of the decompressors (include/codag.h).
//
// Plain per-file launches: one warp per chunk, `warps_per_cta` chunks per CTA, each warp
// with its own slice of dynamic shared memory (TMA input ring + output ring [+ Huffman
// scratch]).  Batched launches: a persistent grid sized to the occupancy limit whose warps
// pull chunk descriptors from a device queue (one atomic per chunk) until it is empty.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <new>
#include <type_traits>
#include <vector>

#include "decode_deflate.cuh"
#include "decode_rle.cuh"
#include "walk_rle.cuh"

using namespace codag_dev;

namespace {

// ---------------------------------------------------------------------------------------
// per-warp shared memory layouts
// ---------------------------------------------------------------------------------------
constexpr uint32_t align_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

using RleOut = OutRing<12, 10, true>;  // 4 KiB ring, 1 KiB drains by TMA bulk stores
// The plain Deflate kernel sizes its window with the literal table (lut_bits), at two
// measured points.  9 bits: 1 KiB window, 256 B drains, 7.5 KiB of shared memory per warp, 28
// warps per SM; more back-references read the flushed output in global memory (a copy whose
// source ends more than 508 bytes back is always flushed already) and more codes miss the
// table, but with many chunks the extra resident warps win: 1 GiB of text in 22.6 ms.  10 or
// 11 bits: 2 KiB window, 512 B drains (10.5 KiB per warp with 10 bits, 20 warps per SM): 25%
// fewer instructions per chunk, faster when there are too few chunks to fill the SMs.  The
// batch kernel uses the same windows: its RLE values never pass through them.
template <int LB>
struct InflateWinOf {
  using T = OutRing<11, 9>;
};
template <>
struct InflateWinOf<9> {
  using T = OutRing<10, 8>;
};

template <int NSLOT>
struct RleLayout {
  static constexpr uint32_t kIn = 0;
  static constexpr uint32_t kOut = kIn + NSLOT * kSlotBytes;
  static constexpr uint32_t kBar = kOut + RleOut::kBytes;
  static constexpr uint32_t kPerWarp = align_up(kBar + NSLOT * 8, 128);
};

// RLE with DirectOut: no output ring
template <int NSLOT>
struct RleDirectLayout {
  static constexpr uint32_t kIn = 0;
  static constexpr uint32_t kBar = kIn + NSLOT * kSlotBytes;
  static constexpr uint32_t kPerWarp = align_up(kBar + NSLOT * 8, 128);
};

template <int NSLOT, int LB, class OUT, class SCR = InflateScratch<LB>>
struct InflateLayout {
  static constexpr uint32_t kIn = 0;
  static constexpr uint32_t kOut = kIn + NSLOT * kSlotBytes;
  static constexpr uint32_t kScratch = kOut + OUT::kBytes;
  static constexpr uint32_t kBar = align_up(kScratch + sizeof(SCR), 16);
  static constexpr uint32_t kPerWarp = align_up(kBar + NSLOT * 8, 128);
};

struct ChunkGeom {
  uint64_t off, len, out_base, store;
};

__device__ __forceinline__ uint64_t store_bytes(uint64_t base, uint64_t chunk_bytes, uint64_t out_bytes) {
  return base < out_bytes ? (chunk_bytes < out_bytes - base ? chunk_bytes : out_bytes - base) : 0;
}

__device__ __forceinline__ bool valid_elem_dev(uint32_t e) { return e == 1 || e == 2 || e == 4 || e == 8; }

__device__ __forceinline__ bool stream_in_bounds(uint64_t off, uint64_t len, uint64_t comp_bytes) {
  return off <= comp_bytes && len <= comp_bytes - off && len < (1ull << 28);
}

// ---------------------------------------------------------------------------------------
// plain kernels: chunk = blockIdx.x * warps + warp
// ---------------------------------------------------------------------------------------
// header walk, one thread per chunk; descriptors and counts go to the workspace
template <int CODEC>
__global__ void __launch_bounds__(128) k_rle_walk(const uint8_t* __restrict__ comp, uint64_t comp_bytes,
                                                  const uint64_t* __restrict__ blk_off,
                                                  const uint64_t* __restrict__ col_len, uint64_t n_chunks,
                                                  uint32_t cap, uint32_t* __restrict__ counts,
                                                  RleDesc* __restrict__ descs) {
  const uint64_t chunk = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (chunk >= n_chunks) return;
  const uint64_t off = blk_off[chunk], len = col_len[chunk];
  uint32_t k = kWalkFallback;
  if (stream_in_bounds(off, len, comp_bytes)) {
    const GStream g{comp + off, static_cast<uint32_t>(len), comp, comp + comp_bytes};
    RleDesc* d = descs + chunk * kDescPerChunk;
    k = CODEC == CODAG_CODEC_RLEV1 ? walk_rlev1(g, cap, d) : walk_rlev2(g, cap, d);
  }
  counts[chunk] = k;
}

template <int NSLOT, int CODEC, int E, bool DIRECT>
__global__ void __launch_bounds__(256) k_rle_plain(const uint8_t* __restrict__ comp, uint64_t comp_bytes,
                                                   const uint64_t* __restrict__ blk_off,
                                                   const uint64_t* __restrict__ col_len, uint64_t n_chunks,
                                                   uint64_t chunk_bytes, uint8_t* __restrict__ out,
                                                   uint64_t out_bytes, int32_t* __restrict__ status,
                                                   uint64_t wait_cycles, const uint32_t* __restrict__ counts,
                                                   const RleDesc* __restrict__ descs) {
  extern __shared__ __align__(128) uint8_t smem[];
  using L = std::conditional_t<DIRECT, RleDirectLayout<NSLOT>, RleLayout<NSLOT>>;
  using OUT = std::conditional_t<DIRECT, DirectOut, RleOut>;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint64_t chunk = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
  if (chunk >= n_chunks) return;
  uint8_t* base = smem + warp * L::kPerWarp;
  InRing<NSLOT> in;
  in.buf = base + L::kIn;
  in.sbuf = smem_u32(in.buf);
  in.bar = reinterpret_cast<uint64_t*>(base + L::kBar);
  in.phase = 0;
  in.wait_cycles = wait_cycles;
  in.lane = lane;
  OUT o;
  if constexpr (!DIRECT) {
    o.buf = base + L::kOut;
    o.sbuf = smem_u32(o.buf);
  }
  o.lane = lane;
  init_ring_barriers<NSLOT>(in.bar, lane);

  const uint64_t off = blk_off[chunk], len = col_len[chunk];
  const uint64_t cbase = chunk * chunk_bytes;
  int st;
  if (!stream_in_bounds(off, len, comp_bytes)) {
    st = CODAG_ECORRUPT;
  } else {
    in.begin(comp + off, static_cast<uint32_t>(len));
    o.begin(out + cbase, store_bytes(cbase, chunk_bytes, out_bytes));
    const uint32_t cap = static_cast<uint32_t>(chunk_bytes / E);
    const uint32_t nd = counts ? counts[chunk] : kWalkFallback;
    if (nd != kWalkFallback) {
      const RleDesc* d = descs + chunk * kDescPerChunk;
      st = CODEC == CODAG_CODEC_RLEV1 ? expand_rlev1<NSLOT, E>(in, o, d, nd) : expand_rlev2<NSLOT, E>(in, o, d, nd);
    } else {
      st = CODEC == CODAG_CODEC_RLEV1 ? decode_rlev1_chunk<NSLOT, E>(in, o, cap) : decode_rlev2_chunk<NSLOT, E>(in, o, cap);
    }
  }
  if (status && lane == 0) status[chunk] = st;
}

template <int NSLOT, int LB>
__global__ void __launch_bounds__(256) k_inflate_plain(const uint8_t* __restrict__ comp, uint64_t comp_bytes,
                                                       const uint64_t* __restrict__ blk_off, uint64_t n_chunks,
                                                       uint64_t chunk_bytes, uint32_t wrapper,
                                                       uint8_t* __restrict__ out, uint64_t out_bytes,
                                                       int32_t* __restrict__ status, uint64_t wait_cycles) {
  extern __shared__ __align__(128) uint8_t smem[];
  using W = typename InflateWinOf<LB>::T;
  using L = InflateLayout<NSLOT, LB, W>;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint64_t chunk = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
  if (chunk >= n_chunks) return;
  uint8_t* base = smem + warp * L::kPerWarp;
  InRing<NSLOT> in;
  in.buf = base + L::kIn;
  in.sbuf = smem_u32(in.buf);
  in.bar = reinterpret_cast<uint64_t*>(base + L::kBar);
  in.phase = 0;
  in.wait_cycles = wait_cycles;
  in.lane = lane;
  W o;
  o.buf = base + L::kOut;
  o.sbuf = smem_u32(o.buf);
  o.lane = lane;
  auto& sc = *reinterpret_cast<InflateScratch<LB>*>(base + L::kScratch);
  init_ring_barriers<NSLOT>(in.bar, lane);

  const uint64_t off = blk_off[chunk], next = blk_off[chunk + 1];
  const uint64_t cbase = chunk * chunk_bytes;
  int st;
  if (next < off || !stream_in_bounds(off, next - off, comp_bytes)) {
    st = CODAG_ECORRUPT;
  } else {
    in.begin(comp + off, static_cast<uint32_t>(next - off));
    o.begin(out + cbase, store_bytes(cbase, chunk_bytes, out_bytes));
    st = decode_deflate_chunk<NSLOT, LB>(in, o, sc, sc.lit_lut, sc.dist_lut, chunk_bytes, wrapper);
  }
  if (status && lane == 0) status[chunk] = st;
}

// One CTA of two warps per Deflate chunk (codag_tune.cta_per_chunk): warp 2p decodes the symbols
// of chunk p of the CTA into tokens, warp 2p+1 expands them (decode_deflate.cuh, TokenPipe /
// expand_tokens); pair p synchronises on named barrier p+1.
template <int NSLOT, int LB>
struct InflatePairLayout {
  using W = typename InflateWinOf<LB>::T;
  static constexpr uint32_t kIn = 0;
  static constexpr uint32_t kBar = kIn + NSLOT * kSlotBytes;
  static constexpr uint32_t kScratch = align_up(kBar + NSLOT * 8, 16);
  static constexpr uint32_t kOut = align_up(kScratch + sizeof(InflateScratch<LB>), 128);
  static constexpr uint32_t kTok = kOut + W::kBytes;
  static constexpr uint32_t kPerPair = align_up(kTok + sizeof(TokenShared), 128);
};

template <int NSLOT, int LB>
__global__ void __launch_bounds__(256) k_inflate_cta(const uint8_t* __restrict__ comp, uint64_t comp_bytes,
                                                     const uint64_t* __restrict__ blk_off, uint64_t n_chunks,
                                                     uint64_t chunk_bytes, uint32_t wrapper, uint8_t* __restrict__ out,
                                                     uint64_t out_bytes, int32_t* __restrict__ status,
                                                     uint64_t wait_cycles) {
  extern __shared__ __align__(128) uint8_t smem[];
  using L = InflatePairLayout<NSLOT, LB>;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, pair = warp >> 1;
  const uint64_t chunk = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 6) + pair;
  uint8_t* base = smem + pair * L::kPerPair;
  TokenShared* sh = reinterpret_cast<TokenShared*>(base + L::kTok);
  if ((warp & 1u) == 0 && lane == 0) sh->done = 0;
  __syncthreads();
  if (chunk >= n_chunks) return;  // both warps of the pair leave together
  const uint32_t bar = pair + 1u;
  const uint64_t off = blk_off[chunk], next = blk_off[chunk + 1];
  const uint64_t cbase = chunk * chunk_bytes;
  const bool bad = next < off || !stream_in_bounds(off, next - off, comp_bytes);
  if ((warp & 1u) == 0) {  // decoder
    InRing<NSLOT> in;
    in.buf = base + L::kIn;
    in.sbuf = smem_u32(in.buf);
    in.bar = reinterpret_cast<uint64_t*>(base + L::kBar);
    in.phase = 0;
    in.wait_cycles = wait_cycles;
    in.lane = lane;
    init_ring_barriers<NSLOT>(in.bar, lane);
    auto& sc = *reinterpret_cast<InflateScratch<LB>*>(base + L::kScratch);
    TokenPipe pipe{sh, bar, 0, 0, lane};
    int st = CODAG_ECORRUPT;
    if (!bad) {
      in.begin(comp + off, static_cast<uint32_t>(next - off));
      NullOut none;
      st = decode_deflate_chunk<NSLOT, LB>(in, none, sc, sc.lit_lut, sc.dist_lut, chunk_bytes, wrapper, &pipe);
    }
    pipe.finish(st);
  } else {  // expander
    typename L::W o;
    o.buf = base + L::kOut;
    o.sbuf = smem_u32(o.buf);
    o.lane = lane;
    o.begin(out + cbase, store_bytes(cbase, chunk_bytes, out_bytes));
    const int est = expand_tokens(sh, bar, o, lane);
    const int dst = sh->status;
    if (status && lane == 0) status[chunk] = dst != CODAG_OK ? dst : est;
  }
}

// ---------------------------------------------------------------------------------------
// batched persistent kernel
// ---------------------------------------------------------------------------------------
// The Deflate window is the plain kernel's (InflateWinOf<LB>), small enough for many resident
// warps; RLE values go straight to global memory (element by element when the output is
// element aligned, byte by byte otherwise), so no RLE header needs the window.
// With n_pair > 0 (a plan made with cta_per_chunk), the first n_pair entries of the work order
// are large Deflate files taken by pairs of warps: warp 2p of a CTA decodes the symbols into
// tokens, warp 2p+1 expands them, the tokens passing through the expander's idle input ring
// (TokenShared), each job fenced by named barrier p+1; the pair counter is queue[1].  When those
// run out, every warp pulls the remaining entries on its own from queue[0].
// GT: the Huffman lookup tables live in global memory (gtab, kLutEntries<LB> words per warp of
// the grid, read through L1) instead of shared memory.
template <int NSLOT, int LB, bool GT>
__global__ void __launch_bounds__(256) k_batch(const codag_chunk_desc* __restrict__ descs,
                                               const uint32_t* __restrict__ order, uint64_t n,
                                               uint32_t* __restrict__ queue, const uint8_t* __restrict__ comp,
                                               uint64_t comp_bytes, uint8_t* __restrict__ out, uint64_t out_bytes,
                                               int32_t* __restrict__ status, uint64_t wait_cycles, uint32_t n_pair,
                                               uint32_t* __restrict__ gtab) {
  extern __shared__ __align__(128) uint8_t smem[];
  using W = typename InflateWinOf<LB>::T;
  using SCR = std::conditional_t<GT, InflateCodes, InflateScratch<LB>>;
  using L = InflateLayout<NSLOT, LB, W, SCR>;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint8_t* base = smem + warp * L::kPerWarp;
  InRing<NSLOT> in;
  in.buf = base + L::kIn;
  in.sbuf = smem_u32(in.buf);
  in.bar = reinterpret_cast<uint64_t*>(base + L::kBar);
  in.phase = 0;
  in.wait_cycles = wait_cycles;
  in.lane = lane;
  W o;
  o.buf = base + L::kOut;
  o.sbuf = smem_u32(o.buf);
  o.lane = lane;
  DirectOut od;
  od.lane = lane;
  ByteOut ob;
  ob.lane = lane;
  auto& sc = *reinterpret_cast<SCR*>(base + L::kScratch);
  uint32_t *lit_lut, *dist_lut;
  if constexpr (GT) {
    lit_lut = gtab + (static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + warp) * kLutEntries<LB>;
    dist_lut = lit_lut + (1u << LB);
  } else {
    lit_lut = sc.lit_lut;
    dist_lut = sc.dist_lut;
  }
  init_ring_barriers<NSLOT>(in.bar, lane);

  if (n_pair) {  // large Deflate files, one pair of warps each
    const uint32_t bar = (warp >> 1) + 1u;
    const bool decoder = (warp & 1u) == 0;
    TokenShared* sh = reinterpret_cast<TokenShared*>(smem + (warp | 1u) * L::kPerWarp + L::kIn);
    for (;;) {
      if (decoder && lane == 0) {
        sh->job = atomicAdd(queue + 1, 1u);
        sh->done = 0;
      }
      pair_barrier(bar);
      const uint32_t k = sh->job;
      if (k >= n_pair) break;
      const uint32_t i = order[k];
      const codag_chunk_desc d = descs[i];
      const bool ok = d.codec == CODAG_CODEC_DEFLATE && d.out_off <= out_bytes && d.out_len <= out_bytes - d.out_off &&
                      stream_in_bounds(d.comp_off, d.comp_len, comp_bytes);
      if (decoder) {
        TokenPipe pipe{sh, bar, 0, 0, lane};
        int st = CODAG_ECORRUPT;
        if (ok) {
          in.begin(comp + d.comp_off, d.comp_len);
          NullOut none;
          st = decode_deflate_chunk<NSLOT, LB, NullOut, TokenPipe, GT>(in, none, sc, lit_lut, dist_lut, d.out_len,
                                                                      d.wrapper_bytes, &pipe);
        }
        pipe.finish(st);
      } else {
        o.begin(out + d.out_off, ok ? d.out_len : 0);
        const int est = expand_tokens(sh, bar, o, lane);
        const int dst = sh->status;
        if (status && lane == 0) status[i] = dst != CODAG_OK ? dst : est;
      }
      const bool timed_out = sh->status == CODAG_ETIMEOUT;
      pair_barrier(bar);  // the expander has read this job's status before the next job begins
      if (timed_out) return;  // ring state unknown: both warps stop
    }
    order += n_pair;
    n -= n_pair;
  }

  for (;;) {
    uint32_t k = 0;
    if (lane == 0) k = atomicAdd(queue, 1u);
    k = __shfl_sync(FULL, k, 0);
    if (k >= n) break;
    const uint32_t i = order ? order[k] : k;
    const codag_chunk_desc d = descs[i];
    int st;
    const bool out_ok = d.out_off <= out_bytes && d.out_len <= out_bytes - d.out_off;
    if (!out_ok || !stream_in_bounds(d.comp_off, d.comp_len, comp_bytes)) {
      st = CODAG_ECORRUPT;
    } else {
      in.begin(comp + d.comp_off, d.comp_len);
      if (d.codec == CODAG_CODEC_DEFLATE) {
        o.begin(out + d.out_off, d.out_len);
        st = decode_deflate_chunk<NSLOT, LB, typename InflateWinOf<LB>::T, NoTokens, GT>(
            in, o, sc, lit_lut, dist_lut, d.out_len, d.wrapper_bytes);
      } else if (d.codec == CODAG_CODEC_RLEV1 || d.codec == CODAG_CODEC_RLEV2) {
        const uint32_t e = d.elem_bytes;
        if (valid_elem_dev(e) && (reinterpret_cast<uintptr_t>(out + d.out_off) % e) == 0 && d.out_len % e == 0) {
          od.begin(out + d.out_off, d.out_len);
          st = decode_rle_any<NSLOT>(d.codec, in, od, d.out_len, static_cast<int>(e));
        } else {
          ob.begin(out + d.out_off, d.out_len);
          st = decode_rle_any<NSLOT>(d.codec, in, ob, d.out_len, d.elem_bytes);
        }
      } else {
        st = CODAG_EINVAL;
      }
    }
    if (status && lane == 0) status[i] = st;
    if (st == CODAG_ETIMEOUT) break;  // ring state unknown: this warp stops pulling work
  }
}

// ---------------------------------------------------------------------------------------
// one CTA per chunk (RLE, values straight to global memory)
// ---------------------------------------------------------------------------------------
// The CTA copies the whole stream into shared memory, warp 0 walks the headers into
// shared-memory descriptors (with each header's first value index), and every warp expands
// an equal share of the descriptors.  A stream larger than the staging buffer, or one whose
// walk gives up (malformed, more headers than the descriptor budget), is decoded by warp 0
// in one pass with the usual TMA ring, which reports the exact error.
constexpr uint32_t kStageBytes = 64u << 10;
constexpr int kStageSlots = static_cast<int>(kStageBytes >> kSlotLog2);
struct CtaLayout {
  static constexpr uint32_t kStage = 0;
  static constexpr uint32_t kDesc = kStage + kStageBytes;
  static constexpr uint32_t kNStart = kDesc + kDescPerChunk * sizeof(RleDesc);
  static constexpr uint32_t kBar = kNStart + kDescPerChunk * 4;
  static constexpr uint32_t kMisc = kBar + 64;
  static constexpr uint32_t kBytes = kMisc + 64;
};

template <int CODEC, int E>
__global__ void __launch_bounds__(256) k_rle_cta(const uint8_t* __restrict__ comp, uint64_t comp_bytes,
                                                 const uint64_t* __restrict__ blk_off,
                                                 const uint64_t* __restrict__ col_len, uint64_t n_chunks,
                                                 uint64_t chunk_bytes, uint8_t* __restrict__ out, uint64_t out_bytes,
                                                 int32_t* __restrict__ status, uint64_t wait_cycles) {
  extern __shared__ __align__(128) uint8_t smem[];
  using L = CtaLayout;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint64_t chunk = blockIdx.x;
  if (chunk >= n_chunks) return;
  uint8_t* stage = smem + L::kStage;
  RleDesc* desc = reinterpret_cast<RleDesc*>(smem + L::kDesc);
  uint32_t* nstart = reinterpret_cast<uint32_t*>(smem + L::kNStart);
  uint32_t* misc = reinterpret_cast<uint32_t*>(smem + L::kMisc);  // [0] descriptors, [1] status, [2] values
  const uint64_t off = blk_off[chunk], len = col_len[chunk];
  const uint64_t cbase = chunk * chunk_bytes;
  const uint32_t cap = static_cast<uint32_t>(chunk_bytes / E);
  const bool inb = stream_in_bounds(off, len, comp_bytes);
  const uintptr_t a = reinterpret_cast<uintptr_t>(comp + off);
  const uint8_t* g0 = reinterpret_cast<const uint8_t*>(a & ~static_cast<uintptr_t>(15));
  const uint32_t lo = static_cast<uint32_t>(a & 15);
  const uint32_t hi = inb ? lo + static_cast<uint32_t>(len) : 0u;
  const bool staged = inb && hi <= kStageBytes;
  if (threadIdx.x == 0) {
    misc[0] = kWalkFallback;
    misc[1] = CODAG_OK;
    misc[2] = 0;
  }
  if (staged) {  // 16-byte granules covering [lo, hi); bytes outside the buffer read as 0
    const uint8_t* end = comp + comp_bytes;
    for (uint32_t g = threadIdx.x; g < (hi + 15u) >> 4; g += blockDim.x) {
      const uint8_t* q = g0 + 16u * g;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (q >= comp && q + 16 <= end) {
        v = __ldg(reinterpret_cast<const uint4*>(q));
      } else {
        uint32_t w[4] = {0, 0, 0, 0};
        for (int i = 0; i < 16; i++)
          if (q + i >= comp && q + i < end) w[i >> 2] |= static_cast<uint32_t>(__ldg(q + i)) << (8 * (i & 3));
        v = make_uint4(w[0], w[1], w[2], w[3]);
      }
      *reinterpret_cast<uint4*>(stage + 16u * g) = v;
    }
  }
  fence_proxy_async_smem();  // the one-pass fallback may refill the stage by TMA
  // a fully resident view of the stage (every slot counted as arrived, nothing to release)
  InRing<kStageSlots> in;
  in.buf = stage;
  in.sbuf = smem_u32(stage);
  in.bar = nullptr;
  in.gbase = g0;
  in.lo = lo;
  in.hi = hi;
  in.nslots = (hi + kSlotBytes - 1) >> kSlotLog2;
  in.issued = in.waited = in.nslots;
  in.ready = in.nslots << kSlotLog2;
  in.release_at = 0xffffffffu;
  in.phase = 0;
  in.wait_cycles = wait_cycles;
  in.lane = lane;
  __syncthreads();
  if (staged && warp == 0) {  // RLE v1: the whole warp walks; RLE v2: one thread
    uint32_t k;
    if constexpr (CODEC == CODAG_CODEC_RLEV1) {
      k = walk_rlev1_warp(in, static_cast<uint32_t>(len), cap, desc, nstart, lane);
    } else {
      k = 0;
      if (lane == 0) {
        const SStream sv{smem_u32(stage), lo, static_cast<uint32_t>(len), kStageBytes - 1u};
        k = walk_rlev2(sv, cap, desc, nstart);
      }
    }
    __syncwarp();
    if (lane == 0) {
      misc[0] = k;
      if (k != kWalkFallback && k) misc[2] = nstart[k - 1] + ((desc[k - 1].info >> 7) & 0x1ffu);
    }
  }
  __syncthreads();
  const uint32_t nd = misc[0];
  DirectOut o;
  o.lane = lane;
  if (nd == kWalkFallback) {
    if (warp == 0) {  // one pass through a TMA ring in the (unused) staging buffer
      InRing<4> ring;
      ring.buf = stage;
      ring.sbuf = smem_u32(stage);
      ring.bar = reinterpret_cast<uint64_t*>(smem + L::kBar);
      ring.phase = 0;
      ring.wait_cycles = wait_cycles;
      ring.lane = lane;
      init_ring_barriers<4>(ring.bar, lane);
      int st = CODAG_ECORRUPT;
      if (inb) {
        ring.begin(comp + off, static_cast<uint32_t>(len));
        o.begin(out + cbase, store_bytes(cbase, chunk_bytes, out_bytes));
        st = CODEC == CODAG_CODEC_RLEV1 ? decode_rlev1_chunk<4, E>(ring, o, cap) : decode_rlev2_chunk<4, E>(ring, o, cap);
      }
      if (status && lane == 0) status[chunk] = st;
    }
    return;
  }
  // every warp expands descriptors [k0, k1)
  o.begin(out + cbase, store_bytes(cbase, chunk_bytes, out_bytes));
  const uint32_t k0 = static_cast<uint32_t>((static_cast<uint64_t>(nd) * warp) / nw);
  const uint32_t k1 = static_cast<uint32_t>((static_cast<uint64_t>(nd) * (warp + 1)) / nw);
  if (k0 < k1) {
    uint32_t n = nstart[k0];
    const int st = CODEC == CODAG_CODEC_RLEV1 ? expand_rlev1_range<kStageSlots, E, true>(in, o, desc, k0, k1, n)
                                              : expand_rlev2_range<kStageSlots, E, true>(in, o, desc, k0, k1, n);
    if (st && lane == 0) atomicMax(&misc[1], static_cast<uint32_t>(st));
  }
  __syncthreads();
  if (threadIdx.x == 0 && status) {
    int st = static_cast<int>(misc[1]);
    if (st == CODAG_OK && static_cast<uint64_t>(misc[2]) * E < o.store) st = CODAG_ECORRUPT;
    status[chunk] = st;
  }
}

// A wait that no copy ever completes: exercises the bounded-wait path of InRing.
__global__ void k_selftest_timeout(int32_t* status, uint64_t wait_cycles) {
  __shared__ __align__(128) uint8_t buf[kSlotBytes];
  __shared__ uint64_t bar[1];
  const uint32_t lane = threadIdx.x & 31u;
  InRing<1> in;
  in.buf = buf;
  in.sbuf = smem_u32(buf);
  in.bar = bar;
  in.phase = 0;
  in.wait_cycles = wait_cycles;
  in.lane = lane;
  init_ring_barriers<1>(bar, lane);
  if (lane == 0) mbar_arrive_expect_tx(&bar[0], 16);  // 16 bytes are expected, none is sent
  __syncwarp();
  const bool ok = in.wait_slot(0);
  if (lane == 0) *status = ok ? CODAG_OK : CODAG_ETIMEOUT;
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
std::mutex g_mu;
codag_tune g_tune[3] = {{8, 4, 10, 0, 0}, {8, 4, 10, 0, 0}, {2, 2, 9, 0, 0}};
uint64_t g_wait_cycles = 2000000000ull;  // about one second at 2 GHz

bool valid_slots(int s) { return s == 2 || s == 4 || s == 8; }
bool valid_lut(int b) { return b == 9 || b == 10 || b == 11; }
bool valid_warps(int w) { return w >= 1 && w <= 8; }
bool valid_elem(int e) { return e == 1 || e == 2 || e == 4 || e == 8; }

codag_tune tune_of(int codec) {
  std::lock_guard<std::mutex> g(g_mu);
  return g_tune[codec];
}
uint64_t wait_of() {
  std::lock_guard<std::mutex> g(g_mu);
  return g_wait_cycles;
}

// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the current device.  The
// limit is per kernel, and one instantiation serves shapes of different sizes (a batched plan
// of 8 warps per CTA and one of 2 share k_batch<4, 10>), so it is only ever raised: lowering it
// for a small shape would make a later launch of a larger one, or a plan made earlier, fail.
std::mutex g_smem_mu;
std::vector<std::pair<std::pair<const void*, int>, uint32_t>> g_smem_max;  // (kernel, device) -> limit set
template <class K>
cudaError_t allow_smem(K kernel, uint32_t bytes) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  const void* key = reinterpret_cast<const void*>(kernel);
  std::lock_guard<std::mutex> g(g_smem_mu);
  for (auto& e : g_smem_max)
    if (e.first.first == key && e.first.second == dev) {
      if (e.second >= bytes) return cudaSuccess;
      err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
      if (err == cudaSuccess) e.second = bytes;
      return err;
    }
  err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  if (err == cudaSuccess) g_smem_max.push_back({{key, dev}, bytes});
  return err;
}

// An entry point clears a CUDA error that earlier work of the process left pending (for
// example an allocation that a caching allocator retried after freeing memory), so that the
// check after its own launches reports only errors of those launches.
void clear_stale_error() { (void)cudaGetLastError(); }

codag_status finish_launch() {
  const cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) return CODAG_OK;
  std::fprintf(stderr, "codag: kernel launch failed: %s\n", cudaGetErrorName(err));
  return CODAG_ECUDA;
}

// workspace of the two-pass RLE path: per-chunk descriptor counts, then descriptor tables
constexpr uint64_t rle_ws_counts_bytes(uint64_t n) { return (n * 4 + 255) / 256 * 256; }
constexpr uint64_t rle_ws_bytes(uint64_t n) { return rle_ws_counts_bytes(n) + n * kDescPerChunk * sizeof(RleDesc); }

template <int NSLOT, int CODEC, int E, bool DIRECT>
codag_status launch_rle_out(const codag_tune& t, const uint8_t* comp, uint64_t comp_bytes, const uint64_t* blk_off,
                            const uint64_t* col_len, uint64_t n, uint64_t chunk_bytes, uint8_t* out,
                            uint64_t out_bytes, int32_t* status, void* ws, uint64_t ws_bytes, cudaStream_t s) {
  using L = std::conditional_t<DIRECT, RleDirectLayout<NSLOT>, RleLayout<NSLOT>>;
  const uint32_t smem = L::kPerWarp * t.warps_per_cta;
  auto kern = k_rle_plain<NSLOT, CODEC, E, DIRECT>;
  if (allow_smem(kern, smem) != cudaSuccess) return CODAG_ECUDA;
  const uint64_t grid = (n + t.warps_per_cta - 1) / t.warps_per_cta;
  if (grid > 0x7fffffffull) return CODAG_EINVAL;
  uint32_t* counts = nullptr;
  RleDesc* descs = nullptr;
  if (ws && ws_bytes >= rle_ws_bytes(n) && (reinterpret_cast<uintptr_t>(ws) & 255) == 0) {
    counts = static_cast<uint32_t*>(ws);
    descs = reinterpret_cast<RleDesc*>(static_cast<uint8_t*>(ws) + rle_ws_counts_bytes(n));
    k_rle_walk<CODEC><<<static_cast<unsigned>((n + 127) / 128), 128, 0, s>>>(
        comp, comp_bytes, blk_off, col_len, n, static_cast<uint32_t>(chunk_bytes / E), counts, descs);
  }
  kern<<<static_cast<unsigned>(grid), 32 * t.warps_per_cta, smem, s>>>(comp, comp_bytes, blk_off, col_len, n,
                                                                         chunk_bytes, out, out_bytes, status,
                                                                         wait_of(), counts, descs);
  return finish_launch();
}

template <int CODEC, int E>
codag_status launch_rle_cta(const codag_tune& t, const uint8_t* comp, uint64_t comp_bytes, const uint64_t* blk_off,
                            const uint64_t* col_len, uint64_t n, uint64_t chunk_bytes, uint8_t* out,
                            uint64_t out_bytes, int32_t* status, cudaStream_t s) {
  auto kern = k_rle_cta<CODEC, E>;
  if (allow_smem(kern, CtaLayout::kBytes) != cudaSuccess) return CODAG_ECUDA;
  if (n > 0x7fffffffull) return CODAG_EINVAL;
  kern<<<static_cast<unsigned>(n), 32 * t.warps_per_cta, CtaLayout::kBytes, s>>>(
      comp, comp_bytes, blk_off, col_len, n, chunk_bytes, out, out_bytes, status, wait_of());
  return finish_launch();
}

// Values go straight to global memory when the output is element aligned (DirectOut),
// through the shared-memory ring otherwise; with cta_per_chunk (and no workspace) a whole
// CTA decodes each chunk.
template <int NSLOT, int CODEC, int E>
codag_status launch_rle(const codag_tune& t, const uint8_t* comp, uint64_t comp_bytes, const uint64_t* blk_off,
                        const uint64_t* col_len, uint64_t n, uint64_t chunk_bytes, uint8_t* out, uint64_t out_bytes,
                        int32_t* status, void* ws, uint64_t ws_bytes, cudaStream_t s) {
  // direct stores write whole elements: the output and out_bytes must be element aligned
  const bool direct = (reinterpret_cast<uintptr_t>(out) % E) == 0 && out_bytes % E == 0;
  if (direct && t.cta_per_chunk && !ws)
    return launch_rle_cta<CODEC, E>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, out, out_bytes, status, s);
  if (direct)
    return launch_rle_out<NSLOT, CODEC, E, true>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, out,
                                                 out_bytes, status, ws, ws_bytes, s);
  return launch_rle_out<NSLOT, CODEC, E, false>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, out, out_bytes,
                                                status, ws, ws_bytes, s);
}

template <int NSLOT, int CODEC>
codag_status launch_rle_e(const codag_tune& t, const uint8_t* comp, uint64_t comp_bytes, const uint64_t* blk_off,
                          const uint64_t* col_len, uint64_t n, uint64_t chunk_bytes, int e, uint8_t* out,
                          uint64_t out_bytes, int32_t* status, void* ws, uint64_t wsb, cudaStream_t s) {
  switch (e) {
    case 8: return launch_rle<NSLOT, CODEC, 8>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, out, out_bytes, status, ws, wsb, s);
    case 4: return launch_rle<NSLOT, CODEC, 4>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, out, out_bytes, status, ws, wsb, s);
    case 2: return launch_rle<NSLOT, CODEC, 2>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, out, out_bytes, status, ws, wsb, s);
    default: return launch_rle<NSLOT, CODEC, 1>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, out, out_bytes, status, ws, wsb, s);
  }
}

template <int NSLOT, int LB>
codag_status launch_inflate(const codag_tune& t, const uint8_t* comp, uint64_t comp_bytes, const uint64_t* blk_off,
                            uint64_t n, uint64_t chunk_bytes, int wrapper, uint8_t* out, uint64_t out_bytes,
                            int32_t* status, cudaStream_t s) {
  using L = InflateLayout<NSLOT, LB, typename InflateWinOf<LB>::T>;
  const uint32_t smem = L::kPerWarp * t.warps_per_cta;
  auto kern = k_inflate_plain<NSLOT, LB>;
  if (allow_smem(kern, smem) != cudaSuccess) return CODAG_ECUDA;
  const uint64_t grid = (n + t.warps_per_cta - 1) / t.warps_per_cta;
  if (grid > 0x7fffffffull) return CODAG_EINVAL;
  kern<<<static_cast<unsigned>(grid), 32 * t.warps_per_cta, smem, s>>>(comp, comp_bytes, blk_off, n, chunk_bytes,
                                                                         static_cast<uint32_t>(wrapper), out,
                                                                         out_bytes, status, wait_of());
  return finish_launch();
}

template <int NSLOT, int LB>
codag_status launch_inflate_cta(const codag_tune& t, const uint8_t* comp, uint64_t comp_bytes, const uint64_t* blk_off,
                                uint64_t n, uint64_t chunk_bytes, int wrapper, uint8_t* out, uint64_t out_bytes,
                                int32_t* status, cudaStream_t s) {
  using L = InflatePairLayout<NSLOT, LB>;
  const uint32_t pairs = static_cast<uint32_t>(t.warps_per_cta) / 2u;
  const uint32_t smem = L::kPerPair * pairs;
  auto kern = k_inflate_cta<NSLOT, LB>;
  if (allow_smem(kern, smem) != cudaSuccess) return CODAG_ECUDA;
  const uint64_t grid = (n + pairs - 1) / pairs;
  if (grid > 0x7fffffffull) return CODAG_EINVAL;
  kern<<<static_cast<unsigned>(grid), 64 * pairs, smem, s>>>(comp, comp_bytes, blk_off, n, chunk_bytes,
                                                             static_cast<uint32_t>(wrapper), out, out_bytes, status,
                                                             wait_of());
  return finish_launch();
}

template <int CODEC>
codag_status dispatch_rle(const uint8_t* comp, uint64_t comp_bytes, const uint64_t* blk_off, const uint64_t* col_len,
                          uint64_t n, uint64_t chunk_bytes, int e, uint8_t* out, uint64_t out_bytes, int32_t* status,
                          void* ws, uint64_t wsb, cudaStream_t s) {
  if (!comp || !blk_off || !col_len || (!out && out_bytes) || !valid_elem(e) || chunk_bytes == 0 ||
      chunk_bytes % static_cast<uint64_t>(e) || chunk_bytes >= (1ull << 31))
    return CODAG_EINVAL;
  if (n == 0) return CODAG_OK;
  clear_stale_error();
  const codag_tune t = tune_of(CODEC);
  if (t.ring_slots == 4)
    return launch_rle_e<4, CODEC>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, e, out, out_bytes, status, ws, wsb, s);
  return launch_rle_e<8, CODEC>(t, comp, comp_bytes, blk_off, col_len, n, chunk_bytes, e, out, out_bytes, status, ws, wsb, s);
}

}  // namespace

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
extern "C" uint64_t codag_workspace_bytes(int codec, uint64_t n_chunks) {
  return (codec == CODAG_CODEC_RLEV1 || codec == CODAG_CODEC_RLEV2) ? rle_ws_bytes(n_chunks) : 0;
}

extern "C" codag_status codag_decompress_rlev1(const uint8_t* d_comp, uint64_t comp_bytes, const uint64_t* d_blk_off,
                                               const uint64_t* d_col_len, uint64_t n_chunks, uint64_t chunk_bytes,
                                               int elem_bytes, uint8_t* d_out, uint64_t out_bytes,
                                               int32_t* d_chunk_status, void* d_workspace, uint64_t workspace_bytes,
                                               codag_stream_t stream) {
  return dispatch_rle<CODAG_CODEC_RLEV1>(d_comp, comp_bytes, d_blk_off, d_col_len, n_chunks, chunk_bytes, elem_bytes,
                                         d_out, out_bytes, d_chunk_status, d_workspace, workspace_bytes,
                                         reinterpret_cast<cudaStream_t>(stream));
}

extern "C" codag_status codag_decompress_rlev2(const uint8_t* d_comp, uint64_t comp_bytes, const uint64_t* d_blk_off,
                                               const uint64_t* d_col_len, uint64_t n_chunks, uint64_t chunk_bytes,
                                               int elem_bytes, uint8_t* d_out, uint64_t out_bytes,
                                               int32_t* d_chunk_status, void* d_workspace, uint64_t workspace_bytes,
                                               codag_stream_t stream) {
  return dispatch_rle<CODAG_CODEC_RLEV2>(d_comp, comp_bytes, d_blk_off, d_col_len, n_chunks, chunk_bytes, elem_bytes,
                                         d_out, out_bytes, d_chunk_status, d_workspace, workspace_bytes,
                                         reinterpret_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------------------
// Two-pass RLE v2 decode for callers that cannot allocate device memory.
//
// The scratch is a fixed array in the module's device memory, sized for
// CODAG_NOALLOC_MAX_CHUNKS chunks; every device that loads this library holds it until the
// process exits.  In host code `g_noalloc_ws` only names a host-side shadow, so the device
// address is looked up once per device with cudaGetSymbolAddress (on the first call made
// with that device current) and passed to the kernels.  All calls share the array: the
// header walk rewrites the count of every chunk it is given before the expansion reads it,
// so no clearing is needed, and calls that overlap on the GPU race on the array.
// ---------------------------------------------------------------------------------------
namespace {
constexpr uint64_t kNoAllocScratchBytes = rle_ws_bytes(CODAG_NOALLOC_MAX_CHUNKS);
__device__ __align__(256) uint8_t g_noalloc_ws[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};

codag_status noalloc_scratch(void** addr) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return CODAG_ECUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return CODAG_EINVAL;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_ws) != cudaSuccess || !p) return CODAG_ECUDA;
    g_noalloc_addr[dev] = p;
  }
  *addr = g_noalloc_addr[dev];
  return CODAG_OK;
}
}  // namespace

extern "C" codag_status codag_decompress_rlev2_noalloc(const uint8_t* d_comp, uint64_t comp_bytes,
                                                       const uint64_t* d_blk_off, const uint64_t* d_col_len,
                                                       uint64_t n_chunks, uint64_t chunk_bytes, int elem_bytes,
                                                       uint8_t* d_out, uint64_t out_bytes, int32_t* d_chunk_status,
                                                       codag_stream_t stream) {
  if (!d_comp || !d_blk_off || !d_col_len || (!d_out && out_bytes) || !valid_elem(elem_bytes) || chunk_bytes == 0 ||
      chunk_bytes % static_cast<uint64_t>(elem_bytes) || chunk_bytes >= (1ull << 31))
    return CODAG_EINVAL;  // the checks of dispatch_rle, made before the capacity check
  if (n_chunks > CODAG_NOALLOC_MAX_CHUNKS) return CODAG_ELIMIT;
  if (n_chunks == 0) return CODAG_OK;
  void* ws = nullptr;
  const codag_status st = noalloc_scratch(&ws);
  if (st != CODAG_OK) return st;
  // The two-pass launch takes a workspace only when it is large and 256-byte aligned enough
  // (launch_rle_out); both hold by construction, and if either did not, this call reports it
  // instead of quietly decoding in one pass.
  if ((reinterpret_cast<uintptr_t>(ws) & 255u) != 0 || kNoAllocScratchBytes < rle_ws_bytes(n_chunks)) return CODAG_ECUDA;
  return dispatch_rle<CODAG_CODEC_RLEV2>(d_comp, comp_bytes, d_blk_off, d_col_len, n_chunks, chunk_bytes, elem_bytes,
                                         d_out, out_bytes, d_chunk_status, ws, kNoAllocScratchBytes,
                                         reinterpret_cast<cudaStream_t>(stream));
}

extern "C" codag_status codag_decompress_deflate(const uint8_t* d_comp, uint64_t comp_bytes, const uint64_t* d_blk_off,
                                                 uint64_t n_chunks, uint64_t chunk_bytes, int wrapper_bytes,
                                                 uint8_t* d_out, uint64_t out_bytes, int32_t* d_chunk_status,
                                                 codag_stream_t stream) {
  if (!d_comp || !d_blk_off || (!d_out && out_bytes) || chunk_bytes == 0 || chunk_bytes >= (1ull << 31) ||
      wrapper_bytes < 0 || wrapper_bytes > 16)
    return CODAG_EINVAL;
  if (n_chunks == 0) return CODAG_OK;
  clear_stale_error();
  const codag_tune t = tune_of(CODAG_CODEC_DEFLATE);
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
#define CODAG_INF(NS, LB)                                                                                               \
  return t.cta_per_chunk                                                                                                \
             ? launch_inflate_cta<NS, LB>(t, d_comp, comp_bytes, d_blk_off, n_chunks, chunk_bytes, wrapper_bytes, d_out, \
                                          out_bytes, d_chunk_status, s)                                                 \
             : launch_inflate<NS, LB>(t, d_comp, comp_bytes, d_blk_off, n_chunks, chunk_bytes, wrapper_bytes, d_out,     \
                                      out_bytes, d_chunk_status, s)
  if (t.ring_slots == 2) {
    if (t.lut_bits == 9) CODAG_INF(2, 9);
    if (t.lut_bits == 10) CODAG_INF(2, 10);
    CODAG_INF(2, 11);
  }
  if (t.ring_slots == 4) {
    if (t.lut_bits == 9) CODAG_INF(4, 9);
    if (t.lut_bits == 10) CODAG_INF(4, 10);
    CODAG_INF(4, 11);
  }
  if (t.lut_bits == 9) CODAG_INF(8, 9);
  if (t.lut_bits == 10) CODAG_INF(8, 10);
  CODAG_INF(8, 11);
#undef CODAG_INF
}

extern "C" codag_status codag_set_tune(int codec, const codag_tune* tune) {
  if (codec < 0 || codec > 2 || !tune || !valid_warps(tune->warps_per_cta) || !valid_slots(tune->ring_slots) ||
      !valid_lut(tune->lut_bits))
    return CODAG_EINVAL;
  // an RLE v2 header with its data spans up to 2060 bytes; it must fit the window of
  // (slots - 1) KiB ahead of the read position
  if (codec != CODAG_CODEC_DEFLATE && tune->ring_slots < 4) return CODAG_EINVAL;
  if (tune->cta_per_chunk != 0 && tune->cta_per_chunk != 1) return CODAG_EINVAL;
  if (tune->table_global != 0) return CODAG_EINVAL;  // per-file calls: tables in shared memory (no workspace)
  // a Deflate chunk per CTA takes a decoder and an expander warp: an even count, up to 4 pairs
  if (codec == CODAG_CODEC_DEFLATE && tune->cta_per_chunk && (tune->warps_per_cta & 1)) return CODAG_EINVAL;
  std::lock_guard<std::mutex> g(g_mu);
  g_tune[codec] = *tune;
  return CODAG_OK;
}

extern "C" codag_status codag_get_tune(int codec, codag_tune* tune) {
  if (codec < 0 || codec > 2 || !tune) return CODAG_EINVAL;
  *tune = tune_of(codec);
  return CODAG_OK;
}

extern "C" codag_status codag_set_wait_limit(uint64_t cycles) {
  if (cycles == 0) return CODAG_EINVAL;
  std::lock_guard<std::mutex> g(g_mu);
  g_wait_cycles = cycles;
  return CODAG_OK;
}

extern "C" codag_status codag_selftest_wait_timeout(int32_t* d_status, codag_stream_t stream) {
  if (!d_status) return CODAG_EINVAL;
  clear_stale_error();
  k_selftest_timeout<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_status, wait_of());
  return finish_launch();
}

// ---------------------------------------------------------------------------------------
// batched plans
// ---------------------------------------------------------------------------------------
struct codag_plan {
  uint64_t n = 0;
  uint32_t n_pair = 0;  // leading entries of the order decoded by warp pairs (large Deflate files)
  codag_tune tune{};
  codag_chunk_desc* d_descs = nullptr;
  uint32_t* d_order = nullptr;
  uint32_t* d_queue = nullptr;
  uint32_t* d_tab = nullptr;  // Huffman lookup tables of every warp (tune.table_global)
  int grid = 0;
  // captured graph and the arguments it was captured with
  cudaGraphExec_t exec = nullptr;
  const void* g_comp = nullptr;
  const void* g_out = nullptr;
  const void* g_status = nullptr;
  uint64_t g_comp_bytes = 0, g_out_bytes = 0;
};

namespace {

template <int NSLOT, int LB, bool GT>
using BatchLayout = InflateLayout<NSLOT, LB, typename InflateWinOf<LB>::T,
                                  std::conditional_t<GT, InflateCodes, InflateScratch<LB>>>;

template <int NSLOT, int LB, bool GT>
codag_status batch_setup(codag_plan* p) {
  using L = BatchLayout<NSLOT, LB, GT>;
  const uint32_t smem = L::kPerWarp * p->tune.warps_per_cta;
  auto kern = k_batch<NSLOT, LB, GT>;
  if (allow_smem(kern, smem) != cudaSuccess) return CODAG_ECUDA;
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return CODAG_ECUDA;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * p->tune.warps_per_cta, smem) != cudaSuccess)
    return CODAG_ECUDA;
  per_sm = std::max(per_sm, 1);
  const uint64_t need = (p->n + p->tune.warps_per_cta - 1) / p->tune.warps_per_cta;
  p->grid = static_cast<int>(std::min<uint64_t>(need, static_cast<uint64_t>(sms) * per_sm));
  return CODAG_OK;
}

template <int NSLOT, int LB, bool GT>
codag_status batch_launch(codag_plan* p, const uint8_t* comp, uint64_t comp_bytes, uint8_t* out, uint64_t out_bytes,
                          int32_t* status, cudaStream_t s) {
  using L = BatchLayout<NSLOT, LB, GT>;
  const uint32_t smem = L::kPerWarp * p->tune.warps_per_cta;
  k_batch<NSLOT, LB, GT><<<p->grid, 32 * p->tune.warps_per_cta, smem, s>>>(
      p->d_descs, p->d_order, p->n, p->d_queue, comp, comp_bytes, out, out_bytes, status, wait_of(), p->n_pair,
      p->d_tab);
  return CODAG_OK;
}

// Calls f.template operator()<NSLOT, LB, GT>() for the plan's launch shape.
template <class F>
codag_status batch_dispatch(const codag_tune& t, F&& f) {
  const int key = t.ring_slots * 100 + t.lut_bits;
#define CODAG_BATCH_CASE(NS, LB)                                                               \
  case NS * 100 + LB:                                                                          \
    return t.table_global ? f.template operator()<NS, LB, true>() : f.template operator()<NS, LB, false>();
  switch (key) {
    CODAG_BATCH_CASE(2, 9)
    CODAG_BATCH_CASE(2, 10)
    CODAG_BATCH_CASE(2, 11)
    CODAG_BATCH_CASE(4, 9)
    CODAG_BATCH_CASE(4, 10)
    CODAG_BATCH_CASE(4, 11)
    CODAG_BATCH_CASE(8, 9)
    CODAG_BATCH_CASE(8, 10)
    default:
      return t.table_global ? f.template operator()<8, 11, true>() : f.template operator()<8, 11, false>();
  }
#undef CODAG_BATCH_CASE
}

codag_status batch_setup_any(codag_plan* p) {
  return batch_dispatch(p->tune, [&]<int NS, int LB, bool GT>() { return batch_setup<NS, LB, GT>(p); });
}

void batch_enqueue(codag_plan* p, const uint8_t* comp, uint64_t comp_bytes, uint8_t* out, uint64_t out_bytes,
                   int32_t* status, cudaStream_t s) {
  cudaMemsetAsync(p->d_queue, 0, (p->n_pair ? 2 : 1) * sizeof(uint32_t), s);
  batch_dispatch(p->tune, [&]<int NS, int LB, bool GT>() {
    return batch_launch<NS, LB, GT>(p, comp, comp_bytes, out, out_bytes, status, s);
  });
}

// lookup-table words of a plan whose tables live in global memory (every warp of the grid)
uint64_t table_words(const codag_plan* p) {
  const uint64_t per = p->tune.lut_bits == 9 ? kLutEntries<9> : p->tune.lut_bits == 10 ? kLutEntries<10> : kLutEntries<11>;
  return static_cast<uint64_t>(p->grid) * p->tune.warps_per_cta * per;
}

// work estimate used to order the queue: compressed bytes, Deflate weighted by its
// per-byte decode cost relative to the RLE codecs
// Launch shape of a batched call given no tune: 8 warps per CTA, 4 ring slots, 10-bit tables.
// The per-file Deflate default (2 warps per CTA) keeps too few warps per SM for a launch over
// thousands of chunks: a serving loop on one B200 sustained 36.6 GB/s with it, 60 GB/s with this.
constexpr codag_tune kBatchDefault = {8, 4, 10, 0, 0};

// In a plan made with cta_per_chunk = k (1..4), Deflate files of at least k x 256 KiB go to
// warp pairs
constexpr uint64_t kPairStepBytes = 256u << 10;

uint64_t chunk_cost(const codag_chunk_desc& d) {
  return d.codec == CODAG_CODEC_DEFLATE ? 8ull * d.comp_len + d.out_len : static_cast<uint64_t>(d.comp_len) + d.out_len / 4;
}

}  // namespace

extern "C" codag_status codag_batch_plan(const codag_chunk_desc* h_descs, uint64_t n, const codag_tune* tune,
                                         codag_plan** plan) {
  if (!h_descs || !plan || n == 0 || n > 0xffffffffull) return CODAG_EINVAL;
  codag_tune t = tune ? *tune : kBatchDefault;
  if (!valid_warps(t.warps_per_cta) || !valid_slots(t.ring_slots) || !valid_lut(t.lut_bits)) return CODAG_EINVAL;
  if (t.cta_per_chunk < 0 || t.cta_per_chunk > 4 || (t.cta_per_chunk && (t.warps_per_cta & 1))) return CODAG_EINVAL;
  if (t.table_global != 0 && t.table_global != 1) return CODAG_EINVAL;
  if (t.ring_slots < 4) t.ring_slots = 4;  // mixed batches include RLE chunks (and the token batches need 4 KiB)
  for (uint64_t i = 0; i < n; i++) {
    const codag_chunk_desc& d = h_descs[i];
    if (d.codec > CODAG_CODEC_DEFLATE) return CODAG_EINVAL;
    if (d.codec != CODAG_CODEC_DEFLATE && (!valid_elem(d.elem_bytes) || d.out_len % d.elem_bytes)) return CODAG_EINVAL;
  }
  codag_plan* p = new (std::nothrow) codag_plan();
  if (!p) return CODAG_ENOMEM;
  p->n = n;
  p->tune = t;
  std::vector<uint32_t> order(n);
  for (uint64_t i = 0; i < n; i++) order[i] = static_cast<uint32_t>(i);
  // with cta_per_chunk, the Deflate files of at least cta_per_chunk x 256 KiB go first, to warp pairs
  const uint64_t pair_min = static_cast<uint64_t>(t.cta_per_chunk) * kPairStepBytes;
  auto paired = [&](uint32_t i) {
    return t.cta_per_chunk && h_descs[i].codec == CODAG_CODEC_DEFLATE && h_descs[i].out_len >= pair_min;
  };
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    const bool pa = paired(a), pb = paired(b);
    if (pa != pb) return pa;
    return chunk_cost(h_descs[a]) > chunk_cost(h_descs[b]);
  });
  for (uint64_t i = 0; i < n && paired(order[i]); i++) p->n_pair++;
  if (cudaMalloc(&p->d_descs, n * sizeof(codag_chunk_desc)) != cudaSuccess ||
      cudaMalloc(&p->d_order, n * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&p->d_queue, 2 * sizeof(uint32_t)) != cudaSuccess ||
      cudaMemcpy(p->d_descs, h_descs, n * sizeof(codag_chunk_desc), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_order, order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
    codag_batch_destroy(p);
    return CODAG_ECUDA;
  }
  const codag_status st = batch_setup_any(p);
  if (st != CODAG_OK) {
    codag_batch_destroy(p);
    return st;
  }
  if (t.table_global && cudaMalloc(&p->d_tab, table_words(p) * sizeof(uint32_t)) != cudaSuccess) {
    codag_batch_destroy(p);
    return CODAG_ECUDA;
  }
  *plan = p;
  return CODAG_OK;
}

extern "C" codag_status codag_batch_run(codag_plan* p, const uint8_t* d_comp, uint64_t comp_bytes, uint8_t* d_out,
                                        uint64_t out_bytes, int32_t* d_status, int use_graph, codag_stream_t stream) {
  if (!p || !d_comp || !d_out) return CODAG_EINVAL;
  clear_stale_error();
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (!use_graph) {
    batch_enqueue(p, d_comp, comp_bytes, d_out, out_bytes, d_status, s);
    return finish_launch();
  }
  const bool same = p->exec && p->g_comp == d_comp && p->g_out == d_out && p->g_status == d_status &&
                    p->g_comp_bytes == comp_bytes && p->g_out_bytes == out_bytes;
  if (!same) {
    if (p->exec) {
      cudaGraphExecDestroy(p->exec);
      p->exec = nullptr;
    }
    cudaStream_t cap;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) return CODAG_ECUDA;
    cudaGraph_t g = nullptr;
    cudaError_t err = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      batch_enqueue(p, d_comp, comp_bytes, d_out, out_bytes, d_status, cap);
      err = cudaStreamEndCapture(cap, &g);
    }
    if (err == cudaSuccess) err = cudaGraphInstantiate(&p->exec, g, 0);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cap);
    if (err != cudaSuccess) {
      p->exec = nullptr;
      cudaGetLastError();
      return CODAG_ECUDA;
    }
    p->g_comp = d_comp;
    p->g_out = d_out;
    p->g_status = d_status;
    p->g_comp_bytes = comp_bytes;
    p->g_out_bytes = out_bytes;
  }
  return cudaGraphLaunch(p->exec, s) == cudaSuccess ? CODAG_OK : CODAG_ECUDA;
}

extern "C" codag_status codag_batch_destroy(codag_plan* p) {
  if (!p) return CODAG_EINVAL;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->d_descs) cudaFree(p->d_descs);
  if (p->d_order) cudaFree(p->d_order);
  if (p->d_queue) cudaFree(p->d_queue);
  if (p->d_tab) cudaFree(p->d_tab);
  delete p;
  return CODAG_OK;
}

// ---------------------------------------------------------------------------------------
// launches over caller-owned descriptor lists (continuous batching)
// ---------------------------------------------------------------------------------------
namespace {
struct LaunchShape {
  codag_tune tune;
  int grid_cap;  // SMs x resident CTAs of k_batch for this shape on the current device
  int dev;
};
std::mutex g_shape_mu;
std::vector<LaunchShape> g_shapes;

codag_status launch_shape(const codag_tune& t, int* grid_cap) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CODAG_ECUDA;
  {
    std::lock_guard<std::mutex> g(g_shape_mu);
    for (const LaunchShape& s : g_shapes)
      if (s.dev == dev && s.tune.warps_per_cta == t.warps_per_cta && s.tune.ring_slots == t.ring_slots &&
          s.tune.lut_bits == t.lut_bits) {
        *grid_cap = s.grid_cap;
        return CODAG_OK;
      }
  }
  codag_plan probe;
  probe.n = 0xffffffffull;
  probe.tune = t;
  const codag_status st = batch_setup_any(&probe);
  if (st != CODAG_OK) return st;
  std::lock_guard<std::mutex> g(g_shape_mu);
  g_shapes.push_back({t, probe.grid, dev});
  *grid_cap = probe.grid;
  return CODAG_OK;
}
}  // namespace

extern "C" codag_status codag_batch_launch(const codag_chunk_desc* d_descs, const uint32_t* d_order, uint64_t n,
                                           uint32_t* d_queue, const codag_tune* tune, const uint8_t* d_comp,
                                           uint64_t comp_bytes, uint8_t* d_out, uint64_t out_bytes,
                                           int32_t* d_status, codag_stream_t stream) {
  if (!d_descs || !d_queue || !d_comp || !d_out || n > 0xffffffffull) return CODAG_EINVAL;
  if (n == 0) return CODAG_OK;
  clear_stale_error();
  codag_plan p;
  p.n = n;
  p.tune = tune ? *tune : kBatchDefault;
  if (!valid_warps(p.tune.warps_per_cta) || !valid_slots(p.tune.ring_slots) || !valid_lut(p.tune.lut_bits))
    return CODAG_EINVAL;
  if (p.tune.ring_slots < 4) p.tune.ring_slots = 4;  // mixed batches include RLE chunks
  if (p.tune.table_global) return CODAG_EINVAL;         // no plan, so no global table scratch
  int cap = 0;
  const codag_status st = launch_shape(p.tune, &cap);
  if (st != CODAG_OK) return st;
  const uint64_t need = (n + p.tune.warps_per_cta - 1) / p.tune.warps_per_cta;
  p.grid = static_cast<int>(std::min<uint64_t>(need, static_cast<uint64_t>(cap)));
  p.d_descs = const_cast<codag_chunk_desc*>(d_descs);
  p.d_order = const_cast<uint32_t*>(d_order);
  p.d_queue = d_queue;
  batch_enqueue(&p, d_comp, comp_bytes, d_out, out_bytes, d_status, reinterpret_cast<cudaStream_t>(stream));
  p.d_descs = nullptr;  // borrowed: the destructor-free plan owns nothing
  p.d_order = nullptr;
  p.d_queue = nullptr;
  return finish_launch();
}
