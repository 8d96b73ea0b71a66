// Device building blocks shared by the chunk decoders (sm_100a).
//
//   InRing   the compressed stream of one chunk, staged into a shared-memory ring of 1 KiB
//            slots by TMA bulk copies (cp.async.bulk ... mbarrier::complete_tx).  The warp
//            that decodes the chunk is both producer and consumer: it issues the copies
//            for the slots ahead of its read position and waits on each slot's mbarrier
//            (bounded, see wait_slot) before reading it.  This replaces CODAG's
//            warp-cooperative refill (include/common_warp.h:730-950) and its spin queues
//            (common_warp.h:72-372).  Every copy is a plain single-CTA bulk copy.
//   OutRing  a shared-memory staging ring for decoded bytes, drained to global memory in
//            fixed-size pieces with coalesced 16-byte vector stores.
//
// Conventions: one warp decodes one chunk; every lane keeps an identical copy of the
// decoder state (control flow is warp-uniform); lane 0 issues the TMA copies.
#pragma once
#include <cstdint>

#include "../../../include/codag.h"

namespace codag_dev {

constexpr uint32_t FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t tx_bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(tx_bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Async-proxy ordering for shared memory that generic loads read before a TMA overwrites it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 1-D bulk copy global -> shared, completion counted on `bar` (this CTA only).
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// 1-D bulk copy shared -> global (TMA store), tracked in this thread's bulk async-group.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_s2g(void* gdst, uint32_t ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(ssrc), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until at most N of this thread's committed bulk groups still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Shared-memory accessors on 32-bit shared addresses (explicit ld/st.shared, no generic
// addressing).  Loads are volatile asm, so they stay ordered after the (volatile) barrier
// waits without pinning surrounding arithmetic; stores also clobber memory.
__device__ __forceinline__ uint32_t ld_s8(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ uint32_t ld_s16(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.u16 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ uint32_t ld_s32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ uint64_t ld_s64(uint32_t a) {
  uint64_t v;
  asm volatile("ld.shared.u64 %0, [%1];" : "=l"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ uint4 ld_s128(uint32_t a) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ void st_s8(uint32_t a, uint32_t v) {
  asm volatile("st.shared.u8 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void st_s16(uint32_t a, uint32_t v) {
  asm volatile("st.shared.u16 [%0], %1;" ::"r"(a), "h"(static_cast<unsigned short>(v)) : "memory");
}
__device__ __forceinline__ void st_s32(uint32_t a, uint32_t v) {
  asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void st_s64(uint32_t a, uint64_t v) {
  asm volatile("st.shared.u64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
}
__device__ __forceinline__ void st_g128(void* p, uint4 v) {
  asm volatile("st.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w) : "memory");
}

__device__ __forceinline__ uint64_t bswap64(uint64_t v) {
  const uint32_t lo = static_cast<uint32_t>(v), hi = static_cast<uint32_t>(v >> 32);
  return (static_cast<uint64_t>(__byte_perm(lo, 0, 0x0123)) << 32) | __byte_perm(hi, 0, 0x0123);
}

// shifts that give 0 for amounts >= 64 (the clamped PTX semantics the reference relies on)
__device__ __forceinline__ uint64_t shl64(uint64_t v, uint32_t s) { return s >= 64 ? 0ull : (v << s); }
__device__ __forceinline__ uint64_t shr64(uint64_t v, uint32_t s) { return s >= 64 ? 0ull : (v >> s); }

__device__ __forceinline__ uint64_t warp_or64(uint64_t v) {
  const uint32_t lo = __reduce_or_sync(FULL, static_cast<uint32_t>(v));
  const uint32_t hi = __reduce_or_sync(FULL, static_cast<uint32_t>(v >> 32));
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
  const uint32_t lo = __shfl_sync(FULL, static_cast<uint32_t>(v), src);
  const uint32_t hi = __shfl_sync(FULL, static_cast<uint32_t>(v >> 32), src);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

__device__ __forceinline__ uint64_t shfl_up64(uint64_t v, int d) {
  const uint32_t lo = __shfl_up_sync(FULL, static_cast<uint32_t>(v), d);
  const uint32_t hi = __shfl_up_sync(FULL, static_cast<uint32_t>(v >> 32), d);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

__device__ __forceinline__ uint64_t shfl_down64(uint64_t v, int d) {
  const uint32_t lo = __shfl_down_sync(FULL, static_cast<uint32_t>(v), d);
  const uint32_t hi = __shfl_down_sync(FULL, static_cast<uint32_t>(v >> 32), d);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

// inclusive warp prefix sum of 64-bit values
__device__ __forceinline__ uint64_t warp_scan_add64(uint64_t v, uint32_t lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint64_t o = shfl_up64(v, d);
    if (lane >= static_cast<uint32_t>(d)) v += o;
  }
  return v;
}

__device__ __forceinline__ uint32_t lanemask_lt(uint32_t lane) { return (1u << lane) - 1u; }

// ---------------------------------------------------------------------------------------
// TMA input ring
// ---------------------------------------------------------------------------------------
constexpr uint32_t kSlotLog2 = 10;
constexpr uint32_t kSlotBytes = 1u << kSlotLog2;

template <int NSLOT>
struct InRing {
  static constexpr uint32_t kBytes = NSLOT * kSlotBytes;
  static constexpr uint32_t kMask = kBytes - 1;
  static_assert((NSLOT & (NSLOT - 1)) == 0, "ring depth must be a power of two");

  uint8_t* buf;            // kBytes of shared memory, 16-byte aligned
  uint32_t sbuf;           // shared-space address of buf
  uint64_t* bar;           // NSLOT mbarriers
  const uint8_t* gbase;    // stream start rounded down to 16 bytes
  uint32_t lo, hi;         // stream bytes are [lo, hi) relative to gbase
  uint32_t nslots;         // slots covering [0, hi)
  uint32_t issued, waited; // slots issued / known complete for this chunk
  uint32_t ready;          // bytes below `ready` are resident (waited << kSlotLog2)
  uint32_t release_at;     // read position from which release() can issue another slot
  uint32_t phase;          // expected parity per barrier; persists across chunks
  uint64_t wait_cycles;    // bound of one wait
  uint32_t lane;

  // Binds the ring to the stream [src, src+len).  The barriers must be initialised.
  __device__ __forceinline__ void begin(const uint8_t* src, uint32_t len) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    gbase = reinterpret_cast<const uint8_t*>(a & ~static_cast<uintptr_t>(15));
    lo = static_cast<uint32_t>(a & 15);
    hi = lo + len;
    nslots = (hi + kSlotBytes - 1) >> kSlotLog2;
    issued = 0;
    waited = 0;
    ready = 0;
    release_at = 0;
  }

  // Cheap per-header bookkeeping: refill behind `pos` and make [.., end) resident.
  __device__ __forceinline__ int advance(uint32_t pos, uint32_t end) {
    if (pos >= release_at && !release(pos)) return CODAG_ETIMEOUT;
    return end <= ready ? CODAG_OK : ensure(end);
  }

  // Fill slot s: the 16-byte aligned body by TMA, the unaligned head/tail bytes by lanes.
  __device__ __forceinline__ void issue(uint32_t s) {
    const uint32_t r = s & (NSLOT - 1);
    const uint32_t slot_lo = s << kSlotLog2, slot_hi = slot_lo + kSlotBytes;
    const uint32_t body_lo = (lo + 15) & ~15u, body_hi = hi & ~15u;
    const uint32_t a = slot_lo > body_lo ? slot_lo : body_lo;
    const uint32_t b = slot_hi < body_hi ? slot_hi : body_hi;
    const uint32_t bytes = b > a ? b - a : 0;
    // head fragment [lo, min(body_lo, hi)) and tail fragment [max(body_hi, body_lo), hi)
    if (s == 0 && lane < 16) {
      const uint32_t p = lo + lane;
      const uint32_t head_end = body_lo < hi ? body_lo : hi;
      if (p < head_end) st_s8(sbuf + (p & kMask), gbase[p]);
    }
    const uint32_t tail_lo = body_hi > body_lo ? body_hi : body_lo;
    if (tail_lo < hi && s == ((hi - 1) >> kSlotLog2) && lane < 16) {
      const uint32_t p = tail_lo + lane;
      if (p < hi) st_s8(sbuf + (p & kMask), gbase[p]);
    }
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&bar[r], bytes);
      if (bytes) bulk_g2s(buf + (a & kMask), gbase + a, bytes, &bar[r]);
    }
  }

  // Bounded wait for slot s; false on timeout.
  __device__ __forceinline__ bool wait_slot(uint32_t s) {
    const uint32_t r = s & (NSLOT - 1);
    const uint32_t parity = (phase >> r) & 1u;
    bool ok = mbar_try_wait(&bar[r], parity);
    if (!ok) {
      const long long t0 = clock64();
      while (!(ok = mbar_try_wait(&bar[r], parity))) {
        if (static_cast<uint64_t>(clock64() - t0) > wait_cycles) break;
      }
    }
    ok = __all_sync(FULL, ok);
    if (ok) phase ^= 1u << r;
    return ok;
  }

  // Issues the slots ahead of read position `pos` (everything below pos is consumed).
  __device__ __forceinline__ bool release(uint32_t pos) {
    const uint32_t free_below = pos >> kSlotLog2;
    if (!(issued < nslots && issued < free_below + NSLOT)) return true;
    __syncwarp();  // every lane is done reading the slots about to be refilled
    while (issued < nslots && issued < free_below + NSLOT) {
      if (issued >= NSLOT && waited <= issued - NSLOT) {  // previous occupant never waited
        if (!wait_slot(waited)) return false;
        waited++;
        ready = waited << kSlotLog2;
      }
      issue(issued);
      issued++;
    }
    release_at = issued >= nslots ? 0xffffffffu : (issued + 1 - NSLOT) << kSlotLog2;
    __syncwarp();
    return true;
  }

  // Makes bytes [.., end) readable.  Returns CODAG_OK, CODAG_ECORRUPT (beyond the window)
  // or CODAG_ETIMEOUT.
  __device__ __forceinline__ int ensure(uint32_t end) {
    if (end == 0) return CODAG_OK;
    const uint32_t need = (end - 1) >> kSlotLog2;
    if (need >= issued) return CODAG_ECORRUPT;
    while (waited <= need) {
      if (!wait_slot(waited)) return CODAG_ETIMEOUT;
      waited++;
    }
    ready = waited << kSlotLog2;
    return CODAG_OK;
  }

  // Waits for every issued copy so the barriers and the ring can be reused.
  __device__ __forceinline__ bool drain() {
    bool ok = true;
    while (waited < issued) {
      if (!wait_slot(waited)) {
        ok = false;
        break;
      }
      waited++;
    }
    return ok;
  }

  __device__ __forceinline__ uint32_t rd8(uint32_t p) const { return ld_s8(sbuf + (p & kMask)); }
  __device__ __forceinline__ uint32_t rd32(uint32_t p4) const { return ld_s32(sbuf + (p4 & kMask)); }
  // bytes p..p+7, little-endian
  __device__ __forceinline__ uint64_t peek_le64(uint32_t p) const {
    const uint32_t a = p & ~3u;
    const uint32_t w0 = rd32(a), w1 = rd32(a + 4), w2 = rd32(a + 8);
    const uint64_t v = (static_cast<uint64_t>(w1) << 32) | w0;
    const uint32_t sh = (p & 3u) * 8u;
    return sh ? (v >> sh) | (static_cast<uint64_t>(w2) << (64 - sh)) : v;
  }
  // bytes p..p+7 as a big-endian value (byte p on top): two byte permutes of three aligned words
  __device__ __forceinline__ uint64_t peek_be64(uint32_t p) const {
    const uint32_t a = p & ~3u, sel = 0x0123u + 0x1111u * (p & 3u);
    const uint32_t w0 = rd32(a), w1 = rd32(a + 4), w2 = rd32(a + 8);
    return (static_cast<uint64_t>(__byte_perm(w0, w1, sel)) << 32) | __byte_perm(w1, w2, sel);
  }
  // bytes p..p+3 as a big-endian word (byte p on top): one byte permute of two aligned words
  __device__ __forceinline__ uint32_t peek_be32(uint32_t p) const {
    const uint32_t a = p & ~3u;
    return __byte_perm(rd32(a), rd32(a + 4), 0x0123u + 0x1111u * (p & 3u));
  }
  // bytes p..p+3, little-endian (two aligned loads)
  __device__ __forceinline__ uint32_t peek_le32(uint32_t p) const {
    const uint32_t a = p & ~3u;
    return __funnelshift_r(rd32(a), rd32(a + 4), (p & 3u) * 8u);
  }
  // big-endian 32-bit word at a 4-byte aligned position
  __device__ __forceinline__ uint32_t be32(uint32_t p4) const { return __byte_perm(rd32(p4), 0, 0x0123); }
  // w (1..32) bits at stream bit bitpos, most significant bit first (two aligned loads)
  __device__ __forceinline__ uint32_t msb_bits32(uint32_t bitpos, uint32_t w) const {
    const uint32_t a = (bitpos >> 5) << 2;
    const uint32_t top = __funnelshift_l(be32(a + 4), be32(a), bitpos & 31u);
    return top >> (32u - w);
  }
  // w (1..64) bits at stream bit bitpos, most significant bit first (three aligned loads
  // cover the 64 bits that start anywhere within the first word)
  __device__ __forceinline__ uint64_t msb_bits64(uint32_t bitpos, uint32_t w) const {
    const uint32_t a = (bitpos >> 5) << 2, s = bitpos & 31u;
    const uint32_t w0 = be32(a), w1 = be32(a + 4), w2 = be32(a + 8);
    const uint64_t v = (static_cast<uint64_t>(__funnelshift_l(w1, w0, s)) << 32) | __funnelshift_l(w2, w1, s);
    return v >> (64u - w);
  }
  // `w` (1..64) bits starting at stream bit `bitpos`, most significant bit first; the field
  // must fit in the 8 bytes at bitpos/8, which holds for every ORC RLE v2 width.
  __device__ __forceinline__ uint64_t bits_be(uint32_t bitpos, uint32_t w) const {
    const uint64_t be = peek_be64(bitpos >> 3);
    return (be << (bitpos & 7u)) >> (64u - w);
  }
};

template <int NSLOT>
__device__ __forceinline__ void init_ring_barriers(uint64_t* bar, uint32_t lane) {
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NSLOT; i++) mbar_init(&bar[i], 1);
    fence_mbar_init();
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------------------
// output staging ring
// ---------------------------------------------------------------------------------------
template <int LOG2_BYTES, int LOG2_FLUSH, bool BULK = false>
struct OutRing {
  static constexpr uint32_t kBytes = 1u << LOG2_BYTES;
  static constexpr uint32_t kMask = kBytes - 1;
  static constexpr uint32_t kFlush = 1u << LOG2_FLUSH;
  static constexpr bool kDirect = false;
  // BULK: complete pieces leave by TMA bulk stores issued by lane 0; no decoder may read
  // the chunk's output back from global memory while the stores are in flight.  A piece
  // may be rewritten once the store of the piece after it has been issued (the stores are
  // waited for down to one in flight), which holds while a header writes at most
  // kBytes - 2 * kFlush bytes past the last complete piece.
  static_assert(LOG2_BYTES >= LOG2_FLUSH + 2, "ring must hold four flush pieces");

  uint8_t* buf;     // kBytes of shared memory, 16-byte aligned
  uint32_t sbuf;    // shared-space address of buf
  uint8_t* gdst;    // chunk output base
  uint32_t store;   // bytes of this chunk that may be stored (chunks are < 2 GiB)
  uint32_t flushed; // bytes already copied out (multiple of kFlush until the end)
  uint32_t lane;

  __device__ __forceinline__ void begin(uint8_t* dst, uint64_t store_bytes) {
    gdst = dst;
    store = static_cast<uint32_t>(store_bytes);
    flushed = 0;
  }

  // copy [a, a+len) of the stream out of the ring; the range never wraps the ring
  __device__ __forceinline__ void copy_out(uint32_t a, uint32_t len) {
    if (a >= store) return;
    if (len > store - a) len = store - a;
    const uint32_t src = sbuf + static_cast<uint32_t>(a & kMask);
    uint8_t* dst = gdst + a;
    const uintptr_t al = reinterpret_cast<uintptr_t>(dst);
    uint32_t done = 0;
    if constexpr (BULK) {
      if ((al & 15u) == 0 && len >= 16) {
        fence_proxy_async_smem();  // this lane's ring writes become visible to the bulk copy
        __syncwarp();
        done = len & ~15u;
        if (lane == 0) {
          bulk_s2g(dst, src, done);
          bulk_commit();
          bulk_wait_read<1>();
        }
      }
    }
    if (!done) {
      if ((al & 15u) == 0) {
        const uint32_t n16 = len >> 4;
        for (uint32_t k = lane; k < n16; k += 32) st_g128(dst + 16 * k, ld_s128(src + 16 * k));
        done = n16 << 4;
      } else if ((al & 7u) == 0) {
        const uint32_t n8 = len >> 3;
        for (uint32_t k = lane; k < n8; k += 32) reinterpret_cast<uint64_t*>(dst)[k] = ld_s64(src + 8 * k);
        done = n8 << 3;
      } else if ((al & 3u) == 0) {
        const uint32_t n4 = len >> 2;
        for (uint32_t k = lane; k < n4; k += 32) reinterpret_cast<uint32_t*>(dst)[k] = ld_s32(src + 4 * k);
        done = n4 << 2;
      }
    }
    for (uint32_t k = done + lane; k < len; k += 32) dst[k] = static_cast<uint8_t>(ld_s8(src + k));
  }

  // drains every complete flush piece below `pos`
  __device__ __forceinline__ void flush_to(uint32_t pos) {
    if (pos - flushed < kFlush) return;
    __syncwarp();
    do {
      copy_out(flushed, kFlush);
      flushed += kFlush;
    } while (pos - flushed >= kFlush);
    __syncwarp();
  }

  __device__ __forceinline__ void finish(uint32_t pos) {
    __syncwarp();
    if (pos > flushed) copy_out(flushed, pos - flushed);
    flushed = pos;
    if constexpr (BULK) {
      if (lane == 0) bulk_wait_read<0>();  // the ring is reused by the next chunk
    }
    __syncwarp();
  }

  // byte at stream position p of the window
  __device__ __forceinline__ uint32_t get8(uint32_t p) const { return ld_s8(sbuf + (p & kMask)); }
  __device__ __forceinline__ void put8(uint32_t p, uint32_t v) { st_s8(sbuf + (p & kMask), v); }

  // E-byte element at byte offset `off` of the chunk (a stream position of the window)
  template <int E>
  __device__ __forceinline__ void put(uint32_t off, uint64_t v) {
    const uint32_t a = sbuf + (off & kMask);
    if constexpr (E == 8) st_s64(a, v);
    else if constexpr (E == 4) st_s32(a, static_cast<uint32_t>(v));
    else if constexpr (E == 2) st_s16(a, static_cast<uint32_t>(v));
    else st_s8(a, static_cast<uint32_t>(v));
  }
  template <int E>
  __device__ __forceinline__ uint64_t get(uint32_t off) const {
    const uint32_t a = sbuf + (off & kMask);
    if constexpr (E == 8) return ld_s64(a);
    else if constexpr (E == 4) return ld_s32(a);
    else if constexpr (E == 2) return ld_s16(a);
    else return ld_s8(a);
  }
};

// Output straight to global memory: lane i of a warp store writes element n + i, so one warp
// store covers 32 consecutive elements (256 bytes for 8-byte values).  Needs the chunk's
// output base aligned to the element width; elements at or beyond `store` are not written.
// No staging, so nothing to drain.
struct DirectOut {
  static constexpr uint32_t kFlush = 0xffffffffu;
  static constexpr bool kDirect = true;
  uint8_t* gdst;   // chunk output base (element aligned)
  uint32_t store;  // bytes of this chunk that may be stored
  uint32_t flushed;
  uint32_t lane;

  __device__ __forceinline__ void begin(uint8_t* dst, uint64_t store_bytes) {
    gdst = dst;
    store = static_cast<uint32_t>(store_bytes);
    flushed = 0;
  }
  __device__ __forceinline__ void flush_to(uint32_t) {}
  __device__ __forceinline__ void finish(uint32_t pos) { flushed = pos; }
  // how many of the cnt E-byte elements from element n may be stored (store is a multiple of E)
  template <int E>
  __device__ __forceinline__ uint32_t storable(uint32_t n, uint32_t cnt) const {
    const uint32_t se = store / static_cast<uint32_t>(E);
    return n >= se ? 0u : (cnt < se - n ? cnt : se - n);
  }

  template <int E>
  __device__ __forceinline__ void put(uint32_t off, uint64_t v) {
    if (off >= store) return;
    uint8_t* a = gdst + off;
    if constexpr (E == 8) *reinterpret_cast<uint64_t*>(a) = v;
    else if constexpr (E == 4) *reinterpret_cast<uint32_t*>(a) = static_cast<uint32_t>(v);
    else if constexpr (E == 2) *reinterpret_cast<uint16_t*>(a) = static_cast<uint16_t>(v);
    else *a = static_cast<uint8_t>(v);
  }
  template <int E>
  __device__ __forceinline__ uint64_t get(uint32_t off) const {
    if (off >= store) return 0;  // never stored: the patch result is dropped as well
    const uint8_t* a = gdst + off;
    if constexpr (E == 8) return *reinterpret_cast<const uint64_t*>(a);
    else if constexpr (E == 4) return *reinterpret_cast<const uint32_t*>(a);
    else if constexpr (E == 2) return *reinterpret_cast<const uint16_t*>(a);
    else return *a;
  }
};

// Output that is not element aligned, stored straight to global memory byte by byte (a
// fallback for rare unaligned outputs that have no shared-memory ring to go through).
struct ByteOut {
  static constexpr uint32_t kFlush = 0xffffffffu;
  static constexpr bool kDirect = false;
  uint8_t* gdst;
  uint32_t store;
  uint32_t flushed;
  uint32_t lane;

  __device__ __forceinline__ void begin(uint8_t* dst, uint64_t store_bytes) {
    gdst = dst;
    store = static_cast<uint32_t>(store_bytes);
    flushed = 0;
  }
  __device__ __forceinline__ void flush_to(uint32_t) {}
  __device__ __forceinline__ void finish(uint32_t pos) { flushed = pos; }
  template <int E>
  __device__ __forceinline__ void put(uint32_t off, uint64_t v) {
#pragma unroll
    for (int i = 0; i < E; i++)
      if (off + i < store) gdst[off + i] = static_cast<uint8_t>(v >> (8 * i));
  }
  template <int E>
  __device__ __forceinline__ uint64_t get(uint32_t off) const {
    uint64_t v = 0;
#pragma unroll
    for (int i = 0; i < E; i++)
      if (off + i < store) v |= static_cast<uint64_t>(gdst[off + i]) << (8 * i);
    return v;
  }
};

}  // namespace codag_dev
