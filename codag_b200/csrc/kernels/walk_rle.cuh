// Two-pass RLE decoding: a thread-per-chunk header walk, then warp-per-chunk expansion.
//
// The serial part of RLE decoding is finding where each header starts.  Done by the warp
// that decodes the chunk, every lane repeats it (about 300 warp instructions per RLE v2
// header).  The walk below runs one thread per chunk instead, so one warp instruction
// advances 32 chunks; it reads only header bytes (literal groups are skipped 16 bytes at a
// time by counting varint ends) straight from global memory through the read-only cache,
// and writes one 32-byte descriptor per header.  The expansion pass then loads the
// descriptors 32 at a time with one coalesced load per lane and spends a few instructions
// per header before its lane-parallel value loop.
//
// A chunk whose walk finds anything unexpected (a malformed header, more headers than the
// descriptor budget) is marked for the single-pass decoder, which reports the exact error.
#pragma once
#include "decode_rle.cuh"

namespace codag_dev {

// One header.  pos/data/total are stream-relative bytes.
//   RLE v2: info = kind | width code << 2 | values << 7 | third << 16 | fourth << 24;
//           a = SHORT_REPEAT value, DELTA base or PATCHED base; b = DELTA base delta
//   RLE v1: info = (literal group ? 1 : 0) | values << 7; a = run base; b = run delta
struct __align__(16) RleDesc {
  uint32_t pos, info, data, total;
  uint64_t a, b;
};
static_assert(sizeof(RleDesc) == 32, "descriptor layout");

constexpr uint32_t kDescPerChunk = 512;          // descriptor budget of one chunk
constexpr uint32_t kWalkFallback = 0xffffffffu;  // walk gave up: decode in one pass

// bounded, read-only view of one stream in global memory
struct GStream {
  const uint8_t* s;   // stream start
  uint32_t len;
  const uint8_t* lo;  // readable range of the whole buffer
  const uint8_t* hi;

  __device__ __forceinline__ uint4 load16(const uint8_t* a) const {  // a is 16-byte aligned
    if (a >= lo && a + 16 <= hi) return __ldg(reinterpret_cast<const uint4*>(a));
    uint32_t w[4] = {0, 0, 0, 0};
    for (int i = 0; i < 16; i++) {
      const uint8_t* q = a + i;
      if (q >= lo && q < hi) w[i >> 2] |= static_cast<uint32_t>(__ldg(q)) << (8 * (i & 3));
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
  }
  // the 16 bytes at stream offset p, little-endian (bytes outside the buffer read as 0)
  __device__ __forceinline__ void peek16(uint32_t p, uint64_t& lo8, uint64_t& hi8) const {
    const uintptr_t abs = reinterpret_cast<uintptr_t>(s + p);
    const uint8_t* base = reinterpret_cast<const uint8_t*>(abs & ~static_cast<uintptr_t>(15));
    const uint32_t o = static_cast<uint32_t>(abs & 15);
    const uint4 q0 = load16(base), q1 = load16(base + 16);
    uint64_t w0 = (static_cast<uint64_t>(q0.y) << 32) | q0.x, w1 = (static_cast<uint64_t>(q0.w) << 32) | q0.z;
    uint64_t w2 = (static_cast<uint64_t>(q1.y) << 32) | q1.x;
    if (o >= 8) {
      w0 = w1;
      w1 = w2;
      w2 = (static_cast<uint64_t>(q1.w) << 32) | q1.z;
    }
    const uint32_t sh = (o & 7u) * 8u;
    lo8 = sh ? (w0 >> sh) | (w1 << (64 - sh)) : w0;
    hi8 = sh ? (w1 >> sh) | (w2 << (64 - sh)) : w1;
  }
};

// the same view of a stream staged whole in shared memory (stream byte 0 at sbuf + lo)
struct SStream {
  uint32_t sbuf;  // shared address of the staging buffer
  uint32_t lo;    // offset of the stream's first byte in it
  uint32_t len;
  uint32_t mask;  // staging buffer bytes - 1 (a power of two)
  __device__ __forceinline__ void peek16(uint32_t p, uint64_t& lo8, uint64_t& hi8) const {
    const uint32_t a = lo + p;
    const uint32_t w = a & ~3u, sh = (a & 3u) * 8u;
    uint32_t x[5];
#pragma unroll
    for (int i = 0; i < 5; i++) x[i] = ld_s32(sbuf + ((w + 4u * i) & mask));
    const uint32_t y0 = __funnelshift_r(x[0], x[1], sh), y1 = __funnelshift_r(x[1], x[2], sh);
    const uint32_t y2 = __funnelshift_r(x[2], x[3], sh), y3 = __funnelshift_r(x[3], x[4], sh);
    lo8 = (static_cast<uint64_t>(y1) << 32) | y0;
    hi8 = (static_cast<uint64_t>(y3) << 32) | y2;
    // bytes past the stream read as zero, as in GStream outside the buffer
    if (p + 16u > len) {
      const uint32_t valid = p >= len ? 0u : len - p;
      if (valid < 8) {
        lo8 &= valid ? ((1ull << (8 * valid)) - 1ull) : 0ull;
        hi8 = 0;
      } else {
        hi8 &= valid == 8 ? 0ull : ((1ull << (8 * (valid - 8))) - 1ull);
      }
    }
  }
};

__device__ __forceinline__ uint64_t be_bytes(uint64_t le, uint32_t nb) {  // first nb bytes, big-endian
  return bswap64(le) >> (64u - 8u * nb);
}

// ---------------------------------------------------------------------------------------
// walks (one thread per chunk); return the descriptor count or kWalkFallback
// ---------------------------------------------------------------------------------------
template <class S>
__device__ uint32_t walk_rlev2(const S& g, uint32_t cap, RleDesc* __restrict__ d, uint32_t* __restrict__ nstart = nullptr,
                               uint32_t budget = kDescPerChunk) {
  uint32_t pos = 0, n = 0, k = 0;
  while (pos < g.len) {
    if (k == budget) return kWalkFallback;
    uint64_t lo8, hi8;
    g.peek16(pos, lo8, hi8);
    const uint32_t first = static_cast<uint32_t>(lo8 & 0xff);
    const uint32_t kind = first >> 6;
    const uint32_t code = (first >> 1) & 0x1fu;
    const uint32_t len8 = ((((first & 1u) << 8) | static_cast<uint32_t>((lo8 >> 8) & 0xff)) + 1u) & 0xffu;
    RleDesc h;
    h.pos = pos;
    h.a = 0;
    h.b = 0;
    uint32_t cnt, extra = 0;
    if (kind == 0) {  // SHORT_REPEAT
      const uint32_t nb = ((first >> 3) & 7u) + 1u;
      cnt = (first & 7u) + 3u;
      h.total = 1u + nb;
      h.data = pos + 1u;
      h.a = be_bytes((lo8 >> 8) | (hi8 << 56), nb);
    } else if (kind == 1) {  // DIRECT
      cnt = len8;
      h.data = pos + 2u;
      h.total = 2u + (len8 * v2_width(code) + 7u) / 8u;
    } else if (kind == 3) {  // DELTA: two varints from byte 2
      const uint64_t v_lo = (lo8 >> 16) | (hi8 << 48), v_hi = hi8 >> 16;
      const uint32_t l1 = leb_len(v_lo, v_hi);
      if (!l1 || l1 > 10) return kWalkFallback;
      uint64_t w_lo, w_hi;
      g.peek16(pos + 2 + l1, w_lo, w_hi);
      const uint32_t l2 = leb_len(w_lo, w_hi);
      if (!l2 || l2 > 10) return kWalkFallback;
      h.a = leb_value(v_lo, v_hi, l1);
      const int64_t sd = static_cast<int64_t>(leb_value(w_lo, w_hi, l2));
      h.b = static_cast<uint64_t>((sd >> 1) ^ -(sd & 1));
      const uint32_t nd = (len8 - 2u) & 0xffu;
      cnt = nd + 2u;
      h.data = pos + 2u + l1 + l2;
      h.total = (h.data - pos) + (code ? (nd * v2_width(code) + 7u) / 8u : 0u);
    } else {  // PATCHED_BASE
      const uint32_t third = static_cast<uint32_t>((lo8 >> 16) & 0xff), fourth = static_cast<uint32_t>((lo8 >> 24) & 0xff);
      const uint32_t bw = ((third >> 5) & 7u) + 1u, pw = v2_width(third & 0x1fu), pgw = ((fourth >> 5) & 7u) + 1u;
      const uint32_t pll = fourth & 0x1fu;
      if (pw + pgw > 64u) return kWalkFallback;
      cnt = len8;
      h.a = be_bytes((lo8 >> 32) | (hi8 << 32), bw);
      h.data = pos + 4u + bw;
      h.total = (h.data - pos) + (len8 * v2_width(code) + 7u) / 8u + (pll * v2_closest(pw + pgw) + 7u) / 8u;
      extra = (third << 16) | (fourth << 24);
    }
    if (pos + h.total > g.len || h.total > 3000u || n + cnt > cap) return kWalkFallback;
    h.info = kind | (code << 2) | (cnt << 7) | extra;
    if (nstart) nstart[k] = n;
    d[k++] = h;
    pos += h.total;
    n += cnt;
  }
  return k;
}

// position just past the `cnt`-th varint end at or after p, or 0 if the stream ends first
template <class S>
__device__ __forceinline__ uint32_t skip_varints(const S& g, uint32_t p, uint32_t cnt) {
  while (p < g.len) {
    uint64_t lo8, hi8;
    g.peek16(p, lo8, hi8);
    const uint32_t valid = g.len - p < 16u ? g.len - p : 16u;
    uint64_t t0 = ~lo8 & 0x8080808080808080ull, t1 = ~hi8 & 0x8080808080808080ull;
    if (valid < 16) {
      if (valid <= 8) {
        t0 &= valid == 8 ? ~0ull : ((1ull << (8 * valid)) - 1ull);
        t1 = 0;
      } else {
        t1 &= (1ull << (8 * (valid - 8))) - 1ull;
      }
    }
    const uint32_t c0 = __popcll(t0), c1 = __popcll(t1);
    if (c0 + c1 >= cnt) {
      uint64_t t = c0 >= cnt ? t0 : t1;
      uint32_t k = c0 >= cnt ? cnt : cnt - c0;
      while (--k) t &= t - 1;
      return p + (c0 >= cnt ? 0u : 8u) + (ctz64(t) >> 3) + 1u;
    }
    cnt -= c0 + c1;
    p += valid;
  }
  return 0;
}

template <class S>
__device__ uint32_t walk_rlev1(const S& g, uint32_t cap, RleDesc* __restrict__ d, uint32_t* __restrict__ nstart = nullptr,
                               uint32_t budget = kDescPerChunk) {
  uint32_t pos = 0, n = 0, k = 0;
  while (n < cap) {
    if (k == budget || pos >= g.len) return kWalkFallback;
    uint64_t lo8, hi8;
    g.peek16(pos, lo8, hi8);
    const int h = static_cast<int8_t>(lo8 & 0xff);
    RleDesc r;
    r.pos = pos;
    uint32_t cnt;
    if (h >= 0) {  // run
      const uint64_t v_lo = (lo8 >> 16) | (hi8 << 48), v_hi = hi8 >> 16;
      const uint32_t l = leb_len(v_lo, v_hi);
      if (!l || l > 12) return kWalkFallback;
      cnt = static_cast<uint32_t>(h) + 3u;
      r.a = leb_value(v_lo, v_hi, l);
      r.b = static_cast<uint64_t>(static_cast<int64_t>(static_cast<int8_t>((lo8 >> 8) & 0xff)));
      r.data = pos + 2u;
      r.total = 2u + l;
      r.info = cnt << 7;
    } else {  // literal group
      cnt = static_cast<uint32_t>(-h);
      const uint32_t e = skip_varints(g, pos + 1, cnt);
      if (!e) return kWalkFallback;
      r.a = 0;
      r.b = 0;
      r.data = pos + 1u;
      r.total = e - pos;
      r.info = 1u | (cnt << 7);
    }
    if (pos + r.total > g.len || n + cnt > cap) return kWalkFallback;
    if (nstart) nstart[k] = n;
    d[k++] = r;
    pos += r.total;
    n += cnt;
  }
  return k;
}

// RLE v1 walk by a whole warp over a stream resident in `in` (stream byte 0 at in.lo): the
// same descriptors as walk_rlev1, but literal groups are skipped 128 bytes per step (each
// lane counts the varint ends in its 4 bytes, a warp scan finds the lane holding the end).
template <int NSLOT>
__device__ uint32_t walk_rlev1_warp(const InRing<NSLOT>& in, uint32_t len, uint32_t cap, RleDesc* __restrict__ d,
                                    uint32_t* __restrict__ nstart, uint32_t lane) {
  const uint32_t base = in.lo;
  uint32_t pos = 0, n = 0, k = 0;
  while (n < cap) {
    if (k == kDescPerChunk || pos >= len) return kWalkFallback;
    const uint64_t lo8 = in.peek_le64(base + pos), hi8 = in.peek_le64(base + pos + 8);
    const int h = static_cast<int8_t>(lo8 & 0xff);
    RleDesc r;
    r.pos = pos;
    uint32_t cnt;
    if (h >= 0) {  // run
      const uint64_t v_lo = (lo8 >> 16) | (hi8 << 48), v_hi = hi8 >> 16;
      const uint32_t l = leb_len(v_lo, v_hi);
      if (!l || l > 12) return kWalkFallback;
      cnt = static_cast<uint32_t>(h) + 3u;
      r.a = leb_value(v_lo, v_hi, l);
      r.b = static_cast<uint64_t>(static_cast<int64_t>(static_cast<int8_t>((lo8 >> 8) & 0xff)));
      r.data = pos + 2u;
      r.total = 2u + l;
      r.info = cnt << 7;
    } else {  // literal group: find the end of its cnt varints
      cnt = static_cast<uint32_t>(-h);
      uint32_t p = pos + 1, rem = cnt, e = 0;
      for (;;) {
        if (p >= len) return kWalkFallback;
        const uint32_t q0 = p + 4u * lane;
        const uint32_t tb = ~in.peek_le32(base + q0) & 0x80808080u;
        uint32_t nib = ((tb >> 7) & 1u) | ((tb >> 14) & 2u) | ((tb >> 21) & 4u) | ((tb >> 28) & 8u);
        if (q0 + 4 > len) nib &= q0 >= len ? 0u : ((1u << (len - q0)) - 1u);
        const uint32_t c = __popc(nib);
        uint32_t incl = c;
#pragma unroll
        for (int dd = 1; dd < 32; dd <<= 1) {
          const uint32_t o = __shfl_up_sync(FULL, incl, dd);
          if (lane >= static_cast<uint32_t>(dd)) incl += o;
        }
        const uint32_t total = __shfl_sync(FULL, incl, 31);
        if (total >= rem) {
          uint32_t endp = 0;
          if (incl >= rem && incl - c < rem) {  // this lane holds the rem-th end
            uint32_t m = nib;
            for (uint32_t t = rem - (incl - c); t > 1; t--) m &= m - 1;
            endp = q0 + static_cast<uint32_t>(__ffs(m));  // one past the end byte
          }
          e = __reduce_max_sync(FULL, endp);
          break;
        }
        rem -= total;
        p += 128;
      }
      r.a = 0;
      r.b = 0;
      r.data = pos + 1u;
      r.total = e - pos;
      r.info = 1u | (cnt << 7);
    }
    if (pos + r.total > len || n + cnt > cap) return kWalkFallback;
    if (lane == 0) {
      nstart[k] = n;
      d[k] = r;
    }
    k++;
    pos += r.total;
    n += cnt;
  }
  return k;
}

// ---------------------------------------------------------------------------------------
// expansion (one warp per chunk) driven by the descriptors
// ---------------------------------------------------------------------------------------
struct DescCache {  // descriptors [base, base+32) spread over the lanes
  uint4 c0, c1;
  // d in global memory (read-only path) or, with SMEM, in shared memory
  template <bool SMEM = false>
  __device__ __forceinline__ void load(const RleDesc* __restrict__ d, uint32_t first, uint32_t nd, uint32_t lane) {
    const uint32_t k = first + lane;
    if (k < nd) {
      const uint4* p = reinterpret_cast<const uint4*>(d + k);
      if constexpr (SMEM) {
        c0 = p[0];
        c1 = p[1];
      } else {
        c0 = __ldg(p);
        c1 = __ldg(p + 1);
      }
    }
  }
};

// Descriptors [k0, k1), whose first value is value n of the chunk; n is advanced.
template <int NSLOT, int E, bool SMEM, class OUT>
__device__ int expand_rlev2_range(InRing<NSLOT>& in, OUT& out, const RleDesc* __restrict__ d, uint32_t k0, uint32_t k1,
                                  uint32_t& n) {
  constexpr uint64_t M = emask<E>();
  const uint32_t lane = in.lane;
  const uint32_t lo = in.lo;
  int st = CODAG_OK;
  DescCache cur, nxt;
  cur.template load<SMEM>(d, k0, k1, lane);
  nxt.template load<SMEM>(d, k0 + 32, k1, lane);
  for (uint32_t k = k0; k < k1; k++) {
    const uint32_t src = (k - k0) & 31u;
    if (src == 0 && k != k0) {
      cur = nxt;
      nxt.template load<SMEM>(d, k + 32, k1, lane);
    }
    const uint32_t pos = lo + __shfl_sync(FULL, cur.c0.x, src);
    const uint32_t info = __shfl_sync(FULL, cur.c0.y, src);
    const uint32_t data = lo + __shfl_sync(FULL, cur.c0.z, src);
    const uint32_t total = __shfl_sync(FULL, cur.c0.w, src);
    const uint32_t kind = info & 3u, fbw = v2_width((info >> 2) & 0x1fu), cnt = (info >> 7) & 0x1ffu;
    st = in.advance(pos, pos + total);
    if (st) break;
    if (kind == 1) {
      body_unpack<NSLOT, E>(in, out, n, cnt, data * 8u, fbw, 0ull, lane);
    } else {
      const uint64_t a = (static_cast<uint64_t>(__shfl_sync(FULL, cur.c1.y, src)) << 32) | __shfl_sync(FULL, cur.c1.x, src);
      if (kind == 0) {
        if (lane < cnt) put_elem<E>(out, n + lane, a & M);
      } else if (kind == 3) {
        const uint64_t b = ((static_cast<uint64_t>(__shfl_sync(FULL, cur.c1.w, src)) << 32) | __shfl_sync(FULL, cur.c1.z, src)) & M;
        if (((info >> 2) & 0x1fu) == 0) body_fill<E>(out, n, cnt, a & M, b, lane);
        else body_delta_packed<NSLOT, E>(in, out, n, cnt - 2u, fbw, a & M, b, data * 8u, lane);
      } else {
        const uint32_t third = (info >> 16) & 0xffu, fourth = info >> 24;
        const uint32_t pw = v2_width(third & 0x1fu), pll = fourth & 0x1fu;
        body_unpack<NSLOT, E>(in, out, n, cnt, data * 8u, fbw, a, lane);
        if (pll) {
          __syncwarp();
          const uint32_t cfb = v2_closest(pw + ((fourth >> 5) & 7u) + 1u);
          st = body_patches<NSLOT, E>(in, out, n, cnt, fbw, pw, cfb, pll, a, (data + (cnt * fbw + 7u) / 8u) * 8u, lane);
          if (st) break;
        }
      }
    }
    n += cnt;
    __syncwarp();
    out.flush_to(n * E);
  }
  return st;
}

template <int NSLOT, int E, class OUT>
__device__ int expand_rlev2(InRing<NSLOT>& in, OUT& out, const RleDesc* __restrict__ d, uint32_t nd) {
  uint32_t n = 0;
  int st = expand_rlev2_range<NSLOT, E, false>(in, out, d, 0, nd, n);
  if (!in.drain() && st == CODAG_OK) st = CODAG_ETIMEOUT;
  out.finish(n * E);
  if (st == CODAG_OK && n * E < out.store) st = CODAG_ECORRUPT;
  return st;
}

// Descriptors [k0, k1), whose first value is value n of the chunk; n is advanced.
template <int NSLOT, int E, bool SMEM, class OUT>
__device__ int expand_rlev1_range(InRing<NSLOT>& in, OUT& out, const RleDesc* __restrict__ d, uint32_t k0, uint32_t k1,
                                  uint32_t& n) {
  const uint32_t lane = in.lane;
  const uint32_t lo = in.lo;
  int st = CODAG_OK;
  DescCache cur, nxt;
  cur.template load<SMEM>(d, k0, k1, lane);
  nxt.template load<SMEM>(d, k0 + 32, k1, lane);
  for (uint32_t k = k0; k < k1; k++) {
    const uint32_t src = (k - k0) & 31u;
    if (src == 0 && k != k0) {
      cur = nxt;
      nxt.template load<SMEM>(d, k + 32, k1, lane);
    }
    const uint32_t pos = lo + __shfl_sync(FULL, cur.c0.x, src);
    const uint32_t info = __shfl_sync(FULL, cur.c0.y, src);
    const uint32_t total = __shfl_sync(FULL, cur.c0.w, src);
    const uint32_t cnt = (info >> 7) & 0x1ffu;
    if (info & 1u) {
      uint32_t p = pos + 1;
      st = body_literals<NSLOT, E>(in, out, n, cnt, p, pos + total, lane);
      if (st) break;
    } else {
      st = in.advance(pos, pos + total);
      if (st) break;
      const uint64_t a = (static_cast<uint64_t>(__shfl_sync(FULL, cur.c1.y, src)) << 32) | __shfl_sync(FULL, cur.c1.x, src);
      const uint64_t b = (static_cast<uint64_t>(__shfl_sync(FULL, cur.c1.w, src)) << 32) | __shfl_sync(FULL, cur.c1.z, src);
      body_fill<E>(out, n, cnt, a, b, lane);
    }
    n += cnt;
    __syncwarp();
    out.flush_to(n * E);
  }
  return st;
}

template <int NSLOT, int E, class OUT>
__device__ int expand_rlev1(InRing<NSLOT>& in, OUT& out, const RleDesc* __restrict__ d, uint32_t nd) {
  uint32_t n = 0;
  int st = expand_rlev1_range<NSLOT, E, false>(in, out, d, 0, nd, n);
  if (!in.drain() && st == CODAG_OK) st = CODAG_ETIMEOUT;
  out.finish(n * E);
  if (st == CODAG_OK && n * E < out.store) st = CODAG_ECORRUPT;
  return st;
}

}  // namespace codag_dev
