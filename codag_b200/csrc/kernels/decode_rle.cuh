// Warp decoders for ORC RLE v1 and ORC RLE v2 chunks.
//
// CODAG decodes these with one lane walking the stream byte by byte while the other lanes
// idle or store the same addresses (include/rlev1/decoder.h:588-798,
// include/rlev2/decoder_new.h:909-1187).  Here each chunk is decoded in two passes when a
// workspace is available (walk_rle.cuh):
//   1. a header walk, one THREAD per chunk (so one warp instruction advances 32 chunks),
//      writes a 32-byte descriptor per header;
//   2. one WARP per chunk expands the headers: descriptors arrive 32 at a time with one
//      coalesced load, and each header's values are produced lane-parallel.
// Without a workspace the same warp parses the headers itself (decode_rlev*_chunk).
// Lane-parallel value expansion, shared by both paths:
//   - RLE v1 runs, RLE v2 SHORT_REPEAT and fixed-step DELTA: one arithmetic value per lane;
//   - RLE v1 literal groups: 128 stream bytes per step, 4 bytes per lane; one ballot per byte
//     lane finds the varint ends and the lane holding an end decodes that varint in registers
//     (7-bit groups compacted with shifts and masks);
//   - RLE v2 DIRECT/PATCHED_BASE: one value per lane by direct bit addressing (two or three
//     aligned shared-memory words and a funnel shift);
//   - RLE v2 packed DELTA: deltas unpacked per lane and accumulated with a warp scan;
//   - PATCHED_BASE patches: gaps prefix-summed across the patch lanes, patches applied by
//     those lanes (a group hitting one value is OR-combined first).
// Values go either to the shared-memory output ring (OutRing, drained by TMA bulk stores) or,
// when the output is element aligned, straight to global memory (DirectOut), 32 consecutive
// elements per warp store.
// Element arithmetic is modulo 2^(8*E), keeping the reference's quirks (oracle/oracle.c).
#pragma once
#include "../rlev2_widths.h"
#include "device_common.cuh"

namespace codag_dev {

template <int E>
struct ElemType;
template <>
struct ElemType<1> { using T = uint8_t; };
template <>
struct ElemType<2> { using T = uint16_t; };
template <>
struct ElemType<4> { using T = uint32_t; };
template <>
struct ElemType<8> { using T = uint64_t; };

template <int E>
__device__ __forceinline__ constexpr uint64_t emask() {
  return E == 8 ? ~0ull : ((1ull << (8 * E)) - 1ull);
}

template <int E, class OUT>
__device__ __forceinline__ void put_elem(OUT& o, uint32_t idx, uint64_t v) {
  o.template put<E>(idx * static_cast<uint32_t>(E), v);
}

template <int E, class OUT>
__device__ __forceinline__ uint64_t get_elem(const OUT& o, uint32_t idx) {
  return o.template get<E>(idx * static_cast<uint32_t>(E));
}

// LEB128 payload of the first `len` bytes of a little-endian window (len 1..8)
__host__ __device__ __forceinline__ uint64_t leb_compact(uint64_t x, uint32_t len) {
  if (len < 8) x &= (1ull << (8 * len)) - 1ull;
  x &= 0x7F7F7F7F7F7F7F7Full;
  x = (x & 0x007F007F007F007Full) | ((x >> 1) & 0x3F803F803F803F80ull);
  x = (x & 0x00003FFF00003FFFull) | ((x >> 2) & 0x0FFFC0000FFFC000ull);
  x = (x & 0x000000000FFFFFFFull) | ((x >> 4) & 0x00FFFFFFF0000000ull);
  return x;
}
// the same for len 1..4 in 32-bit arithmetic
__device__ __forceinline__ uint32_t leb_compact32(uint32_t x, uint32_t len) {
  if (len < 4) x &= (1u << (8 * len)) - 1u;
  x &= 0x7F7F7F7Fu;
  x = (x & 0x007F007Fu) | ((x >> 1) & 0x3F803F80u);
  return (x & 0x00003FFFu) | ((x >> 2) & 0x0FFFC000u);
}
// value of a LEB128 varint of `len` bytes whose first 16 bytes are lo8, hi8; bytes past
// the 10th only feed bits above 63 and vanish, as with the reference's clamped shifts
__host__ __device__ __forceinline__ uint64_t leb_value(uint64_t lo8, uint64_t hi8, uint32_t len) {
  if (len <= 8) return leb_compact(lo8, len);
  return leb_compact(lo8, 8) | (leb_compact(hi8, len - 8 < 8 ? len - 8 : 8) << 56);
}
__host__ __device__ __forceinline__ uint32_t ctz64(uint64_t t) {
#ifdef __CUDA_ARCH__
  return static_cast<uint32_t>(__ffsll(static_cast<long long>(t)) - 1);
#else
  return static_cast<uint32_t>(__builtin_ctzll(t));
#endif
}
// length (1..16) of the varint that starts a 16-byte window, or 0 if it is longer
__host__ __device__ __forceinline__ uint32_t leb_len(uint64_t lo8, uint64_t hi8) {
  uint64_t t = ~lo8 & 0x8080808080808080ull;
  if (t) return (ctz64(t) >> 3) + 1;
  t = ~hi8 & 0x8080808080808080ull;
  return t ? (ctz64(t) >> 3) + 9 : 0u;
}

// Reads the unsigned varint at `p` (all lanes, same data); false if it is truncated or
// longer than the resident window allows (1 KiB).
template <int NSLOT>
__device__ __forceinline__ bool read_uvarint(InRing<NSLOT>& in, uint32_t p, uint32_t end, uint32_t& len,
                                             uint64_t& val) {
  if (p + 20 > in.ready && in.ensure(min(p + 20, end))) return false;
  const uint64_t lo8 = in.peek_le64(p);
  const uint64_t t = ~lo8 & 0x8080808080808080ull;
  if (t) {
    len = (static_cast<uint32_t>(__ffsll(t)) >> 3);
    val = leb_compact(lo8, len);
  } else {
    const uint64_t hi8 = in.peek_le64(p + 8);
    len = leb_len(lo8, hi8);
    if (!len) {  // longer than 16 bytes: only the first 16 carry bits; find the end
      uint32_t q = p + 16;
      const uint32_t lim = min(end, p + 1024);
      if (in.ensure(lim)) return false;
      while (q < lim && in.rd8(q) >= 0x80u) q++;
      if (q >= lim) return false;
      len = q - p + 1;
    }
    val = leb_value(lo8, hi8, len);
  }
  return p + len <= end;
}

// ---------------------------------------------------------------------------------------
// per-header value expansion (warp-cooperative; all lanes call with identical arguments)
// ---------------------------------------------------------------------------------------
// value i = v + i*step, i < cnt
template <int E, class OUT>
__device__ __forceinline__ void body_fill(OUT& out, uint32_t n, uint32_t cnt, uint64_t v, uint64_t step, uint32_t lane) {
  if (lane >= cnt) return;
  uint64_t x = v + static_cast<uint64_t>(lane) * step;
  const uint64_t s32 = step << 5;
  if constexpr (OUT::kDirect) {  // bounds hoisted out of the loop, a running element pointer
    using T = typename ElemType<E>::T;
    const uint32_t lim = out.template storable<E>(n, cnt);
    T* dst = reinterpret_cast<T*>(out.gdst) + n + lane;
#pragma unroll 4  // independent iterations: unrolled they overlap their latencies
    for (uint32_t i = lane; i < lim; i += 32, x += s32, dst += 32) *dst = static_cast<T>(x);
  } else {
    uint32_t oa = (n + lane) * E;
    for (uint32_t i = lane; i < cnt; i += 32, x += s32, oa += 32 * E) out.template put<E>(oa, x);
  }
}

// value i = (fbw-bit field i at bit0, most significant bit first) + add, i < cnt
template <int NSLOT, int E, class OUT>
__device__ __forceinline__ void body_unpack(const InRing<NSLOT>& in, OUT& out, uint32_t n, uint32_t cnt, uint32_t bit0,
                                            uint32_t fbw, uint64_t add, uint32_t lane) {
  constexpr uint32_t IM = InRing<NSLOT>::kMask;
  const uint32_t ib = in.sbuf;
  if (lane >= cnt) return;
  uint32_t bp = bit0 + lane * fbw;
  const uint32_t bstep = fbw << 5;
  uint32_t oa = (n + lane) * E;
  if (fbw <= 32) {
    const uint32_t rs = 32u - fbw;
    if constexpr (OUT::kDirect) {  // bounds hoisted out of the loop, a running element pointer
      using T = typename ElemType<E>::T;
      const uint32_t lim = out.template storable<E>(n, cnt);
      T* dst = reinterpret_cast<T*>(out.gdst) + n + lane;
#pragma unroll 4
      for (uint32_t j = lane; j < lim; j += 32, bp += bstep, dst += 32) {
        const uint32_t wa = (bp >> 3) & ~3u;
        const uint32_t w0 = __byte_perm(ld_s32(ib + (wa & IM)), 0, 0x0123);
        const uint32_t w1 = __byte_perm(ld_s32(ib + ((wa + 4) & IM)), 0, 0x0123);
        const uint32_t v = __funnelshift_l(w1, w0, bp & 31u) >> rs;
        *dst = static_cast<T>(static_cast<uint64_t>(v) + add);
      }
      return;
    }
    for (uint32_t j = lane; j < cnt; j += 32, bp += bstep, oa += 32 * E) {
      const uint32_t wa = (bp >> 3) & ~3u;
      const uint32_t w0 = __byte_perm(ld_s32(ib + (wa & IM)), 0, 0x0123);
      const uint32_t w1 = __byte_perm(ld_s32(ib + ((wa + 4) & IM)), 0, 0x0123);
      const uint32_t v = __funnelshift_l(w1, w0, bp & 31u) >> rs;
      out.template put<E>(oa, static_cast<uint64_t>(v) + add);
    }
  } else {
    const uint32_t rs = 64u - fbw;
    if constexpr (OUT::kDirect) {
      using T = typename ElemType<E>::T;
      const uint32_t lim = out.template storable<E>(n, cnt);
      T* dst = reinterpret_cast<T*>(out.gdst) + n + lane;
#pragma unroll 4
      for (uint32_t j = lane; j < lim; j += 32, bp += bstep, dst += 32) {
        const uint32_t wa = (bp >> 3) & ~3u, s = bp & 31u;
        const uint32_t w0 = __byte_perm(ld_s32(ib + (wa & IM)), 0, 0x0123);
        const uint32_t w1 = __byte_perm(ld_s32(ib + ((wa + 4) & IM)), 0, 0x0123);
        const uint32_t w2 = __byte_perm(ld_s32(ib + ((wa + 8) & IM)), 0, 0x0123);
        const uint64_t v = ((static_cast<uint64_t>(__funnelshift_l(w1, w0, s)) << 32) | __funnelshift_l(w2, w1, s)) >> rs;
        *dst = static_cast<T>(v + add);
      }
      return;
    }
    for (uint32_t j = lane; j < cnt; j += 32, bp += bstep, oa += 32 * E) {
      const uint32_t wa = (bp >> 3) & ~3u, s = bp & 31u;
      const uint32_t w0 = __byte_perm(ld_s32(ib + (wa & IM)), 0, 0x0123);
      const uint32_t w1 = __byte_perm(ld_s32(ib + ((wa + 4) & IM)), 0, 0x0123);
      const uint32_t w2 = __byte_perm(ld_s32(ib + ((wa + 8) & IM)), 0, 0x0123);
      const uint64_t v = ((static_cast<uint64_t>(__funnelshift_l(w1, w0, s)) << 32) | __funnelshift_l(w2, w1, s)) >> rs;
      out.template put<E>(oa, v + add);
    }
  }
}

// packed DELTA: values base, base+bd, then += (or -=) each of nd packed deltas
template <int NSLOT, int E, class OUT>
__device__ __forceinline__ void body_delta_packed(const InRing<NSLOT>& in, OUT& out, uint32_t n, uint32_t nd,
                                                  uint32_t fbw, uint64_t base, uint64_t bd, uint32_t bit0,
                                                  uint32_t lane) {
  constexpr uint64_t M = emask<E>();
  const bool plus = bd != 0;  // multiplier = base_delta > 0 ? 1 : -1 on the unsigned type
  const uint64_t v1 = (base + bd) & M;
  if (lane == 0) put_elem<E>(out, n, base);
  if (lane == 1) put_elem<E>(out, n + 1, v1);
  uint64_t carry = v1;
  for (uint32_t k0 = 0; k0 < nd; k0 += 32) {
    const uint32_t k = k0 + lane;
    const uint64_t d = k < nd ? (in.msb_bits64(bit0 + k * fbw, fbw) & M) : 0ull;
    const uint64_t s = warp_scan_add64(d, lane);
    const uint64_t v = (plus ? carry + s : carry - s) & M;
    if (k < nd) put_elem<E>(out, n + 2 + k, v);
    carry = shfl64(v, 31);
  }
}

// PATCHED_BASE patch list (decoder_new.h:1142-1182), applied to the len8 values at n
template <int NSLOT, int E, class OUT>
__device__ __forceinline__ int body_patches(const InRing<NSLOT>& in, OUT& out, uint32_t n, uint32_t len8, uint32_t fbw,
                                            uint32_t pw, uint32_t cfb, uint32_t pll, uint64_t base, uint32_t bit0,
                                            uint32_t lane) {
  constexpr uint64_t M = emask<E>();
  // the reference masks patches with a 32-bit mask (decoder_new.h:1103)
  const uint64_t pmask = pw >= 32 ? 0xffffffffull : ((1ull << pw) - 1ull);
  uint64_t patch = 0;
  uint32_t gap = 0;
  if (lane < pll) {
    const uint64_t ent = in.msb_bits64(bit0 + lane * cfb, cfb);
    gap = static_cast<uint32_t>(shr64(ent, pw));
    patch = shl64((ent & pmask) & M, fbw) & M;
  }
  uint32_t off = gap;  // inclusive scan of the gaps
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(FULL, off, d);
    if (lane >= static_cast<uint32_t>(d)) off += o;
  }
  if (__any_sync(FULL, lane < pll && off >= len8)) return CODAG_ECORRUPT;
  const uint32_t prev = __shfl_up_sync(FULL, off, 1);
  if (__any_sync(FULL, lane > 0 && lane < pll && prev == off)) {
    // several patches on one value: OR the group into its first lane
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t o = shfl_down64(patch, d);
      const uint32_t ooff = __shfl_down_sync(FULL, off, d);
      if (lane + d < pll && ooff == off) patch |= o;
    }
  }
  __syncwarp();
  if (lane < pll && (lane == 0 || prev != off)) {
    const uint64_t v = get_elem<E>(out, n + off);
    put_elem<E>(out, n + off, ((((v - base) & M) | patch) + base) & M);
  }
  return CODAG_OK;
}

// RLE v1 literal group: `remaining` varints from pos (decoder.h:686-727); advances pos
template <int NSLOT, int E, class OUT>
__device__ __forceinline__ int body_literals(InRing<NSLOT>& in, OUT& out, uint32_t n, uint32_t remaining, uint32_t& pos,
                                             uint32_t end, uint32_t lane) {
  constexpr uint64_t M = emask<E>();
  while (remaining) {
    int st = in.advance(pos, min(pos + 148, end));
    if (st) return st;
    const uint32_t q0 = pos + 4 * lane;
    const uint32_t tb = ~in.peek_le32(q0) & 0x80808080u;
    uint32_t nib = ((tb >> 7) & 1u) | ((tb >> 14) & 2u) | ((tb >> 21) & 4u) | ((tb >> 28) & 8u);
    if (q0 + 4 > end) nib &= q0 >= end ? 0u : ((1u << (end - q0)) - 1u);
    const uint32_t b0 = __ballot_sync(FULL, nib & 1u), b1 = __ballot_sync(FULL, nib & 2u);
    const uint32_t b2 = __ballot_sync(FULL, nib & 4u), b3 = __ballot_sync(FULL, nib & 8u);
    const uint32_t lt = lanemask_lt(lane);
    const uint32_t before = __popc(b0 & lt) + __popc(b1 & lt) + __popc(b2 & lt) + __popc(b3 & lt);
    const uint32_t total = __popc(b0) + __popc(b1) + __popc(b2) + __popc(b3);
    if (!total) return CODAG_ECORRUPT;  // a varint longer than 128 bytes
    const uint32_t take = total < remaining ? total : remaining;
    // end of the previous varint: the last end in a lower lane, or the window start
    const uint32_t nz = __ballot_sync(FULL, nib != 0) & lt;
    const uint32_t src = nz ? 31u - __clz(nz) : lane;
    const uint32_t pnib = __shfl_sync(FULL, nib, src);
    uint32_t start = nz ? pos + 4 * src + (32u - __clz(pnib)) : pos;
    uint32_t m = nib, idx = before, last_end = 0;
    while (m && idx < take) {
      const uint32_t q = q0 + __ffs(m) - 1;
      m &= m - 1;
      const uint32_t len = q - start + 1;
      uint64_t v;
      if (len <= 4) {
        v = leb_compact32(in.peek_le32(start), len);
      } else {
        const uint64_t lo8 = in.peek_le64(start);
        v = leb_value(lo8, len > 8 ? in.peek_le64(start + 8) : 0ull, len);
      }
      put_elem<E>(out, n + idx, v & M);
      if (idx == take - 1) last_end = q + 1;
      idx++;
      start = q + 1;
    }
    pos = __reduce_max_sync(FULL, last_end);
    n += take;
    remaining -= take;
  }
  return CODAG_OK;
}

// ---------------------------------------------------------------------------------------
// single-pass decoders: the warp walks the headers itself
// ---------------------------------------------------------------------------------------
// RLE v1, one header at pos (all lanes on the same data): expands it and advances pos and n.
template <int NSLOT, int E, class OUT>
__device__ __forceinline__ int rlev1_header(InRing<NSLOT>& in, OUT& out, uint32_t& pos, uint32_t& n, uint32_t cap,
                                            uint32_t end, uint32_t lane) {
  int st = in.advance(pos, min(pos + 32, end));
  if (st) return st;
  const int h = static_cast<int8_t>(in.rd8(pos));
  uint32_t cnt;
  if (h >= 0) {  // run: count h+3, int8 delta, varint base (decoder.h:731-790)
    if (pos + 2 >= end) return CODAG_ECORRUPT;
    const int64_t delta = static_cast<int8_t>(in.rd8(pos + 1));
    uint32_t len;
    uint64_t base;
    if (!read_uvarint(in, pos + 2, end, len, base)) return CODAG_ECORRUPT;
    cnt = static_cast<uint32_t>(h) + 3u;
    if (n + cnt > cap) return CODAG_ECORRUPT;
    body_fill<E>(out, n, cnt, base, static_cast<uint64_t>(delta), lane);
    pos += 2 + len;
  } else {
    cnt = static_cast<uint32_t>(-h);
    if (n + cnt > cap) return CODAG_ECORRUPT;
    pos += 1;
    st = body_literals<NSLOT, E>(in, out, n, cnt, pos, end, lane);
    if (st) return st;
  }
  n += cnt;
  __syncwarp();
  out.flush_to(n * E);
  return CODAG_OK;
}

// RLE v1: loops while fewer than cap elements were produced, as the reference does
// (decoder.h:669); the warp parses one header at a time.
template <int NSLOT, int E, class OUT>
__device__ int decode_rlev1_chunk(InRing<NSLOT>& in, OUT& out, uint32_t cap) {
  const uint32_t lane = in.lane, end = in.hi;
  uint32_t pos = in.lo, n = 0;
  int st = CODAG_OK;
  while (n < cap) {
    if (pos >= end) { st = CODAG_ECORRUPT; break; }
    st = rlev1_header<NSLOT, E>(in, out, pos, n, cap, end, lane);
    if (st) break;
  }
  if (!in.drain() && st == CODAG_OK) st = CODAG_ETIMEOUT;
  out.finish(n * E);
  if (st == CODAG_OK && n * E < out.store) st = CODAG_ECORRUPT;
  return st;
}

// RLE v2 (unsigned values, include/rlev2/decoder_new.h:909-1187)
//
// One header at pos, all lanes on the same data: expands it and advances pos and n.  Used
// for headers the batched parse below does not size (a varint longer than its 16-byte look,
// a malformed or truncated header).
template <int NSLOT, int E, class OUT>
__device__ __forceinline__ int rlev2_header(InRing<NSLOT>& in, OUT& out, uint32_t& pos, uint32_t& n, uint32_t cap,
                                            uint32_t end, uint32_t lane) {
  constexpr uint64_t M = emask<E>();
  int st = in.advance(pos, min(pos + 32, end));
  if (st) return st;
  const uint64_t hdr = in.peek_be64(pos);
  const uint32_t first = static_cast<uint32_t>(hdr >> 56);
  // the length field is held in a uint8_t (decoder_new.h:1019,1048,1095)
  const uint32_t len8 = ((static_cast<uint32_t>(hdr >> 48) & 0x1ffu) + 1u) & 0xffu;
  uint32_t cnt, total;
  if ((first >> 6) == 0) {  // SHORT_REPEAT (decoder_new.h:1004-1014)
    const uint32_t nb = ((first >> 3) & 7u) + 1u;
    cnt = (first & 7u) + 3u;
    total = 1u + nb;
    if (pos + total > end || n + cnt > cap) return CODAG_ECORRUPT;
    const uint64_t v = nb < 8 ? (hdr << 8) >> (64u - 8u * nb) : in.peek_be64(pos + 1);
    if (lane < cnt) put_elem<E>(out, n + lane, v & M);
  } else if ((first >> 6) == 1) {  // DIRECT (decoder_new.h:1015-1043)
    const uint32_t fbw = v2_width((first >> 1) & 0x1fu);
    cnt = len8;
    total = 2u + (len8 * fbw + 7u) / 8u;
    if (pos + total > end || n + cnt > cap) return CODAG_ECORRUPT;
    st = in.advance(pos, pos + total);
    if (st) return st;
    body_unpack<NSLOT, E>(in, out, n, cnt, (pos + 2u) * 8u, fbw, 0ull, lane);
  } else if ((first >> 6) == 3) {  // DELTA (decoder_new.h:1044-1091)
    const uint32_t enc = (first >> 1) & 0x1fu;
    const uint32_t fbw = v2_width(enc);
    uint32_t l1, l2;
    uint64_t ub, ud;
    if (!read_uvarint(in, pos + 2, end, l1, ub) || !read_uvarint(in, pos + 2 + l1, end, l2, ud)) {
      return CODAG_ECORRUPT;
    }
    const uint64_t base = ub & M;
    const int64_t sd = static_cast<int64_t>(ud);
    const uint64_t bd = static_cast<uint64_t>((sd >> 1) ^ -(sd & 1)) & M;  // arithmetic shift (decoder_new.h:990)
    const uint32_t nd = (len8 - 2u) & 0xffu;                              // "len -= 2" on a uint8_t
    const uint32_t data = pos + 2u + l1 + l2;
    cnt = nd + 2u;
    total = (data - pos) + (enc ? (nd * fbw + 7u) / 8u : 0u);
    if (pos + total > end || n + cnt > cap) return CODAG_ECORRUPT;
    st = in.advance(pos, pos + total);
    if (st) return st;
    if (enc == 0) body_fill<E>(out, n, cnt, base, bd, lane);
    else body_delta_packed<NSLOT, E>(in, out, n, nd, fbw, base, bd, data * 8u, lane);
  } else {  // PATCHED_BASE (decoder_new.h:1092-1183)
    const uint32_t fbw = v2_width((first >> 1) & 0x1fu);
    const uint32_t third = static_cast<uint32_t>(hdr >> 40) & 0xffu;
    const uint32_t fourth = static_cast<uint32_t>(hdr >> 32) & 0xffu;
    const uint32_t bw = ((third >> 5) & 7u) + 1u;
    const uint32_t pw = v2_width(third & 0x1fu);
    const uint32_t pgw = ((fourth >> 5) & 7u) + 1u;
    const uint32_t pll = fourth & 0x1fu;
    if (pw + pgw > 64u) return CODAG_ECORRUPT;
    const uint32_t cfb = v2_closest(pw + pgw);
    const uint32_t vals = pos + 4u + bw;
    const uint32_t patches = vals + (len8 * fbw + 7u) / 8u;
    cnt = len8;
    total = (patches - pos) + (pll * cfb + 7u) / 8u;
    if (pos + total > end || n + cnt > cap) return CODAG_ECORRUPT;
    st = in.advance(pos, pos + total);
    if (st) return st;
    const uint64_t base = in.peek_be64(pos + 4) >> (64u - 8u * bw);
    body_unpack<NSLOT, E>(in, out, n, cnt, vals * 8u, fbw, base, lane);
    if (pll) {
      __syncwarp();
      st = body_patches<NSLOT, E>(in, out, n, len8, fbw, pw, cfb, pll, base, patches * 8u, lane);
      if (st) return st;
    }
  }
  n += cnt;
  pos += total;
  out.flush_to(n * E);
  return CODAG_OK;
}

// Byte size of the RLE v2 header at p from its leading bytes, or 0 when this look cannot
// size it (DELTA varints not both inside the 8 bytes after the header, or a PATCHED_BASE
// header whose patch width exceeds 64 bits).
template <int NSLOT>
__device__ __forceinline__ uint32_t rlev2_size(const InRing<NSLOT>& in, uint32_t p) {
  const uint32_t w = in.peek_be32(p);  // bytes p..p+3, first byte on top
  const uint32_t first = w >> 24;
  const uint32_t len8 = (((w >> 16) & 0x1ffu) + 1u) & 0xffu;
  const uint32_t fbw = v2_width((first >> 1) & 0x1fu);
  switch (first >> 6) {
    case 0: return 2u + ((first >> 3) & 7u);
    case 1: return 2u + (len8 * fbw + 7u) / 8u;
    case 3: {
      const uint64_t t = ~in.peek_le64(p + 2) & 0x8080808080808080ull;
      const uint64_t t2 = t & (t - 1ull);  // the second varint's last byte
      if (!t2) return 0u;
      const uint32_t nd = (len8 - 2u) & 0xffu;
      return 2u + (ctz64(t2) >> 3) + 1u + (((first >> 1) & 0x1fu) ? (nd * fbw + 7u) / 8u : 0u);
    }
    default: {
      const uint32_t third = (w >> 8) & 0xffu, fourth = w & 0xffu;
      const uint32_t pw = v2_width(third & 0x1fu), pgw = ((fourth >> 5) & 7u) + 1u;
      if (pw + pgw > 64u) return 0u;
      return 4u + ((third >> 5) & 7u) + 1u + (len8 * fbw + 7u) / 8u + ((fourth & 0x1fu) * v2_closest(pw + pgw) + 7u) / 8u;
    }
  }
}

// Batched parse: the warp sizes up to 32 consecutive headers whose bytes are resident (a
// short serial walk over their leading bytes), lane j then decodes header j's fields on
// its own, and the headers are expanded in order with their fields taken from lane j by
// shuffles.  Header decoding thus costs one lane-parallel pass per 32 headers instead of
// a warp-uniform pass per header.
template <int NSLOT, int E, class OUT>
__device__ int decode_rlev2_chunk(InRing<NSLOT>& in, OUT& out, uint32_t cap) {
  constexpr uint64_t M = emask<E>();
  const uint32_t lane = in.lane;
  const uint32_t end = in.hi;
  uint32_t pos = in.lo;
  uint32_t n = 0;
  int st = CODAG_OK;
  while (pos < end) {
    // the largest header spans 4 + 8 + 2040 + 248 bytes; make at least that much resident
    if (pos >= in.release_at || min(pos + 2304u, end) > in.ready) {
      st = in.advance(pos, min(pos + 2304u, end));
      if (st) break;
    }
    const uint32_t ready = in.ready;
    const uint32_t lim = min(ready, end);
    // 1. sizes of the next headers (warp-uniform walk over leading bytes only)
    uint32_t k = 0, p = pos, mine = 0;
    while (k < 32 && p < end && (p + 24u <= ready || ready >= end)) {
      const uint32_t sz = rlev2_size(in, p);
      if (!sz || p + sz > lim) break;
      if (lane == k) mine = p;
      p += sz;
      k++;
    }
    if (k == 0) {  // not sizable here: the one-header path decodes it or reports the error
      st = rlev2_header<NSLOT, E>(in, out, pos, n, cap, end, lane);
      if (st) break;
      continue;
    }
    // 2. lane j < k decodes header j
    uint32_t kc = 0, bit = 0, pinfo = 0, pbit = 0;
    uint64_t va = 0, vb = 0;
    if (lane < k) {
      const uint32_t w = in.peek_be32(mine);
      const uint32_t first = w >> 24;
      const uint32_t len8 = (((w >> 16) & 0x1ffu) + 1u) & 0xffu;
      const uint32_t kind = first >> 6;
      uint32_t cnt, fbw = v2_width((first >> 1) & 0x1fu);
      if (kind == 0) {  // SHORT_REPEAT: big-endian value of nb bytes
        const uint32_t nb = ((first >> 3) & 7u) + 1u;
        cnt = (first & 7u) + 3u;
        va = in.peek_be64(mine + 1) >> (64u - 8u * nb);
      } else if (kind == 1) {  // DIRECT
        cnt = len8;
        bit = (mine + 2u) * 8u;
      } else if (kind == 3) {  // DELTA: base and zigzag delta varints, both in these 8 bytes
        const uint64_t lo = in.peek_le64(mine + 2);
        const uint64_t t = ~lo & 0x8080808080808080ull;
        const uint32_t l1 = (ctz64(t) >> 3) + 1u;
        const uint32_t l12 = (ctz64(t & (t - 1ull)) >> 3) + 1u;
        va = leb_compact(lo, l1) & M;
        const int64_t sd = static_cast<int64_t>(leb_compact(lo >> (8u * l1), l12 - l1));
        vb = static_cast<uint64_t>((sd >> 1) ^ -(sd & 1)) & M;  // arithmetic shift (decoder_new.h:990)
        const uint32_t nd = (len8 - 2u) & 0xffu;                // "len -= 2" on a uint8_t
        cnt = nd + 2u;
        if (!((first >> 1) & 0x1fu)) fbw = 0;  // fixed delta
        bit = (mine + 2u + l12) * 8u;
      } else {  // PATCHED_BASE
        const uint32_t third = (w >> 8) & 0xffu, fourth = w & 0xffu;
        const uint32_t bw = ((third >> 5) & 7u) + 1u;
        const uint32_t pw = v2_width(third & 0x1fu);
        const uint32_t cfb = v2_closest(pw + ((fourth >> 5) & 7u) + 1u);
        cnt = len8;
        va = in.peek_be64(mine + 4) >> (64u - 8u * bw);
        bit = (mine + 4u + bw) * 8u;
        pbit = bit + ((len8 * fbw + 7u) / 8u) * 8u;
        pinfo = pw | (cfb << 8) | ((fourth & 0x1fu) << 16);
      }
      kc = kind | (cnt << 2) | (fbw << 12);
    }
    // 3. expand the headers in order
    for (uint32_t j = 0; j < k; j++) {
      const uint32_t c = __shfl_sync(FULL, kc, j);
      const uint32_t kind = c & 3u, cnt = (c >> 2) & 0x3ffu, fbw = c >> 12;
      if (n + cnt > cap) { st = CODAG_ECORRUPT; break; }
      if (kind == 0) {
        const uint64_t v = shfl64(va, j);
        if (lane < cnt) put_elem<E>(out, n + lane, v & M);
      } else if (kind == 1) {
        body_unpack<NSLOT, E>(in, out, n, cnt, __shfl_sync(FULL, bit, j), fbw, 0ull, lane);
      } else if (kind == 3) {
        const uint64_t base = shfl64(va, j), bd = shfl64(vb, j);
        if (fbw == 0) body_fill<E>(out, n, cnt, base, bd, lane);
        else body_delta_packed<NSLOT, E>(in, out, n, cnt - 2u, fbw, base, bd, __shfl_sync(FULL, bit, j), lane);
      } else {
        const uint64_t base = shfl64(va, j);
        const uint32_t pi = __shfl_sync(FULL, pinfo, j);
        body_unpack<NSLOT, E>(in, out, n, cnt, __shfl_sync(FULL, bit, j), fbw, base, lane);
        if (pi >> 16) {
          const uint32_t pb = __shfl_sync(FULL, pbit, j);
          __syncwarp();
          st = body_patches<NSLOT, E>(in, out, n, cnt, fbw, pi & 0xffu, (pi >> 8) & 0xffu, pi >> 16, base, pb, lane);
          if (st) break;
        }
      }
      n += cnt;
      out.flush_to(n * E);
    }
    if (st) break;
    pos = p;
  }
  if (!in.drain() && st == CODAG_OK) st = CODAG_ETIMEOUT;
  out.finish(n * E);
  if (st == CODAG_OK && n * E < out.store) st = CODAG_ECORRUPT;
  return st;
}

// Element-width dispatch for callers that know the width only at run time.
template <int NSLOT, class OUT>
__device__ __noinline__ int decode_rle_any(int codec, InRing<NSLOT>& in, OUT& out, uint64_t chunk_bytes, int e) {
  const uint32_t cap = static_cast<uint32_t>(chunk_bytes / static_cast<uint32_t>(e));
  if (codec == CODAG_CODEC_RLEV1) {
    switch (e) {
      case 8: return decode_rlev1_chunk<NSLOT, 8>(in, out, cap);
      case 4: return decode_rlev1_chunk<NSLOT, 4>(in, out, cap);
      case 2: return decode_rlev1_chunk<NSLOT, 2>(in, out, cap);
      default: return decode_rlev1_chunk<NSLOT, 1>(in, out, cap);
    }
  }
  switch (e) {
    case 8: return decode_rlev2_chunk<NSLOT, 8>(in, out, cap);
    case 4: return decode_rlev2_chunk<NSLOT, 4>(in, out, cap);
    case 2: return decode_rlev2_chunk<NSLOT, 2>(in, out, cap);
    default: return decode_rlev2_chunk<NSLOT, 1>(in, out, cap);
  }
}

}  // namespace codag_dev
