// Warp decoders for ORC RLE v1 and ORC RLE v2 chunks.
//
// CODAG decodes these with one lane walking the stream byte by byte and the other 31 lanes
// idle or storing the same addresses (include/rlev1/decoder.h:588-798,
// include/rlev2/decoder_new.h:909-1187).  Here the header walk stays sequential (each
// header's size depends on its contents) but everything inside a header is lane-parallel:
//   RLE v1  literal groups: 32 stream bytes per step, varint ends found with one ballot of
//           the byte MSBs, values assembled by a segmented OR scan; runs: one value per lane.
//   RLE v2  DIRECT/PATCHED_BASE values unpacked one per lane by direct bit addressing;
//           DELTA deltas unpacked one per lane and accumulated with a warp scan;
//           PATCHED_BASE patch gaps accumulated with a warp scan and applied by the first
//           lane of each group of patches that hit the same value.
// Decoded values go to the shared-memory output ring (OutRing) and leave it as 16-byte stores.
// Arithmetic on values is modulo 2^(8*elem_bytes), with the reference's quirks kept
// (see oracle/oracle.c for the list).
#pragma once
#include "device_common.cuh"

namespace codag_dev {

__device__ __forceinline__ uint64_t elem_mask(int e) { return e == 8 ? ~0ull : ((1ull << (8 * e)) - 1ull); }

__constant__ uint8_t kV2WidthDecode[32] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11,
                                           12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22,
                                           23, 24, 26, 28, 30, 32, 40, 48, 56, 64};
__constant__ uint8_t kV2Closest[65] = {
    1,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21,
    22, 23, 24, 26, 26, 28, 28, 30, 30, 32, 32, 40, 40, 40, 40, 40, 40, 40, 40, 48, 48, 48,
    48, 48, 48, 48, 48, 56, 56, 56, 56, 56, 56, 56, 56, 64, 64, 64, 64, 64, 64, 64, 64};

// ---------------------------------------------------------------------------------------
// ORC RLE v1
// ---------------------------------------------------------------------------------------
// Decodes one chunk.  Loops while fewer than chunk_bytes bytes were produced, as the
// reference does (decoder.h:669).
template <int NSLOT, class OUT>
__device__ int decode_rlev1_chunk(InRing<NSLOT>& in, OUT& out, uint64_t chunk_bytes, int e) {
  const uint32_t lane = in.lane;
  const uint64_t m = elem_mask(e);
  const uint64_t cap = chunk_bytes / static_cast<uint32_t>(e);
  uint32_t pos = in.lo;
  const uint32_t end = in.hi;
  uint64_t n = 0;
  int st = CODAG_OK;

  while (n < cap) {
    if (pos >= end) { st = CODAG_ECORRUPT; break; }
    if (!in.release(pos)) { st = CODAG_ETIMEOUT; break; }
    // header, delta and base varint, or the start of a literal group
    st = in.ensure(min(pos + 34, end));
    if (st) break;
    const int h = static_cast<int8_t>(in.rd8(pos));
    if (h >= 0) {
      // run: count h+3, int8 delta, varint base (decoder.h:731-790)
      if (pos + 2 >= end) { st = CODAG_ECORRUPT; break; }
      const int64_t delta = static_cast<int8_t>(in.rd8(pos + 1));
      const uint32_t q = pos + 2 + lane;
      const uint32_t b = q < end ? in.rd8(q) : 0x80u;
      const uint32_t term = __ballot_sync(FULL, b < 0x80u);
      if (!term) { st = CODAG_ECORRUPT; break; }
      const uint32_t len = __ffs(term);  // bytes of the base varint
      const uint64_t base = warp_or64(lane < len ? shl64(b & 0x7fu, 7u * lane) : 0ull);
      const uint32_t cnt = static_cast<uint32_t>(h) + 3u;
      if (n + cnt > cap) { st = CODAG_ECORRUPT; break; }
      for (uint32_t i = lane; i < cnt; i += 32)
        out.put(n + i, (base + static_cast<uint64_t>(static_cast<int64_t>(i) * delta)) & m, e);
      n += cnt;
      pos += 2 + len;
    } else {
      // literal group of -h varints (decoder.h:686-727)
      uint32_t remaining = static_cast<uint32_t>(-h);
      if (n + remaining > cap) { st = CODAG_ECORRUPT; break; }
      pos += 1;
      while (remaining) {
        if (!in.release(pos)) { st = CODAG_ETIMEOUT; break; }
        st = in.ensure(min(pos + 32, end));
        if (st) break;
        const uint32_t q = pos + lane;
        const bool valid = q < end;
        const uint32_t b = valid ? in.rd8(q) : 0x80u;
        const uint32_t term = __ballot_sync(FULL, valid && b < 0x80u);
        if (!term) { st = CODAG_ECORRUPT; break; }
        // byte `lane` belongs to varint number `seg`, which started after the previous end
        const uint32_t below = term & lanemask_lt(lane);
        const uint32_t seg = __popc(below);
        const uint32_t start = below ? 32u - __clz(below) : 0u;
        uint64_t v = shl64(b & 0x7fu, 7u * (lane - start));
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {  // segmented inclusive OR scan
          const uint64_t o = shfl_up64(v, d);
          const uint32_t oseg = __shfl_up_sync(FULL, seg, d);
          if (lane >= static_cast<uint32_t>(d) && oseg == seg) v |= o;
        }
        const uint32_t avail = __popc(term);
        const uint32_t take = avail < remaining ? avail : remaining;
        if (((term >> lane) & 1u) && seg < take) out.put(n + seg, v & m, e);
        // position after the take-th varint end
        const uint32_t last_end = __ballot_sync(FULL, ((term >> lane) & 1u) && seg == take - 1u);
        pos += static_cast<uint32_t>(__ffs(last_end));
        n += take;
        remaining -= take;
        __syncwarp();
        out.flush_to(n * static_cast<uint32_t>(e));
      }
      if (st) break;
    }
    __syncwarp();
    out.flush_to(n * static_cast<uint32_t>(e));
  }
  if (!in.drain() && st == CODAG_OK) st = CODAG_ETIMEOUT;
  out.finish(n * static_cast<uint32_t>(e));
  if (st == CODAG_OK && n * static_cast<uint32_t>(e) < out.store) st = CODAG_ECORRUPT;
  return st;
}

// ---------------------------------------------------------------------------------------
// ORC RLE v2 (unsigned values, include/rlev2/decoder_new.h:909-1187)
// ---------------------------------------------------------------------------------------
template <int NSLOT, class OUT>
__device__ int decode_rlev2_chunk(InRing<NSLOT>& in, OUT& out, uint64_t chunk_bytes, int e) {
  const uint32_t lane = in.lane;
  const uint64_t m = elem_mask(e);
  const uint64_t cap = chunk_bytes / static_cast<uint32_t>(e);
  uint32_t pos = in.lo;
  const uint32_t end = in.hi;
  uint64_t n = 0;
  int st = CODAG_OK;

  while (pos < end) {
    if (!in.release(pos)) { st = CODAG_ETIMEOUT; break; }
    st = in.ensure(min(pos + 32, end));
    if (st) break;
    const uint64_t hdr = in.peek_be64(pos);
    const uint32_t first = static_cast<uint32_t>(hdr >> 56);
    const uint32_t second = static_cast<uint32_t>(hdr >> 48) & 0xffu;
    const uint32_t kind = first & 0xC0u;
    // the length field is held in a uint8_t (decoder_new.h:1019,1048,1095)
    const uint32_t len8 = ((((first & 1u) << 8) | second) + 1u) & 0xffu;

    if (kind == 0x00u) {  // SHORT_REPEAT (decoder_new.h:1004-1014)
      const uint32_t nb = ((first >> 3) & 7u) + 1u;
      const uint32_t cnt = (first & 7u) + 3u;
      if (pos + 1 + nb > end) { st = CODAG_ECORRUPT; break; }
      if (n + cnt > cap) { st = CODAG_ECORRUPT; break; }
      const uint64_t v = (in.peek_be64(pos + 1) >> (64u - 8u * nb)) & m;
      if (lane < cnt) out.put(n + lane, v, e);
      n += cnt;
      pos += 1 + nb;
    } else if (kind == 0x40u) {  // DIRECT (decoder_new.h:1015-1043)
      const uint32_t fbw = kV2WidthDecode[(first >> 1) & 0x1fu];
      const uint32_t total = 2u + (len8 * fbw + 7u) / 8u;
      if (pos + total > end || n + len8 > cap) { st = CODAG_ECORRUPT; break; }
      st = in.ensure(pos + total);
      if (st) break;
      const uint32_t bit0 = (pos + 2u) * 8u;
      for (uint32_t j = lane; j < len8; j += 32) out.put(n + j, in.bits_be(bit0 + j * fbw, fbw) & m, e);
      n += len8;
      pos += total;
    } else if (kind == 0xC0u) {  // DELTA (decoder_new.h:1044-1091)
      const uint32_t enc = (first >> 1) & 0x1fu;
      const uint32_t fbw = kV2WidthDecode[enc];
      // base (unsigned varint) and base delta (signed varint), one byte per lane
      const uint32_t q = pos + 2 + lane;
      const uint32_t b = (lane < 30 && q < end) ? in.rd8(q) : 0x80u;
      const uint32_t term = __ballot_sync(FULL, b < 0x80u);
      const uint32_t l1 = __ffs(term);
      const uint32_t rest = l1 ? (term & (~0u << l1)) : 0u;
      const uint32_t l2end = __ffs(rest);
      if (!l1 || !l2end) { st = CODAG_ECORRUPT; break; }
      const uint64_t base = warp_or64(lane < l1 ? shl64(b & 0x7fu, 7u * lane) : 0ull) & m;
      const uint64_t ud = warp_or64((lane >= l1 && lane < l2end) ? shl64(b & 0x7fu, 7u * (lane - l1)) : 0ull);
      const int64_t sd = static_cast<int64_t>(ud);
      const uint64_t bd = static_cast<uint64_t>((sd >> 1) ^ -(sd & 1)) & m;  // arithmetic shift
      const uint32_t nd = (len8 - 2u) & 0xffu;                              // "len -= 2" on a uint8_t
      const uint32_t data = pos + 2u + l2end;
      const uint32_t total = (data - pos) + (enc ? (nd * fbw + 7u) / 8u : 0u);
      const uint32_t cnt = nd + 2u;
      if (pos + total > end || n + cnt > cap) { st = CODAG_ECORRUPT; break; }
      st = in.ensure(pos + total);
      if (st) break;
      if (enc == 0) {
        for (uint32_t t = lane; t < cnt; t += 32) out.put(n + t, (base + static_cast<uint64_t>(t) * bd) & m, e);
      } else {
        const bool plus = bd != 0;  // multiplier = base_delta > 0 ? 1 : -1 on the unsigned type
        const uint64_t v1 = (base + bd) & m;
        if (lane == 0) out.put(n, base, e);
        if (lane == 1) out.put(n + 1, v1, e);
        uint64_t carry = v1;
        const uint32_t bit0 = data * 8u;
        for (uint32_t k0 = 0; k0 < nd; k0 += 32) {
          const uint32_t k = k0 + lane;
          const uint64_t d = k < nd ? (in.bits_be(bit0 + k * fbw, fbw) & m) : 0ull;
          const uint64_t s = warp_scan_add64(d, lane);
          const uint64_t v = (plus ? carry + s : carry - s) & m;
          if (k < nd) out.put(n + 2 + k, v, e);
          carry = shfl64(v, 31);
        }
      }
      n += cnt;
      pos += total;
    } else {  // PATCHED_BASE (decoder_new.h:1092-1183)
      const uint32_t fbw = kV2WidthDecode[(first >> 1) & 0x1fu];
      const uint32_t third = static_cast<uint32_t>(hdr >> 40) & 0xffu;
      const uint32_t fourth = static_cast<uint32_t>(hdr >> 32) & 0xffu;
      const uint32_t bw = ((third >> 5) & 7u) + 1u;
      const uint32_t pw = kV2WidthDecode[third & 0x1fu];
      const uint32_t pgw = ((fourth >> 5) & 7u) + 1u;
      const uint32_t pll = fourth & 0x1fu;
      if (pw + pgw > 64u) { st = CODAG_ECORRUPT; break; }
      const uint32_t cfb = kV2Closest[pw + pgw];
      const uint32_t vals = pos + 4u + bw;
      const uint32_t patches = vals + (len8 * fbw + 7u) / 8u;
      const uint32_t total = (patches - pos) + (pll * cfb + 7u) / 8u;
      if (pos + total > end || n + len8 > cap) { st = CODAG_ECORRUPT; break; }
      st = in.ensure(pos + total);
      if (st) break;
      const uint64_t base = in.peek_be64(pos + 4) >> (64u - 8u * bw);
      for (uint32_t j = lane; j < len8; j += 32)
        out.put(n + j, (in.bits_be(vals * 8u + j * fbw, fbw) + base) & m, e);
      __syncwarp();
      if (pll) {
        // the reference masks patches with a 32-bit mask (decoder_new.h:1103)
        const uint64_t pmask = pw >= 32 ? 0xffffffffull : ((1ull << pw) - 1ull);
        uint64_t ent = 0, gap = 0, patch = 0;
        if (lane < pll) {
          ent = in.bits_be(patches * 8u + lane * cfb, cfb);
          gap = shr64(ent, pw);
          patch = shl64((ent & pmask) & m, fbw) & m;
        }
        const uint64_t off = warp_scan_add64(gap, lane);
        const bool bad = __any_sync(FULL, lane < pll && off >= len8);
        if (bad) { st = CODAG_ECORRUPT; break; }
        // OR together the patches of a group of equal offsets into its first lane
        uint64_t acc = patch;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint64_t o = shfl_down64(acc, d);
          const uint64_t ooff = shfl_down64(off, d);
          if (lane + d < pll && ooff == off) acc |= o;
        }
        const uint64_t prev_off = shfl_up64(off, 1);
        const bool head = lane < pll && (lane == 0 || prev_off != off);
        if (head) {
          const uint64_t idx = n + off;
          const uint64_t v = out.get(idx, e);
          out.put(idx, ((((v - base) & m) | acc) + base) & m, e);
        }
      }
      n += len8;
      pos += total;
    }
    __syncwarp();
    out.flush_to(n * static_cast<uint32_t>(e));
  }
  if (!in.drain() && st == CODAG_OK) st = CODAG_ETIMEOUT;
  out.finish(n * static_cast<uint32_t>(e));
  if (st == CODAG_OK && n * static_cast<uint32_t>(e) < out.store) st = CODAG_ECORRUPT;
  return st;
}

}  // namespace codag_dev
