// Warp decoder for one Deflate (RFC 1951) chunk.
//
// CODAG's decoder (include/zlib/zlib.h:807-902) decodes with 5-bit literal/length and 8-bit
// distance lookup tables, walks code lengths 6..15 serially on a miss, copies
// back-references with 4-byte pieces and ignores stored blocks.  This decoder keeps the
// same one-warp-per-chunk shape but:
//   - builds per-block lookup tables in shared memory of LB (9..11) bits for literals and
//     lengths and 8 bits for distances, in parallel over the warp (canonical codes are
//     tiled in MSB-first order, so each table slot finds its code by walking lengths);
//   - keeps a 64-bit bit buffer refilled 32 bits at a time from the TMA input ring;
//   - decodes a length or distance code together with its extra bits (one table entry
//     gives both widths) and two literals per step where the table slot holds both codes;
//   - expands back-references warp-cooperatively out of a shared-memory window of the
//     output (the OUT ring: 1 or 2 KiB in the kernels here); older sources are read back
//     from the chunk's already-written output, and such a load (length <= 32) is left in
//     flight while the next symbols decode;
//   - drains output in quarter-window pieces with vector stores;
//   - decodes stored blocks.
// Every lane runs the same symbol loop on the same data (shared-memory reads broadcast), so
// control flow stays uniform and only the stores are lane-specific.
#pragma once
#include "device_common.cuh"

namespace codag_dev {

__constant__ uint16_t kLenBase[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                      31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
__constant__ uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                      2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
__constant__ uint16_t kDistBase[30] = {1,    2,    3,    4,    5,    7,     9,     13,    17,  25,
                                       33,   49,   65,   97,   129,  193,   257,   385,   513, 769,
                                       1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
__constant__ uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2,  3,  3,  4,  4,  5,  5,  6,
                                       6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
__constant__ uint8_t kCodeLenOrder[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

constexpr uint32_t kDistLB = 8;
constexpr uint32_t kCodeLenLB = 7;

// Table entry (32 bits):
//   [0,5)   bits consumed in all: code length + extra bits, or both codes of a literal pair
//   [5,9)   code length of the (first) symbol
//   [9,11)  kind: literal(s), length, end of block, other (invalid, or not in the table)
//   [11]    a second literal follows in [24,32) (literal/length tables only)
//   [12]    the code is longer than the table: decode it with slow_entry
//   [16,32) literal byte in [16,24) / length or distance base / code-length symbol
enum : uint32_t {
  kKindShift = 9,
  kKindMask = 3u << kKindShift,
  kKindLitBits = 0u,
  kKindLenBits = 1u << kKindShift,
  kKindEndBits = 2u << kKindShift,
  kKindBadBits = 3u << kKindShift,
  kPairFlag = 1u << 11,
  kSlowFlag = 1u << 12,
  kSlowEntry = kKindBadBits | kSlowFlag,
};
enum : int { kAlphaLitLen = 0, kAlphaDist = 1, kAlphaCodeLen = 2 };

__device__ __forceinline__ uint32_t entry_bits(uint32_t total, uint32_t len) { return total | (len << 5); }

__device__ __forceinline__ uint32_t make_entry(uint32_t sym, uint32_t len, int alpha) {
  if (alpha == kAlphaLitLen) {
    if (sym < 256) return entry_bits(len, len) | kKindLitBits | (sym << 16);
    if (sym == 256) return entry_bits(len, len) | kKindEndBits;
    if (sym <= 285) {
      const uint32_t k = sym - 257;
      return entry_bits(len + kLenExtra[k], len) | kKindLenBits | (static_cast<uint32_t>(kLenBase[k]) << 16);
    }
    return entry_bits(len, len) | kKindBadBits;
  }
  if (alpha == kAlphaDist) {
    if (sym < 30) return entry_bits(len + kDistExtra[sym], len) | (static_cast<uint32_t>(kDistBase[sym]) << 16);
    return entry_bits(len, len) | kKindBadBits;
  }
  return entry_bits(len, len) | (sym << 16);
}

// `n` bits of `x` starting at bit `pos` (pos + n <= 32; n may be 0)
__device__ __forceinline__ uint32_t bfe32(uint32_t x, uint32_t pos, uint32_t n) {
  uint32_t r;
  asm("bfe.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(pos), "r"(n));
  return r;
}

struct HuffTable {
  uint32_t* lut;     // 1 << lb entries
  uint16_t* sorted;  // symbols ordered by (code length, symbol)
  uint32_t* cnt;     // [16] codes per length
  uint32_t* first;   // [16] first canonical code per length
  uint32_t* index;   // [16] position of the first code of each length in `sorted`
  uint32_t lb;
};

// Builds `t` from code lengths lens[0..nsym).  False when the lengths over-subscribe the
// code space.  Incomplete codes are accepted; their unused codes decode as invalid.
__device__ bool build_table(const uint8_t* lens, uint32_t nsym, const HuffTable& t, int alpha,
                            uint32_t* fill, uint32_t lane) {
  if (lane < 16) t.cnt[lane] = 0;
  __syncwarp();
  for (uint32_t s = lane; s < nsym; s += 32) {
    const uint32_t l = lens[s];
    if (l) atomicAdd(&t.cnt[l], 1u);
  }
  __syncwarp();
  uint32_t ok = 1;
  if (lane == 0) {
    uint32_t code = 0, idx = 0;
    int left = 1;
    for (uint32_t l = 1; l < 16; l++) {
      t.first[l] = code;
      code = (code + t.cnt[l]) << 1;
      t.index[l] = idx;
      fill[l] = idx;
      idx += t.cnt[l];
      left = (left << 1) - static_cast<int>(t.cnt[l]);
      if (left < 0) ok = 0;
    }
  }
  ok = __shfl_sync(FULL, ok, 0);
  __syncwarp();
  if (!ok) return false;
  for (uint32_t s0 = 0; s0 < nsym; s0 += 32) {
    const uint32_t s = s0 + lane;
    const uint32_t l = s < nsym ? lens[s] : 0u;
    const uint32_t grp = __match_any_sync(FULL, l);
    const uint32_t rank = __popc(grp & lanemask_lt(lane));
    if (l) t.sorted[fill[l] + rank] = static_cast<uint16_t>(s);
    __syncwarp();
    if (l && rank == 0) fill[l] += __popc(grp);
    __syncwarp();
  }
  const uint32_t n = 1u << t.lb;
  for (uint32_t x = lane; x < n; x += 32) {
    const uint32_t v = __brev(x) >> (32 - t.lb);  // MSB-first code prefix of table slot x
    uint32_t entry = kSlowEntry;
    for (uint32_t l = 1; l <= t.lb; l++) {
      const uint32_t k = (v >> (t.lb - l)) - t.first[l];
      if (k < t.cnt[l]) {
        entry = make_entry(t.sorted[t.index[l] + k], l, alpha);
        break;
      }
    }
    t.lut[x] = entry;
  }
  __syncwarp();
  if (alpha == kAlphaLitLen) {
    // literal pairs: when the bits of slot x after its literal code hold a whole literal
    // code too, the entry carries both.  Only the first-literal fields of the other slot
    // are read, and a pair rewrite leaves those fields unchanged, so lanes need no order.
    for (uint32_t x = lane; x < n; x += 32) {
      const uint32_t e1 = t.lut[x];
      const uint32_t l1 = (e1 >> 5) & 15u;
      if ((e1 & kKindMask) != kKindLitBits || l1 >= t.lb) continue;
      const uint32_t e2 = t.lut[x >> l1];
      const uint32_t l2 = (e2 >> 5) & 15u;
      if ((e2 & kKindMask) != kKindLitBits || l1 + l2 > t.lb) continue;
      t.lut[x] = (e1 & ~31u & 0x00ffffffu) | (l1 + l2) | kPairFlag | ((e2 & 0x00ff0000u) << 8);
    }
    __syncwarp();
  }
  return true;
}

// Codes longer than the table width: walk lengths lb+1..15 (zlib.h:459-527 does 6..15).
__device__ __forceinline__ uint32_t slow_entry(uint64_t bb, const HuffTable& t, int alpha) {
  const uint32_t rev = __brev(static_cast<uint32_t>(bb));
  for (uint32_t l = t.lb + 1; l < 16; l++) {
    const uint32_t k = (rev >> (32 - l)) - t.first[l];
    if (k < t.cnt[l]) return make_entry(t.sorted[t.index[l] + k], l, alpha);
  }
  return 0;
}

// Per-warp shared memory of the Deflate decoder: the current block's canonical codes, and
// (InflateScratch) its lookup tables.  The batched kernel can keep the lookup tables in
// global memory instead (read through L1), which frees 3-9 KiB of shared memory per warp.
struct InflateCodes {
  uint32_t lit_cnt[16], lit_first[16], lit_index[16];
  uint32_t dist_cnt[16], dist_first[16], dist_index[16];
  uint32_t fill[16];
  uint16_t lit_sorted[288];
  uint16_t dist_sorted[32];
  uint8_t lens[320];
};
template <int LB>
struct InflateScratch : InflateCodes {
  uint32_t lit_lut[1u << LB];
  uint32_t dist_lut[1u << kDistLB];
};
// entries of the global-memory tables of one warp
template <int LB>
constexpr uint32_t kLutEntries = (1u << LB) + (1u << kDistLB);

// table entry i: a shared-memory table (saddr) or a global one (p)
template <bool GT>
__device__ __forceinline__ uint32_t lut_ld(const uint32_t* p, uint32_t saddr, uint32_t i) {
  if constexpr (GT) return p[i];
  else return ld_s32(saddr + 4u * i);
}

template <int NSLOT>
struct BitReader {
  uint64_t bb;    // pending bits, next bit in bit 0
  uint32_t bc;    // number of pending bits
  uint32_t wpos;  // ring position of the next 32-bit word (multiple of 4)

  // append one word; returns a status (corruption = read far beyond the stream)
  __device__ __forceinline__ int refill(InRing<NSLOT>& in) {
    if (wpos < in.hi) {
      const uint32_t end = min(wpos + 4, in.hi);
      if (end > (in.waited << kSlotLog2)) {
        // the buffer holds at most 8 bytes before wpos; everything older is consumed
        if (!in.release(wpos >= 8 ? wpos - 8 : 0)) return CODAG_ETIMEOUT;
        const int st = in.ensure(end);
        if (st) return st;
      }
    } else if (wpos > in.hi + 16) {
      return CODAG_ECORRUPT;
    }
    bb |= static_cast<uint64_t>(in.rd32(wpos)) << bc;
    bc += 32;
    wpos += 4;
    return CODAG_OK;
  }

  __device__ __forceinline__ void start(InRing<NSLOT>& in, uint32_t p) {
    wpos = p & ~3u;
    bb = 0;
    bc = 0;
    (void)in;
  }
  __device__ __forceinline__ void drop(uint32_t n) {
    bb >>= n;
    bc -= n;
  }
  // stream position (ring coordinates) of the next unread bit, times 8
  __device__ __forceinline__ uint64_t bitpos() const { return static_cast<uint64_t>(wpos) * 8u - bc; }
};

// ---------------------------------------------------------------------------------------
// Decoder/expander pairs (one CTA of two warps per chunk)
// ---------------------------------------------------------------------------------------
// The decoder warp runs the block and symbol loops below but emits tokens instead of bytes; the
// expander warp turns the tokens into output through the usual window.  Tokens travel in two
// shared-memory batches handed over with a named barrier of the pair's 64 threads: after
// barrier k the decoder fills one batch while the expander drains the other, and each side
// reaches barrier k+1 only when done with its batch, so neither ever spins.
// Token: bit 31 set = one or two literals (bits 0-7, 8-15; bit 16 = two); clear = a match,
// length in bits 0-8 and distance in bits 9-24.
// 496 tokens a batch: the two batches and their counters fit in 4 KiB (the batched kernel keeps
// them in the expander warp's idle input ring)
constexpr uint32_t kTokBatch = 496;
struct TokenShared {
  uint32_t tok[2][kTokBatch];
  uint32_t cnt[2];
  uint32_t done;
  int32_t status;
  uint32_t job;  // batched kernel: the pair's current job
};
static_assert(sizeof(TokenShared) <= 4096, "token batches must fit a 4 KiB ring");

__device__ __forceinline__ void pair_barrier(uint32_t id) {
  asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory");
}

struct NoTokens {  // single-warp decode: bytes go straight to the window
  static constexpr bool kOn = false;
  __device__ __forceinline__ void literal(uint32_t, uint32_t) {}
  __device__ __forceinline__ void match(uint32_t, uint32_t) {}
};

struct TokenPipe {
  static constexpr bool kOn = true;
  TokenShared* sh;
  uint32_t bar, k, n, lane;
  __device__ __forceinline__ void handoff() {
    __syncwarp();
    if (lane == 0) sh->cnt[k] = n;
    pair_barrier(bar);
    k ^= 1u;
    n = 0;
  }
  __device__ __forceinline__ void push(uint32_t t) {
    // lane 0 writes the token: a predicated store, no branch on the lane
    const uint32_t a = smem_u32(&sh->tok[k][n]);
    asm volatile("{ .reg .pred p; setp.eq.u32 p, %0, 0; @p st.shared.u32 [%1], %2; }" ::"r"(lane), "r"(a), "r"(t)
                 : "memory");
    if (++n == kTokBatch) handoff();
  }
  // one literal, or two (second in bits 8-15 when `two`)
  __device__ __forceinline__ void literal(uint32_t bytes, uint32_t two) { push(0x80000000u | (two << 16) | bytes); }
  __device__ __forceinline__ void match(uint32_t len, uint32_t dist) { push(len | (dist << 9)); }
  // the last batch, with the decoder's status
  __device__ __forceinline__ void finish(int st) {
    __syncwarp();
    if (lane == 0) {
      sh->cnt[k] = n;
      sh->status = st;
      sh->done = 1;
    }
    pair_barrier(bar);
  }
};

// Output stand-in for the decoder warp of a pair, which writes no bytes itself.
struct NullOut {
  static constexpr uint32_t kBytes = 4096, kFlush = 1024;
  uint32_t flushed = 0, store = 0;
  uint8_t* gdst = nullptr;
  __device__ __forceinline__ void put8(uint32_t, uint32_t) {}
  __device__ __forceinline__ uint32_t get8(uint32_t) const { return 0; }
  __device__ __forceinline__ void flush_to(uint32_t) {}
  __device__ __forceinline__ void finish(uint32_t) {}
};

// GT: lit_lut / dist_lut are global memory (else shared memory, e.g. InflateScratch's).
template <int NSLOT, int LB, class OUT, class TOK = NoTokens, bool GT = false>
__device__ int decode_deflate_chunk(InRing<NSLOT>& in, OUT& out, InflateCodes& sc, uint32_t* lit_lut,
                                    uint32_t* dist_lut, uint64_t chunk_bytes, uint32_t wrapper, TOK* tok = nullptr) {
  // Before each symbol fewer than kFlush bytes of the window are unflushed; what is written
  // until the next flush (a match of up to 258 bytes, a piece of a stored block) must not wrap
  // onto them.
  static_assert(OUT::kBytes - OUT::kFlush >= 258, "window too small for a match");
  constexpr uint32_t kStoredPiece = OUT::kBytes - OUT::kFlush < 1024u ? OUT::kBytes - OUT::kFlush : 1024u;
  const uint32_t lane = in.lane;
  const uint32_t cap = static_cast<uint32_t>(chunk_bytes);
  const HuffTable lit{lit_lut, sc.lit_sorted, sc.lit_cnt, sc.lit_first, sc.lit_index, LB};
  const HuffTable dst{dist_lut, sc.dist_sorted, sc.dist_cnt, sc.dist_first, sc.dist_index, kDistLB};
  const HuffTable cl{dist_lut, sc.dist_sorted, sc.dist_cnt, sc.dist_first, sc.dist_index, kCodeLenLB};
  const uint32_t s_lit = GT ? 0u : smem_u32(lit_lut), s_dist = GT ? 0u : smem_u32(dist_lut);

  uint32_t op = 0;  // bytes produced (chunks are < 2 GiB)
  int st = CODAG_OK;
  BitReader<NSLOT> br;
  const uint32_t lit_sh = 16u + 8u * (lane & 1u);  // first literal in bits 16-23, second in 24-31
  bool fixed_ready = false;

  if (in.lo + wrapper > in.hi) st = CODAG_ECORRUPT;
  if (!st && !in.release(in.lo)) st = CODAG_ETIMEOUT;
  const uint32_t start = in.lo + wrapper;
  br.start(in, start);
  if (!st) st = br.refill(in);
  if (!st) br.drop((start & 3u) * 8u);

#define CODAG_REFILL()                   \
  if (br.bc < 32) {                      \
    st = br.refill(in);                  \
    if (st) break;                       \
  }
  // one deferred far copy: pend_len bytes for [pend_op, pend_end), byte `lane` in pend_val
  uint32_t pend_op = 0, pend_len = 0, pend_end = 0, pend_val = 0;
#define CODAG_COMPLETE()                                              \
  if (pend_len) {                                                     \
    if (lane < pend_len) out.put8(pend_op + lane, pend_val);          \
    pend_len = 0;                                                     \
    pend_end = 0;                                                     \
  }
#define CODAG_FLUSH()   \
  {                     \
    CODAG_COMPLETE();   \
    out.flush_to(op);   \
  }

  bool last = false;
  while (!st && !last) {
    if (br.bitpos() > static_cast<uint64_t>(in.hi) * 8u) { st = CODAG_ECORRUPT; break; }
    CODAG_REFILL();
    last = br.bb & 1u;
    const uint32_t btype = static_cast<uint32_t>(br.bb >> 1) & 3u;
    br.drop(3);
    if (btype == 0) {  // stored block
      br.drop(br.bc & 7u);
      CODAG_REFILL();
      const uint32_t len = static_cast<uint32_t>(br.bb) & 0xffffu;
      const uint32_t nlen = static_cast<uint32_t>(br.bb >> 16) & 0xffffu;
      br.drop(32);
      if (len != (~nlen & 0xffffu)) { st = CODAG_ECORRUPT; break; }
      uint32_t p = br.wpos - br.bc / 8u;
      if (p + len > in.hi || op + len > cap) { st = CODAG_ECORRUPT; break; }
      uint32_t left = len;
      while (left) {
        const uint32_t piece = left < kStoredPiece ? left : kStoredPiece;
        if (!in.release(p)) { st = CODAG_ETIMEOUT; break; }
        st = in.ensure(p + piece);
        if (st) break;
        if constexpr (TOK::kOn) {  // two bytes per literal token
          for (uint32_t t = 0; t < piece; t += 2) {
            const uint32_t two = t + 1 < piece ? 1u : 0u;
            tok->literal(in.rd8(p + t) | (two ? in.rd8(p + t + 1) << 8 : 0u), two);
          }
        } else {
          for (uint32_t t = lane; t < piece; t += 32) out.put8(op + t, in.rd8(p + t));
        }
        op += piece;
        p += piece;
        left -= piece;
        __syncwarp();
        CODAG_FLUSH();
      }
      if (st) break;
      br.start(in, p);
      st = br.refill(in);
      if (st) break;
      br.drop((p & 3u) * 8u);
      continue;
    }
    if (btype == 3) { st = CODAG_ECORRUPT; break; }
    if (btype == 1) {  // fixed Huffman codes (RFC 1951 3.2.6)
      if (!fixed_ready) {
        for (uint32_t s = lane; s < 320; s += 32)
          sc.lens[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : s < 288 ? 8 : 5;
        __syncwarp();
        build_table(sc.lens, 288, lit, kAlphaLitLen, sc.fill, lane);
        build_table(sc.lens + 288, 30, dst, kAlphaDist, sc.fill, lane);
        fixed_ready = true;
      }
    } else {  // dynamic Huffman codes (zlib.h:607-707)
      fixed_ready = false;
      CODAG_REFILL();
      const uint32_t hlit = (static_cast<uint32_t>(br.bb) & 31u) + 257u;
      const uint32_t hdist = (static_cast<uint32_t>(br.bb >> 5) & 31u) + 1u;
      const uint32_t hclen = (static_cast<uint32_t>(br.bb >> 10) & 15u) + 4u;
      br.drop(14);
      if (hlit > 286 || hdist > 30) { st = CODAG_ECORRUPT; break; }
      // code length code lengths, 3 bits each in kCodeLenOrder order
      for (uint32_t i0 = 0; i0 < 19; i0 += 10) {
        CODAG_REFILL();
        const uint32_t i = i0 + lane;
        if (lane < 10 && i < 19) {
          const uint32_t v = i < hclen ? static_cast<uint32_t>(br.bb >> (3 * lane)) & 7u : 0u;
          sc.lens[kCodeLenOrder[i]] = static_cast<uint8_t>(v);
        }
        const uint32_t took = hclen > i0 ? min(hclen - i0, 10u) : 0u;
        br.drop(3 * took);
      }
      if (st) break;
      __syncwarp();
      if (!build_table(sc.lens, 19, cl, kAlphaCodeLen, sc.fill, lane)) { st = CODAG_ECORRUPT; break; }
      // literal/length and distance code lengths, run-length coded with symbols 16..18
      uint32_t idx = 0, prev = 0;
      const uint32_t total = hlit + hdist;
      while (idx < total) {
        CODAG_REFILL();
        const uint32_t e = lut_ld<GT>(dist_lut, s_dist, static_cast<uint32_t>(br.bb & ((1u << kCodeLenLB) - 1u)));
        if (e & kSlowFlag) { st = CODAG_ECORRUPT; break; }  // code lengths are at most 7 bits
        br.drop(e & 31u);
        const uint32_t sym = e >> 16;
        if (sym < 16) {
          if (lane == 0) sc.lens[idx] = static_cast<uint8_t>(sym);
          prev = sym;
          idx++;
          continue;
        }
        uint32_t rep, val = 0;
        if (sym == 16) {
          if (idx == 0) { st = CODAG_ECORRUPT; break; }
          val = prev;
          rep = 3u + (static_cast<uint32_t>(br.bb) & 3u);
          br.drop(2);
        } else if (sym == 17) {
          rep = 3u + (static_cast<uint32_t>(br.bb) & 7u);
          br.drop(3);
        } else {
          rep = 11u + (static_cast<uint32_t>(br.bb) & 127u);
          br.drop(7);
        }
        if (idx + rep > total) { st = CODAG_ECORRUPT; break; }
        for (uint32_t t = lane; t < rep; t += 32) sc.lens[idx + t] = static_cast<uint8_t>(val);
        prev = val;
        idx += rep;
      }
      if (st) break;
      __syncwarp();
      if (sc.lens[256] == 0) { st = CODAG_ECORRUPT; break; }
      // the distance lengths follow the literal/length lengths; move them to their slot
      uint8_t dl = 0;
      if (lane < hdist) dl = sc.lens[hlit + lane];
      __syncwarp();
      for (uint32_t s = hlit + lane; s < 288; s += 32) sc.lens[s] = 0;
      __syncwarp();
      if (lane < 32) sc.lens[288 + lane] = lane < hdist ? dl : 0;
      __syncwarp();
      if (!build_table(sc.lens, hlit, lit, kAlphaLitLen, sc.fill, lane)) { st = CODAG_ECORRUPT; break; }
      if (!build_table(sc.lens + 288, hdist, dst, kAlphaDist, sc.fill, lane)) { st = CODAG_ECORRUPT; break; }
    }

    // symbol loop (zlib.h:712-805)
    for (;;) {
      CODAG_REFILL();
      uint32_t e = lut_ld<GT>(lit_lut, s_lit, static_cast<uint32_t>(br.bb) & ((1u << LB) - 1u));
      if ((e & kKindMask) == kKindLitBits) {  // one literal or a pair
        const uint32_t pair = (e >> 11) & 1u;
        br.drop(e & 31u);
        if constexpr (TOK::kOn) {
          tok->literal(((e >> 16) & 0xffu) | ((e >> 16) & 0xff00u), pair);
          op += 1u + pair;
          continue;
        } else {
          // lane 0 stores the literal, lane 1 the second of a pair: one predicated byte store
          // of the entry shifted by lit_sh, with no branch on the lane
          const uint32_t a = out.sbuf + ((op + lane) & OUT::kMask);
          asm volatile("{ .reg .pred p; setp.le.u32 p, %0, %1; @p st.shared.u8 [%2], %3; }" ::"r"(lane), "r"(pair),
                       "r"(a), "r"(e >> lit_sh)
                       : "memory");
          op += 1u + pair;
          if (op - out.flushed >= OUT::kFlush) CODAG_FLUSH();
          continue;
        }
      }
      if (e & kSlowFlag) {
        e = slow_entry(br.bb, lit, kAlphaLitLen);
        if (!e) { st = CODAG_ECORRUPT; break; }
        if ((e & kKindMask) == kKindLitBits) {
          br.drop(e & 31u);
          if constexpr (TOK::kOn) {
            tok->literal((e >> 16) & 0xffu, 0u);
            op++;
            continue;
          }
          if (lane == 0) out.put8(op, (e >> 16) & 0xffu);
          op++;
          if (op - out.flushed >= OUT::kFlush) CODAG_FLUSH();
          continue;
        }
      }
      if ((e & kKindMask) == kKindEndBits) {
        br.drop(e & 31u);
        break;
      }
      if ((e & kKindMask) != kKindLenBits) { st = CODAG_ECORRUPT; break; }
      // length: code and extra bits in one step (at most 20 bits; 32 are buffered)
      const uint32_t ln = (e >> 5) & 15u, lt = e & 31u;
      const uint32_t len = (e >> 16) + bfe32(static_cast<uint32_t>(br.bb), ln, lt - ln);
      br.drop(lt);
      if (br.bc < 28) {  // distance code and extra bits take at most 28 bits
        st = br.refill(in);
        if (st) break;
      }
      uint32_t d = lut_ld<GT>(dist_lut, s_dist, static_cast<uint32_t>(br.bb) & ((1u << kDistLB) - 1u));
      if (d & kSlowFlag) {
        d = slow_entry(br.bb, dst, kAlphaDist);
        if (!d) { st = CODAG_ECORRUPT; break; }
      }
      if (d & kKindMask) { st = CODAG_ECORRUPT; break; }
      const uint32_t dn = (d >> 5) & 15u, dt = d & 31u;
      const uint32_t dist = (d >> 16) + bfe32(static_cast<uint32_t>(br.bb), dn, dt - dn);
      br.drop(dt);
      if (dist > op || op + len > cap) { st = CODAG_ECORRUPT; break; }
      if constexpr (TOK::kOn) {
        tok->match(len, dist);
        op += len;
        continue;
      }
      const uint32_t src = op - dist;
      if (dist + len <= OUT::kBytes) {  // source still in the shared-memory window
        if (src < pend_end) CODAG_COMPLETE();
        __syncwarp();
        if (dist >= len) {
          for (uint32_t t = lane; t < len; t += 32) out.put8(op + t, out.get8(src + t));
        } else {
          uint32_t r = lane % dist;
          const uint32_t step = 32u % dist;
          for (uint32_t t = lane; t < len; t += 32) {
            out.put8(op + t, out.get8(src + r));
            r += step;
            if (r >= dist) r -= dist;
          }
        }
      } else if (len <= 32) {
        // older than the window: the bytes were flushed to the chunk's output already.  The
        // load is issued now and its bytes enter the window later (CODAG_COMPLETE), so the
        // memory latency overlaps the next symbols.
        CODAG_COMPLETE();
        pend_val = (lane < len && src + lane < out.store) ? static_cast<uint32_t>(out.gdst[src + lane]) : 0u;
        pend_op = op;
        pend_len = len;
        pend_end = op + len;
      } else {
        CODAG_COMPLETE();
        const uint32_t r0 = dist >= len ? lane : lane % dist;
        const uint32_t step = dist >= len ? 32u : 32u % dist;
        uint32_t r = r0;
        for (uint32_t t = lane; t < len; t += 32) {
          const uint32_t sp = src + r;
          out.put8(op + t, sp < out.store ? out.gdst[sp] : 0u);  // unstored bytes are never stored either
          r += step;
          if (dist < len && r >= dist) r -= dist;
        }
      }
      op += len;
      if (op - out.flushed >= OUT::kFlush) CODAG_FLUSH();
    }
  }
  CODAG_COMPLETE();
#undef CODAG_FLUSH
#undef CODAG_COMPLETE
#undef CODAG_REFILL
  if (!in.drain() && st == CODAG_OK) st = CODAG_ETIMEOUT;
  out.finish(op);
  if (st == CODAG_OK && (op < out.store || op > cap || br.bitpos() > static_cast<uint64_t>(in.hi) * 8u))
    st = CODAG_ECORRUPT;
  return st;
}

// Expander warp of a pair: drains the decoder's token batches into `out` (the window and far
// copies of decode_deflate_chunk).  Returns CODAG_OK or CODAG_ECORRUPT (fewer bytes than the
// stored part); the decoder's status arrives in sh->status.
template <class OUT>
__device__ int expand_tokens(TokenShared* sh, uint32_t bar, OUT& out, uint32_t lane) {
  static_assert(OUT::kBytes - OUT::kFlush >= 258, "window too small for a match");
  uint32_t op = 0, k = 0;
  const uint32_t tok_sh = 8u * (lane & 1u);  // a literal token: first byte in bits 0-7, second in 8-15
  uint32_t pend_op = 0, pend_len = 0, pend_end = 0, pend_val = 0;
#define CODAG_COMPLETE()                                     \
  if (pend_len) {                                            \
    if (lane < pend_len) out.put8(pend_op + lane, pend_val); \
    pend_len = 0;                                            \
    pend_end = 0;                                            \
  }
  for (;;) {
    pair_barrier(bar);
    const uint32_t cnt = sh->cnt[k], done = sh->done;
    const uint32_t s_tok = smem_u32(sh->tok[k]);
    for (uint32_t i = 0; i < cnt; i++) {
      const uint32_t t = ld_s32(s_tok + 4u * i);
      if (t >> 31) {  // literals: lane 0 stores the first, lane 1 the second (predicated)
        const uint32_t two = (t >> 16) & 1u;
        const uint32_t a = out.sbuf + ((op + lane) & OUT::kMask);
        asm volatile("{ .reg .pred p; setp.le.u32 p, %0, %1; @p st.shared.u8 [%2], %3; }" ::"r"(lane), "r"(two),
                     "r"(a), "r"(t >> tok_sh)
                     : "memory");
        op += 1u + two;
      } else {
        const uint32_t len = t & 0x1ffu, dist = (t >> 9) & 0xffffu;
        const uint32_t src = op - dist;
        if (dist + len <= OUT::kBytes) {  // source still in the shared-memory window
          if (src < pend_end) CODAG_COMPLETE();
          __syncwarp();
          if (dist >= len) {
            for (uint32_t q = lane; q < len; q += 32) out.put8(op + q, out.get8(src + q));
          } else {
            uint32_t r = lane % dist;
            const uint32_t step = 32u % dist;
            for (uint32_t q = lane; q < len; q += 32) {
              out.put8(op + q, out.get8(src + r));
              r += step;
              if (r >= dist) r -= dist;
            }
          }
        } else if (len <= 32) {  // flushed already: load now, write into the window later
          CODAG_COMPLETE();
          pend_val = (lane < len && src + lane < out.store) ? static_cast<uint32_t>(out.gdst[src + lane]) : 0u;
          pend_op = op;
          pend_len = len;
          pend_end = op + len;
        } else {
          CODAG_COMPLETE();
          const uint32_t r0 = dist >= len ? lane : lane % dist;
          const uint32_t step = dist >= len ? 32u : 32u % dist;
          uint32_t r = r0;
          for (uint32_t q = lane; q < len; q += 32) {
            const uint32_t sp = src + r;
            out.put8(op + q, sp < out.store ? out.gdst[sp] : 0u);
            r += step;
            if (dist < len && r >= dist) r -= dist;
          }
        }
        op += len;
      }
      if (op - out.flushed >= OUT::kFlush) {
        CODAG_COMPLETE();
        out.flush_to(op);
      }
    }
    k ^= 1u;
    if (done) break;
  }
  CODAG_COMPLETE();
#undef CODAG_COMPLETE
  out.finish(op);
  return op < out.store ? CODAG_ECORRUPT : CODAG_OK;
}

}  // namespace codag_dev
