// Decoder of CODAG's transposed RLE v2 layout (include/codag.h, codag_decompress_rlev2_transposed).
//
// In that layout (include/rlev2/encoder_trans.h:8-182 and 359-391) a chunk is 32 substreams,
// substream t holding the values t*ru + k*32*ru + j (j < ru), and the chunk's bytes interleave
// the substreams in 4-byte words: word w of every substream longer than 4w, in substream
// order, then word w+1.  CODAG decodes it with one lane per substream fed by a reader warp
// through spin queues (include/rlev2/decoder_new.h:375-632, 1193-1230).  Here one warp
// decodes a chunk with no queue.  The set of substreams that still have a word w only shrinks
// as w grows, so it changes at most 32 times: the warp tabulates those segments of rows (first
// and last row, the mask of substreams present, the words before the segment; at most 32
// entries, 512 bytes of shared memory per warp), and lane t finds its word w at
// start + (w - first row) * popc(mask) + popc(mask & lanes below t) by itself.  Then every
// lane decodes its own substream and writes its values straight to their interleaved places
// in global memory.  The small table leaves occupancy to the registers, so many chunks' lanes
// wait on their word loads at once.  Header semantics are CODAG's (the oracle's restatement of
// decoder_new.h:1000-1184, quirks included: the uint8_t run length, the 32-bit patch mask, the
// arithmetic-shift zigzag and the DELTA direction taken from the base delta).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../../include/codag.h"
#include "../rlev2_widths.h"

namespace {

constexpr uint32_t FULL = 0xffffffffu;

__device__ __forceinline__ uint64_t shl64(uint64_t v, uint32_t s) { return s >= 64 ? 0ull : v << s; }
__device__ __forceinline__ uint64_t shr64(uint64_t v, uint32_t s) { return s >= 64 ? 0ull : v >> s; }

// bytes of one lane's substream, read word by word from the interleaved region
// row segments of one chunk (shared memory): rows lo[s] <= w < hi[s] hold a word of exactly the
// substreams in mask[s], and words[s] words of the region come before row lo[s]
struct Segments {
  uint32_t hi[32], lo[32], mask[32], words[32];
};

constexpr uint32_t kWarps = 4;  // chunks (warps) per block

struct LaneReader {
  const uint32_t* region;  // the chunk's region (128-byte aligned)
  const Segments* seg;
  uint32_t total;          // words in the region
  uint32_t lt;             // lanes below this one
  uint32_t len;            // substream bytes
  uint32_t p;              // next byte
  uint32_t cw, cv;         // cached word index and value
  uint32_t s;              // segment of cw (rows only grow, so it only moves forward)
  bool bad;

  // where word w of this substream sits in the region; w < its word count <= the last
  // segment's hi keeps the walk inside the table, and the region has `total` words
  __device__ __forceinline__ uint32_t start(uint32_t w) {
    while (w >= seg->hi[s]) s++;
    const uint32_t m = seg->mask[s];
    const uint32_t at = seg->words[s] + (w - seg->lo[s]) * __popc(m) + __popc(m & lt);
    if (at >= total) {
      bad = true;
      return 0;
    }
    return at;
  }

  __device__ __forceinline__ uint32_t byte() {
    if (p >= len) {
      bad = true;
      return 0;
    }
    const uint32_t w = p >> 2;
    if (w != cw) {
      cw = w;
      cv = __ldg(region + start(w));
    }
    return (cv >> (8u * (p++ & 3u))) & 0xffu;
  }

  // the next k (1..8) bytes as one big-endian number, a word's worth of bytes per step
  __device__ __forceinline__ uint64_t take(uint32_t k) {
    if (k > len - p) {
      bad = true;
      return 0;
    }
    uint64_t v = 0;
    while (k) {
      const uint32_t w = p >> 2;
      if (w != cw) {
        cw = w;
        cv = __ldg(region + start(w));
      }
      const uint32_t o = p & 3u, m = k < 4u - o ? k : 4u - o;
      const uint32_t be = __byte_perm(cv, 0u, 0x0123u) << (8u * o);  // stream bytes o.. at the top
      v = (v << (8u * m)) | (be >> (32u - 8u * m));
      p += m;
      k -= m;
    }
    return v;
  }
};

// MSB-first bits local to one header (decoder_new.h:1024-1040): `cur` holds the last byte
// taken, its low `left` bits not yet read
struct HeaderBits {
  uint32_t cur, left;
  __device__ __forceinline__ uint64_t read(LaneReader& r, uint32_t n) {  // n <= 64
    if (n <= left) {
      left -= n;
      return (cur >> left) & ((1u << n) - 1u);
    }
    const uint32_t need = n - left, k = (need + 7u) >> 3;
    const uint64_t hi = cur & ((1u << left) - 1u);
    const uint64_t lo = r.take(k);
    left = 8u * k - need;
    cur = static_cast<uint32_t>(lo) & 0xffu;
    return shl64(hi, need) | (lo >> left);
  }
};

// value k of substream t lands on element t*ru + (k/ru)*32*ru + k%ru of the chunk
template <typename T>
struct LaneOut {
  T* chunk;
  uint32_t t, ru, cap, store;  // cap: values per substream; store: elements of the chunk to store
  uint32_t n;
  uint32_t e, j;  // element of value n, and n % ru (stepped without a division)
  bool over;
  __device__ __forceinline__ uint32_t elem(uint32_t k) const { return t * ru + (k / ru) * 32u * ru + k % ru; }
  __device__ __forceinline__ void put(uint64_t v) {
    if (n >= cap) {
      over = true;
      return;
    }
    if (e < store) chunk[e] = static_cast<T>(v);
    n++;
    if (++j == ru) {  // next group of ru values, 32 * ru elements on
      j = 0;
      e += 31u * ru + 1u;
    } else {
      e++;
    }
  }
  __device__ __forceinline__ uint64_t get(uint32_t k) const {
    const uint32_t e = elem(k);
    return e < store ? static_cast<uint64_t>(chunk[e]) : 0ull;
  }
  __device__ __forceinline__ void set(uint32_t k, uint64_t v) {
    const uint32_t e = elem(k);
    if (e < store) chunk[e] = static_cast<T>(v);
  }
};

__device__ __forceinline__ uint64_t uvarint(LaneReader& r) {
  uint64_t v = 0;
  uint32_t off = 0, b;
  do {
    b = r.byte();
    if (r.bad) return 0;
    v |= shl64(b & 0x7fu, off);
    off += 7;
  } while (b >= 0x80u);
  return v;
}

// One lane's substream as a state machine that yields one value per pass: a lane whose run
// ends reads its next header while the other lanes go on with theirs, so the warp's lanes
// meet again after every value instead of waiting for the longest run among them.  Every run
// kind yields its next value by one step, x = v + d or v - d (v kept as x for the kinds that
// accumulate), d being the run's next bit field or a constant, so the only fork inside the
// step is whether the lane reads bits.

template <typename T>
__device__ int decode_substream(LaneReader& r, LaneOut<T>& o) {
  constexpr uint64_t M = sizeof(T) == 8 ? ~0ull : ((1ull << (8 * sizeof(T))) - 1ull);
  uint32_t rem = 0, fbw = 0;
  uint64_t v = 0, bd = 0;  // repeat: the value; delta: running value and base delta; patched: base
  bool bits = false, acc = false, sub = false, patched = false;
  uint32_t pw = 0, pgw = 0, pll = 0, base_out = 0;  // patched: patch width, gap width, list length
  HeaderBits b{0, 0};
  for (;;) {
    if (rem == 0) {
      if (patched) {  // the run's values are out: patch them (decoder_new.h:1166-1183)
        if (pw + pgw > 64) return CODAG_ECORRUPT;
        const uint64_t pmask = pw >= 32 ? 0xFFFFFFFFull : ((1ull << pw) - 1ull);  // 32-bit mask (:1103)
        const uint32_t cfb = v2_closest(pw + pgw);
        b = HeaderBits{0, 0};
        uint64_t gap = 0;
        while (pll-- > 0) {
          const uint64_t ent = b.read(r, cfb);
          gap += shr64(ent, pw);
          const uint64_t idx = base_out + gap;
          if (r.bad || idx >= o.n || o.over) return CODAG_ECORRUPT;
          const uint64_t patch = shl64((ent & pmask) & M, fbw) & M;
          const uint64_t x = o.get(static_cast<uint32_t>(idx));
          o.set(static_cast<uint32_t>(idx), ((((x - v) & M) | patch) + v) & M);
        }
        if (r.bad || o.over) return CODAG_ECORRUPT;
      }
      patched = false;
      if (r.p >= r.len) break;
      const uint32_t first = r.byte();
      b = HeaderBits{0, 0};
      switch (first & 0xC0u) {
        case 0x00: {  // SHORT_REPEAT (decoder_new.h:1004-1014)
          rem = (first & 7u) + 3u;
          v = r.take(((first >> 3) & 7u) + 1u) & M;  // a big-endian value of 1..8 bytes
          bd = 0;
          bits = sub = false;
          acc = true;
        } break;
        case 0x40:  // DIRECT (decoder_new.h:1015-1043)
          fbw = v2_width((first >> 1) & 0x1fu);
          rem = static_cast<uint8_t>((((first & 1u) << 8) | r.byte()) + 1u);  // a uint8_t length (:1018)
          v = 0;
          bits = true;
          acc = sub = false;
          break;
        case 0xC0: {  // DELTA (decoder_new.h:1044-1091)
          const uint32_t enc = (first >> 1) & 0x1fu;
          fbw = v2_width(enc);
          const uint8_t len = static_cast<uint8_t>((((first & 1u) << 8) | r.byte()) + 1u);
          v = uvarint(r) & M;
          const int64_t u = static_cast<int64_t>(uvarint(r));
          bd = static_cast<uint64_t>((u >> 1) ^ -(u & 1)) & M;  // arithmetic shift (:990)
          o.put(v);
          v = (v + bd) & M;
          o.put(v);
          rem = static_cast<uint8_t>(len - 2);
          bits = enc != 0;  // else every step adds the base delta
          sub = bits && bd == 0;  // multiplier = base_delta > 0 ? 1 : -1 on the unsigned type (:1057)
          acc = true;
        } break;
        default: {  // PATCHED_BASE (decoder_new.h:1092-1165)
          fbw = v2_width((first >> 1) & 0x1fu);
          rem = static_cast<uint8_t>((((first & 1u) << 8) | r.byte()) + 1u);
          const uint32_t h = static_cast<uint32_t>(r.take(2));  // third and fourth header bytes
          pw = v2_width((h >> 8) & 0x1fu);
          pgw = ((h >> 5) & 7u) + 1u;
          pll = h & 0x1fu;
          base_out = o.n;
          v = r.take(((h >> 13) & 7u) + 1u);  // the big-endian base, 1..8 bytes
          bits = patched = true;
          acc = sub = false;
        } break;
      }
      if (r.bad || o.over) return CODAG_ECORRUPT;
      if (rem == 0) continue;
    }
    const uint64_t d = bits ? b.read(r, fbw) & M : bd;
    const uint64_t x = (sub ? v - d : v + d) & M;
    if (acc) v = x;
    o.put(x);
    rem--;
    if (r.bad || o.over) return CODAG_ECORRUPT;
  }
  return CODAG_OK;
}

// values of substream t whose elements fall below `store`
__device__ __forceinline__ uint32_t needed(uint32_t t, uint32_t ru, uint32_t store) {
  const uint32_t grp = 32u * ru, g = store / grp, rem = store % grp;
  const uint32_t lo = t * ru;
  return g * ru + (rem > lo ? (rem - lo < ru ? rem - lo : ru) : 0u);
}

template <typename T>
__global__ void __launch_bounds__(32 * kWarps)
    k_rlev2_transposed(const uint8_t* __restrict__ comp, uint64_t comp_bytes, const uint64_t* __restrict__ blk_off,
                       const uint64_t* __restrict__ col_len, uint64_t n_chunks, uint64_t chunk_bytes, uint32_t ru,
                       uint8_t* __restrict__ out, uint64_t out_bytes, int32_t* __restrict__ status,
                       uint32_t max_words) {
  __shared__ Segments segs[kWarps];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint64_t c = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
  if (c >= n_chunks) return;
  Segments* seg = segs + warp;
  const uint64_t len64 = col_len[32 * c + lane];
  const uint32_t words = static_cast<uint32_t>(len64 < (1ull << 34) ? (len64 + 3) / 4 : 0xffffffffu);
  const uint32_t maxw = __reduce_max_sync(FULL, words);
  const uint64_t total = 4ull * __reduce_add_sync(FULL, words);
  const uint64_t off = blk_off[c];
  int st = CODAG_OK;
  if (maxw > max_words || (off & 3u) || off > comp_bytes || total > comp_bytes - off) st = CODAG_ECORRUPT;
  const uint64_t base_e = c * (chunk_bytes / sizeof(T));
  const uint64_t store_b = c * chunk_bytes < out_bytes ? (out_bytes - c * chunk_bytes < chunk_bytes
                                                             ? out_bytes - c * chunk_bytes : chunk_bytes) : 0;
  const uint32_t store = static_cast<uint32_t>(store_b / sizeof(T));
  if (st == CODAG_OK) {
    // one segment per distinct word count: each pass drops at least one substream, so at most 32
    uint32_t run = 0, row = 0, ns = 0;
    for (uint32_t m = __ballot_sync(FULL, words > 0); m; m = __ballot_sync(FULL, words > row)) {
      const uint32_t nxt = __reduce_min_sync(FULL, words > row ? words : 0xffffffffu);
      if (lane == 0) {
        seg->hi[ns] = nxt;
        seg->lo[ns] = row;
        seg->mask[ns] = m;
        seg->words[ns] = run;
      }
      run += (nxt - row) * __popc(m);
      row = nxt;
      ns++;
    }
    __syncwarp();
    LaneReader r{reinterpret_cast<const uint32_t*>(comp + off), seg, run, (1u << lane) - 1u,
                 static_cast<uint32_t>(len64), 0, 0xffffffffu, 0, 0, false};
    LaneOut<T> o{reinterpret_cast<T*>(out) + base_e, lane, ru,
                 static_cast<uint32_t>(chunk_bytes / sizeof(T) / 32), store, 0, lane * ru, 0, false};
    int s = decode_substream<T>(r, o);
    if (s == CODAG_OK && o.n < needed(lane, ru, store)) s = CODAG_ECORRUPT;
    st = __reduce_max_sync(FULL, static_cast<uint32_t>(s));
  }
  if (status && lane == 0) status[c] = st;
}

bool valid_elem(int e) { return e == 1 || e == 2 || e == 4 || e == 8; }

template <typename T>
codag_status launch(const uint8_t* comp, uint64_t comp_bytes, const uint64_t* blk_off, const uint64_t* col_len,
                    uint64_t n, uint64_t chunk, uint32_t ru, uint8_t* out, uint64_t out_bytes, int32_t* status,
                    cudaStream_t s) {
  // a substream is at most about twice its share of the chunk (the encoders' bound), in words
  const uint32_t max_words = static_cast<uint32_t>((chunk / 32 * 2 + 1024) / 4);
  const uint64_t grid = (n + kWarps - 1) / kWarps;
  if (grid > 0x7fffffffull) return CODAG_EINVAL;
  k_rlev2_transposed<T><<<static_cast<unsigned>(grid), 32 * kWarps, 0, s>>>(comp, comp_bytes, blk_off, col_len, n,
                                                                            chunk, ru, out, out_bytes, status,
                                                                            max_words);
  return cudaGetLastError() == cudaSuccess ? CODAG_OK : CODAG_ECUDA;
}

}  // namespace

extern "C" codag_status codag_decompress_rlev2_transposed(const uint8_t* d_comp, uint64_t comp_bytes,
                                                          const uint64_t* d_blk_off, const uint64_t* d_col_len,
                                                          uint64_t n_chunks, uint64_t chunk_bytes, int elem_bytes,
                                                          int read_unit, uint8_t* d_out, uint64_t out_bytes,
                                                          int32_t* d_chunk_status, codag_stream_t stream) {
  if (!d_comp || !d_blk_off || !d_col_len || (!d_out && out_bytes) || !valid_elem(elem_bytes) || read_unit <= 0 ||
      chunk_bytes == 0 || chunk_bytes >= (1ull << 31) ||
      chunk_bytes % (32ull * static_cast<uint64_t>(read_unit) * static_cast<uint64_t>(elem_bytes)) ||
      (reinterpret_cast<uintptr_t>(d_out) % elem_bytes) || (reinterpret_cast<uintptr_t>(d_comp) & 3u))
    return CODAG_EINVAL;
  if (n_chunks == 0) return CODAG_OK;
  (void)cudaGetLastError();  // an error earlier work left pending is not this call's
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const uint32_t ru = static_cast<uint32_t>(read_unit);
  switch (elem_bytes) {
    case 8: return launch<uint64_t>(d_comp, comp_bytes, d_blk_off, d_col_len, n_chunks, chunk_bytes, ru, d_out, out_bytes, d_chunk_status, s);
    case 4: return launch<uint32_t>(d_comp, comp_bytes, d_blk_off, d_col_len, n_chunks, chunk_bytes, ru, d_out, out_bytes, d_chunk_status, s);
    case 2: return launch<uint16_t>(d_comp, comp_bytes, d_blk_off, d_col_len, n_chunks, chunk_bytes, ru, d_out, out_bytes, d_chunk_status, s);
    default: return launch<uint8_t>(d_comp, comp_bytes, d_blk_off, d_col_len, n_chunks, chunk_bytes, ru, d_out, out_bytes, d_chunk_status, s);
  }
}
