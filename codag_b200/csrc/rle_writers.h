// ORC RLE v1 and RLE v2 chunk writers, shared by the host producers (host/encode_rle*.cpp) and
// the GPU encoders (kernels/encode_capi.cu), so both emit the same bytes.
//
// RleV1Writer produces the byte stream of CODAG's encoder include/rlev1/encoder.h:1352-1695
// (compression_warp_orig, driven by deflate_orig :1800-1840).  Format, one stream per chunk:
//   literal group: header (int8) -n, then n unsigned LEB128 varints          (n <= 127)
//   run:           header h in [0,126], int8 delta, varint base; h+3 values  (<= 129 values)
// The writer holds the last two values, opens a literal group whose header byte is a
// placeholder (later patched to -count), and switches to a run once three values share one
// step in [-128,127].  All comparisons and differences are evaluated in the element type's own
// C++ arithmetic (uint32 differences are never negative, uint8/uint16 promote to int),
// because that is what the reference computes.
//
// RleV2Writer produces the byte stream of CODAG's encoder include/rlev2/encoder_trans.h:184-357
// (block_encode_orig) with the helpers of include/rlev2/encoder.h:56-591 (determineEncoding,
// the four header writers, the patch-list builder and the bit/percentile helpers), except for
// one header (a run of 128 zeros, see write_direct).  It keeps up to 128 pending values,
// tracks a fixed run (equal values) and a variable run, and when a run is closed chooses among
//   SHORT_REPEAT  3..10 equal values, value in 1..8 big-endian bytes
//   DELTA         fixed step (width code 0) or monotonic packed deltas
//   DIRECT        values bit packed at an aligned width
//   PATCHED_BASE  base-reduced values at the 95th-percentile width plus (gap, patch) pairs
// Values are zero-extended to 64 bits and are never zigzagged (include/rlev2/utils.h:8); only
// the DELTA base delta is a signed varint.  Kept behaviours of the reference encoder: runs are
// cut at 128 values; a pending group with minimum 0 and maximum <= 128 is written DIRECT
// (is_safe_subtract, encoder.h:55-60); the width of DELTA deltas is computed on the unsigned
// deltas.
//
// A Sink has put(byte), size() and set(position, byte).
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "rlev2_widths.h"

namespace codag_fmt {

// The RLE v1 writer's bulk steps: none when one thread runs the writer (host producers).  A warp
// whose lanes all run the writer on the same values (the GPU encoder) supplies lane(), ballot(),
// shuffles and an exclusive sum, and takes the values of a literal stream or of a run going on
// many at a time (RleV1Writer::bulk).
struct SerialV1 {
  static constexpr bool kBulk = false;
};

template <typename T, class Sink, class G = SerialV1>
class RleV1Writer {
 public:
  CODAG_HD explicit RleV1Writer(Sink& out) : out_(out) {}
  CODAG_HD RleV1Writer(Sink& out, const G& g) : out_(out), g_(g) {}

  // n >= 2 values, value i read as get(i)
  template <class Get>
  CODAG_HD void encode(const Get& get, uint64_t n) {
    // first value
    uint64_t i = 0;
    T x = get(i++);
    run_len_ = 1;
    prev_ = x;
    push_hist(x);
    held_ = 1;

    // second value
    x = get(i++);
    int64_t d = static_cast<int64_t>(x - prev_);
    if (d > 127 || d < -128) {
      in_run_ = false;
      lit_hdr_ = out_.size();
      put_varint(static_cast<T>(1));
      lit_n_ = 1;
      put_varint(hist_[0]);
      held_--;
    } else {
      in_run_ = true;
      step_ = static_cast<int8_t>(d);
      run_len_++;
    }
    prev_ = x;
    push_hist(x);
    held_++;

    for (; i < n; i++) {
      if constexpr (G::kBulk) {
        const uint32_t took = bulk(get, i, n);
        if (took) {
          i += took - 1;  // the loop's increment moves to the first value not taken
          continue;
        }
      }
      if (lit_n_ == 127) close_literals();
      x = get(i);

      if (run_len_ == 1) {
        d = static_cast<int64_t>(x - prev_);
        if (d > 127 || d < -128) {
          in_run_ = false;
          if (lit_n_ == 0) open_literals(1);
          put_varint(hist_[head_ ^ 1]);
          lit_n_++;
          held_--;
        } else {
          in_run_ = true;
          step_ = static_cast<int8_t>(d);
          run_len_++;
        }
        prev_ = x;
        push_hist(x);
        held_++;
        continue;
      }

      if (prev_ + step_ == x && in_run_) {
        run_len_++;
        if (run_len_ == 3) {
          run_first_ = hist_[head_];
          if (lit_n_ != 0) close_literals();
        } else if (run_len_ == 130) {
          put(static_cast<uint8_t>(static_cast<int8_t>(run_len_ - 4)));
          put(static_cast<uint8_t>(step_));
          put_varint(run_first_);
          run_len_ = 1;
          held_ = 0;
          lit_n_ = 0;
        }
        push_hist(x);
        held_ = held_ + 1 < 2 ? held_ + 1 : 2;
        prev_ = x;
        continue;
      }

      if (run_len_ >= 3) {
        put(static_cast<uint8_t>(static_cast<int8_t>(run_len_ - 3)));
        put(static_cast<uint8_t>(step_));
        put_varint(run_first_);
        run_len_ = 1;
        held_ = 0;
        lit_n_ = 0;
        push_hist(x);
        held_ = held_ + 1 < 2 ? held_ + 1 : 2;
        prev_ = x;
        continue;
      }

      // a two-value prefix that did not become a run: the older value is a literal
      if (lit_n_ == 0) open_literals(3);
      lit_n_++;
      put_varint(hist_[head_]);
      if (lit_n_ == 127) close_literals();
      int64_t d2 = static_cast<int64_t>(x - prev_);
      if (d2 > 127 || d2 < -128) {
        if (lit_n_ == 0) open_literals(3);
        in_run_ = false;
        held_ = 0;
        put_varint(hist_[head_ ^ 1]);
        lit_n_++;
        run_len_ = 1;
      } else {
        held_ = 1;
        in_run_ = true;
        step_ = static_cast<int8_t>(d2);
        run_len_ = 2;
      }
      prev_ = x;
      push_hist(x);
      held_ = held_ + 1 < 2 ? held_ + 1 : 2;
    }

    // flush
    if (run_len_ >= 3 && in_run_) {
      put(static_cast<uint8_t>(static_cast<int8_t>(run_len_ - 3)));
      put(static_cast<uint8_t>(step_));
      put_varint(run_first_);
      return;
    }
    if (held_ == 1) {
      if (lit_n_ == 127) close_literals();
      if (lit_n_ == 0) {
        lit_hdr_ = out_.size();
        put_varint(static_cast<T>(1));
      }
      put_varint(hist_[head_ ^ 1]);
      lit_n_++;
    }
    if (held_ == 2) {
      if (lit_n_ == 127) close_literals();
      if (lit_n_ == 0) open_literals(1);
      put_varint(hist_[head_]);
      lit_n_++;
      if (lit_n_ == 127) close_literals();
      if (lit_n_ == 0) open_literals(1);
      head_ ^= 1;
      put_varint(hist_[head_]);
      lit_n_++;
    }
    out_.set(lit_hdr_, static_cast<uint8_t>(static_cast<int8_t>(-static_cast<int>(lit_n_))));
  }

 private:
  // Values i, i+1, ... (at most one per lane) that take the same steps as the value before them:
  // in a run going on (three or more values, step in range), values that continue it, while the
  // run stays below 130 values; in a literal stream (one value held), values whose step from the
  // one before is out of range, each writing the value before it as a literal.  The steps are
  // the per-value ones of encode() below, done for all taken values at once; returns the count
  // (0: encode() takes value i).
  template <class Get>
  CODAG_HD uint32_t bulk(const Get& get, uint64_t i, uint64_t n) {
    const uint32_t lane = g_.lane();
    const uint64_t j = i + lane;
    const bool in = j < n;
    const T x = in ? static_cast<T>(get(j)) : T(0);
    T before = g_.template shfl_up<T>(x);
    if (lane == 0) before = prev_;
    uint32_t take;
    if (run_len_ >= 3 && in_run_) {
      const uint32_t stop = g_.ballot(!(in && before + step_ == x));
      take = stop ? g_.ffs(stop) - 1u : 32u;
      const uint32_t room = 129u - run_len_;  // the value making 130 writes the run (encode())
      if (take > room) take = room;
      if (!take) return 0;
      run_len_ = static_cast<uint16_t>(run_len_ + take);
      held_ = static_cast<uint8_t>(held_ + take < 2 ? held_ + take : 2);
    } else if (run_len_ == 1) {
      const int64_t d = static_cast<int64_t>(x - before);
      const uint32_t stop = g_.ballot(!(in && (d > 127 || d < -128)));
      take = stop ? g_.ffs(stop) - 1u : 32u;
      if (!take) return 0;
      // literal k writes `before`; a group header goes before literal k when L0 + k is a multiple
      // of 127 (at most once in 32 literals): a close of the full group and an open, or only an
      // open when nothing was pending
      const uint32_t l0 = lit_n_;
      const uint32_t ev = l0 == 0 ? 0u : (127u - l0) % 127u;  // literal index of the header
      const bool has_ev = ev < take;
      const bool mine = lane < take;
      const uint32_t hdr = (mine && has_ev && lane == ev) ? 1u : 0u;
      uint32_t vlen = 0;
      if (mine) {
        T w = before;
        do {
          vlen++;
          w = static_cast<T>(w >> 7);
        } while (w != 0);
      }
      const uint32_t at = g_.excl_sum(hdr + vlen);
      const uint32_t total = g_.template shfl<uint32_t>(at + hdr + vlen, 31);
      if (has_ev && l0 != 0) out_.set(lit_hdr_, static_cast<uint8_t>(static_cast<int8_t>(-127)));
      if (mine) {
        uint32_t p = at;
        if (hdr) out_.put_at(p++, 1);  // the placeholder open_literals(1) writes
        T w = before;
        do {
          int8_t b = static_cast<int8_t>(w & 0x7F);
          if ((w & (~0x7f)) != 0) b = static_cast<int8_t>(b | 0x80);
          out_.put_at(p++, static_cast<uint8_t>(b));
          w = static_cast<T>(w >> 7);
        } while (w != 0);
      }
      if (has_ev) {
        lit_hdr_ = out_.size() + g_.template shfl<uint32_t>(at, static_cast<int>(ev));
        lit_n_ = static_cast<uint16_t>(take - ev);
      } else {
        lit_n_ = static_cast<uint16_t>(l0 + take);
      }
      out_.advance(total);
      in_run_ = false;
    } else {
      return 0;
    }
    // the last two values taken become the history (push_hist per value)
    const T last = g_.template shfl<T>(x, static_cast<int>(take - 1));
    const T second = take >= 2 ? g_.template shfl<T>(x, static_cast<int>(take - 2)) : prev_;
    head_ = static_cast<uint8_t>(head_ ^ (take & 1u));
    hist_[head_ ^ 1] = last;
    hist_[head_] = second;
    prev_ = last;
    g_.sync();
    return take;
  }

  CODAG_HD void put(uint8_t b) { out_.put(b); }

  // unsigned LEB128 in the element type's arithmetic (encoder.h:839-853)
  CODAG_HD void put_varint(T val) {
    T w = val;
    do {
      int8_t b = static_cast<int8_t>(w & 0x7F);
      if ((w & (~0x7f)) != 0) b = static_cast<int8_t>(b | 0x80);
      put(static_cast<uint8_t>(b));
      w = static_cast<T>(w >> 7);
    } while (w != 0);
  }

  CODAG_HD void open_literals(uint8_t placeholder) {
    lit_hdr_ = out_.size();
    put(placeholder);
  }

  CODAG_HD void close_literals() {
    out_.set(lit_hdr_, static_cast<uint8_t>(static_cast<int8_t>(-static_cast<int>(lit_n_))));
    lit_n_ = 0;
  }

  CODAG_HD void push_hist(T x) {
    hist_[head_] = x;
    head_ ^= 1;
  }

  Sink& out_;
  G g_;
  T hist_[2] = {0, 0};
  uint8_t head_ = 0;
  uint8_t held_ = 0;
  T run_first_ = 0;
  uint16_t run_len_ = 0;
  int8_t step_ = 0;
  bool in_run_ = false;
  uint64_t lit_hdr_ = 0;
  uint16_t lit_n_ = 0;
  T prev_ = 0;
};


constexpr int kMaxLiterals = 128;  // utils.h:64
constexpr int kMinRepeat = 3;      // utils.h:65
constexpr int kMaxShortRepeat = 10;

// number of significant bits rounded up to a representable width (find_closes_num_bits)
CODAG_HD uint8_t closest_width(uint64_t v) {
  // bits needed for v (0 for 0): a leading-zero count rather than a 64-step shift loop
#if defined(__CUDA_ARCH__)
  const uint32_t c = 64u - static_cast<uint32_t>(__clzll(static_cast<long long>(v)));
#else
  const uint32_t c = v ? 64u - static_cast<uint32_t>(__builtin_clzll(v)) : 0u;
#endif
  return static_cast<uint8_t>(v2_closest(c));
}

// The RLE v2 writer's work on a closed group of up to 128 pending values, run by one thread: the
// host producers.  A warp can stand in for it (the GPU encoder, one warp per chunk): it keeps
// the pending values and the patch list where all its lanes see them and splits each operation
// over its lanes, while every lane runs the writer's decisions on the same data.
struct SerialGroups {
  // no bulk path: every value takes the writer's per-value steps (see RleV2Writer::encode)
  static constexpr bool kBulk = false;
  template <class Get>
  CODAG_HD uint32_t append_run(const Get&, uint64_t, uint64_t, uint64_t*, uint32_t, uint64_t&, uint32_t) const {
    return 0;
  }
  template <class Get>
  CODAG_HD uint32_t append_equal(const Get&, uint64_t, uint64_t, uint64_t*, uint32_t, uint32_t) const {
    return 0;
  }
  uint64_t lit[kMaxLiterals] = {};
  uint64_t list[kMaxLiterals];
  CODAG_HD uint64_t* lits() { return lit; }
  CODAG_HD uint64_t* lists() { return list; }

  struct Scan {
    uint64_t lmin, lmax, max_delta;
    bool increasing, decreasing, fixed;
  };
  // over l[0..n), n >= 2: extremes, monotonicity, whether every step equals the first, the largest
  // step (steps as unsigned differences)
  CODAG_HD Scan scan(const uint64_t* l, uint32_t n) const {
    Scan r{l[0], l[0], 0, true, true, true};
    const uint64_t initial = l[1] - l[0];
    for (uint32_t i = 1; i < n; i++) {
      const uint64_t l1 = l[i], l0 = l[i - 1];
      const uint64_t d = l1 - l0;
      r.lmin = l1 < r.lmin ? l1 : r.lmin;
      r.lmax = l1 > r.lmax ? l1 : r.lmax;
      r.increasing &= (l0 <= l1);
      r.decreasing &= (l0 >= l1);
      r.fixed &= (d == initial);
      r.max_delta = d > r.max_delta ? d : r.max_delta;
    }
    return r;
  }

  // histogram of representable widths (compute_bit_width)
  template <class D>
  CODAG_HD void hist(const D& d, uint32_t n, uint8_t* h) const {
    for (int i = 0; i < 32; i++) h[i] = 0;
    for (uint32_t i = 0; i < n; ++i) h[v2_code(closest_width(d(i)))]++;
  }

  // fixed width big-endian packing used by DIRECT and DELTA (write_aligned_ints)
  template <class S, class D>
  CODAG_HD void pack_aligned(S& out, const D& d, uint32_t n, uint8_t bits) const {
    if (bits < 8) {
      const uint8_t mask = static_cast<uint8_t>((1 << bits) - 1);
      const uint32_t per_byte = 8 / bits;
      const uint32_t rem = n % per_byte;
      const uint32_t full = n - rem;
      for (uint32_t i = 0; i < full; i += per_byte) {
        uint8_t b = 0;
        for (uint32_t j = 0; j < per_byte; ++j)
          b |= static_cast<uint8_t>((d(i + j) & mask) << (8 - (j + 1) * bits));
        out.put(b);
      }
      if (rem > 0) {
        uint32_t shift = 8 - bits;
        uint8_t b = 0;
        for (uint32_t i = full; i < n; ++i) {
          b |= static_cast<uint8_t>((d(i) & mask) << shift);
          shift -= bits;
        }
        out.put(b);
      }
    } else {
      const int bytes = bits / 8;
      for (uint32_t i = 0; i < n; ++i)
        for (int j = bytes - 1; j >= 0; --j) out.put(static_cast<uint8_t>((d(i) >> (j * 8)) & 0xff));
    }
  }

  // MSB-first packing at any width (write_unaligned_ints)
  template <class S, class D>
  CODAG_HD void pack_unaligned(S& out, const D& d, uint32_t n, uint8_t bits) const {
    uint32_t room = 8;
    uint8_t cur = 0;
    for (uint32_t i = 0; i < n; ++i) {
      uint64_t value = d(i);
      uint32_t todo = bits;
      while (todo > room) {
        cur |= static_cast<uint8_t>(value >> (todo - room));
        todo -= room;
        value &= (static_cast<uint64_t>(1) << todo) - 1;
        out.put(cur);
        cur = 0;
        room = 8;
      }
      room -= todo;
      cur |= static_cast<uint8_t>(value << room);
      if (room == 0) {
        out.put(cur);
        cur = 0;
        room = 8;
      }
    }
    if (room != 8) out.put(cur);
  }

  // patch list of a PATCHED_BASE group (preparePatchedBlob1, encoder.h:182-268): one entry
  // (gap << pwidth) | (value >> b95) per base-reduced value above mask, gaps from the previous
  // patched position (0 before the first); a group holds at most 128 values, so every gap is
  // below 256 and takes one entry.  Returns the entry count and the largest gap.
  CODAG_HD uint32_t patches(const uint64_t* l, uint32_t n, uint64_t lmin, uint64_t mask, uint32_t b95,
                            uint32_t pwidth, uint64_t* out, uint64_t* max_gap) const {
    uint32_t np = 0;
    uint64_t prev = 0, mg = 0;
    for (uint32_t i = 0; i < n; i++) {
      const uint64_t r = l[i] - lmin;
      if (r > mask) {
        const uint64_t gap = i - prev;
        if (gap > mg) mg = gap;
        prev = i;
        out[np++] = (gap << pwidth) | (r >> b95);
      }
    }
    *max_gap = mg;
    return np;
  }
};

template <class Sink, class G = SerialGroups>
class RleV2Writer {
 public:
  CODAG_HD explicit RleV2Writer(Sink& out) : out_(out), lit_(g_.lits()) {}
  // a group executor with its own storage (one warp per chunk)
  CODAG_HD RleV2Writer(Sink& out, const G& g) : out_(out), g_(g), lit_(g_.lits()) {}
  RleV2Writer(const RleV2Writer&) = delete;  // lit_ points into g_
  RleV2Writer& operator=(const RleV2Writer&) = delete;

  // n values, value i read as get(i) (zero-extended to 64 bits)
  template <class Get>
  CODAG_HD void encode(const Get& get, uint64_t n) {
    uint64_t prev_delta = 0;
    for (uint64_t i = 0; i < n; i++) {
      if constexpr (G::kBulk) {
        // Inside a variable run (no fixed run pending, two or more values held) a value only
        // appends to the pending values, until two zero steps in a row start a fixed run or the
        // group reaches 128 values: the executor may take such values many at a time.
        if (fix_ == 0 && nlit_ >= 2) {
          const uint32_t lim_v = static_cast<uint32_t>(kMaxLiterals) - var_;
          const uint32_t lim_n = static_cast<uint32_t>(kMaxLiterals) - nlit_;
          const uint32_t took = g_.append_run(get, i, n, lit_, nlit_, prev_delta, lim_v < lim_n ? lim_v : lim_n);
          if (took) {
            nlit_ += took;
            var_ += took;
            if (var_ == static_cast<uint32_t>(kMaxLiterals)) choose_encoding();
            i += took - 1;  // the loop's increment moves to the first value not taken
            continue;
          }
        }
        // Inside a fixed run (no variable values pending) a value equal to the last only appends,
        // until the run reaches 128 values.
        if (var_ == 0 && fix_ >= static_cast<uint32_t>(kMinRepeat) && prev_delta == 0 && nlit_ >= 1) {
          const uint32_t lim_f = static_cast<uint32_t>(kMaxLiterals) - fix_;
          const uint32_t lim_n = static_cast<uint32_t>(kMaxLiterals) - nlit_;
          const uint32_t took = g_.append_equal(get, i, n, lit_, nlit_, lim_f < lim_n ? lim_f : lim_n);
          if (took) {
            nlit_ += took;
            fix_ += took;
            if (fix_ == static_cast<uint32_t>(kMaxLiterals)) choose_encoding();
            i += took - 1;
            continue;
          }
        }
      }
      const uint64_t val = get(i);
      if (nlit_ == 0) {
        lit_[nlit_++] = val;
        fix_ = 1;
        var_ = 1;
        continue;
      }
      if (nlit_ == 1) {
        lit_[nlit_++] = val;
        prev_delta = val - lit_[0];
        if (val == lit_[0]) {
          fix_ = 2;
          var_ = 0;
        } else {
          fix_ = 0;
          var_ = 2;
        }
        continue;
      }
      const uint64_t cur_delta = val - lit_[nlit_ - 1];
      if (prev_delta == 0 && cur_delta == 0) {
        lit_[nlit_++] = val;
        if (var_ > 0) fix_ = 2;  // the fixed run is the tail of the pending values
        fix_++;
        if (fix_ >= kMinRepeat && var_ > 0) {
          nlit_ -= kMinRepeat;
          var_ -= kMinRepeat - 1;
          choose_encoding();
          prev_delta = 0;
          for (int k = 0; k < kMinRepeat; ++k) lit_[k] = val;
          nlit_ = kMinRepeat;
        }
        if (fix_ == kMaxLiterals) choose_encoding();
        continue;
      }
      if (fix_ >= kMinRepeat) {
        if (fix_ <= kMaxShortRepeat) {
          write_short_repeat();
        } else {
          fixed_delta_ = true;
          write_delta();
        }
      }
      if (fix_ > 0 && fix_ < kMinRepeat && val != lit_[nlit_ - 1]) {
        var_ = fix_;
        fix_ = 0;
      }
      if (nlit_ == 0) {
        lit_[nlit_++] = val;
        fix_ = 1;
        var_ = 1;
      } else {
        prev_delta = val - lit_[nlit_ - 1];
        lit_[nlit_++] = val;
        var_++;
        if (var_ == kMaxLiterals) choose_encoding();
      }
    }
    if (nlit_ != 0) {
      if (var_ != 0) {
        choose_encoding();
      } else if (fix_ != 0) {
        if (fix_ < kMinRepeat) {
          var_ = fix_;
          fix_ = 0;
          choose_encoding();
        } else if (fix_ <= kMaxShortRepeat) {
          write_short_repeat();
        } else {
          fixed_delta_ = true;
          write_delta();
        }
      }
    }
  }

 private:
  CODAG_HD void put(uint8_t b) { out_.put(b); }

  // The writer keeps only the pending values (lit_) and the patch list: deltas and base-reduced
  // values are derived from lit_ where they are read, which keeps a GPU thread's state small.

  // smallest width covering all but the top (100-p)% of values (compute_percentile_bit_width)
  CODAG_HD static uint8_t percentile_width(const uint8_t* hist, uint32_t n, uint8_t p) {
    p = static_cast<uint8_t>(100 - p);
    int32_t left = (p == 0 ? 0 : static_cast<int32_t>((n * p - 1) / 100 + 1));
    for (int8_t i = 31; i >= 0; --i) {
      left -= hist[i];
      if (left < 0) return v2_width(i);
    }
    return 0;
  }

  CODAG_HD void put_uvarint(int64_t val) {
    for (;;) {
      if ((val & ~0x7f) == 0) {
        put(static_cast<uint8_t>(val));
        return;
      }
      put(static_cast<uint8_t>(0x80 | (val & 0x7f)));
      val = static_cast<int64_t>(static_cast<uint64_t>(val) >> 7);
    }
  }
  CODAG_HD void put_svarint(int64_t val) { put_uvarint((val << 1) ^ (val >> 63)); }

  CODAG_HD_CALL void write_short_repeat() {
    const uint64_t val = lit_[0];
    const uint8_t nbytes = static_cast<uint8_t>((closest_width(val) - 1) / 8 + 1);
    put(static_cast<uint8_t>(((nbytes - 1) << 3) | (fix_ - kMinRepeat)));
    for (int i = nbytes - 1; i >= 0; i--) put(static_cast<uint8_t>((val >> (i * 8)) & 0xff));
    fix_ = 0;
    nlit_ = 0;
    var_ = 0;
  }

  CODAG_HD_CALL void write_direct() {
    uint8_t hist[32];
    const uint64_t* l = lit_;
    const auto lit = [l](uint32_t i) { return l[i]; };
    g_.hist(lit, nlit_, hist);
    const uint8_t bits = v2_closest_aligned(percentile_width(hist, nlit_, 100));
    const uint16_t enc = v2_code(bits);
    // The reference writes var_runlen-1 here.  On every path var_runlen equals the number
    // of pending values except one: a 128-value run of zeros reaches this writer through
    // is_safe_subtract with var_runlen == 0, and the reference emits a length field of 511
    // over 128 packed values, a stream no decoder reads back.  Counting the pending values
    // gives the same bytes everywhere else and a decodable header there.
    const uint16_t len = static_cast<uint16_t>(nlit_ - 1);
    put(static_cast<uint8_t>(0x40 | (enc << 1) | ((len & 0x100) >> 8)));
    put(static_cast<uint8_t>(len & 0xff));
    g_.pack_aligned(out_, lit, nlit_, bits);
    var_ = 0;
    nlit_ = 0;
  }

  CODAG_HD_CALL void write_delta() {
    uint16_t len;
    uint8_t enc = 0;
    uint8_t bits = v2_closest_aligned(delta_bits_);
    if (fixed_delta_) {
      if (fix_ > kMinRepeat) {
        len = static_cast<uint16_t>(fix_ - 1);
        fix_ = 0;
      } else {
        len = static_cast<uint16_t>(var_ - 1);
        var_ = 0;
      }
    } else {
      if (bits == 1) bits = 2;
      enc = v2_code(bits);
      len = static_cast<uint16_t>(var_ - 1);
      var_ = 0;
    }
    put(static_cast<uint8_t>(0xC0 | (enc << 1) | ((len & 0x100) >> 8)));
    put(static_cast<uint8_t>(len & 0xff));
    put_uvarint(static_cast<int64_t>(lit_[0]));
    // every path here has at least three pending values; a fixed run's deltas are all zero
    put_svarint(static_cast<int64_t>(lit_[1] - lit_[0]));
    if (!fixed_delta_) {
      const uint64_t* l = lit_;
      g_.pack_aligned(out_, [l](uint32_t i) { return l[i + 2] - l[i + 1]; }, nlit_ - 2, bits);
    }
    nlit_ = 0;
    var_ = 0;
  }

  CODAG_HD_CALL void write_patched(uint64_t lit_min, uint8_t b95, uint8_t b100) {
    // patch list (preparePatchedBlob1, encoder.h:182-268); a group holds at most 128 values, so
    // every gap is below 256 and each patch takes one list entry
    int64_t mask = static_cast<int64_t>((static_cast<uint64_t>(1) << b95) - 1);
    uint32_t pwidth = v2_closest(b100 - b95);
    if (pwidth == 64) {
      pwidth = 56;
      b95 = 8;
      mask = static_cast<int64_t>((static_cast<uint64_t>(1) << b95) - 1);
    }
    uint64_t* list = g_.lists();
    uint64_t max_gap = 0;
    const uint32_t npatch = g_.patches(lit_, nlit_, lit_min, static_cast<uint64_t>(mask), b95, pwidth, list, &max_gap);
    const uint32_t gap_width = (max_gap == 0 && npatch != 0) ? 1u : closest_width(max_gap);
    const uint32_t nlist = npatch;

    // header and body (writePatchedBasedValues, encoder.h:527-591)
    uint32_t len = var_ - 1;
    const uint8_t h0 = static_cast<uint8_t>(0x80 | (v2_code(b95) << 1) | ((len & 0x100) >> 8));
    const uint8_t h1 = static_cast<uint8_t>(len & 0xff);
    const uint32_t base_bits = closest_width(lit_min) + 1;
    const uint32_t base_bytes = (base_bits - 1) / 8 + 1;
    const uint8_t h2 = static_cast<uint8_t>(((base_bytes - 1) << 5) | v2_code(pwidth));
    const uint8_t h3 = static_cast<uint8_t>((gap_width - 1) << 5 | nlist);
    put(h0);
    put(h1);
    put(h2);
    put(h3);
    for (int i = static_cast<int>(base_bytes) - 1; i >= 0; i--) put(static_cast<uint8_t>((lit_min >> (i * 8)) & 0xff));
    // base-reduced values; the patched ones keep their low b95 bits
    const uint64_t* l = lit_;
    const uint64_t um = static_cast<uint64_t>(mask);
    g_.pack_unaligned(out_, [l, lit_min, um](uint32_t i) { return (l[i] - lit_min) & um; }, nlit_, v2_closest(b95));
    g_.pack_unaligned(out_, [list](uint32_t i) { return list[i]; }, nlist, v2_closest(gap_width + pwidth));
    var_ = 0;
    nlit_ = 0;
  }

  // determineEncoding (encoder.h:270-387)
  CODAG_HD_CALL void choose_encoding() {
    if (nlit_ <= static_cast<uint32_t>(kMinRepeat)) {
      write_direct();
      return;
    }
    const typename G::Scan sc = g_.scan(lit_, nlit_);
    const uint64_t lmin = sc.lmin, lmax = sc.lmax, max_delta = sc.max_delta;
    const uint64_t initial = lit_[1] - lit_[0];
    const bool increasing = sc.increasing, decreasing = sc.decreasing;
    fixed_delta_ = sc.fixed;
    // is_safe_subtract on unsigned values: only a minimum of 0 with maximum <= 128 fails
    const bool safe = (lmin > 0) || (lmax > static_cast<uint64_t>(lmin - INT8_MIN));
    if (!safe) {
      write_direct();
      return;
    }
    if (lmin == lmax || fixed_delta_) {
      write_delta();
      return;
    }
    if (initial != 0) {
      delta_bits_ = closest_width(max_delta);
      if (increasing || decreasing) {
        write_delta();
        return;
      }
    }
    uint8_t hist[32];
    const uint64_t* l = lit_;
    g_.hist([l](uint32_t i) { return l[i]; }, nlit_, hist);
    const uint8_t b100 = percentile_width(hist, nlit_, 100);
    const uint8_t b90 = percentile_width(hist, nlit_, 90);
    if (static_cast<uint32_t>(b100 - b90) > 1) {
      g_.hist([l, lmin](uint32_t i) { return l[i] - lmin; }, nlit_, hist);
      const uint8_t r95 = percentile_width(hist, nlit_, 95);
      const uint8_t r100 = percentile_width(hist, nlit_, 100);
      if (r100 - r95 != 0) {
        write_patched(lmin, r95, r100);
      } else {
        write_direct();
      }
      return;
    }
    write_direct();
  }

  Sink& out_;
  G g_;
  uint64_t* lit_;
  uint32_t nlit_ = 0, fix_ = 0, var_ = 0;
  uint8_t delta_bits_ = 0;
  bool fixed_delta_ = false;
};


}  // namespace codag_fmt
