// ORC RLE v1 chunk encoder (host).  Produces the exact byte stream of CODAG's GPU encoder
// include/rlev1/encoder.h:1352-1695 (compression_warp_orig, driven by deflate_orig :1800-1840),
// so files written here decode identically with CODAG's decoder and with ours.
//
// Format (one stream per chunk of chunk_bytes bytes, i.e. chunk_bytes/sizeof(T) values):
//   literal group: header (int8) -n, then n unsigned LEB128 varints          (n <= 127)
//   run:           header h in [0,126], int8 delta, varint base; h+3 values  (<= 129 values)
// The encoder holds the last two values, opens a literal group whose header byte is a
// placeholder (later patched to -count), and switches to a run once three values share
// one step in [-128,127].  All comparisons and differences are evaluated in the element
// type's own C++ arithmetic (uint32 differences are never negative, uint8/uint16 promote
// to int), because that is what the reference computes.
//
// File layout (include/rlev1/rlev1.h:103-192):
//   n_chunks_pad = ceil(bytes / (chunk*32)) * 32, input zero padded to n_chunks_pad*chunk;
//   blob = [u64 original_bytes][stream_0 ...]; stream i starts at 8 + blk_off[i];
//   blk_off[0] = 0, blk_off[i+1] = blk_off[i] + round_up4(col_len[i]).
#include <cstdint>
#include <cstring>
#include <vector>

#include "host_common.hpp"

namespace codag_host {
namespace {

template <typename T>
class RleV1Writer {
 public:
  explicit RleV1Writer(std::vector<uint8_t>& out) : out_(out) {}

  void encode(const T* v, uint64_t n) {
    // first value
    uint64_t i = 0;
    T x = v[i++];
    run_len_ = 1;
    prev_ = x;
    push_hist(x);
    held_ = 1;

    // second value
    x = v[i++];
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
      if (lit_n_ == 127) close_literals();
      x = v[i];

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
    out_[lit_hdr_] = static_cast<uint8_t>(static_cast<int8_t>(-static_cast<int>(lit_n_)));
  }

 private:
  void put(uint8_t b) { out_.push_back(b); }

  // unsigned LEB128 in the element type's arithmetic (encoder.h:839-853)
  void put_varint(T val) {
    T w = val;
    do {
      int8_t b = static_cast<int8_t>(w & 0x7F);
      if ((w & (~0x7f)) != 0) b = static_cast<int8_t>(b | 0x80);
      put(static_cast<uint8_t>(b));
      w = static_cast<T>(w >> 7);
    } while (w != 0);
  }

  void open_literals(uint8_t placeholder) {
    lit_hdr_ = out_.size();
    put(placeholder);
  }

  void close_literals() {
    out_[lit_hdr_] = static_cast<uint8_t>(static_cast<int8_t>(-static_cast<int>(lit_n_)));
    lit_n_ = 0;
  }

  void push_hist(T x) {
    hist_[head_] = x;
    head_ ^= 1;
  }

  std::vector<uint8_t>& out_;
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

template <typename T>
void encode_chunk_t(const uint8_t* chunk, uint64_t chunk_bytes, std::vector<uint8_t>& out) {
  const uint64_t n = chunk_bytes / sizeof(T);
  std::vector<T> vals(n);
  std::memcpy(vals.data(), chunk, n * sizeof(T));
  RleV1Writer<T> w(out);
  w.encode(vals.data(), n);
}

}  // namespace

int rlev1_encode_chunk(const uint8_t* chunk, uint64_t chunk_bytes, int elem_bytes,
                       std::vector<uint8_t>& out) {
  if (chunk_bytes % elem_bytes || chunk_bytes / elem_bytes < 2) return CODAG_EINVAL;
  switch (elem_bytes) {
    case 1: encode_chunk_t<uint8_t>(chunk, chunk_bytes, out); break;
    case 2: encode_chunk_t<uint16_t>(chunk, chunk_bytes, out); break;
    case 4: encode_chunk_t<uint32_t>(chunk, chunk_bytes, out); break;
    case 8: encode_chunk_t<uint64_t>(chunk, chunk_bytes, out); break;
    default: return CODAG_EINVAL;
  }
  return CODAG_OK;
}

}  // namespace codag_host
