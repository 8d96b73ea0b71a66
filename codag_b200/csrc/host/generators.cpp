// Seeded synthetic columns standing in for CODAG's paper datasets (mortgage/taxi columns and
// text files that are not distributed with the code).  Each generator fills its output in
// independent 1 Mi-element (or 4 MiB text) blocks, each with its own derived seed, so the
// result depends only on (n, seed) and the blocks can be generated in parallel.
//
//   rlev1 column: segments, 50/50 run or literal.  Run: length U{3..130}, base U[0,2^20),
//                 step U{-3..3}, value i = base + i*step (two's complement).  Literal:
//                 length U{1..128}, values U[0,2^20).
//   rlev2 column: segments of length U{3..512}, one of four kinds with probability 1/4:
//                 constant U[0,2^31); arithmetic base U[4096,2^31) step U{-8..8} (the base
//                 floor keeps every value non-negative); uniform U[0,2^b) with b U{1..32};
//                 small U[0,2^8) with 2% outliers U[0,2^31).
//   text:         8192-word vocabulary of random lowercase words of length U{2..12}; words
//                 drawn Zipf(s=1.1) over ranks 1..8192, separated by single spaces, with a
//                 newline in place of the space after every U{12..20} words.
// Narrower element widths keep the low bytes of each value.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "host_common.hpp"

namespace codag_host {

static inline uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

Rng::Rng(uint64_t seed) {
  uint64_t x = seed;
  for (auto& w : s) w = splitmix64(x);
}

uint64_t Rng::next() {
  const uint64_t r = rotl(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return r;
}

uint64_t Rng::below(uint64_t n) { return n ? static_cast<uint64_t>((static_cast<unsigned __int128>(next()) * n) >> 64) : 0; }
int64_t Rng::range(int64_t lo, int64_t hi) { return lo + static_cast<int64_t>(below(static_cast<uint64_t>(hi - lo + 1))); }
double Rng::uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }

uint64_t derive_seed(uint64_t base, uint64_t stream) {
  uint64_t x = base ^ (0xD1B54A32D192ED03ull * (stream + 1));
  return splitmix64(x);
}

namespace {

constexpr uint64_t kBlockElems = 1ull << 20;
constexpr uint64_t kTextBlock = 4ull << 20;

inline void store_elem(uint8_t* out, uint64_t idx, int e, uint64_t v) { std::memcpy(out + idx * e, &v, e); }

void gen_rlev1_block(Rng& r, uint8_t* out, uint64_t start, uint64_t n, int e) {
  uint64_t i = 0;
  while (i < n) {
    if (r.below(2) == 0) {
      const uint64_t len = r.range(3, 130);
      const uint64_t base = r.below(1ull << 20);
      const int64_t step = r.range(-3, 3);
      for (uint64_t k = 0; k < len && i < n; k++, i++)
        store_elem(out, start + i, e, base + static_cast<uint64_t>(static_cast<int64_t>(k) * step));
    } else {
      const uint64_t len = r.range(1, 128);
      for (uint64_t k = 0; k < len && i < n; k++, i++) store_elem(out, start + i, e, r.below(1ull << 20));
    }
  }
}

void gen_rlev2_block(Rng& r, uint8_t* out, uint64_t start, uint64_t n, int e) {
  uint64_t i = 0;
  while (i < n) {
    const uint64_t len = r.range(3, 512);
    const int kind = static_cast<int>(r.below(4));
    if (kind == 0) {
      const uint64_t v = r.below(1ull << 31);
      for (uint64_t k = 0; k < len && i < n; k++, i++) store_elem(out, start + i, e, v);
    } else if (kind == 1) {
      const uint64_t base = 4096 + r.below((1ull << 31) - 4096);
      const int64_t step = r.range(-8, 8);
      for (uint64_t k = 0; k < len && i < n; k++, i++)
        store_elem(out, start + i, e, base + static_cast<uint64_t>(static_cast<int64_t>(k) * step));
    } else if (kind == 2) {
      const int b = static_cast<int>(r.range(1, 32));
      for (uint64_t k = 0; k < len && i < n; k++, i++) store_elem(out, start + i, e, r.below(1ull << b));
    } else {
      for (uint64_t k = 0; k < len && i < n; k++, i++) {
        const uint64_t v = (r.below(100) < 2) ? r.below(1ull << 31) : r.below(256);
        store_elem(out, start + i, e, v);
      }
    }
  }
}

struct TextModel {
  std::vector<std::string> words;
  std::vector<double> cdf;
  explicit TextModel(uint64_t seed) {
    Rng r(derive_seed(seed, 0xC0FFEE));
    words.resize(8192);
    for (auto& w : words) {
      const int len = static_cast<int>(r.range(2, 12));
      w.resize(len);
      for (auto& c : w) c = static_cast<char>('a' + r.below(26));
    }
    cdf.resize(8192);
    double acc = 0;
    for (int k = 0; k < 8192; k++) {
      acc += std::pow(static_cast<double>(k + 1), -1.1);
      cdf[k] = acc;
    }
    for (auto& c : cdf) c /= acc;
  }
  const std::string& draw(Rng& r) const {
    const double u = r.uniform();
    const size_t k = std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin();
    return words[std::min<size_t>(k, 8191)];
  }
};

}  // namespace
}  // namespace codag_host

using namespace codag_host;

extern "C" void codag_gen_rlev1_column(uint64_t n, uint64_t seed, int elem_bytes, uint8_t* out) {
  const int64_t nblk = static_cast<int64_t>((n + kBlockElems - 1) / kBlockElems);
#pragma omp parallel for schedule(dynamic)
  for (int64_t b = 0; b < nblk; b++) {
    Rng r(derive_seed(seed, static_cast<uint64_t>(b)));
    const uint64_t start = b * kBlockElems;
    gen_rlev1_block(r, out, start, std::min(kBlockElems, n - start), elem_bytes);
  }
}

extern "C" void codag_gen_rlev2_column(uint64_t n, uint64_t seed, int elem_bytes, uint8_t* out) {
  const int64_t nblk = static_cast<int64_t>((n + kBlockElems - 1) / kBlockElems);
#pragma omp parallel for schedule(dynamic)
  for (int64_t b = 0; b < nblk; b++) {
    Rng r(derive_seed(seed, static_cast<uint64_t>(b)));
    const uint64_t start = b * kBlockElems;
    gen_rlev2_block(r, out, start, std::min(kBlockElems, n - start), elem_bytes);
  }
}

extern "C" void codag_gen_text(uint64_t bytes, uint64_t seed, uint8_t* out) {
  const TextModel model(seed);
  const int64_t nblk = static_cast<int64_t>((bytes + kTextBlock - 1) / kTextBlock);
#pragma omp parallel for schedule(dynamic)
  for (int64_t b = 0; b < nblk; b++) {
    Rng r(derive_seed(seed, static_cast<uint64_t>(b)));
    uint8_t* dst = out + b * kTextBlock;
    const uint64_t n = std::min(kTextBlock, bytes - b * kTextBlock);
    uint64_t i = 0;
    int64_t until_newline = r.range(12, 20);
    while (i < n) {
      const std::string& w = model.draw(r);
      for (size_t k = 0; k < w.size() && i < n; k++) dst[i++] = static_cast<uint8_t>(w[k]);
      if (i < n) {
        if (--until_newline == 0) {
          dst[i++] = '\n';
          until_newline = r.range(12, 20);
        } else {
          dst[i++] = ' ';
        }
      }
    }
  }
}
