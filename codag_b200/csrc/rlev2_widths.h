// ORC RLE v2 bit-width codes, shared by the CUDA decoders and the host writer.
//
// A header stores a bit width as a 5-bit code.  Widths 1..24 are exact; above that only
// 26, 28, 30, 32, 40, 48, 56 and 64 exist, so a value needing b bits is stored at the
// closest representable width >= b.  These are CODAG's four lookup tables
// (include/rlev2/utils.h:28-59), computed here instead of looked up; tests/test_golden_rlev2.py
// checks every entry against CODAG's tables.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define CODAG_HD __host__ __device__ __forceinline__
// a large step called from many places, kept out of line on the device: its registers then
// do not add to those of every loop that calls it
#define CODAG_HD_CALL __host__ __device__ __noinline__
#else
#define CODAG_HD inline
#define CODAG_HD_CALL inline
#endif

// width of 5-bit code c (__BIT_WIDTH_DECODE_MAP)
CODAG_HD uint32_t v2_width(uint32_t c) { return c < 24 ? c + 1 : (c < 28 ? 2 * c - 22 : 8 * c - 184); }

// 5-bit code of a representable width b, 0..64; 0 and 1 give code 0 (__BIT_WIDTH_ENCODE_MAP)
CODAG_HD uint32_t v2_code(uint32_t b) { return b <= 1 ? 0u : (b <= 24 ? b - 1 : (b <= 32 ? 24 + (b - 25) / 2 : 28 + (b - 33) / 8)); }

// smallest representable width >= b, for b in 0..64 (__CLOSEST_FIXED_BIT_MAP)
CODAG_HD uint32_t v2_closest(uint32_t b) { return b <= 24 ? (b ? b : 1u) : (b <= 32 ? (b + 1) & ~1u : (b + 7) & ~7u); }

// smallest width >= b among 1, 2, 4, 8 and the multiples of 8 (__CLOSEST_ALIGNED_FIXED_BIT_MAP)
CODAG_HD uint32_t v2_closest_aligned(uint32_t b) {
  return b <= 2 ? (b ? b : 1u) : (b <= 4 ? 4u : (b + 7) & ~7u);
}
