/*
 * codag_format.h -- host-side producers of CODAG's on-disk chunk layouts, and seeded
 * synthetic columns (libcodag_fmt.so; CPU only, no CUDA).
 *
 * These write the files CODAG's tools read (include/rlev1/rlev1.h:103-192,
 * include/rlev2/encoder_trans.h:482-564, deflate_compressor.py:44-125) and are used by the
 * command-line tools, the tests and the benchmarks to make inputs for the decoders of
 * codag.h.  They live in their own library so that a caller that only writes or inspects
 * files (or times a CPU decoder) does not load the CUDA decoders.
 */
#ifndef CODAG_FORMAT_H
#define CODAG_FORMAT_H

#include "codag.h" /* codag_status, codag_chunk_desc, CODAG_CODEC_* */

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint8_t *data;
    uint64_t bytes;
} codag_hbuf; /* malloc'd by the library; release with codag_hbuf_free */
void codag_hbuf_free(codag_hbuf *b);

/* CODAG's RLE v1 layout (include/rlev1/rlev1.h:103-192): blob = [u64 in_bytes][streams],
 * blk_off = n_pad+1 u64 (stream i at blob+8+blk_off[i], 4-byte aligned), col_len = n_pad u64,
 * n_pad = ceil(in_bytes/(chunk*32))*32 chunks over the zero-padded input. */
codag_status codag_encode_rlev1(const uint8_t *in, uint64_t in_bytes, uint64_t chunk_bytes,
                                int elem_bytes, codag_hbuf *blob, codag_hbuf *blk_off,
                                codag_hbuf *col_len);
/* CODAG's RLE v2 layout (include/rlev2/encoder_trans.h:482-564): streams at 128-byte aligned
 * blk_off[i]; blk_off has n_pad+1 entries with blk_off[n_pad] = in_bytes; col_len n_pad. */
codag_status codag_encode_rlev2(const uint8_t *in, uint64_t in_bytes, uint64_t chunk_bytes,
                                int elem_bytes, codag_hbuf *comp, codag_hbuf *blk_off,
                                codag_hbuf *col_len);
/* CODAG's Deflate layout (deflate_compressor.py:44-125): input zero padded to a multiple of
 * chunk_bytes; comp = zlib streams each padded to 8 bytes; blk_offset = n+2 u64
 * [in_bytes, 0, cum_1 .. cum_n]; col_len = n padded sizes.  zlib_wrapper=1 writes RFC 1950
 * streams (CODAG's format), 0 raw Deflate.  Fails with CODAG_EINVAL if require_no_stored and
 * zlib emitted a stored block. */
codag_status codag_encode_deflate(const uint8_t *in, uint64_t in_bytes, uint64_t chunk_bytes,
                                  int level, int zlib_wrapper, int require_no_stored,
                                  codag_hbuf *comp, codag_hbuf *blk_offset, codag_hbuf *col_len);
/* CODAG's transposed RLE v2 layout (include/rlev2/encoder_trans.h:8-182 and 359-391,
 * rlev2::compress_gpu_transpose :411-480): n = ceil(in_bytes/chunk_bytes) chunks, each split into
 * 32 substreams (substream t = values t*read_unit + k*32*read_unit + j, j < read_unit) encoded on
 * their own and interleaved in 4-byte words; blk_off has n+1 entries (128-byte aligned regions,
 * blk_off[n] = in_bytes), col_len n*32 exact substream lengths.  chunk_bytes must be a multiple
 * of 32 * read_unit * elem_bytes. */
codag_status codag_encode_rlev2_transposed(const uint8_t *in, uint64_t in_bytes, uint64_t chunk_bytes,
                                           int elem_bytes, int read_unit, codag_hbuf *comp,
                                           codag_hbuf *blk_off, codag_hbuf *col_len);
/* CODAG's cuDF-comparison layout (rapids_compressor.py:222-275, read by
 * include/base_deflate.h:20-130): file = [u64 chunk_bytes][u64 n][u64 size_i x n] then the n
 * zlib-wrapped streams back to back, one per chunk of the input zero padded to a multiple of
 * chunk_bytes (the script uses 64 KiB chunks and level 9).  Decode with
 * codag_decompress_deflate(file + data_offset, ..., blk_off, n, chunk_bytes, wrapper_bytes = 2). */
codag_status codag_encode_cudf_deflate(const uint8_t *in, uint64_t in_bytes, uint64_t chunk_bytes,
                                       int level, codag_hbuf *file);
/* Parses that layout: chunk size, chunk count, byte offset of the first stream, and (blk_off
 * non-NULL) n+1 stream offsets relative to it.  CODAG_EINVAL if a size runs past the file. */
codag_status codag_cudf_deflate_layout(const uint8_t *file, uint64_t file_bytes, uint64_t *chunk_bytes,
                                       uint64_t *n_chunks, uint64_t *data_offset, uint64_t *blk_off);
/* One stream of a single buffer (the batched workload's per-chunk files). */
codag_status codag_encode_one(int codec, const uint8_t *in, uint64_t in_bytes, int elem_bytes,
                              int level, codag_hbuf *stream);

/* A set of n independent files, file i = in[in_off[i] .. +in_len[i]), each encoded as ONE
 * stream of codecs[i] (Deflate: zlib level `level` with the 2-byte zlib wrapper; RLE:
 * elem_bytes[i]-wide values) and packed for codag_batch_plan: streams 16-byte aligned in
 * `comp`, outputs 256-byte aligned in an output buffer of *out_bytes; descs[i] is filled.
 * OpenMP over files. */
codag_status codag_encode_set(const uint8_t *in, const uint64_t *in_off, const uint64_t *in_len,
                              const uint8_t *codecs, const uint8_t *elem_bytes, uint64_t n, int level,
                              codag_chunk_desc *descs, codag_hbuf *comp, uint64_t *out_bytes);

/* Seeded synthetic columns (splitmix64/xoshiro256**). */
void codag_gen_rlev1_column(uint64_t n, uint64_t seed, int elem_bytes, uint8_t *out);
void codag_gen_rlev2_column(uint64_t n, uint64_t seed, int elem_bytes, uint8_t *out);
void codag_gen_text(uint64_t bytes, uint64_t seed, uint8_t *out);

#ifdef __cplusplus
}
#endif
#endif /* CODAG_FORMAT_H */
