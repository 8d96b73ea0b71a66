/*
 * codag.h -- C ABI of the B200-native CODAG chunk decompressors.
 *
 * Every pointer named d_* is a DEVICE pointer owned by the caller.  Calls are asynchronous
 * on `stream` (a cudaStream_t; NULL = legacy default stream), allocate no device memory
 * (scratch comes from the caller's workspace), never print and never exit.  The return value reports argument and launch errors only;
 * stream corruption and bounded-wait timeouts are reported per chunk in d_chunk_status
 * (CODAG_OK / CODAG_ECORRUPT / CODAG_ETIMEOUT), which may be NULL when not wanted.
 * Distinct streams may be used from distinct host threads concurrently.
 *
 * Output contract shared by the three decoders: chunk i decodes to
 * d_out + i*chunk_bytes; bytes beyond out_bytes are decoded but not stored, so out_bytes
 * may be the exact original size.  A chunk is OK when its stream is well formed and the
 * bytes it produced cover its stored part without exceeding chunk_bytes.
 */
#ifndef CODAG_H
#define CODAG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *codag_stream_t; /* same type as cudaStream_t */

typedef enum {
    CODAG_OK = 0,
    CODAG_EINVAL = 1,   /* bad argument (null pointer, size, alignment, element width) */
    CODAG_ECORRUPT = 2, /* malformed stream (per chunk) */
    CODAG_ETIMEOUT = 3, /* a bounded device wait ran out (per chunk) */
    CODAG_ECUDA = 4,    /* a CUDA runtime call or launch failed */
    CODAG_ENOMEM = 5,   /* host allocation failed (planning calls only) */
    CODAG_ELIMIT = 6    /* request exceeds a fixed capacity (codag_decompress_rlev2_noalloc) */
} codag_status;

enum { CODAG_CODEC_RLEV1 = 0, CODAG_CODEC_RLEV2 = 1, CODAG_CODEC_DEFLATE = 2 };

/*
 * ORC RLE v1, one stream per chunk.
 * Replaces rle_v1::decompress_gpu_orig<...> (include/rlev1/rlev1.h:419-592), which takes the
 * host blob [u64 original_bytes][streams] and reads ./input_data/rle_v1_{col_len,blk_offset}.bin.
 *   d_comp      stream base, i.e. blob + 8 (the kernel argument d_in+8 at rlev1.h:513)
 *   comp_bytes  readable bytes at d_comp (every stream must lie inside)
 *   d_blk_off   n_chunks offsets: stream i starts at d_comp + d_blk_off[i]
 *   d_col_len   n_chunks exact stream lengths in bytes
 *   chunk_bytes decoded bytes per chunk (131072 in CODAG), a multiple of elem_bytes, < 2^31
 *   elem_bytes  1, 2, 4 or 8 (the DATA_TYPE template argument)
 *   d_workspace optional scratch of codag_workspace_bytes(codec, n_chunks) bytes, 256-byte
 *               aligned; with it the headers are walked one thread per chunk before the
 *               warp-per-chunk expansion; NULL decodes each chunk in a single warp pass,
 *               which measures faster on B200 (the walk is bound by dependent global loads)
 */
codag_status codag_decompress_rlev1(const uint8_t *d_comp, uint64_t comp_bytes,
                                    const uint64_t *d_blk_off, const uint64_t *d_col_len,
                                    uint64_t n_chunks, uint64_t chunk_bytes, int elem_bytes,
                                    uint8_t *d_out, uint64_t out_bytes, int32_t *d_chunk_status,
                                    void *d_workspace, uint64_t workspace_bytes,
                                    codag_stream_t stream);

/*
 * ORC RLE v2 (unsigned variant), one stream per chunk.
 * Replaces rlev2::decompress_gpu_orig<...> (include/rlev2/decoder_trans.h:57-133), whose
 * arguments (in, n_chunks, blk_off, col_len, CHUNK_SIZE) map one to one onto these.
 *   d_blk_off   n_chunks offsets (128-byte aligned in CODAG's layout)
 *   d_col_len   n_chunks exact stream lengths
 *   d_workspace as for codag_decompress_rlev1
 */
codag_status codag_decompress_rlev2(const uint8_t *d_comp, uint64_t comp_bytes,
                                    const uint64_t *d_blk_off, const uint64_t *d_col_len,
                                    uint64_t n_chunks, uint64_t chunk_bytes, int elem_bytes,
                                    uint8_t *d_out, uint64_t out_bytes, int32_t *d_chunk_status,
                                    void *d_workspace, uint64_t workspace_bytes,
                                    codag_stream_t stream);

/*
 * ORC RLE v2 in CODAG's transposed layout: each chunk is 32 substreams interleaved in 4-byte
 * words (codag_encode_rlev2_transposed of codag_format.h writes it).  Replaces
 * rlev2::decompress_gpu<READ_UNIT,...> (include/rlev2/decoder_trans.h:10-56, the inflate kernel of
 * decoder_new.h:1193-1230 with decoder_warp :375-632).
 *   d_blk_off   n_chunks offsets of the chunks' regions (4-byte aligned; 128 in CODAG's layout)
 *   d_col_len   n_chunks*32 exact substream lengths
 *   read_unit   values per substream turn (the READ_UNIT template argument); chunk_bytes must
 *               be a multiple of 32 * read_unit * elem_bytes
 * Output as for the other decoders: chunk i at d_out + i*chunk_bytes, stored up to out_bytes.
 */
codag_status codag_decompress_rlev2_transposed(const uint8_t *d_comp, uint64_t comp_bytes,
                                               const uint64_t *d_blk_off, const uint64_t *d_col_len,
                                               uint64_t n_chunks, uint64_t chunk_bytes, int elem_bytes,
                                               int read_unit, uint8_t *d_out, uint64_t out_bytes,
                                               int32_t *d_chunk_status, codag_stream_t stream);

/* Workspace bytes the two-pass RLE decode of n_chunks chunks uses (0 for Deflate). */
uint64_t codag_workspace_bytes(int codec, uint64_t n_chunks);

/*
 * RLE v2 two-pass decode that allocates nothing.  No counterpart in CODAG: it exists for
 * callers that cannot call cudaMalloc -- a plugin inside a host engine whose device memory
 * is all reserved by that engine's own pool, or code that must not allocate at all on its
 * path -- and so cannot hand codag_decompress_rlev2 a workspace.
 * Arguments and output are those of codag_decompress_rlev2 without the workspace.  The
 * scratch is a fixed array of codag_workspace_bytes(CODAG_CODEC_RLEV2,
 * CODAG_NOALLOC_MAX_CHUNKS) bytes (about 8 MiB) in the library's device memory, which every
 * device that loads the library holds until the process exits.
 *   - n_chunks above CODAG_NOALLOC_MAX_CHUNKS returns CODAG_ELIMIT (split the request).
 *   - The first call on a device looks up the array's device address on that device
 *     (cudaGetSymbolAddress); make that first call before any stream capture.  The address
 *     is kept per device number for the device's primary context (the runtime's own
 *     context); it is not valid after cudaDeviceReset, nor in another context made current
 *     on that device.
 *   - Arguments are checked as codag_decompress_rlev2 checks them (CODAG_EINVAL), before
 *     the chunk-count limit.
 *   - Every call shares the one array and leaves its contents behind.  Calls whose work
 *     overlaps on the GPU (different streams, or different host threads) race on it:
 *     order them on one stream or with events.
 */
#define CODAG_NOALLOC_MAX_CHUNKS 512
codag_status codag_decompress_rlev2_noalloc(const uint8_t *d_comp, uint64_t comp_bytes,
                                            const uint64_t *d_blk_off, const uint64_t *d_col_len,
                                            uint64_t n_chunks, uint64_t chunk_bytes, int elem_bytes,
                                            uint8_t *d_out, uint64_t out_bytes,
                                            int32_t *d_chunk_status, codag_stream_t stream);

/*
 * Deflate, one stream per chunk.
 * Replaces deflate::decompress_gpu<...> (include/zlib/zlib.h:1583-1700), which reads the
 * <name>_blk_offset.bin array [original_bytes, 0, cum_1 .. cum_n] and passes blk_offset+1.
 *   d_blk_off     n_chunks+1 relative offsets (the array above without its first entry);
 *                 stream i is d_comp[d_blk_off[i] .. d_blk_off[i+1])
 *   wrapper_bytes header bytes skipped before the Deflate data: 2 for zlib-wrapped streams
 *                 (what CODAG's decoder assumes, zlib.h:819), 0 for raw Deflate
 * Stored blocks are decoded (CODAG's decoder ignores them, zlib.h:840-842).
 */
codag_status codag_decompress_deflate(const uint8_t *d_comp, uint64_t comp_bytes,
                                      const uint64_t *d_blk_off, uint64_t n_chunks,
                                      uint64_t chunk_bytes, int wrapper_bytes, uint8_t *d_out,
                                      uint64_t out_bytes, int32_t *d_chunk_status,
                                      codag_stream_t stream);

/* --- GPU encoders -----------------------------------------------------------------------
 * CODAG's rlev1/rlev2 tools encode on the GPU, one thread per chunk, before they decode
 * (rle_v1::compress_gpu_orig, include/rlev1/rlev1.h:103-192 with rlev1/encoder.h:1728-1847;
 * rlev2::compress_gpu_orig, include/rlev2/encoder_trans.h:482-564).  These write the same
 * files, byte for byte, as the host producers of codag_format.h (codag_encode_rlev1/_rlev2),
 * from a column in device memory, asynchronously on `stream`, allocating nothing:
 *   n = codag_compress_chunks(in_bytes, chunk_bytes) chunks (a multiple of 32, the input zero
 *       padded to n * chunk_bytes);
 *   d_blk_off  n+1 u64: RLE v1 stream i at d_blob + 8 + d_blk_off[i] (4-byte aligned),
 *              RLE v2 stream i at d_comp + d_blk_off[i] (128-byte aligned), d_blk_off[n] = in_bytes;
 *   d_col_len  n u64 exact stream lengths;
 *   d_blob/d_comp  16-byte aligned, capacity bytes (codag_compress_bound always suffices);
 *              the RLE v1 blob starts with the u64 original size;
 *   d_out_bytes    (nullable) receives the file length in bytes;
 *   d_status       (nullable) receives CODAG_OK, CODAG_ELIMIT (capacity too small: nothing
 *              written) or CODAG_ECORRUPT (a stream outgrew its workspace slot);
 *   d_workspace    codag_compress_workspace_bytes(...) bytes, 256-byte aligned; d_in is
 *              aligned to elem_bytes. */
uint64_t codag_compress_chunks(uint64_t in_bytes, uint64_t chunk_bytes);
uint64_t codag_compress_bound(int codec, uint64_t in_bytes, uint64_t chunk_bytes, int elem_bytes);
uint64_t codag_compress_workspace_bytes(int codec, uint64_t in_bytes, uint64_t chunk_bytes, int elem_bytes);
codag_status codag_compress_rlev1(const uint8_t *d_in, uint64_t in_bytes, uint64_t chunk_bytes, int elem_bytes,
                                  uint8_t *d_blob, uint64_t blob_capacity, uint64_t *d_blk_off,
                                  uint64_t *d_col_len, uint64_t *d_out_bytes, int32_t *d_status,
                                  void *d_workspace, uint64_t workspace_bytes, codag_stream_t stream);
codag_status codag_compress_rlev2(const uint8_t *d_in, uint64_t in_bytes, uint64_t chunk_bytes, int elem_bytes,
                                  uint8_t *d_comp, uint64_t comp_capacity, uint64_t *d_blk_off,
                                  uint64_t *d_col_len, uint64_t *d_out_bytes, int32_t *d_status,
                                  void *d_workspace, uint64_t workspace_bytes, codag_stream_t stream);

/* --- launch tuning --------------------------------------------------------------------
 * Process-wide launch shape for the per-file calls above, per codec.  warps_per_cta is
 * the number of chunks one CTA decodes (one warp per chunk, 1..8); ring_slots the depth of
 * the TMA input ring (2, 4 or 8 slots of 1 KiB; the RLE codecs need at least 4 because an
 * RLE v2 header with its data spans up to 2060 bytes); lut_bits the primary Huffman table width
 * (Deflate only: 9, 10 or 11), which also sizes the shared-memory history window of the
 * Deflate call (9: 1 KiB, so more warps fit per SM, for many chunks; 10 and 11: 2 KiB, fewer
 * instructions per chunk, for few chunks).  cta_per_chunk (0 or 1) shortens the decode of a single
 * chunk (few chunks, e.g. an 8 MiB column, or large files) at the cost of throughput on many:
 * for the RLE calls without a workspace it runs one CTA of warps_per_cta warps per chunk (the
 * CTA stages the chunk's stream in shared memory, one warp walks its headers and all warps
 * expand them; applies when the output and out_bytes are element aligned); for Deflate a
 * chunk takes two warps, one decoding its symbols into tokens and one expanding them into
 * bytes, warps_per_cta/2 chunks per CTA (warps_per_cta even).  Values outside the supported
 * sets return CODAG_EINVAL. */
typedef struct {
    int32_t warps_per_cta;
    int32_t ring_slots;
    int32_t lut_bits;
    int32_t cta_per_chunk;
    int32_t table_global; /* batched plans only (0 or 1): the Huffman lookup tables of every warp in
                             global memory, read through L1, instead of shared memory; frees
                             3-9 KiB of shared memory per warp for more resident warps.  The
                             per-file calls and codag_batch_launch keep them in shared memory
                             (0; other values give CODAG_EINVAL). */
} codag_tune;

codag_status codag_set_tune(int codec, const codag_tune *tune);
codag_status codag_get_tune(int codec, codag_tune *tune);

/* Upper bound, in GPU clock cycles, of every device-side wait (default about one second).
 * A wait that runs out marks its chunk CODAG_ETIMEOUT and the warp stops cleanly. */
codag_status codag_set_wait_limit(uint64_t cycles);

/* Launch a kernel whose only warp waits on a TMA barrier that no copy ever completes,
 * bounded by the wait limit, and writes the resulting status (CODAG_ETIMEOUT) to
 * *d_status.  Used to test the timeout path without faulting or hanging a GPU. */
codag_status codag_selftest_wait_timeout(int32_t *d_status, codag_stream_t stream);

/* --- batched persistent decompression ------------------------------------------------
 * Thousands of independently compressed chunks of uneven size and mixed codec, decoded
 * by one persistent launch that pulls work from a device queue ordered by estimated cost
 * (largest first).  There is no counterpart in CODAG, whose kernels assume one uniform
 * chunk size per launch; the per-chunk decoders are the ones behind the calls above. */
typedef struct {
    uint64_t comp_off;     /* stream byte offset in d_comp */
    uint64_t out_off;      /* output byte offset in d_out */
    uint32_t comp_len;     /* stream bytes */
    uint32_t out_len;      /* decoded bytes */
    uint8_t codec;         /* CODAG_CODEC_* */
    uint8_t elem_bytes;    /* RLE element width */
    uint8_t wrapper_bytes; /* Deflate header bytes to skip */
    uint8_t reserved[5];
} codag_chunk_desc;

typedef struct codag_plan codag_plan;

/* Copies the descriptors to the device (the only allocating call), orders the queue and
 * picks the launch shape (tune may be NULL: 8 warps per CTA, 4 ring slots, 10-bit tables).  In a plan,
 * tune->cta_per_chunk = k (1..4, warps_per_cta even) sends the Deflate chunks of at least
 * k x 256 KiB to warp pairs (a symbol decoder and a byte expander each), decoded first. */
codag_status codag_batch_plan(const codag_chunk_desc *h_descs, uint64_t n, const codag_tune *tune,
                              codag_plan **plan);
/* One persistent launch over all planned chunks; d_status has n entries (may be NULL).
 * With use_graph != 0 the launch is captured once into a CUDA graph for these pointers
 * and replayed on later calls with the same pointers. */
codag_status codag_batch_run(codag_plan *plan, const uint8_t *d_comp, uint64_t comp_bytes,
                             uint8_t *d_out, uint64_t out_bytes, int32_t *d_status, int use_graph,
                             codag_stream_t stream);
codag_status codag_batch_destroy(codag_plan *plan);

/* One persistent launch over n descriptors that already sit in device memory, for callers
 * that rebuild the chunk list for every launch (continuous batching).  d_order (n u32,
 * may be NULL = descriptor order) is the order the warps take chunks in; d_queue is 4 bytes
 * of device memory that this call resets on `stream`; d_status has n entries (may be NULL)
 * and entry i reports descriptor i.  tune may be NULL (8 warps per CTA, 4 ring slots, 10-bit
 * tables, as codag_batch_plan).  Allocates
 * nothing; the launch shape of each tune is measured once per device and cached. */
codag_status codag_batch_launch(const codag_chunk_desc *d_descs, const uint32_t *d_order, uint64_t n,
                                uint32_t *d_queue, const codag_tune *tune, const uint8_t *d_comp,
                                uint64_t comp_bytes, uint8_t *d_out, uint64_t out_bytes,
                                int32_t *d_status, codag_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* CODAG_H */
