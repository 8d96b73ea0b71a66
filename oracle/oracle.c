/*
 * oracle.c -- CPU restatement of CODAG's chunk decoders.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is the parity checker for the CUDA decoders in codag_b200/csrc.  Only the
 * test-suite, the smoke test and the CPU-baseline leg of bench.py load it.  The product
 * path never calls into it.
 *
 * What it restates (paths are relative to the illinois-impact/codag tree):
 *   - ORC RLE v1 chunk decoder: include/rlev1/decoder.h:588-798
 *     (decoder_warp_orig_rdw_fsm, launched by inflate_orig_rdw at :906-936).
 *   - ORC RLE v2 chunk decoder: include/rlev2/decoder_new.h:909-1187
 *     (decoder_warp_orig_rdw, launched by inflate_orig_rdw at :1344-1377),
 *     with the header masks and bit-width tables of include/rlev2/utils.h:22-59.
 *   - Deflate chunk decoder: include/zlib/zlib.h:807-902 (full_warp_shared_lut / inflate).
 *     Two CPU decoders are provided: the system zlib (third-party; zlibVersion() is
 *     reported by oracle_zlib_version) and a small RFC 1951 restatement
 *     (oracle_deflate_rfc_chunk) that also reports which block types a stream uses.
 *
 * Pinning (CODAG's repository has no tests, golden vectors or known-answer data):
 *   - RLE v1: pinned to CODAG's own GPU decoder -- tests/golden/ref_rlev1_*.npz hold its
 *     per-chunk digests on seeded chunks (oracle/ref_harness.cu, tests/golden/make_ref_golden.py).
 *   - Deflate: pinned to zlib (the system zlib decodes the same streams) and to files written
 *     by CODAG's own Python compressor (tests/golden/deflate_ref_*).
 *   - RLE v2: parity unpinned against CODAG's decoder output (its kernel did not finish on
 *     well-formed chunks and is not run); checked by hand-built known-answer streams for
 *     every header kind and quirk and by round trips through the restated encoder.
 *
 * Integer semantics follow what the reference kernels compute on the GPU, value by value:
 * element arithmetic is modulo 2^(8*elem_bytes); a shift by at least the register width
 * gives 0 (PTX shl/shr clamp the shift amount).  Reference quirks that are kept on purpose:
 *   - RLE v2 run lengths are held in a uint8_t (decoder_new.h:1019,1048,1095), so a 9-bit
 *     length field of 255 decodes to 0 values and DELTA's "len -= 2" wraps modulo 256.
 *   - RLE v2 PATCHED_BASE masks patch values with a 32-bit mask (decoder_new.h:1103):
 *     patch widths above 32 bits are truncated to their low 32 bits.
 *   - RLE v2 signed varints are decoded with an arithmetic right shift (decoder_new.h:990).
 *   - RLE v2 DELTA multiplies packed deltas by (base_delta > 0 ? 1 : -1) on the unsigned
 *     element type (decoder_new.h:1057).
 * Where the reference would read or write out of bounds on a malformed stream, the oracle
 * stops and returns ORC_ECORRUPT instead.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { ORC_OK = 0, ORC_EINVAL = 1, ORC_ECORRUPT = 2 };

/* ------------------------------------------------------------------------------------ */
/* element helpers                                                                       */
/* ------------------------------------------------------------------------------------ */

static inline uint64_t elem_mask(int e) { return e == 8 ? ~0ull : ((1ull << (8 * e)) - 1ull); }

/* shift that yields 0 for amounts >= 64, as a clamped PTX shift does */
static inline uint64_t shl64(uint64_t v, unsigned s) { return s >= 64 ? 0ull : (v << s); }
static inline uint64_t shr64(uint64_t v, unsigned s) { return s >= 64 ? 0ull : (v >> s); }

typedef struct {
    uint8_t *out;        /* chunk output base */
    uint64_t store_cap;  /* elements that may be stored (clip of the last chunk) */
    uint64_t limit;      /* logical chunk capacity in elements */
    uint64_t n;          /* elements produced */
    int e;               /* element bytes */
    int overflow;        /* a value fell beyond the logical capacity */
} elem_sink;

static inline void sink_put(elem_sink *s, uint64_t v) {
    if (s->n >= s->limit) { s->overflow = 1; s->n++; return; }
    if (s->n < s->store_cap) {
        uint8_t *p = s->out + s->n * (uint64_t)s->e;
        for (int i = 0; i < s->e; i++) p[i] = (uint8_t)(v >> (8 * i));
    }
    s->n++;
}

static inline uint64_t sink_get(const elem_sink *s, uint64_t idx) {
    const uint8_t *p = s->out + idx * (uint64_t)s->e;
    uint64_t v = 0;
    for (int i = 0; i < s->e; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

static inline void sink_set(elem_sink *s, uint64_t idx, uint64_t v) {
    uint8_t *p = s->out + idx * (uint64_t)s->e;
    for (int i = 0; i < s->e; i++) p[i] = (uint8_t)(v >> (8 * i));
}

/* ------------------------------------------------------------------------------------ */
/* ORC RLE v1 (include/rlev1/decoder.h:588-798)                                          */
/* ------------------------------------------------------------------------------------ */
/*
 * Stream grammar: a header byte h (int8).  h < 0: -h literals follow, each an unsigned
 * LEB128 varint (decoder.h:686-727).  h >= 0: a run of h+3 values; an int8 delta byte and
 * an unsigned varint base follow, and value i is base + i*delta (decoder.h:731-790).
 * The decoder loops while fewer than chunk_bytes bytes were produced (decoder.h:669).
 */
static int rlev1_varint(const uint8_t *in, uint64_t len, uint64_t *p, uint64_t *val) {
    uint64_t v = 0;
    unsigned off = 0;
    for (;;) {
        if (*p >= len) return ORC_ECORRUPT;
        uint8_t b = in[(*p)++];
        if (b < 0x80) { v |= shl64(b, off); break; }
        v |= shl64(b & 0x7f, off);
        off += 7;
    }
    *val = v;
    return ORC_OK;
}

int oracle_rlev1_decode_chunk(const uint8_t *in, uint64_t in_len, uint8_t *out,
                              uint64_t chunk_bytes, uint64_t store_bytes, int e) {
    if (!(e == 1 || e == 2 || e == 4 || e == 8) || chunk_bytes % e || store_bytes > chunk_bytes)
        return ORC_EINVAL;
    const uint64_t m = elem_mask(e);
    elem_sink s = {out, store_bytes / e, chunk_bytes / e, 0, e, 0};
    uint64_t p = 0;
    while (s.n * (uint64_t)e < chunk_bytes) {
        if (p >= in_len) return ORC_ECORRUPT;
        int8_t h = (int8_t)in[p++];
        if (h < 0) {
            int cnt = -(int)h;
            for (int i = 0; i < cnt; i++) {
                uint64_t v;
                if (rlev1_varint(in, in_len, &p, &v)) return ORC_ECORRUPT;
                sink_put(&s, v & m);
            }
        } else {
            if (p >= in_len) return ORC_ECORRUPT;
            int8_t delta = (int8_t)in[p++];
            uint64_t base;
            if (rlev1_varint(in, in_len, &p, &base)) return ORC_ECORRUPT;
            int cnt = (int)h + 3;
            for (int i = 0; i < cnt; i++)
                sink_put(&s, (base + (uint64_t)((int64_t)i * (int64_t)delta)) & m);
        }
        if (s.overflow) return ORC_ECORRUPT;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------ */
/* ORC RLE v2 (include/rlev2/decoder_new.h:909-1187, include/rlev2/utils.h:22-59)        */
/* ------------------------------------------------------------------------------------ */
static const uint8_t V2_WIDTH_DECODE[32] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11,
                                            12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22,
                                            23, 24, 26, 28, 30, 32, 40, 48, 56, 64};
static const uint8_t V2_CLOSEST_WIDTH[65] = {
    1,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21,
    22, 23, 24, 26, 26, 28, 28, 30, 30, 32, 32, 40, 40, 40, 40, 40, 40, 40, 40, 48, 48, 48,
    48, 48, 48, 48, 48, 56, 56, 56, 56, 56, 56, 56, 56, 64, 64, 64, 64, 64, 64, 64, 64};

typedef struct {
    const uint8_t *in;
    uint64_t len, p;
    int bad;
} v2_src;

static inline uint8_t v2_byte(v2_src *r) {
    if (r->p >= r->len) { r->bad = 1; return 0; }
    return r->in[r->p++];
}

/* MSB-first bit reader local to one header (decoder_new.h:1024-1040) */
typedef struct { uint8_t cur; unsigned left; } v2_bits;

static inline uint64_t v2_read_bits(v2_src *r, v2_bits *b, unsigned n) {
    uint64_t v = 0;
    while (n > b->left) {
        v = shl64(v, b->left) | (b->cur & ((1u << b->left) - 1u));
        n -= b->left;
        b->cur = v2_byte(r);
        b->left = 8;
    }
    if (n) {
        v = shl64(v, n);
        b->left -= n;
        v |= (b->cur >> b->left) & ((1u << n) - 1u);
    }
    return v;
}

static uint64_t v2_uvarint(v2_src *r) {
    uint64_t v = 0;
    unsigned off = 0;
    uint8_t b;
    do {
        b = v2_byte(r);
        if (r->bad) return 0;
        v |= shl64((uint64_t)(b & 0x7f), off);
        off += 7;
    } while (b >= 0x80);
    return v;
}

static int64_t v2_svarint(v2_src *r) {
    int64_t u = (int64_t)v2_uvarint(r);
    return (u >> 1) ^ -(u & 1); /* arithmetic shift, as decoder_new.h:990 */
}

int oracle_rlev2_decode_chunk(const uint8_t *in, uint64_t in_len, uint8_t *out,
                              uint64_t chunk_bytes, uint64_t store_bytes, int e,
                              uint64_t *produced_bytes) {
    if (!(e == 1 || e == 2 || e == 4 || e == 8) || chunk_bytes % e || store_bytes > chunk_bytes)
        return ORC_EINVAL;
    const uint64_t m = elem_mask(e);
    elem_sink s = {out, store_bytes / e, chunk_bytes / e, 0, e, 0};
    v2_src r = {in, in_len, 0, 0};
    int st = ORC_OK;
    while (r.p < in_len) {
        uint8_t first = v2_byte(&r);
        switch (first & 0xC0) {
        case 0x00: { /* SHORT_REPEAT (decoder_new.h:1004-1014) */
            unsigned nbytes = ((first >> 3) & 7) + 1;
            unsigned count = (first & 7) + 3;
            uint64_t v = 0;
            while (nbytes-- > 0) v |= shl64(v2_byte(&r), nbytes * 8);
            v &= m;
            while (count-- > 0) sink_put(&s, v);
        } break;
        case 0x40: { /* DIRECT (decoder_new.h:1015-1043) */
            unsigned fbw = V2_WIDTH_DECODE[(first >> 1) & 0x1f];
            uint8_t len = (uint8_t)(((((unsigned)first & 1u) << 8) | v2_byte(&r)) + 1u);
            v2_bits b = {0, 0};
            while (len-- > 0) sink_put(&s, v2_read_bits(&r, &b, fbw) & m);
        } break;
        case 0xC0: { /* DELTA (decoder_new.h:1044-1091) */
            unsigned enc = (first >> 1) & 0x1f;
            unsigned fbw = V2_WIDTH_DECODE[enc];
            uint8_t len = (uint8_t)(((((unsigned)first & 1u) << 8) | v2_byte(&r)) + 1u);
            uint64_t base = v2_uvarint(&r) & m;
            uint64_t bdelta = (uint64_t)v2_svarint(&r) & m;
            sink_put(&s, base);
            base = (base + bdelta) & m;
            sink_put(&s, base);
            len = (uint8_t)(len - 2);
            int positive = bdelta > 0; /* multiplier = base_delta > 0 ? 1 : -1 */
            if (enc != 0) {
                v2_bits b = {0, 0};
                while (len-- > 0) {
                    uint64_t d = v2_read_bits(&r, &b, fbw) & m;
                    base = (positive ? base + d : base - d) & m;
                    sink_put(&s, base);
                }
            } else {
                while (len-- > 0) {
                    base = (base + bdelta) & m;
                    sink_put(&s, base);
                }
            }
        } break;
        default: { /* PATCHED_BASE (decoder_new.h:1092-1183) */
            unsigned fbw = V2_WIDTH_DECODE[(first >> 1) & 0x1f];
            uint8_t len = (uint8_t)(((((unsigned)first & 1u) << 8) | v2_byte(&r)) + 1u);
            uint8_t third = v2_byte(&r), fourth = v2_byte(&r);
            unsigned bw = ((third >> 5) & 7) + 1;
            unsigned pw = V2_WIDTH_DECODE[third & 0x1f];
            unsigned pgw = ((fourth >> 5) & 7) + 1;
            unsigned pll = fourth & 0x1f;
            uint64_t pmask = pw >= 32 ? 0xFFFFFFFFull : ((1ull << pw) - 1ull);
            uint64_t base_out = s.n;
            uint64_t base = 0;
            while (bw-- > 0) base |= shl64(v2_byte(&r), bw * 8);
            v2_bits b = {0, 0};
            while (len-- > 0) sink_put(&s, (v2_read_bits(&r, &b, fbw) + base) & m);
            if (pw + pgw > 64) { st = ORC_ECORRUPT; break; }
            unsigned cfb = V2_CLOSEST_WIDTH[pw + pgw];
            b.cur = 0; b.left = 0;
            uint64_t gap = 0;
            while (pll-- > 0) {
                uint64_t ent = v2_read_bits(&r, &b, cfb);
                gap += shr64(ent, pw);
                uint64_t idx = base_out + gap;
                if (r.bad || idx >= s.n || s.overflow) { st = ORC_ECORRUPT; break; }
                uint64_t patch = shl64((ent & pmask) & m, fbw) & m;
                if (idx < s.store_cap) {
                    uint64_t v = sink_get(&s, idx);
                    sink_set(&s, idx, (((v - base) & m) | patch) + base);
                }
            }
        } break;
        }
        if (st || r.bad || s.overflow) return ORC_ECORRUPT;
    }
    if (produced_bytes) *produced_bytes = s.n * (uint64_t)e;
    if (s.n * (uint64_t)e < store_bytes) return ORC_ECORRUPT;
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------ */
/* Deflate                                                                               */
/* ------------------------------------------------------------------------------------ */

const char *oracle_zlib_version(void) { return zlibVersion(); }

/* System zlib, raw inflate after skipping the wrapper bytes the reference skips
 * (zlib.h:819 skips the 2-byte zlib header; the adler32 trailer is not checked). */
int oracle_deflate_decode_chunk(const uint8_t *in, uint64_t in_len, int wrapper, uint8_t *out,
                                uint64_t chunk_bytes, uint64_t store_bytes,
                                uint64_t *produced_bytes) {
    if (wrapper < 0 || (uint64_t)wrapper > in_len || store_bytes > chunk_bytes) return ORC_EINVAL;
    uint8_t *dst = out;
    uint8_t *tmp = NULL;
    if (store_bytes < chunk_bytes) {
        tmp = (uint8_t *)malloc(chunk_bytes ? chunk_bytes : 1);
        if (!tmp) return ORC_EINVAL;
        dst = tmp;
    }
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (inflateInit2(&zs, -15) != Z_OK) { free(tmp); return ORC_EINVAL; }
    zs.next_in = (Bytef *)(in + wrapper);
    zs.avail_in = (uInt)(in_len - wrapper);
    zs.next_out = dst;
    zs.avail_out = (uInt)chunk_bytes;
    int rc = inflate(&zs, Z_FINISH);
    uint64_t produced = zs.total_out;
    inflateEnd(&zs);
    if (tmp) { memcpy(out, tmp, store_bytes); free(tmp); }
    if (produced_bytes) *produced_bytes = produced;
    if (rc != Z_STREAM_END || produced < store_bytes) return ORC_ECORRUPT;
    return ORC_OK;
}

/* A compact RFC 1951 decoder restating the block loop of zlib.h:807-866 (BFINAL/BTYPE,
 * fixed tables zlib.h:1622-1650, dynamic header zlib.h:607-707, symbol loop zlib.h:712-805,
 * length/distance tables zlib.h:35-57).  Unlike the reference it decodes stored blocks
 * (the reference skips them, zlib.h:840-842).  Bit 0/1/2 of *types is set when a stored,
 * fixed or dynamic block is seen. */
typedef struct {
    const uint8_t *in;
    uint64_t len, pos;
    uint32_t bitbuf;
    int bitcnt;
    int bad;
} rfc_state;

static int rfc_bits(rfc_state *s, int need) {
    uint64_t val = s->bitbuf;
    while (s->bitcnt < need) {
        if (s->pos >= s->len) { s->bad = 1; return 0; }
        val |= (uint64_t)s->in[s->pos++] << s->bitcnt;
        s->bitcnt += 8;
    }
    s->bitbuf = (uint32_t)(val >> need);
    s->bitcnt -= need;
    return (int)(val & ((1ull << need) - 1));
}

typedef struct { short count[16]; short symbol[320]; } rfc_huff;

static int rfc_build(rfc_huff *h, const short *length, int n) {
    short offs[16];
    for (int l = 0; l < 16; l++) h->count[l] = 0;
    for (int s = 0; s < n; s++) h->count[length[s]]++;
    if (h->count[0] == n) return 0;
    int left = 1;
    for (int l = 1; l < 16; l++) { left <<= 1; left -= h->count[l]; if (left < 0) return -1; }
    offs[1] = 0;
    for (int l = 1; l < 15; l++) offs[l + 1] = offs[l] + h->count[l];
    for (int s = 0; s < n; s++) if (length[s]) h->symbol[offs[length[s]]++] = (short)s;
    return left;
}

static int rfc_decode(rfc_state *s, const rfc_huff *h) {
    int code = 0, first = 0, index = 0;
    for (int l = 1; l < 16; l++) {
        code |= rfc_bits(s, 1);
        if (s->bad) return -1;
        int count = h->count[l];
        if (code - count < first) return h->symbol[index + (code - first)];
        index += count;
        first += count;
        first <<= 1;
        code <<= 1;
    }
    return -1;
}

static const short RFC_LBASE[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                    31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
static const short RFC_LEXT[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                   2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
static const short RFC_DBASE[30] = {1,    2,    3,    4,    5,    7,     9,     13,    17,  25,
                                    33,   49,   65,   97,   129,  193,   257,   385,   513, 769,
                                    1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
static const short RFC_DEXT[30] = {0, 0, 0, 0, 1, 1, 2, 2,  3,  3,  4,  4,  5,  5,  6,
                                   6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

static int rfc_codes(rfc_state *s, const rfc_huff *lc, const rfc_huff *dc, uint8_t *out,
                     uint64_t cap, uint64_t *n) {
    for (;;) {
        int sym = rfc_decode(s, lc);
        if (sym < 0) return ORC_ECORRUPT;
        if (sym < 256) {
            if (*n >= cap) return ORC_ECORRUPT;
            out[(*n)++] = (uint8_t)sym;
        } else if (sym == 256) {
            return ORC_OK;
        } else {
            sym -= 257;
            if (sym >= 29) return ORC_ECORRUPT;
            int len = RFC_LBASE[sym] + rfc_bits(s, RFC_LEXT[sym]);
            int ds = rfc_decode(s, dc);
            if (ds < 0 || ds >= 30) return ORC_ECORRUPT;
            uint64_t dist = (uint64_t)RFC_DBASE[ds] + (uint64_t)rfc_bits(s, RFC_DEXT[ds]);
            if (s->bad || dist > *n || *n + (uint64_t)len > cap) return ORC_ECORRUPT;
            for (int i = 0; i < len; i++, (*n)++) out[*n] = out[*n - dist];
        }
    }
}

int oracle_deflate_rfc_chunk(const uint8_t *in, uint64_t in_len, int wrapper, uint8_t *out,
                             uint64_t cap, uint64_t *produced, uint32_t *types) {
    static const short order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
    if (wrapper < 0 || (uint64_t)wrapper > in_len) return ORC_EINVAL;
    rfc_state s = {in, in_len, (uint64_t)wrapper, 0, 0, 0};
    uint64_t n = 0;
    uint32_t seen = 0;
    int last;
    rfc_huff lc, dc;
    short lengths[320];
    do {
        last = rfc_bits(&s, 1);
        int type = rfc_bits(&s, 2);
        if (s.bad) return ORC_ECORRUPT;
        if (type == 0) {
            seen |= 1;
            s.bitbuf = 0;
            s.bitcnt = 0;
            if (s.pos + 4 > s.len) return ORC_ECORRUPT;
            unsigned len = s.in[s.pos] | (s.in[s.pos + 1] << 8);
            unsigned nlen = s.in[s.pos + 2] | (s.in[s.pos + 3] << 8);
            s.pos += 4;
            if (len != (~nlen & 0xffff) || s.pos + len > s.len || n + len > cap) return ORC_ECORRUPT;
            memcpy(out + n, s.in + s.pos, len);
            s.pos += len;
            n += len;
        } else if (type == 1) {
            seen |= 2;
            int sym = 0;
            for (; sym < 144; sym++) lengths[sym] = 8;
            for (; sym < 256; sym++) lengths[sym] = 9;
            for (; sym < 280; sym++) lengths[sym] = 7;
            for (; sym < 288; sym++) lengths[sym] = 8;
            rfc_build(&lc, lengths, 288);
            for (sym = 0; sym < 30; sym++) lengths[sym] = 5;
            rfc_build(&dc, lengths, 30);
            if (rfc_codes(&s, &lc, &dc, out, cap, &n)) return ORC_ECORRUPT;
        } else if (type == 2) {
            seen |= 4;
            int nlen = rfc_bits(&s, 5) + 257, ndist = rfc_bits(&s, 5) + 1, ncode = rfc_bits(&s, 4) + 4;
            if (s.bad || nlen > 286 || ndist > 30) return ORC_ECORRUPT;
            int idx;
            for (idx = 0; idx < ncode; idx++) lengths[order[idx]] = (short)rfc_bits(&s, 3);
            for (; idx < 19; idx++) lengths[order[idx]] = 0;
            if (rfc_build(&lc, lengths, 19) != 0) return ORC_ECORRUPT;
            idx = 0;
            while (idx < nlen + ndist) {
                int sym = rfc_decode(&s, &lc);
                if (sym < 0) return ORC_ECORRUPT;
                if (sym < 16) {
                    lengths[idx++] = (short)sym;
                } else {
                    int len = 0, rep;
                    if (sym == 16) {
                        if (idx == 0) return ORC_ECORRUPT;
                        len = lengths[idx - 1];
                        rep = 3 + rfc_bits(&s, 2);
                    } else if (sym == 17) {
                        rep = 3 + rfc_bits(&s, 3);
                    } else {
                        rep = 11 + rfc_bits(&s, 7);
                    }
                    if (idx + rep > nlen + ndist) return ORC_ECORRUPT;
                    while (rep--) lengths[idx++] = (short)len;
                }
            }
            if (s.bad || lengths[256] == 0) return ORC_ECORRUPT;
            int err = rfc_build(&lc, lengths, nlen);
            if (err < 0 || (err > 0 && nlen - lc.count[0] != 1)) return ORC_ECORRUPT;
            err = rfc_build(&dc, lengths + nlen, ndist);
            if (err < 0 || (err > 0 && ndist - dc.count[0] != 1)) return ORC_ECORRUPT;
            if (rfc_codes(&s, &lc, &dc, out, cap, &n)) return ORC_ECORRUPT;
        } else {
            return ORC_ECORRUPT;
        }
    } while (!last);
    if (produced) *produced = n;
    if (types) *types = seen;
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------ */
/* chunk batches (OpenMP over chunks): the CPU baseline and the test checker             */
/* ------------------------------------------------------------------------------------ */
enum { ORC_RLEV1 = 0, ORC_RLEV2 = 1, ORC_DEFLATE = 2 };

/* Decode n independent chunks.  Chunk i reads comp[comp_off[i] .. + comp_len[i]) and writes
 * out[out_off[i] .. + store_len[i]); its logical decoded size is chunk_len[i].  codec[i],
 * elem[i] and wrapper[i] select the decoder per chunk (wrapper is the Deflate header size
 * to skip).  status[i] receives ORC_OK / ORC_ECORRUPT.  Returns the number of failed chunks. */
int64_t oracle_decode_batch(const uint8_t *comp, const uint64_t *comp_off, const uint64_t *comp_len,
                            uint8_t *out, const uint64_t *out_off, const uint64_t *chunk_len,
                            const uint64_t *store_len, const uint8_t *codec, const uint8_t *elem,
                            const uint8_t *wrapper, int32_t *status, int64_t n, int nthreads) {
    int64_t bad = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(+ : bad)
#endif
    for (int64_t i = 0; i < n; i++) {
        const uint8_t *src = comp + comp_off[i];
        uint8_t *dst = out + out_off[i];
        int st;
        uint64_t produced = 0;
        switch (codec[i]) {
        case ORC_RLEV1:
            st = oracle_rlev1_decode_chunk(src, comp_len[i], dst, chunk_len[i], store_len[i], elem[i]);
            break;
        case ORC_RLEV2:
            st = oracle_rlev2_decode_chunk(src, comp_len[i], dst, chunk_len[i], store_len[i], elem[i],
                                           &produced);
            break;
        case ORC_DEFLATE:
            st = oracle_deflate_decode_chunk(src, comp_len[i], wrapper[i], dst, chunk_len[i],
                                             store_len[i], &produced);
            break;
        default:
            st = ORC_EINVAL;
        }
        if (status) status[i] = st;
        if (st) bad++;
    }
    return bad;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
