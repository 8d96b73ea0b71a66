"""A plain walk over the headers of a well-formed ORC RLE v2 stream (test helper).

Sizes every header by the format definition, reading the DIRECT / PATCHED_BASE / DELTA
length fields with their full 9 bits, so it follows a stream as its writer laid it out.
Used by the golden-file generator and tests to name the two places where CODAG's own
encoder and decoder disagree:

  zero_run  a DIRECT header whose length field says 512 values (CODAG's encoder writes it for
            a run of 128 zeros, include/rlev2/encoder.h:424-440); CODAG's decoder keeps the
            length in a uint8_t (decoder_new.h:1019) and reads 0 values;
  wide_patch a PATCHED_BASE patch whose value has bits at or above bit 32; CODAG's decoder
            masks patches with a 32-bit mask (decoder_new.h:1103) and drops those bits.
"""
from __future__ import annotations

WIDTH = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 26, 28, 30, 32, 40, 48,
         56, 64]
KINDS = ("short_repeat", "direct", "patched_base", "delta_fixed", "delta_packed")


def closest(b: int) -> int:
    return (b if b else 1) if b <= 24 else ((b + 1) // 2 * 2 if b <= 32 else (b + 7) // 8 * 8)


def _bits(s: bytes, bitpos: int, w: int) -> int:
    """w bits at bitpos, most significant first."""
    v = 0
    for k in range(w):
        p = bitpos + k
        v = (v << 1) | ((s[p >> 3] >> (7 - (p & 7))) & 1)
    return v


def walk(stream) -> dict:
    """Header counts per kind and the two quirk flags of one stream."""
    s = bytes(stream)
    out = {k: 0 for k in KINDS}
    out.update(zero_run=False, wide_patch=False)
    p = 0
    while p < len(s):
        f = s[p]
        kind = f >> 6
        ln = (((f & 1) << 8) | s[p + 1]) + 1 if p + 1 < len(s) else 0
        if kind == 0:
            out["short_repeat"] += 1
            p += 2 + ((f >> 3) & 7)
        elif kind == 1:
            out["direct"] += 1
            out["zero_run"] |= ln == 512
            n = 128 if ln == 512 else ln  # the quirk header is followed by 128 values
            p += 2 + (n * WIDTH[(f >> 1) & 31] + 7) // 8
        elif kind == 2:
            out["patched_base"] += 1
            t, fo = s[p + 2], s[p + 3]
            fbw, pw, pgw, pll = WIDTH[(f >> 1) & 31], WIDTH[t & 31], ((fo >> 5) & 7) + 1, fo & 31
            vals = p + 4 + ((t >> 5) & 7) + 1
            pat = vals + (ln * fbw + 7) // 8
            cfb = closest(pw + pgw)
            for k in range(pll):
                if _bits(s, pat * 8 + k * cfb, cfb) & ((1 << pw) - 1) >= 1 << 32:
                    out["wide_patch"] = True
            p = pat + (pll * cfb + 7) // 8
        else:
            q = p + 2
            for _ in range(2):
                while s[q] >= 0x80:
                    q += 1
                q += 1
            enc = (f >> 1) & 31
            out["delta_packed" if enc else "delta_fixed"] += 1
            p = q + ((ln - 2) * WIDTH[enc] + 7) // 8 if enc else q
    return out


def detranspose(region, lens) -> list:
    """The 32 substreams of one chunk of CODAG's transposed RLE v2 layout: the region interleaves
    them in 4-byte words, row w holding word w of every substream longer than 4w, in substream
    order (include/rlev2/encoder_trans.h:359-391)."""
    r = bytes(region)
    words = [(int(x) + 3) // 4 for x in lens]
    subs = [bytearray() for _ in lens]
    p = 0
    for w in range(max(words, default=0)):
        for t, n in enumerate(words):
            if n > w:
                subs[t] += r[p:p + 4]
                p += 4
    return [bytes(s[:int(x)]) for s, x in zip(subs, lens)]


def interleave_values(subvals, ru: int, elem: int) -> bytes:
    """Chunk bytes from the 32 substreams' decoded values (bytes, elem-byte little-endian
    values): value k of substream t is element t*ru + (k//ru)*32*ru + k%ru."""
    import numpy as np
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[elem]
    per = len(subvals[0]) // elem
    out = np.zeros(32 * per, dt)
    k = np.arange(per)
    for t, sv in enumerate(subvals):
        out[t * ru + (k // ru) * 32 * ru + k % ru] = np.frombuffer(sv, dt)
    return out.tobytes()
