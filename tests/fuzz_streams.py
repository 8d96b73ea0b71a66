"""Random RLE v1 / RLE v2 chunk streams written header by header from the format definition,
together with the values each must decode to: a model of the formats that shares nothing with
the encoders in codag_b200 or with the oracle.

RLE v1 (include/rlev1/decoder.h:686-790): an int8 header h; h < 0 is followed by -h unsigned
LEB128 literals; h >= 0 by an int8 delta and an unsigned LEB128 base, for h + 3 values
base + i * delta.
RLE v2, unsigned variant (include/rlev2/decoder_new.h:1000-1091): SHORT_REPEAT, DIRECT and
DELTA headers (fixed and packed).  Header lengths stay at or below 255 values, below the 8-bit
wrap of the reference's length counter, so the only quirk the model restates is DELTA's sign
rule: packed deltas are added when the base delta (taken modulo the element width) is non-zero
and subtracted when it is zero.  Every value is taken modulo 2^(8 * elem).

The generators draw every form the decoders branch on: all 32 width codes, varints of 1 to 10
bytes, 1 to 8 byte SHORT_REPEAT values, negative and zero deltas, 1-value literal groups and
130-value runs.
"""
from __future__ import annotations

import numpy as np

WIDTHS = [c + 1 if c < 24 else (2 * c - 22 if c < 28 else 8 * c - 184) for c in range(32)]
U64 = (1 << 64) - 1


def uleb(v: int) -> bytes:
    out = bytearray()
    while True:
        b = v & 0x7F
        v >>= 7
        if v:
            out.append(b | 0x80)
        else:
            out.append(b)
            return bytes(out)


def pack_msb(values: np.ndarray, width: int) -> bytes:
    """Values packed MSB first, `width` bits each, the last byte padded with zero bits."""
    if values.size == 0:
        return b""
    shifts = np.arange(width - 1, -1, -1, dtype=np.uint64)
    bits = ((values.astype(np.uint64)[:, None] >> shifts) & np.uint64(1)).astype(np.uint8)
    return np.packbits(bits.reshape(-1)).tobytes()


def _wide(rng: np.random.Generator, n: int) -> np.ndarray:
    """n 64-bit values whose magnitudes spread over every varint length."""
    v = rng.integers(0, 2**63, size=n, dtype=np.uint64) | (rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63))
    return v >> rng.integers(0, 64, size=n, dtype=np.uint64)


def rlev1_chunk(rng: np.random.Generator, cap: int, elem: int):
    mask = np.uint64((1 << (8 * elem)) - 1)
    s, vals, n = bytearray(), [], 0
    while n < cap:
        room = cap - n
        if room >= 3 and rng.random() < 0.5:
            cnt = int(rng.integers(3, min(130, room) + 1))
            delta = int(rng.integers(-128, 128))
            base = int(_wide(rng, 1)[0])
            s += bytes([cnt - 3, delta & 0xFF]) + uleb(base)
            v = np.uint64(base) + np.arange(cnt, dtype=np.uint64) * np.uint64(delta & U64)
        else:
            cnt = int(rng.integers(1, min(128, room) + 1))
            s.append((-cnt) & 0xFF)
            v = _wide(rng, cnt)
            for x in v.tolist():
                s += uleb(x)
        vals.append(v & mask)
        n += cnt
    return bytes(s), np.concatenate(vals)


def rlev2_chunk(rng: np.random.Generator, cap: int, elem: int):
    mask = np.uint64((1 << (8 * elem)) - 1)
    s, vals, n = bytearray(), [], 0
    while n < cap:
        room = cap - n
        kind = int(rng.integers(0, 4)) if room >= 3 else 1
        if kind == 0:  # SHORT_REPEAT: 3..10 copies of a 1..8 byte big-endian value
            cnt = int(rng.integers(3, min(10, room) + 1))
            nb = int(rng.integers(1, 9))
            x = int(_wide(rng, 1)[0]) & ((1 << (8 * nb)) - 1)
            s.append(((nb - 1) << 3) | (cnt - 3))
            s += x.to_bytes(nb, "big")
            v = np.full(cnt, x, dtype=np.uint64)
        elif kind == 1:  # DIRECT: 1..255 values of one of the 32 widths
            cnt = int(rng.integers(1, min(255, room) + 1))
            code = int(rng.integers(0, 32))
            w = WIDTHS[code]
            v = _wide(rng, cnt) & np.uint64((1 << w) - 1)
            field = cnt - 1
            s += bytes([0x40 | (code << 1) | (field >> 8), field & 0xFF]) + pack_msb(v, w)
        else:  # DELTA: fixed (width code 0) or packed deltas after the first two values
            cnt = int(rng.integers(2 if kind == 2 else 3, min(255, room) + 1))
            code = 0 if kind == 2 else int(rng.integers(1, 32))
            base = int(_wide(rng, 1)[0])
            d = int(rng.integers(-2**20, 2**20)) if rng.random() < 0.9 else 0
            zz = ((d << 1) ^ -1 if d < 0 else d << 1) & U64
            field = cnt - 1
            s += bytes([0xC0 | (code << 1) | (field >> 8), field & 0xFF]) + uleb(base) + uleb(zz)
            bd = np.uint64(d & U64) & mask
            if code == 0:
                v = np.uint64(base) + np.arange(cnt, dtype=np.uint64) * bd
            else:
                w = WIDTHS[code]
                ds = _wide(rng, cnt - 2) & np.uint64((1 << w) - 1)
                s += pack_msb(ds, w)
                first2 = np.array([base, (base + int(bd)) & U64], dtype=np.uint64)
                walk = np.cumsum(ds & mask, dtype=np.uint64)
                rest = first2[1] + walk if bd != 0 else first2[1] - walk
                v = np.concatenate([first2, rest])
        vals.append(v & mask)
        n += cnt
    return bytes(s), np.concatenate(vals)


def chunk_set(codec: str, n: int, chunk_bytes: int, elem: int, seed: int):
    """n random chunks of chunk_bytes decoded bytes each: (streams, each starting on a 16-byte
    boundary, stream offsets, stream lengths, the expected decoded bytes of all chunks)."""
    assert chunk_bytes % elem == 0
    rng = np.random.default_rng(seed)
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[elem]
    gen = rlev1_chunk if codec == "rlev1" else rlev2_chunk
    parts, offs, lens, outs = [], [], [], []
    pos = 0
    for _ in range(n):
        st, vals = gen(rng, chunk_bytes // elem, elem)
        offs.append(pos)
        lens.append(len(st))
        pad = (-len(st)) % 16
        parts.append(st + b"\0" * pad)
        pos += len(st) + pad
        outs.append(vals.astype(dt).view(np.uint8))
    comp = np.frombuffer(b"".join(parts) + b"\0" * 16, np.uint8).copy()
    return comp, np.array(offs, np.uint64), np.array(lens, np.uint64), np.concatenate(outs)
