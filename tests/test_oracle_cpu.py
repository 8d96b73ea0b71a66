"""CPU tests of the oracle and of the host format producers (no GPU).

The oracle is pinned by: hand-built known-answer streams for every header type and kept
quirk (tests/vectors.py), round trips through the product encoders, agreement of two
independent Deflate decoders, and golden files written by CODAG's own compressor.
"""
import numpy as np
import pytest

from tests.vectors import VECTORS, RLEV1, RLEV2

CH = 131072


def _values_to_bytes(values, e):
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[e]
    return np.array([v % (1 << (8 * e)) for v in values], dtype=np.uint64).astype(dt).view(np.uint8)


@pytest.mark.parametrize("name", sorted(VECTORS))
def test_known_answer_vectors(oracle, name):
    codec, e, stream, expected = VECTORS[name]
    s = np.array(stream, dtype=np.uint8)
    want = _values_to_bytes(expected, e)
    if codec == RLEV1:
        st, out = oracle.rlev1_chunk(s, want.size, e)
    else:
        st, out = oracle.rlev2_chunk(s, want.size, e)
    assert st == oracle.OK
    assert np.array_equal(out, want)


@pytest.mark.parametrize("codec", ["rlev1", "rlev2"])
@pytest.mark.parametrize("e", [1, 2, 4, 8])
def test_rle_round_trip(native, oracle, codec, e):
    n = (1 << 20) // e * 2
    if codec == "rlev1":
        col = native.gen_rlev1_column(n, 20260101 + e, e)
        blob, off, ln = native.encode_rlev1(col, CH, e)
        comp, base = blob, 8
    else:
        col = native.gen_rlev2_column(n, 20260102 + e, e)
        comp, off, ln = native.encode_rlev2(col, CH, e)
        base = 0
        assert off[-1] == col.size  # the last blk_off entry carries the original size
    nch = ln.size
    assert nch % 32 == 0 and nch * CH >= col.size
    out = np.zeros(nch * CH, np.uint8)
    status = oracle.decode_batch(comp, off[:nch] + base, ln, out, np.arange(nch) * CH, [CH] * nch, [CH] * nch,
                                 [0 if codec == "rlev1" else 1] * nch, [e] * nch, [0] * nch)
    assert not status.any()
    assert np.array_equal(out[:col.size], col)
    assert not out[col.size:].any()


def test_rlev1_layout(native):
    col = native.gen_rlev1_column(300_000, 5, 8)
    blob, off, ln = native.encode_rlev1(col, CH, 8)
    assert int(blob[:8].view(np.uint64)[0]) == col.size
    n = ln.size
    assert off.size == n + 1 and off[0] == 0
    assert np.all(np.diff(off) == (ln + 3) // 4 * 4)  # 4-byte aligned streams
    assert blob.size == 8 + off[-1]


def test_rlev2_layout(native):
    col = native.gen_rlev2_column(300_000, 5, 8)
    comp, off, ln = native.encode_rlev2(col, CH, 8)
    n = ln.size
    assert np.all(off[:n] % 128 == 0)
    assert np.all(np.diff(off[:n]) == ((ln[:-1] + 127) // 128 * 128))
    assert comp.size == off[n - 1] + (ln[-1] + 127) // 128 * 128


def test_rlev2_zero_run_header(native, oracle):
    """A 128-value run of zeros: CODAG's encoder writes a length field of 511 there
    (encoder.h writeDirectValues with var_runlen == 0); ours writes 128 and decodes back."""
    col = np.zeros(16384, np.uint64)
    col[:5] = [9, 1, 7, 3, 2]
    s = native.encode_one(1, col.view(np.uint8), 8)
    st, out = oracle.rlev2_chunk(s, col.nbytes, 8)
    assert st == oracle.OK and np.array_equal(out.view(np.uint64), col)


def test_deflate_two_decoders(native, oracle):
    txt = native.gen_text(3 * CH + 777, 11)
    comp, bo, cl = native.encode_deflate(txt, CH, 6)
    assert bo[0] == txt.size and bo[1] == 0 and bo.size == cl.size + 2
    assert np.all(cl % 8 == 0) and np.all(np.diff(bo[1:]) == cl)
    rel = bo[1:]
    pieces = []
    for i in range(cl.size):
        s = comp[int(rel[i]):int(rel[i + 1])]
        st, out = oracle.deflate_chunk(s, CH)
        st2, out2, types = oracle.deflate_rfc_chunk(s, CH)
        assert st == oracle.OK and st2 == oracle.OK
        assert np.array_equal(out, out2)
        assert types == 4  # dynamic blocks only
        pieces.append(out)
    dec = np.concatenate(pieces)
    assert np.array_equal(dec[:txt.size], txt) and not dec[txt.size:].any()


def test_deflate_stored_and_fixed_blocks(native, oracle):
    import zlib
    noise = np.frombuffer(np.random.default_rng(1).bytes(70000), np.uint8)
    text = native.gen_text(70000, 3)
    for data, level, strategy, want in ((noise, 0, zlib.Z_DEFAULT_STRATEGY, 1), (text, 6, zlib.Z_FIXED, 2)):
        co = zlib.compressobj(level, zlib.DEFLATED, 15, 8, strategy)
        s = np.frombuffer(co.compress(data.tobytes()) + co.flush(), np.uint8)
        st, out, types = oracle.deflate_rfc_chunk(s, data.size)
        assert st == oracle.OK and types == want and np.array_equal(out, data)


def test_deflate_layout_matches_codag_compressor(native):
    """Golden files from CODAG's deflate_compressor.py (tests/golden/make_golden.py)."""
    from pathlib import Path
    g = Path(__file__).parent / "golden"
    src = np.fromfile(g / "deflate_src.bin", np.uint8)
    comp, bo, cl = native.encode_deflate(src, CH, 9)
    assert np.array_equal(comp, np.fromfile(g / "deflate_ref_comp.bin", np.uint8))
    assert np.array_equal(bo, np.fromfile(g / "deflate_ref_blk_offset.bin", np.uint64))
    assert np.array_equal(cl, np.fromfile(g / "deflate_ref_col_len.bin", np.uint64))


def test_corrupt_streams_rejected(oracle):
    # truncated varint, header past the end, run overshooting the chunk
    st, _ = oracle.rlev1_chunk(np.array([0xFE, 0x85], np.uint8), 16, 8)
    assert st == oracle.ECORRUPT
    st, _ = oracle.rlev1_chunk(np.array([0x05, 0x01, 0x00], np.uint8), 16, 8)
    assert st == oracle.ECORRUPT
    st, _ = oracle.rlev2_chunk(np.array([0x5E, 0x03, 0x00], np.uint8), 32, 8)
    assert st == oracle.ECORRUPT
    st, _ = oracle.deflate_chunk(np.array([0x78, 0x9C, 0xFF, 0xFF], np.uint8), 64)
    assert st == oracle.ECORRUPT
