"""RLE decode with one CTA per chunk (codag_tune.cta_per_chunk = 1): the CTA stages the
stream in shared memory, one warp walks the headers and all warps expand them.  Results
must equal the oracle's and the source's, including the fallbacks to the one-pass warp
decoder (a stream larger than the 64 KiB stage, more headers than the descriptor budget,
malformed streams) and outputs that are not element aligned (warp path)."""
import contextlib

import numpy as np
import pytest

from codag_b200 import native

CH = 131072
RLEV1, RLEV2 = native.RLEV1, native.RLEV2


@contextlib.contextmanager
def cta_mode(codec, warps):
    old = native.get_tune(codec)
    native.set_tune(codec, warps, 4, 10, 1)
    try:
        yield
    finally:
        native.set_tune(codec, old.warps_per_cta, old.ring_slots, old.lut_bits, old.cta_per_chunk)


def test_tune_accepts_cta_mode(native):
    with cta_mode(RLEV2, 8):
        assert native.get_tune(RLEV2).cta_per_chunk == 1
    assert native.get_tune(RLEV2).cta_per_chunk == 0
    old = native.get_tune(native.DEFLATE)
    try:  # Deflate: a decoder and an expander warp per chunk, so an even warp count
        native.set_tune(native.DEFLATE, 4, 2, 9, 1)
        assert native.get_tune(native.DEFLATE).cta_per_chunk == 1
        with pytest.raises(native.CodagError):
            native.set_tune(native.DEFLATE, 3, 2, 9, 1)
    finally:
        native.set_tune(native.DEFLATE, old.warps_per_cta, old.ring_slots, old.lut_bits, old.cta_per_chunk)
    with pytest.raises(native.CodagError):
        native.set_tune(RLEV1, 8, 4, 10, 2)


def _decode(cuda, codec, comp, off, ln, e, out_bytes=None, out_shift=0):
    from codag_b200 import api
    n = ln.size
    total = n * CH if out_bytes is None else out_bytes
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a).astype(np.uint64).view(np.int64)).to("cuda")
    buf = cuda.full((total + 64 + out_shift,), 0xA5, dtype=cuda.uint8, device="cuda")
    out = buf[out_shift:]
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    fn = api.decompress_rlev1 if codec == RLEV1 else api.decompress_rlev2
    fn(cuda.from_numpy(comp).to("cuda"), t(off[:n]), t(ln), CH, e, out, total, st)
    cuda.cuda.synchronize()
    o = out.cpu().numpy()
    assert np.all(o[total:] == 0xA5), "wrote past out_bytes"
    return st.cpu().numpy(), o[:total]


def _file(codec, n_values, seed, e):
    if codec == RLEV1:
        col = native.gen_rlev1_column(n_values, seed, e)
        blob, off, ln = native.encode_rlev1(col, CH, e)
        return col, blob[8:], off, ln
    col = native.gen_rlev2_column(n_values, seed, e)
    comp, off, ln = native.encode_rlev2(col, CH, e)
    return col, comp, off, ln


@pytest.mark.gpu
@pytest.mark.parametrize("warps", [2, 8])
@pytest.mark.parametrize("e", [1, 2, 4, 8])
@pytest.mark.parametrize("codec", [RLEV1, RLEV2])
def test_cta_parity_with_oracle(cuda, oracle, codec, e, warps):
    col, comp, off, ln = _file(codec, (3 << 20) // e, 50 + e, e)
    n = ln.size
    with cta_mode(codec, warps):
        st, out = _decode(cuda, codec, comp, off, ln, e)
    assert not st.any()
    assert np.array_equal(out[:col.size], col)
    ref = np.zeros(n * CH, np.uint8)
    ost = oracle.decode_batch(comp, off[:n], ln, ref, np.arange(n) * CH, [CH] * n, [CH] * n, [codec] * n, [e] * n,
                              [0] * n)
    assert not ost.any() and np.array_equal(out, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("codec", [RLEV1, RLEV2])
def test_cta_exact_size_and_unaligned_output(cuda, codec):
    col, comp, off, ln = _file(codec, 700_001, 9, 8)
    with cta_mode(codec, 8):
        st, out = _decode(cuda, codec, comp, off, ln, 8, out_bytes=col.size)
        assert not st.any() and np.array_equal(out, col)
        st, out = _decode(cuda, codec, comp, off, ln, 8, out_bytes=col.size, out_shift=3)  # warp path
        assert not st.any() and np.array_equal(out, col)


@pytest.mark.gpu
def test_cta_fallbacks_large_stream_and_many_headers(cuda, oracle):
    rng = np.random.default_rng(3)
    # 64-bit random values: DIRECT at full width, a stream larger than the 64 KiB stage
    big = rng.integers(0, 2**63, size=3 * CH // 8, dtype=np.uint64).view(np.uint8)
    comp, off, ln = native.encode_rlev2(big, CH, 8)
    assert int(ln.max()) > 64 * 1024
    # runs of three: thousands of SHORT_REPEAT headers per chunk, over the descriptor budget
    runs = np.repeat(rng.integers(0, 1000, size=3 * CH // 24, dtype=np.uint64), 3).view(np.uint8)
    comp2, off2, ln2 = native.encode_rlev2(runs, CH, 8)
    # RLE v1 literal groups of one value each
    lit = np.arange(3 * CH // 8, dtype=np.uint64) * np.uint64(1000003)
    lit[1::2] = lit[1::2] ^ np.uint64(0x5555)
    blob, off3, ln3 = native.encode_rlev1(lit.view(np.uint8), CH, 8)
    with cta_mode(RLEV2, 8), cta_mode(RLEV1, 8):
        for codec, c, o, l, src in ((RLEV2, comp, off, ln, big), (RLEV2, comp2, off2, ln2, runs),
                                    (RLEV1, blob[8:], off3, ln3, lit.view(np.uint8))):
            st, out = _decode(cuda, codec, c, o, l, 8)
            assert not st.any()
            assert np.array_equal(out[:src.size], src)


@pytest.mark.gpu
def test_cta_malformed_streams(cuda):
    col = native.gen_rlev2_column(16384 * 4, 5, 8)
    comp, off, ln = native.encode_rlev2(col, CH, 8)
    ln = ln.copy()
    comp = comp.copy()
    ln[1] = ln[1] // 2                   # truncated stream
    comp[int(off[2])] = 0x5E             # DIRECT header asking for more bytes than the stream has
    comp[int(off[2]) + 1] = 0x7F
    ln[2] = 4
    with cta_mode(RLEV2, 8):
        st, out = _decode(cuda, RLEV2, comp, off, ln, 8)
    assert st[1] == 2 and st[2] == 2
    ok = [i for i in range(ln.size) if i not in (1, 2)]
    assert not st[ok].any()
    padded = np.zeros(ln.size * CH, np.uint8)
    padded[:col.size] = col
    for i in ok:
        assert np.array_equal(out[i * CH:(i + 1) * CH], padded[i * CH:(i + 1) * CH])
    rng = np.random.default_rng(7)
    garbage = rng.integers(0, 256, size=64 * 1024, dtype=np.uint8)
    offs = np.arange(0, 64 * 1024, 4096, dtype=np.uint64)
    lens = np.full(offs.size, 4096, np.uint64)
    with cta_mode(RLEV1, 8), cta_mode(RLEV2, 8):
        for codec in (RLEV1, RLEV2):
            st, _ = _decode(cuda, codec, garbage, offs, lens, 8, out_bytes=offs.size * CH)
            assert np.all((st == 0) | (st == 2))
