"""GPU parity: the CUDA decoders, called through the C ABI, against the CPU oracle and the
original data (bit-exact), on the three codecs, every element width, edge cases, the
reference quirks, malformed streams and every launch shape."""
import numpy as np
import pytest

from tests.vectors import VECTORS, RLEV1, RLEV2

pytestmark = pytest.mark.gpu
CH = 131072


def _bytes_of(values, e):
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[e]
    return np.array([v % (1 << (8 * e)) for v in values], dtype=np.uint64).astype(dt).view(np.uint8)


def _t(cuda, a, dtype=None):
    a = np.ascontiguousarray(a)
    if not a.flags.writeable:  # torch.from_numpy warns on read-only arrays
        a = a.copy()
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    return cuda.from_numpy(a).to("cuda")


def _gpu_rle(cuda, api, codec, comp, off, ln, chunk, e, out_bytes=None, comp_shift=0, two_pass=True, out_shift=0):
    """Decode n RLE chunks on the GPU; comp_shift moves the whole stream buffer off 16-byte alignment;
    two_pass=False decodes without a workspace (the warp walks the headers itself); out_shift
    moves the output off element alignment, which routes the values through the shared-memory
    output ring instead of straight to global memory."""
    n = ln.size
    buf = np.zeros(comp.size + comp_shift, np.uint8)
    buf[comp_shift:] = comp
    d_buf = _t(cuda, buf)
    d_comp = d_buf[comp_shift:]
    total = n * chunk if out_bytes is None else out_bytes
    out_all = cuda.full((total + 64 + out_shift,), 0xA5, dtype=cuda.uint8, device="cuda")
    out = out_all[out_shift:]
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    fn = api.decompress_rlev1 if codec == RLEV1 else api.decompress_rlev2
    kw = {"ws": api.AUTO_WORKSPACE} if two_pass else {}
    fn(d_comp, _t(cuda, off[:n]), _t(cuda, ln), chunk, e, out, total, st, **kw)
    cuda.cuda.synchronize()
    o = out.cpu().numpy()
    assert np.all(o[total:] == 0xA5), "wrote past out_bytes"
    assert np.all(out_all.cpu().numpy()[:out_shift] == 0xA5), "wrote before the output"
    return st.cpu().numpy(), o[:total]


@pytest.fixture(scope="module")
def api(native, cuda):
    from codag_b200 import api as a
    return a


# --- known-answer vectors --------------------------------------------------------------------
@pytest.mark.parametrize("two_pass", [True, False])
@pytest.mark.parametrize("name", sorted(VECTORS))
@pytest.mark.parametrize("out_shift", [0, 1])
def test_known_answer_vectors(cuda, api, name, two_pass, out_shift):
    codec, e, stream, expected = VECTORS[name]
    want = _bytes_of(expected, e)
    s = np.array(stream, np.uint8)
    st, out = _gpu_rle(cuda, api, codec, s, np.array([0], np.uint64), np.array([s.size], np.uint64), want.size, e,
                       two_pass=two_pass, out_shift=out_shift)
    assert st.tolist() == [0]
    assert np.array_equal(out, want)


# --- RLE v1 / v2 ----------------------------------------------------------------------------------
@pytest.mark.parametrize("two_pass", [True, False])
@pytest.mark.parametrize("e", [1, 2, 4, 8])
@pytest.mark.parametrize("codec", [RLEV1, RLEV2])
@pytest.mark.parametrize("out_shift", [0, 1])
def test_rle_parity(native, oracle, cuda, api, codec, e, two_pass, out_shift):
    n = (4 << 20) // e
    if codec == RLEV1:
        col = native.gen_rlev1_column(n, 31 + e, e)
        blob, off, ln = native.encode_rlev1(col, CH, e)
        comp = blob[8:]
    else:
        col = native.gen_rlev2_column(n, 37 + e, e)
        comp, off, ln = native.encode_rlev2(col, CH, e)
    nch = ln.size
    st, out = _gpu_rle(cuda, api, codec, comp, off, ln, CH, e, two_pass=two_pass, out_shift=out_shift)
    assert not st.any()
    assert np.array_equal(out[:col.size], col)
    ref = np.zeros(nch * CH, np.uint8)
    ost = oracle.decode_batch(comp, off[:nch], ln, ref, np.arange(nch) * CH, [CH] * nch, [CH] * nch,
                              [codec] * nch, [e] * nch, [0] * nch)
    assert not ost.any()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("codec", [RLEV1, RLEV2])
def test_rle_exact_size_output_and_unaligned_base(native, cuda, api, codec):
    """out_bytes = original size (last chunk clipped); stream buffer 8 bytes off 16-byte
    alignment (the blob+8 pointer of CODAG's RLE v1 layout)."""
    col = (native.gen_rlev1_column if codec == RLEV1 else native.gen_rlev2_column)(700_001, 9, 8)
    comp, off, ln = (native.encode_rlev1 if codec == RLEV1 else native.encode_rlev2)(col, CH, 8)
    if codec == RLEV1:
        comp = comp[8:]
    st, out = _gpu_rle(cuda, api, codec, comp, off, ln, CH, 8, out_bytes=col.size, comp_shift=8)
    assert not st.any()
    assert np.array_equal(out, col)


@pytest.mark.parametrize("cut", [1, 3, 7])
@pytest.mark.parametrize("codec", [RLEV1, RLEV2])
def test_rle_output_size_not_a_multiple_of_the_element(native, cuda, api, codec, cut):
    """out_bytes ending inside an 8-byte element: the bytes up to out_bytes are stored and
    nothing after them (the helper checks the guard bytes)."""
    col = (native.gen_rlev1_column if codec == RLEV1 else native.gen_rlev2_column)(300_000, 19, 8)
    comp, off, ln = (native.encode_rlev1 if codec == RLEV1 else native.encode_rlev2)(col, CH, 8)
    if codec == RLEV1:
        comp = comp[8:]
    size = col.size - cut
    st, out = _gpu_rle(cuda, api, codec, comp, off, ln, CH, 8, out_bytes=size)
    assert not st.any()
    assert np.array_equal(out, col[:size])


def test_rle_odd_chunk_sizes(native, oracle, cuda, api):
    """Chunk sizes that are not multiples of 16 take the unaligned drain path."""
    for chunk, e in ((4104, 8), (1000, 4), (998, 2), (777, 1)):
        col = native.gen_rlev2_column(chunk // e * 5, 3, e)
        comp, off, ln = native.encode_rlev2(col, chunk, e)
        st, out = _gpu_rle(cuda, api, RLEV2, comp, off, ln, chunk, e)
        assert not st.any()
        assert np.array_equal(out[:col.size], col)
        col1 = native.gen_rlev1_column(chunk // e * 5, 4, e)
        blob, off1, ln1 = native.encode_rlev1(col1, chunk, e)
        st1, out1 = _gpu_rle(cuda, api, RLEV1, blob[8:], off1, ln1, chunk, e)
        assert not st1.any()
        assert np.array_equal(out1[:col1.size], col1)


@pytest.mark.parametrize("two_pass", [True, False])
def test_rle_malformed_streams(native, cuda, api, two_pass):
    """Malformed chunks report ECORRUPT; their neighbours still decode; nothing faults."""
    col = native.gen_rlev2_column(16384 * 4, 5, 8)
    comp, off, ln = native.encode_rlev2(col, CH, 8)
    ln = ln.copy()
    comp = comp.copy()
    ln[1] = ln[1] // 2                   # truncated stream
    comp[int(off[2])] = 0x5E             # DIRECT header: 128 16-bit values, more than the stream has
    comp[int(off[2]) + 1] = 0x7F
    ln[2] = 4
    st, out = _gpu_rle(cuda, api, RLEV2, comp, off, ln, CH, 8, two_pass=two_pass)
    assert st[1] == 2 and st[2] == 2
    ok = [i for i in range(ln.size) if i not in (1, 2)]
    assert not st[ok].any()
    padded = np.zeros(ln.size * CH, np.uint8)  # chunks past the column hold the layout's zero padding
    padded[:col.size] = col
    for i in ok:
        assert np.array_equal(out[i * CH:(i + 1) * CH], padded[i * CH:(i + 1) * CH])
    # RLE v1: random garbage bytes never fault and never write past their chunk
    rng = np.random.default_rng(7)
    garbage = rng.integers(0, 256, size=64 * 1024, dtype=np.uint8)
    offs = np.arange(0, 64 * 1024, 4096, dtype=np.uint64)
    lens = np.full(offs.size, 4096, np.uint64)
    st1, _ = _gpu_rle(cuda, api, RLEV1, garbage, offs, lens, 2048, 8, two_pass=two_pass)
    st2, _ = _gpu_rle(cuda, api, RLEV2, garbage, offs, lens, 2048, 8, two_pass=two_pass)
    assert set(st1.tolist()) <= {0, 2} and set(st2.tolist()) <= {0, 2}


def test_rle_stream_out_of_bounds(native, cuda, api):
    col = native.gen_rlev2_column(16384 * 2, 5, 8)
    comp, off, ln = native.encode_rlev2(col, CH, 8)
    off = off.copy()
    off[1] = comp.size + 100  # beyond comp_bytes
    st, _ = _gpu_rle(cuda, api, RLEV2, comp, off, ln, CH, 8)
    assert st[1] == 2 and not np.delete(st, 1).any()


# --- Deflate -------------------------------------------------------------------------------------
def _gpu_deflate(cuda, api, comp, rel, chunk, out_bytes=None, wrapper=2):
    n = rel.size - 1
    total = n * chunk if out_bytes is None else out_bytes
    out = cuda.full((total + 64,), 0xA5, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_deflate(_t(cuda, comp), _t(cuda, rel), chunk, out, wrapper, total, st)
    cuda.cuda.synchronize()
    o = out.cpu().numpy()
    assert np.all(o[total:] == 0xA5)
    return st.cpu().numpy(), o[:total]


def test_deflate_parity(native, oracle, cuda, api):
    txt = native.gen_text(64 * CH + 999, 17)
    comp, bo, cl = native.encode_deflate(txt, CH, 6)
    st, out = _gpu_deflate(cuda, api, comp, bo[1:], CH, out_bytes=txt.size)
    assert not st.any()
    assert np.array_equal(out, txt)
    # and against the oracle, chunk by chunk
    rel = bo[1:]
    for i in (0, 17, rel.size - 2):
        ost, ref = oracle.deflate_chunk(comp[int(rel[i]):int(rel[i + 1])], CH)
        assert ost == 0
        n = min(CH, txt.size - i * CH)
        assert np.array_equal(out[i * CH:i * CH + n], ref[:n])


@pytest.mark.parametrize("level,strategy", [(0, 0), (1, 0), (9, 0), (6, 4), (6, 2), (6, 3)])
def test_deflate_block_kinds(native, oracle, cuda, api, level, strategy):
    """Stored (level 0), fixed (Z_FIXED=4), Huffman-only (2), RLE (3) and dynamic streams;
    zlib and raw wrappers; data of mixed compressibility."""
    import zlib
    rng = np.random.default_rng(level * 10 + strategy)
    parts = [native.gen_text(50_000, 5), rng.integers(0, 256, 30_000, dtype=np.uint8),
             np.zeros(20_000, np.uint8), np.tile(np.arange(7, dtype=np.uint8), 4000)]
    data = np.concatenate(parts)[:CH]
    for wrapper in (2, 0):
        co = zlib.compressobj(level, zlib.DEFLATED, 15 if wrapper else -15, 8, strategy)
        s = np.frombuffer(co.compress(data.tobytes()) + co.flush(), np.uint8)
        rel = np.array([0, s.size], np.uint64)
        st, out = _gpu_deflate(cuda, api, s, rel, data.size, wrapper=wrapper)
        assert st.tolist() == [0]
        assert np.array_equal(out, data)


def test_deflate_malformed(native, cuda, api):
    txt = native.gen_text(8 * CH, 23)
    comp, bo, cl = native.encode_deflate(txt, CH, 6)
    comp = comp.copy()
    rel = bo[1:].copy()
    comp[int(rel[3]) + 2] = 0xFF            # block type 3 (reserved)
    comp[int(rel[5]) + 40:int(rel[5]) + 60] = 0x00  # damaged Huffman data
    rel6 = rel.copy()
    st, out = _gpu_deflate(cuda, api, comp, rel6, CH)
    assert st[3] == 2
    assert st[5] in (0, 2)
    for i in (0, 1, 2, 4, 6, 7):
        assert st[i] == 0
        assert np.array_equal(out[i * CH:(i + 1) * CH], txt[i * CH:(i + 1) * CH])
    rng = np.random.default_rng(3)
    garbage = rng.integers(0, 256, 256 * 1024, dtype=np.uint8)
    st2, _ = _gpu_deflate(cuda, api, garbage, np.arange(0, 256 * 1024 + 1, 4096, dtype=np.uint64), 8192)
    assert set(st2.tolist()) <= {0, 2}


# --- launch shapes ------------------------------------------------------------------------------
@pytest.mark.parametrize("warps,slots,lut", [(1, 4, 9), (4, 8, 11), (8, 4, 10), (2, 8, 10)])
def test_launch_shapes(native, cuda, api, warps, slots, lut):
    from codag_b200 import native as nat
    saved = [nat.get_tune(c) for c in (0, 1, 2)]
    try:
        for c in (0, 1, 2):
            nat.set_tune(c, warps, slots, lut)
        col = native.gen_rlev2_column(16384 * 9, 41, 8)
        comp, off, ln = native.encode_rlev2(col, CH, 8)
        st, out = _gpu_rle(cuda, api, RLEV2, comp, off, ln, CH, 8)
        assert not st.any() and np.array_equal(out[:col.size], col)
        col1 = native.gen_rlev1_column(16384 * 9, 43, 8)
        blob, off1, ln1 = native.encode_rlev1(col1, CH, 8)
        st1, out1 = _gpu_rle(cuda, api, RLEV1, blob[8:], off1, ln1, CH, 8)
        assert not st1.any() and np.array_equal(out1[:col1.size], col1)
        txt = native.gen_text(9 * CH, 47)
        comp2, bo, _ = native.encode_deflate(txt, CH, 6)
        st2, out2 = _gpu_deflate(cuda, api, comp2, bo[1:], CH)
        assert not st2.any() and np.array_equal(out2[:txt.size], txt)
    finally:
        for c, t in zip((0, 1, 2), saved):
            nat.set_tune(c, t.warps_per_cta, t.ring_slots, t.lut_bits)


def test_deflate_two_slot_ring(native, cuda, api):
    from codag_b200 import native as nat
    saved = nat.get_tune(2)
    try:
        nat.set_tune(2, 4, 2, 10)
        txt = native.gen_text(5 * CH, 53)
        comp, bo, _ = native.encode_deflate(txt, CH, 1)
        st, out = _gpu_deflate(cuda, api, comp, bo[1:], CH)
        assert not st.any() and np.array_equal(out[:txt.size], txt)
    finally:
        nat.set_tune(2, saved.warps_per_cta, saved.ring_slots, saved.lut_bits)


# --- bounded waits --------------------------------------------------------------------------------
def test_wait_timeout_returns_status(cuda, api):
    """A TMA barrier that nothing completes: the bounded wait gives up and reports ETIMEOUT;
    the context stays usable afterwards."""
    from codag_b200 import native as nat
    assert api.selftest_wait_timeout(2_000_000) == nat.ETIMEOUT
    x = cuda.arange(10, device="cuda").sum().item()
    assert x == 45


# --- full-size configuration: property test (decoded == original) --------------------------------
def test_full_size_rlev2_1gib(native, cuda, api):
    """CODAG's RLE v2 configuration at full size: 134,217,728 int64 (1 GiB), 8192 chunks."""
    n = 134_217_728
    col = native.gen_rlev2_column(n, 20260102, 8)
    comp, off, ln = native.encode_rlev2(col, CH, 8)
    d_col = _t(cuda, col)
    out = cuda.empty(col.size, dtype=cuda.uint8, device="cuda")
    st = cuda.full((ln.size,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_rlev2(_t(cuda, comp), _t(cuda, off[:ln.size]), _t(cuda, ln), CH, 8, out, col.size, st)
    cuda.cuda.synchronize()
    assert int((st != 0).sum().item()) == 0
    assert bool(cuda.equal(out, d_col))
