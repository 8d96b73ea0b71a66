"""Deflate chunks with adversarial back-references, written by Python's zlib with random
levels, strategies, window sizes and memory levels: periodic data whose period straddles the
decoder's shared-memory windows (1 KiB with a 9-bit literal table, 2 KiB with 10 or 11 bits) or
reaches the 32 KiB maximum distance, byte runs (distance-1, length-258 copies), short periods
(overlapping copies), incompressible bytes (stored blocks) and mixtures of them.

CPU: the oracle must decode every chunk to its source.  GPU: one launch over all chunks must
match the source byte for byte, with every chunk's status OK."""
import zlib

import numpy as np
import pytest

CH = 131072
PERIODS = [1, 2, 3, 5, 31, 255, 256, 257, 1023, 1024, 1025, 2047, 2048, 2049, 4095, 4096, 4097, 8191, 16384,
           32767, 32768]


def _chunk(rng: np.random.Generator, kind: int) -> np.ndarray:
    if kind == 0:  # one period over the whole chunk
        p = int(rng.choice(PERIODS))
        return np.resize(rng.integers(0, 256, p, dtype=np.uint8), CH)
    if kind == 1:  # incompressible
        return rng.integers(0, 256, CH, dtype=np.uint8)
    # segments of runs, periods and noise; periods repeat a block seen earlier in the chunk
    out = np.empty(CH, np.uint8)
    i = 0
    while i < CH:
        n = min(CH - i, int(rng.integers(1, 20000)))
        t = int(rng.integers(0, 4))
        if t == 0:
            out[i:i + n] = rng.integers(0, 256, dtype=np.uint8)
        elif t == 1:
            out[i:i + n] = rng.integers(0, 256, n, dtype=np.uint8)
        elif t == 2 and i >= 4097:
            d = int(rng.choice([1023, 1024, 1025, 2047, 2048, 4095, 4096, 4097, min(i, 32768)]))
            k = 0
            while k < n:  # a copy at distance d (repeating itself when n > d)
                m = min(d, n - k)
                out[i + k:i + k + m] = out[i + k - d:i + k - d + m]
                k += m
        else:
            p = int(rng.choice(PERIODS[:8]))
            out[i:i + n] = np.resize(rng.integers(0, 256, p, dtype=np.uint8), n)
        i += n
    return out


def _streams(seed: int, n: int):
    """n chunks of CH bytes, zlib-wrapped, each padded to 8 bytes: (comp, rel offsets, source)."""
    rng = np.random.default_rng(seed)
    parts, rel, src = [], [0], []
    for c in range(n):
        data = _chunk(rng, c % 3)
        level = int(rng.integers(0, 10))
        strategy = int(rng.choice([0, 1, 2, 3, 4]))
        wbits = int(rng.integers(9, 16))
        mem = int(rng.integers(1, 10))
        co = zlib.compressobj(level, zlib.DEFLATED, wbits, mem, strategy)
        s = co.compress(data.tobytes()) + co.flush()
        s += b"\0" * ((-len(s)) % 8)
        parts.append(s)
        rel.append(rel[-1] + len(s))
        src.append(data)
    return np.frombuffer(b"".join(parts), np.uint8).copy(), np.array(rel, np.uint64), np.concatenate(src)


def test_oracle_decodes_adversarial_chunks(oracle):
    comp, rel, src = _streams(1, 12)
    for i in range(rel.size - 1):
        st, out = oracle.deflate_chunk(comp[int(rel[i]):int(rel[i + 1])], CH)
        assert st == 0, i
        assert np.array_equal(out[:CH], src[i * CH:(i + 1) * CH]), i


@pytest.mark.gpu
@pytest.mark.parametrize("cta", [(0, None), (1, 2), (1, 8)], ids=["warp", "cta_1pair", "cta_4pairs"])
@pytest.mark.parametrize("lut", [9, 10, 11])  # 9 bits: 1 KiB window; 10 and 11: 2 KiB
@pytest.mark.parametrize("seed", [2, 3])
def test_gpu_decodes_adversarial_chunks(cuda, native, seed, lut, cta):
    """One warp per chunk, or a decoder and an expander warp per chunk (cta_per_chunk)."""
    from codag_b200 import api
    comp, rel, src = _streams(seed, 36)
    n = rel.size - 1
    d_comp = cuda.from_numpy(comp).to("cuda")
    d_rel = cuda.from_numpy(rel.view(np.int64)).to("cuda")
    out = cuda.full((n * CH + 64,), 0xA5, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    old = native.get_tune(native.DEFLATE)
    native.set_tune(native.DEFLATE, cta[1] or old.warps_per_cta, old.ring_slots, lut, cta[0])
    try:
        api.decompress_deflate(d_comp, d_rel, CH, out, 2, n * CH, st)
        cuda.cuda.synchronize()
    finally:
        native.set_tune(native.DEFLATE, old.warps_per_cta, old.ring_slots, old.lut_bits)
    o = out.cpu().numpy()
    assert st.cpu().numpy().tolist() == [0] * n
    assert np.all(o[n * CH:] == 0xA5)
    bad = np.flatnonzero(o[:n * CH] != src)
    assert bad.size == 0, (int(bad[0]) // CH, int(bad[0]) % CH)


@pytest.mark.gpu
def test_batch_kernel_decodes_adversarial_chunks(cuda, native):
    """The same streams through the batched persistent launch."""
    from codag_b200 import api
    comp, rel, src = _streams(4, 24)
    n = rel.size - 1
    streams = [comp[int(rel[i]):int(rel[i + 1])] for i in range(n)]
    cs = api.pack_chunks(streams, [native.DEFLATE] * n, [1] * n, [CH] * n)
    plan = api.BatchPlan(cs.descs)
    try:
        out = cuda.zeros(cs.out_bytes, dtype=cuda.uint8, device="cuda")
        st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
        plan.run(cuda.from_numpy(cs.comp).to("cuda"), out, st)
        cuda.cuda.synchronize()
    finally:
        plan.close()
    assert st.cpu().numpy().tolist() == [0] * n
    o = out.cpu().numpy()
    for i in range(n):
        a = int(cs.descs[i]["out_off"])
        assert np.array_equal(o[a:a + CH], src[i * CH:(i + 1) * CH]), i


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [5, 6])
def test_cta_per_chunk_matches_one_warp_on_damaged_streams(cuda, native, seed):
    """Streams with bytes flipped: the decoder/expander pair reports the same status per chunk
    as the one-warp decoder, and the same bytes wherever that status is OK."""
    from codag_b200 import api
    comp, rel, src = _streams(seed, 24)
    rng = np.random.default_rng(seed)
    n = rel.size - 1
    bad = comp.copy()
    for i in range(n):  # flip a few bytes inside most chunks
        lo, hi = int(rel[i]) + 2, int(rel[i + 1])
        if i % 3 and hi > lo:
            for p in rng.integers(lo, hi, 3):
                bad[p] ^= np.uint8(rng.integers(1, 256))
    d_comp = cuda.from_numpy(bad).to("cuda")
    d_rel = cuda.from_numpy(rel.view(np.int64)).to("cuda")
    old = native.get_tune(native.DEFLATE)
    res = []
    try:
        for warps, cta in ((old.warps_per_cta, 0), (4, 1)):
            native.set_tune(native.DEFLATE, warps, old.ring_slots, old.lut_bits, cta)
            out = cuda.zeros(n * CH, dtype=cuda.uint8, device="cuda")
            st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
            api.decompress_deflate(d_comp, d_rel, CH, out, 2, n * CH, st)
            cuda.cuda.synchronize()
            res.append((st.cpu().numpy(), out.cpu().numpy()))
    finally:
        native.set_tune(native.DEFLATE, old.warps_per_cta, old.ring_slots, old.lut_bits, old.cta_per_chunk)
    (s1, o1), (s2, o2) = res
    assert np.array_equal(s1, s2)
    assert (s1 != 0).any() and (s1 == 0).any()
    for i in np.flatnonzero(s1 == 0):
        assert np.array_equal(o1[i * CH:(i + 1) * CH], o2[i * CH:(i + 1) * CH]), i
