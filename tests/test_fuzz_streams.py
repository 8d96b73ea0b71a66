"""Random RLE streams written header by header from the format definition (tests/fuzz_streams.py),
so the decoders meet header forms this project's encoders never emit: every DIRECT and packed
DELTA width, varints of every length, zero and negative deltas, 1-value literal groups.

CPU: the oracle must reproduce the model's values.  GPU: the one-pass warp decoder, the
CTA-per-chunk decoder, the two-pass decoder with a workspace and the shared-memory ring path
(an output that is not element aligned) must all reproduce them too, byte for byte."""
import contextlib

import numpy as np
import pytest

from tests import fuzz_streams as fz

CODECS = {"rlev1": 0, "rlev2": 1}


@pytest.mark.parametrize("elem", [1, 2, 4, 8])
@pytest.mark.parametrize("codec", ["rlev1", "rlev2"])
def test_oracle_matches_stream_model(oracle, codec, elem):
    cb = 4096
    comp, off, ln, want = fz.chunk_set(codec, 24, cb, elem, seed=1000 + 10 * elem + CODECS[codec])
    n = ln.size
    got = np.zeros(n * cb, np.uint8)
    st = oracle.decode_batch(comp, off, ln, got, np.arange(n) * cb, [cb] * n, [cb] * n, [CODECS[codec]] * n,
                             [elem] * n, [0] * n)
    assert not st.any()
    assert np.array_equal(got, want)


def test_model_covers_every_width_code():
    seen = set()
    rng = np.random.default_rng(5)
    for _ in range(24):
        s, _ = fz.rlev2_chunk(rng, 4096, 8)
        # walk the headers to collect the width codes of DIRECT and DELTA
        p = 0
        while p < len(s):
            h = s[p]
            if h >> 6 == 0:
                p += 1 + ((h >> 3) & 7) + 1
                continue
            code, cnt = (h >> 1) & 31, (((h & 1) << 8) | s[p + 1]) + 1
            seen.add((h >> 6, code))
            p += 2
            if h >> 6 == 1:
                p += (cnt * fz.WIDTHS[code] + 7) // 8
            else:
                for _v in range(2):
                    while s[p] & 0x80:
                        p += 1
                    p += 1
                if code:
                    p += ((cnt - 2) * fz.WIDTHS[code] + 7) // 8
    assert {c for k, c in seen if k == 1} == set(range(32))
    assert {c for k, c in seen if k == 3} == set(range(32))


@contextlib.contextmanager
def _tune(native, codec, cta):
    old = native.get_tune(codec)
    native.set_tune(codec, old.warps_per_cta, old.ring_slots, old.lut_bits, cta)
    try:
        yield
    finally:
        native.set_tune(codec, old.warps_per_cta, old.ring_slots, old.lut_bits, old.cta_per_chunk)


@pytest.mark.gpu
@pytest.mark.parametrize("cb", [16384, 131072])
@pytest.mark.parametrize("elem", [1, 2, 4, 8])
@pytest.mark.parametrize("codec", ["rlev1", "rlev2"])
def test_gpu_paths_match_stream_model(cuda, native, codec, elem, cb):
    from codag_b200 import api
    n = 40 if cb == 16384 else 6
    comp, off, ln, want = fz.chunk_set(codec, n, cb, elem, seed=2000 + 10 * elem + CODECS[codec] + cb)
    total = n * cb
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).to("cuda")
    d_comp, d_off, d_len = cuda.from_numpy(comp).to("cuda"), t(off), t(ln)
    fn = api.decompress_rlev1 if codec == "rlev1" else api.decompress_rlev2
    cid = CODECS[codec]
    modes = [("warp", 0, None, 0), ("cta", 1, None, 0), ("two-pass", 0, api.AUTO_WORKSPACE, 0), ("ring", 0, None, 3)]
    for name, cta, ws, shift in modes:
        buf = cuda.full((total + 64 + shift,), 0xA5, dtype=cuda.uint8, device="cuda")
        out = buf[shift:]
        st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
        with _tune(native, cid, cta):
            fn(d_comp, d_off, d_len, cb, elem, out, total, st, ws=ws)
        cuda.cuda.synchronize()
        o = out.cpu().numpy()
        s = st.cpu().numpy()
        assert not s.any(), (name, s)
        assert np.all(o[total:] == 0xA5), name
        bad = np.flatnonzero(o[:total] != want)
        assert bad.size == 0, (name, int(bad[0]) // cb, int(bad[0]) % cb)
