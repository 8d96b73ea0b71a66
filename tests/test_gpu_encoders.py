"""GPU encoders (codag_compress_rlev1/_rlev2): the files they write equal, byte for byte, the
host producers' (codag_encode_rlev1/_rlev2, whose RLE v2 bytes are pinned to CODAG's own
encoder by tests/test_golden_rlev2.py), for every element width, for inputs whose size is not
a multiple of the element or the chunk, and for CODAG-written columns; and they decode back
through the CUDA decoders."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
CH = 131072


def _columns(native, codec, e):
    gen = native.gen_rlev1_column if codec == native.RLEV1 else native.gen_rlev2_column
    rng = np.random.default_rng(e)
    yield gen(3 * CH // e + 5, 300 + e, e)[: 3 * CH + 3]           # ragged: 3 bytes past an element
    yield gen(CH // e, 400 + e, e)                                    # exactly one chunk
    yield rng.integers(0, 256, 2 * CH + 77, dtype=np.uint8)           # random bytes
    yield np.zeros(CH + 16, np.uint8)                                 # long zero runs
    # runs around the 130-value run limit and literal bursts around the 127-literal group limit
    parts = []
    for k, ln in enumerate([128, 129, 130, 131, 260, 126, 127, 128, 254, 255, 3, 1, 2]):
        if k < 5:
            parts.append((np.arange(ln, dtype=np.uint64) * 3 + 1000 * k))
        else:
            parts.append(rng.integers(0, 1 << 62, ln, dtype=np.uint64) * 509)
    vals = np.concatenate(parts * 8)
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[e]
    yield vals.astype(dt).view(np.uint8)


@pytest.mark.parametrize("codec", [0, 1], ids=["rlev1", "rlev2"])
@pytest.mark.parametrize("e", [1, 2, 4, 8])
def test_gpu_encoder_matches_host_producer(cuda, native, codec, e):
    from codag_b200 import api
    for col in _columns(native, codec, e):
        raw = np.ascontiguousarray(col).view(np.uint8)
        if codec == native.RLEV1:
            want, w_off, w_len = native.encode_rlev1(raw, CH, e)
        else:
            want, w_off, w_len = native.encode_rlev2(raw, CH, e)
        f, off, ln = api.compress_rle(codec, cuda.from_numpy(raw.copy()).to("cuda"), CH, e)
        assert np.array_equal(off.cpu().numpy().view(np.uint64), w_off)
        assert np.array_equal(ln.cpu().numpy().view(np.uint64), w_len)
        assert np.array_equal(f.cpu().numpy(), want), (codec, e, raw.size)


GOLDEN = sorted(p.stem for p in (Path(__file__).parent / "golden").glob("ref_rlev2_*.npz") if p.stem != "ref_rlev2_tables")


@pytest.mark.parametrize("name", GOLDEN)
def test_gpu_rlev2_encoder_on_codag_columns(cuda, native, name):
    """The columns of CODAG's golden RLE v2 files (every header kind, patches wider than 32 bits,
    runs of zeros, every element width): one warp per chunk writes the host producer's bytes."""
    from codag_b200 import api
    g = np.load(Path(__file__).parent / "golden" / f"{name}.npz")
    e = int(g["elem"])
    raw = np.ascontiguousarray(g["src"]).view(np.uint8)
    want, w_off, w_len = native.encode_rlev2(raw, CH, e)
    f, off, ln = api.compress_rle(native.RLEV2, cuda.from_numpy(raw.copy()).to("cuda"), CH, e)
    assert np.array_equal(ln.cpu().numpy().view(np.uint64), w_len)
    assert np.array_equal(off.cpu().numpy().view(np.uint64), w_off)
    assert np.array_equal(f.cpu().numpy(), want), name


@pytest.mark.parametrize("codec", [0, 1], ids=["rlev1", "rlev2"])
def test_gpu_encoder_round_trip(cuda, native, codec):
    from codag_b200 import api
    col = (native.gen_rlev1_column if codec == native.RLEV1 else native.gen_rlev2_column)(64 * CH // 8, 77, 8)
    d_col = cuda.from_numpy(col.copy()).to("cuda")
    f, off, ln = api.compress_rle(codec, d_col, CH, 8)
    n = ln.numel()
    out = cuda.empty(col.size, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    if codec == native.RLEV1:
        api.decompress_rlev1(f[8:], off[:n], ln, CH, 8, out, col.size, st)
    else:
        api.decompress_rlev2(f, off[:n], ln, CH, 8, out, col.size, st)
    cuda.cuda.synchronize()
    assert int((st != 0).sum().item()) == 0 and bool(cuda.equal(out, d_col))


def test_gpu_encoder_reports_small_capacity(cuda, native):
    from codag_b200 import native as nat
    lib = nat.lib()
    col = cuda.from_numpy(native.gen_rlev2_column(CH // 8, 5, 8).copy()).to("cuda")
    n = int(lib.codag_compress_chunks(col.numel(), CH))
    need = int(lib.codag_compress_workspace_bytes(nat.RLEV2, col.numel(), CH, 8))
    ws = cuda.empty(need, dtype=cuda.uint8, device="cuda")
    out = cuda.empty(64, dtype=cuda.uint8, device="cuda")
    off = cuda.empty(n + 1, dtype=cuda.int64, device="cuda")
    ln = cuda.empty(n, dtype=cuda.int64, device="cuda")
    meta = cuda.zeros(2, dtype=cuda.int64, device="cuda")
    rc = lib.codag_compress_rlev2(col.data_ptr(), col.numel(), CH, 8, out.data_ptr(), 64, off.data_ptr(), ln.data_ptr(),
                                  meta.data_ptr(), meta.data_ptr() + 8, ws.data_ptr(), need, None)
    assert rc == nat.OK
    cuda.cuda.synchronize()
    assert int(meta[1].item()) == nat.ELIMIT and int(meta[0].item()) > 64
    # argument checks without a launch
    assert lib.codag_compress_rlev2(col.data_ptr(), col.numel(), CH, 3, out.data_ptr(), 64, off.data_ptr(),
                                    ln.data_ptr(), None, None, ws.data_ptr(), need, None) == nat.EINVAL
    assert lib.codag_compress_rlev2(col.data_ptr(), col.numel(), CH, 8, out.data_ptr(), 64, off.data_ptr(),
                                    ln.data_ptr(), None, None, ws.data_ptr(), 16, None) == nat.EINVAL
