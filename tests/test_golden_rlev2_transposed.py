"""CODAG's transposed RLE v2 layout (include/rlev2/encoder_trans.h:8-182, 359-391): 32 substreams
per chunk, interleaved in 4-byte words.  tests/golden/ref_rlev2t_*.npz hold files written by
CODAG's own encoder kernels (block_encode / tranpose_col_len_single run on the host,
tests/golden/make_ref_rlev2.py) for seeded columns.  The format library must write the same
bytes (but for the zero-run header, tests/test_golden_rlev2.py), the oracle must decode every
substream to its values, and codag_decompress_rlev2_transposed must decode the files on the GPU
as the oracle does."""
from pathlib import Path

import numpy as np
import pytest

from tests.rlev2_walk import detranspose, interleave_values, walk

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem[len("ref_rlev2t_"):] for p in GOLDEN.glob("ref_rlev2t_*.npz"))
CH = 131072


def _load(name):
    d = np.load(GOLDEN / f"ref_rlev2t_{name}.npz")
    return {k: d[k] for k in d.files}


def _padded(g):
    n = g["blk_off"].size - 1
    out = np.zeros(n * CH, np.uint8)
    out[:g["src"].size] = g["src"]
    return out


def _subs(g, c):
    region = g["comp"][int(g["blk_off"][c]):]
    return detranspose(region, g["col_len"][32 * c:32 * c + 32])


def _oracle_chunk(oracle, g, c):
    """(status, chunk bytes) from the oracle decoding the 32 substreams of chunk c."""
    e, ru = int(g["elem"]), int(g["read_unit"])
    per = CH // e // 32
    vals, bad = [], 0
    for s in _subs(g, c):
        st, v = oracle.rlev2_chunk(np.frombuffer(s, np.uint8), per * e, e)
        bad |= st
        vals.append(v.tobytes())
    return bad, np.frombuffer(interleave_values(vals, ru, e), np.uint8)


def _quirky(g, c):
    return any(w["zero_run"] or w["wide_patch"] for w in map(walk, _subs(g, c)))


def test_golden_files_present():
    assert CASES == ["c2_u64_ru4", "mix_u16_ru2", "mix_u32_ru8", "mix_u8_ru1"]


@pytest.mark.parametrize("name", CASES)
def test_writer_matches_codag_encoder(native, name):
    g = _load(name)
    e, ru = int(g["elem"]), int(g["read_unit"])
    comp, off, ln = native.encode_rlev2_transposed(g["src"], CH, e, ru)
    assert np.array_equal(off, g["blk_off"]) and np.array_equal(ln, g["col_len"])
    diff = np.nonzero(comp != g["comp"])[0]
    a, b = g["comp"], comp
    # only the zero-run DIRECT headers differ: CODAG (0x41|code<<1, 0xff), ours (0x40|code<<1, 0x7f)
    assert all((a[p] == (b[p] | 1) and (b[p] & 0xc1) == 0x40) or (a[p] == 0xff and b[p] == 0x7f) for p in diff)


@pytest.mark.parametrize("name", CASES)
def test_oracle_decodes_codag_files(oracle, name):
    g = _load(name)
    src = _padded(g)
    n = g["blk_off"].size - 1
    clean = [c for c in range(n) if not _quirky(g, c)]
    assert clean
    for c in clean:
        st, got = _oracle_chunk(oracle, g, c)
        assert st == 0 and np.array_equal(got, src[c * CH:(c + 1) * CH]), c


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cuda_decoder_decodes_codag_files(cuda, oracle, name):
    from codag_b200 import api
    g = _load(name)
    e, ru = int(g["elem"]), int(g["read_unit"])
    n = g["blk_off"].size - 1
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a).astype(np.uint64).view(np.int64)).to("cuda")
    out = cuda.zeros(n * CH, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_rlev2_transposed(cuda.from_numpy(g["comp"].copy()).to("cuda"), t(g["blk_off"][:n]),
                                    t(g["col_len"]), CH, e, ru, out, None, st)
    cuda.cuda.synchronize()
    got, gst = out.cpu().numpy(), st.cpu().numpy()
    src = _padded(g)
    for c in range(n):
        ost, want = _oracle_chunk(oracle, g, c)
        assert (gst[c] == 0) == (ost == 0), c
        if ost == 0:
            assert np.array_equal(got[c * CH:(c + 1) * CH], want), c
        if not _quirky(g, c):
            assert gst[c] == 0 and np.array_equal(got[c * CH:(c + 1) * CH], src[c * CH:(c + 1) * CH]), c


@pytest.mark.gpu
@pytest.mark.parametrize("e,ru", [(8, 1), (8, 8), (4, 4), (2, 16), (1, 32)])
def test_cuda_round_trip_of_writer(cuda, native, e, ru):
    """The format library's transposed files (no zero runs of 128) decode to the column,
    with an output size that ends inside the last chunk."""
    from codag_b200 import api
    col = native.gen_rlev2_column(40 * CH // e + 123, 500 + e, e)
    comp, off, ln = native.encode_rlev2_transposed(col, CH, e, ru)
    n = off.size - 1
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a).astype(np.uint64).view(np.int64)).to("cuda")
    out = cuda.zeros(n * CH, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_rlev2_transposed(cuda.from_numpy(comp).to("cuda"), t(off[:n]), t(ln), CH, e, ru, out, col.size, st)
    cuda.cuda.synchronize()
    ok = st.cpu().numpy() == 0
    got = out.cpu().numpy()[:col.size]
    # the last chunk is mostly zero padding, whose runs of 128 zeros CODAG's decoder misreads
    assert ok[:n - 1].all()
    for c in np.nonzero(ok)[0]:
        hi = min((c + 1) * CH, col.size)
        assert np.array_equal(got[c * CH:hi], col[c * CH:hi]), c


def _damaged(native, seed):
    """A writer's file of 8 int64 chunks, damaged: a byte flipped in chunks 1, 3 and 5, a
    substream cut by 3 bytes in chunk 2, one emptied in chunk 6, and chunk 7 claiming a
    substream far longer than the file (chunks 0 and 4 intact)."""
    col = native.gen_rlev2_column(8 * CH // 8, seed, 8)
    comp, off, ln = native.encode_rlev2_transposed(col, CH, 8, 1)
    comp, ln = comp.copy(), ln.astype(np.uint64).copy()
    rng = np.random.default_rng(seed)
    for c in (1, 3, 5):
        at = int(off[c]) + int(rng.integers(0, int(off[c + 1] - off[c])))
        comp[at] ^= np.uint8(1 << int(rng.integers(0, 8)))
    ln[32 * 2 + 5] -= 3
    ln[32 * 6 + 17] = 0
    ln[32 * 7 + 9] = 1 << 40
    return col, {"comp": comp, "blk_off": off, "col_len": ln, "elem": 8, "read_unit": 1}


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [41, 42, 43])
def test_cuda_decoder_on_damaged_files(cuda, native, oracle, seed):
    """Damaged chunks decode as the oracle decodes them: a chunk the kernel passes, the oracle
    passes with the same bytes, a chunk the oracle rejects the kernel rejects, a substream
    longer than the file is ECORRUPT, and the intact chunks still decode to the column."""
    from codag_b200 import api
    col, g = _damaged(native, seed)
    n = 8
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a).astype(np.uint64).view(np.int64)).to("cuda")
    out = cuda.zeros(n * CH, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_rlev2_transposed(cuda.from_numpy(g["comp"]).to("cuda"), t(g["blk_off"][:n]), t(g["col_len"]),
                                    CH, 8, 1, out, col.nbytes, st)
    cuda.cuda.synchronize()
    got, gst = out.cpu().numpy(), st.cpu().numpy()
    src = col.view(np.uint8)
    for c in (0, 4):
        assert gst[c] == 0 and np.array_equal(got[c * CH:(c + 1) * CH], src[c * CH:(c + 1) * CH]), c
    assert gst[7] == 2  # CODAG_ECORRUPT
    for c in range(7):
        ost, want = _oracle_chunk(oracle, g, c)
        if gst[c] == 0:
            assert ost == 0 and np.array_equal(got[c * CH:(c + 1) * CH], want), c
        if ost != 0:
            assert gst[c] != 0, c
