"""Parity pinned to CODAG's own RLE v2 encoder.

tests/golden/ref_rlev2_*.npz hold seeded columns together with the files CODAG's RLE v2
encoder wrote for them (CODAG's kernels block_encode_orig / orig_col_len_single run on the
host, tests/golden/make_ref_rlev2.py), and ref_rlev2_tables.npz CODAG's four width tables.

Two places where CODAG's own encoder and decoder disagree, named per chunk by
tests/rlev2_walk.py:
  zero_run   for a run of 128 zero values CODAG's encoder writes a DIRECT header whose
             9-bit length field is var_runlen - 1 = -1, i.e. 511, followed by the 128 values
             (include/rlev2/encoder.h:424-440 after the fixed-run flush of
             encoder_trans.h:290-293); its decoder keeps the length in a uint8_t
             (decoder_new.h:1019), reads 0 values and then parses the packed zeros as
             headers.  This project's writer stores the true length (127) there; everywhere
             else the two writers agree byte for byte.
  wide_patch a PATCHED_BASE patch with bits at or above bit 32: CODAG's decoder masks patches
             with a 32-bit mask (decoder_new.h:1103) and loses them.
Chunks with either do not decode to their column in CODAG, in the oracle (which restates
CODAG's decoder) or in the CUDA decoder; all three agree on them."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.rlev2_walk import KINDS, walk

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "golden" if (ROOT / "golden").is_dir() else Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem[len("ref_rlev2_"):] for p in GOLDEN.glob("ref_rlev2_*.npz") if p.stem != "ref_rlev2_tables")
CH = 131072
DT = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def _load(name):
    d = np.load(GOLDEN / f"ref_rlev2_{name}.npz")
    return {k: d[k] for k in d.files}


def _padded_source(g):
    n = g["col_len"].size
    src = np.zeros(n * CH, np.uint8)
    src[:g["src"].size] = g["src"]
    return src


def _stream(comp, off, ln, i):
    return comp[int(off[i]):int(off[i]) + int(ln[i])]


def _longest_zero_run(chunk: np.ndarray, e: int) -> int:
    z = np.concatenate([[0], (chunk.view(DT[e]) == 0).astype(np.int8), [0]])
    d = np.diff(z)
    s, t = np.nonzero(d == 1)[0], np.nonzero(d == -1)[0]
    return int((t - s).max()) if s.size else 0


def _walks(g):
    return [walk(_stream(g["comp"], g["blk_off"], g["col_len"], i)) for i in range(g["col_len"].size)]


def _quirk_chunks(g):
    """Chunks CODAG's decoder does not read as its encoder wrote them."""
    return {i for i, w in enumerate(_walks(g)) if w["zero_run"] or w["wide_patch"]}


def test_golden_files_present():
    assert CASES == ["c2_u32", "c2_u64", "mix_u16", "mix_u32", "mix_u64", "mix_u8", "wide_u64", "zeros_u64"]


@pytest.mark.parametrize("name", CASES)
def test_fixtures_cover_every_header_kind(name):
    """Every case has chunks read as written, holding every header kind (SHORT_REPEAT,
    DIRECT, PATCHED_BASE, DELTA with a fixed step, DELTA with packed deltas)."""
    g = _load(name)
    clean = [w for w in _walks(g) if not (w["zero_run"] or w["wide_patch"])]
    kinds = np.array([sum(w[k] for w in clean) for k in KINDS])
    assert np.array_equal(kinds, g["kinds"]) and (kinds > 0).all()


def test_fixtures_hold_both_quirks():
    walks = [w for name in CASES for w in _walks(_load(name))]
    assert any(w["zero_run"] for w in walks) and any(w["wide_patch"] for w in walks)


def test_width_tables_match_codag(tmp_path):
    """v2_width / v2_code / v2_closest / v2_closest_aligned (shared by the CUDA decoder and the
    host writer) equal CODAG's tables (include/rlev2/utils.h:28-59) at every index."""
    src = tmp_path / "w.cpp"
    src.write_text('#include <cstdio>\n#include "rlev2_widths.h"\n'
                   "int main() {\n"
                   '  for (unsigned c = 0; c < 32; c++) std::printf("%u ", v2_width(c));\n'
                   '  for (unsigned b = 0; b <= 64; b++) std::printf("%u ", v2_code(b));\n'
                   '  for (unsigned b = 0; b <= 64; b++) std::printf("%u ", v2_closest(b));\n'
                   '  for (unsigned b = 0; b <= 64; b++) std::printf("%u ", v2_closest_aligned(b));\n'
                   "}\n")
    exe = tmp_path / "w"
    subprocess.run(["g++", "-std=c++17", "-I", str(ROOT / "codag_b200" / "csrc"), str(src), "-o", str(exe)], check=True)
    got = np.array(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split(), np.int64)
    t = np.load(GOLDEN / "ref_rlev2_tables.npz")
    want = np.concatenate([t["decode"], t["encode"], t["closest"], t["closest_aligned"]]).astype(np.int64)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", CASES)
def test_writer_matches_codag_encoder(native, name):
    g = _load(name)
    e = int(g["elem"])
    comp, off, ln = native.encode_rlev2(g["src"], CH, e)
    assert np.array_equal(off, g["blk_off"])  # 128-byte aligned offsets, last entry = original size
    assert np.array_equal(ln, g["col_len"])
    src = _padded_source(g)
    walks = _walks(g)
    differ = [i for i in range(ln.size)
              if not np.array_equal(_stream(comp, off, ln, i), _stream(g["comp"], g["blk_off"], g["col_len"], i))]
    assert differ == [i for i, w in enumerate(walks) if w["zero_run"]]
    for i in differ:
        assert _longest_zero_run(src[i * CH:(i + 1) * CH], e) >= 128
        a, b = _stream(g["comp"], g["blk_off"], g["col_len"], i), _stream(comp, off, ln, i)
        diff = np.nonzero(a != b)[0]
        heads = diff[::2]
        # only DIRECT length fields differ: CODAG 511 (0x41|code<<1, 0xff), ours 127 (0x40|code<<1, 0x7f)
        assert diff.size % 2 == 0 and np.array_equal(diff[1::2], heads + 1)
        assert (b[heads] & 0xc1 == 0x40).all() and np.array_equal(a[heads], b[heads] | 1)
        assert (a[heads + 1] == 0xff).all() and (b[heads + 1] == 0x7f).all()


@pytest.mark.parametrize("name", CASES)
def test_oracle_decodes_codag_files(oracle, name):
    g = _load(name)
    e, n = int(g["elem"]), int(g["col_len"].size)
    out = np.zeros(n * CH, np.uint8)
    st = oracle.decode_batch(g["comp"], g["blk_off"][:n], g["col_len"], out, np.arange(n, dtype=np.uint64) * CH,
                             [CH] * n, [CH] * n, [1] * n, [e] * n, [0] * n)
    src = _padded_source(g)
    quirk = _quirk_chunks(g)
    good = [i for i in range(n) if i not in quirk]
    assert good
    for i in good:
        assert st[i] == 0 and np.array_equal(out[i * CH:(i + 1) * CH], src[i * CH:(i + 1) * CH]), i
    for i in quirk:  # misread as CODAG's decoder misreads them
        assert st[i] != 0 or not np.array_equal(out[i * CH:(i + 1) * CH], src[i * CH:(i + 1) * CH]), i


@pytest.mark.gpu
@pytest.mark.parametrize("two_pass", [False, True])
@pytest.mark.parametrize("name", CASES)
def test_cuda_decoder_decodes_codag_files(cuda, oracle, name, two_pass):
    """CODAG's own files through codag_decompress_rlev2: every chunk matches the oracle
    (status and bytes), and every chunk outside the zero-run quirk matches the column."""
    from codag_b200 import api
    g = _load(name)
    e, n = int(g["elem"]), int(g["col_len"].size)
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a).astype(np.uint64).view(np.int64)).to("cuda")
    out = cuda.zeros(n * CH, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_rlev2(cuda.from_numpy(g["comp"]).to("cuda"), t(g["blk_off"][:n]), t(g["col_len"]), CH, e, out,
                         None, st, ws=api.AUTO_WORKSPACE if two_pass else None)
    cuda.cuda.synchronize()
    got, gst = out.cpu().numpy(), st.cpu().numpy()
    want = np.zeros(n * CH, np.uint8)
    ost = oracle.decode_batch(g["comp"], g["blk_off"][:n], g["col_len"], want, np.arange(n, dtype=np.uint64) * CH,
                              [CH] * n, [CH] * n, [1] * n, [e] * n, [0] * n)
    src = _padded_source(g)
    quirk = _quirk_chunks(g)
    for i in range(n):
        sl = slice(i * CH, (i + 1) * CH)
        assert (gst[i] == 0) == (ost[i] == 0), i
        if ost[i] == 0:
            assert np.array_equal(got[sl], want[sl]), i
        if i not in quirk:
            assert gst[i] == 0 and np.array_equal(got[sl], src[sl]), i
