"""CODAG's cuDF-comparison layout: [u64 chunk size][u64 n][u64 sizes x n][zlib streams],
written by rapids_compressor.py:222-275 (64 KiB chunks, zlib level 9) and decoded by
include/base_deflate.h:20-130.  tests/golden/cudf_ref_comp.bin is that script's output for
tests/golden/cudf_src.bin (tests/golden/make_golden.py); the format library must write the
same bytes, the oracle and the CUDA decoder must decode it, and the base_deflate tool must
write the decoded chunks."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
CH = 65536


def _golden():
    return np.fromfile(GOLDEN / "cudf_src.bin", np.uint8), np.fromfile(GOLDEN / "cudf_ref_comp.bin", np.uint8)


def _padded(src, chunk):
    n = (src.size + chunk - 1) // chunk
    out = np.zeros(n * chunk, np.uint8)
    out[:src.size] = src
    return out


def test_writer_matches_codag_compressor(native):
    src, ref = _golden()
    assert np.array_equal(native.encode_cudf_deflate(src, CH, 9), ref)


def test_layout_parse(native):
    src, ref = _golden()
    chunk, data, rel = native.cudf_deflate_layout(ref)
    n = (src.size + CH - 1) // CH
    assert (chunk, data, rel.size) == (CH, 16 + 8 * n, n + 1)
    assert int(rel[-1]) == ref.size - data
    bad = ref.copy()
    bad[16:24] = np.frombuffer(np.uint64(1 << 40).tobytes(), np.uint8)  # a size past the end of the file
    with pytest.raises(native.CodagError):
        native.cudf_deflate_layout(bad)


def test_oracle_decodes_codag_file(native, oracle):
    src, ref = _golden()
    chunk, data, rel = native.cudf_deflate_layout(ref)
    want = _padded(src, chunk)
    for i in range(rel.size - 1):
        st, out = oracle.deflate_chunk(ref[data + int(rel[i]):data + int(rel[i + 1])], chunk)
        assert st == 0 and np.array_equal(out, want[i * chunk:(i + 1) * chunk]), i


@pytest.mark.gpu
def test_cuda_decodes_codag_file(cuda, native):
    from codag_b200 import api
    src, ref = _golden()
    assert np.array_equal(api.decompress_cudf_deflate_host(ref), _padded(src, CH))
    # a larger file from the format library, 1 MiB-odd input
    txt = native.gen_text((1 << 20) + 12345, 77)
    f = native.encode_cudf_deflate(txt, CH, 9)
    assert np.array_equal(api.decompress_cudf_deflate_host(f), _padded(txt, CH))


@pytest.mark.gpu
def test_base_deflate_tool(cuda, native, tmp_path):
    exe = ROOT / "build" / "exe" / "src" / "util" / "base_deflate.cu.exe"
    src, ref = _golden()
    out = tmp_path / "out.bin"
    res = subprocess.run([str(exe), str(GOLDEN / "cudf_ref_comp.bin"), str(out)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    assert "num chunks: 4" in res.stdout
    assert np.array_equal(np.fromfile(out, np.uint8), _padded(src, CH))
