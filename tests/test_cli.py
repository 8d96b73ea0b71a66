"""The CODAG-compatible command-line tools and the on-disk layout readers/writers.

CPU: metadata files round trip and match the oracle; the tools reject bad command lines
before touching a GPU.  GPU: each tool decodes a file and its output matches the input."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from codag_b200 import build, formats

EXE = build.EXE


def _exe(name):
    p = EXE / name / f"{name}.cu.exe"
    if not p.exists():
        build.build()
    return p


def test_rlev1_files_round_trip(native, oracle, tmp_path):
    col = native.gen_rlev1_column(100_000, 3, 8)
    blob, off, ln = native.encode_rlev1(col, 131072, 8)
    formats.write_rlev1(tmp_path, blob, off, ln)
    n = ln.size
    assert (tmp_path / "rle_v1_blk_offset.bin").stat().st_size == 8 * (32 * n + 1)
    assert (tmp_path / "rle_v1_col_len.bin").stat().st_size == 8 * 32 * 32 * n
    off2, ln2 = formats.read_rlev1(tmp_path)
    assert np.array_equal(off2, off[:n + 1]) and np.array_equal(ln2, ln)
    st, out = oracle.rlev1_chunk(blob[8 + int(off2[0]):8 + int(off2[0]) + int(ln2[0])], 131072, 8)
    assert st == 0 and np.array_equal(out, col[:131072])


def test_deflate_and_rlev2_files_round_trip(native, tmp_path):
    txt = native.gen_text(300_000, 4)
    comp, bo, cl = native.encode_deflate(txt, 131072, 6)
    formats.write_deflate(tmp_path / "t", comp, bo, cl)
    c2, bo2 = formats.read_deflate(tmp_path / "t")
    assert np.array_equal(c2, comp) and np.array_equal(bo2, bo) and int(bo2[0]) == txt.size
    col = native.gen_rlev2_column(50_000, 4, 8)
    comp, off, ln = native.encode_rlev2(col, 131072, 8)
    formats.write_rlev2(tmp_path / "r", comp, off, ln)
    c3, off3, ln3 = formats.read_rlev2(tmp_path / "r")
    assert np.array_equal(c3, comp) and np.array_equal(off3, off) and np.array_equal(ln3, ln)
    assert int(off3[-1]) == col.size


def test_formats_command_line_writes_codag_deflate_files(native, tmp_path):
    src = tmp_path / "in.txt"
    native.gen_text(200_000, 9).tofile(src)
    assert formats.main(["deflate", str(src), str(tmp_path / "d")]) == 0
    bo = np.fromfile(tmp_path / "d_blk_offset.bin", np.uint64)
    assert bo[0] == 200_000 and bo[1] == 0 and bo.size == 2 + 2
    assert (tmp_path / "d_comp.bin").stat().st_size == int(bo[-1])


@pytest.mark.parametrize("name,args", [("rlev1", []), ("rlev1", ["-t", "3", "-f", "x"]), ("rlev2", []),
                                       ("rlev2", ["x", "5"]), ("zlib", ["a", "b"])])
def test_tools_reject_bad_command_lines(native, name, args):
    r = subprocess.run([str(_exe(name)), *args], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    assert r.stderr or r.stdout


@pytest.mark.gpu
def test_rlev1_tool(native, tmp_path):
    col = tmp_path / "col.bin"
    native.gen_rlev1_column(300_000, 11, 8).tofile(col)
    r = subprocess.run([str(_exe("rlev1")), "-f", str(col), "-t", "8"], capture_output=True, text=True,
                       cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("CHUNK_SIZE\tCOLUMN WIDTH") and lines[1] == "NUM WARP: 1"
    comp_bytes, meta, ratio, secs = lines[2].split("\t")
    assert int(meta) > 0 and 0 < float(ratio) < 1.5 and float(secs) > 0
    assert "File Differ" not in r.stdout
    off, ln = formats.read_rlev1(tmp_path / "input_data")
    assert ln.size == 32 and int(off[-1]) >= int(ln.sum())


@pytest.mark.gpu
def test_rlev2_tool(native, tmp_path):
    col = tmp_path / "c2.bin"
    native.gen_rlev2_column(200_000, 12, 8).tofile(col)
    r = subprocess.run([str(_exe("rlev2")), str(col), "8"], capture_output=True, text=True, cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fail at" not in r.stdout
    assert r.stdout.count(" secs") == 10 and r.stdout.count("131072 \t48\t") == 2
    comp, off, ln = formats.read_rlev2(tmp_path / "input_data" / "c2.bin")
    assert int(off[-1]) == 1_600_000


@pytest.mark.gpu
def test_zlib_tool(native, tmp_path):
    txt = native.gen_text(1_000_003, 13)
    src = tmp_path / "t.txt"
    txt.tofile(src)
    assert formats.main(["deflate", str(src), str(tmp_path / "t")]) == 0
    out = tmp_path / "t.out"
    r = subprocess.run([str(_exe("zlib")), str(tmp_path / "t_comp.bin"), str(out), str(tmp_path / "t_blk_offset.bin"),
                        "131072"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("\t") and float(r.stdout.strip()) > 0
    assert out.read_bytes() == txt.tobytes()
