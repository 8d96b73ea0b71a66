"""CODAG's on-disk chunk layouts: writers, readers and a command-line producer.

RLE v1 (include/rlev1/rlev1.h:103-192): ./input_data/rle_v1_blk_offset.bin holds 32x the
entries the decoder uses (n_pad*32+1 u64, the first n_pad+1 meaningful) and
./input_data/rle_v1_col_len.bin 32*32x (the first n_pad meaningful); the decoder derives
n_pad = (entries - 1) / 32 (rlev1.h:469).  The extra entries are zeros here.
RLE v2 (include/rlev2/encoder_trans.h:482-564, in memory in CODAG): <name>_comp.bin,
<name>_blk_offset.bin (n+1 u64, the last = original size), <name>_col_len.bin (n u64).
Deflate (deflate_compressor.py:44-125): <name>_comp.bin (zlib-wrapped streams padded to 8
bytes), <name>_blk_offset.bin ([size, 0, end_1, ..., end_n] u64), <name>_col_len.bin.

    python -m codag_b200.formats deflate <input> <name> [--level 6] [--raw]
    python -m codag_b200.formats rlev2 <input> <name> [--elem 8]
    python -m codag_b200.formats rlev1 <input> <dir> [--elem 8]
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

from . import native

CH = 131072


def _u64(path: Path) -> np.ndarray:
    return np.fromfile(path, dtype=np.uint64)


# --- RLE v1 ---------------------------------------------------------------------------------------
def write_rlev1(directory: str | Path, blob: np.ndarray, off: np.ndarray, ln: np.ndarray) -> Path:
    """Writes CODAG's two RLE v1 metadata files (the blob stays in memory, as in CODAG)."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    n = ln.size
    off_f = np.zeros(n * 32 + 1, np.uint64)
    off_f[:n + 1] = off[:n + 1]
    len_f = np.zeros(n * 32 * 32, np.uint64)
    len_f[:n] = ln
    len_f.tofile(d / "rle_v1_col_len.bin")
    off_f.tofile(d / "rle_v1_blk_offset.bin")
    return d


def read_rlev1(directory: str | Path):
    """(blk_off[n+1], col_len[n]) from CODAG's RLE v1 metadata files."""
    d = Path(directory)
    off = _u64(d / "rle_v1_blk_offset.bin")
    n = (off.size - 1) // 32
    return off[:n + 1], _u64(d / "rle_v1_col_len.bin")[:n]


# --- RLE v2 ---------------------------------------------------------------------------------------
def write_rlev2(name: str | Path, comp: np.ndarray, off: np.ndarray, ln: np.ndarray) -> None:
    name = str(name)
    comp.tofile(name + "_comp.bin")
    off.astype(np.uint64).tofile(name + "_blk_offset.bin")
    ln.astype(np.uint64).tofile(name + "_col_len.bin")


def read_rlev2(name: str | Path):
    """(comp, blk_off[n+1] with blk_off[n] = size, col_len[n])."""
    name = str(name)
    return np.fromfile(name + "_comp.bin", np.uint8), _u64(Path(name + "_blk_offset.bin")), \
        _u64(Path(name + "_col_len.bin"))


# --- Deflate --------------------------------------------------------------------------------------
def write_deflate(name: str | Path, comp: np.ndarray, blk_offset: np.ndarray, col_len: np.ndarray) -> None:
    name = str(name)
    comp.tofile(name + "_comp.bin")
    blk_offset.astype(np.uint64).tofile(name + "_blk_offset.bin")
    col_len.astype(np.uint64).tofile(name + "_col_len.bin")


def read_deflate(name: str | Path):
    """(comp, blk_offset = [size, 0, end_1 .. end_n])."""
    name = str(name)
    return np.fromfile(name + "_comp.bin", np.uint8), _u64(Path(name + "_blk_offset.bin"))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m codag_b200.formats")
    ap.add_argument("codec", choices=["deflate", "rlev1", "rlev2"])
    ap.add_argument("input")
    ap.add_argument("name", help="output prefix (<name>_comp.bin ...) or, for rlev1, the metadata directory")
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--raw", action="store_true", help="Deflate: raw streams (no 2-byte zlib wrapper)")
    ap.add_argument("--elem", type=int, default=8)
    ap.add_argument("--chunk", type=int, default=CH)
    a = ap.parse_args(argv)
    data = np.fromfile(a.input, np.uint8)
    if a.codec == "deflate":
        comp, bo, cl = native.encode_deflate(data, a.chunk, a.level, zlib_wrapper=not a.raw)
        write_deflate(a.name, comp, bo, cl)
        print(f"{data.size} -> {comp.size} bytes in {cl.size} chunks")
    elif a.codec == "rlev2":
        data = data[:data.size - data.size % a.elem]
        comp, off, ln = native.encode_rlev2(data, a.chunk, a.elem)
        write_rlev2(a.name, comp, off, ln)
        print(f"{data.size} -> {comp.size} bytes in {ln.size} chunks")
    else:
        data = data[:data.size - data.size % a.elem]
        blob, off, ln = native.encode_rlev1(data, a.chunk, a.elem)
        write_rlev1(a.name, blob, off, ln)
        (Path(a.name) / "rle_v1_comp.bin").write_bytes(blob.tobytes())
        print(f"{data.size} -> {blob.size} bytes in {ln.size} chunks")
    return 0


if __name__ == "__main__":
    sys.exit(main())
