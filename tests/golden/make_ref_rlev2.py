"""Regenerates tests/golden/ref_rlev2_*.npz: RLE v2 files written by CODAG's own encoder.

CODAG's RLE v2 encoder kernels (block_encode_orig and orig_col_len_single,
include/rlev2/encoder_trans.h:184-409) are compiled for the host by `oracle/build_ref.sh`
and run by oracle/ref_rlev2_host.cpp with the steps of CODAG's rlev2 tool
(rlev2::compress_gpu_orig, encoder_trans.h:482-564).  For each case this script writes a
seeded column, encodes it with that program and stores the column together with CODAG's
compressed bytes, blk_off and col_len arrays, plus CODAG's width tables
(include/rlev2/utils.h:28-59).  No GPU is needed.

The tests then check, on the CPU, that this project's writer emits the same bytes and that
the oracle decodes CODAG's bytes to the column, and on the GPU that the CUDA decoder does.

    CODAG_REFERENCE_DIR=<CODAG tree> python tests/golden/make_ref_rlev2.py [--out tests/golden]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
from tests.rlev2_walk import KINDS, walk  # noqa: E402

CH = 131072
DT = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def mixed_column(n: int, elem: int, seed: int, zero_run: int = 100, rand_bits: int = 64) -> np.ndarray:
    """Segments of 1-299 values: constant runs (zero, small, boundary and random values),
    ascending and descending steps of 1-8, and random values of random width; no value
    start exceeds `rand_bits` bits.  Constant runs
    of zero are at most `zero_run` long, since CODAG's encoder writes a run of 128 zeros in a
    form its own decoder misreads (the tests treat such chunks separately)."""
    rng = np.random.default_rng(seed)
    top = (1 << min(8 * elem, rand_bits)) - 1
    picks = [0, 1, 5, 127, 128, 129, top]
    parts, have = [], 0
    while have < n:
        L = int(rng.integers(1, 300))
        v = np.uint64(picks[int(rng.integers(0, len(picks)))] if rng.random() < 0.7
                      else int(rng.integers(0, top, dtype=np.uint64, endpoint=True)))
        k = int(rng.integers(0, 4))
        step = np.uint64(int(rng.integers(1, 9)))
        idx = np.arange(L, dtype=np.uint64)
        if k == 0:
            seg = np.full(L if v else min(L, zero_run), v, np.uint64)
        elif k == 1:
            seg = v + idx * step
        elif k == 2:  # descending, wrapping below zero only when the range allows it
            seg = (v if rand_bits >= 8 * elem or v >= L * 8 else v + np.uint64(L * 8)) - idx * step
        else:
            b = int(rng.integers(1, min(8 * elem, rand_bits) + 1))
            seg = rng.integers(0, (1 << b) - 1, L, dtype=np.uint64, endpoint=True)
        parts.append(seg)
        have += seg.size
    with np.errstate(over="ignore"):
        return np.concatenate(parts)[:n].astype(DT[elem])


def transposed_cases():
    """CODAG's transposed layout: (elem, read_unit, column); partial last chunks included."""
    from codag_b200 import native
    return {
        "c2_u64_ru4": (8, 4, native.gen_rlev2_column(2 * CH // 8 + 333, 211, 8).view(np.uint64)),
        "mix_u32_ru8": (4, 8, mixed_column(2 * CH // 4 - 9, 4, 212)),
        "mix_u16_ru2": (2, 2, mixed_column(CH // 2 + 17, 2, 213)),
        "mix_u8_ru1": (1, 1, mixed_column(CH + 5, 1, 214)),
    }


def cases():
    from codag_b200 import native
    # name: column (the product's seeded generator of the RLE v2 benchmark column, and the
    # mixed generator above)
    return {
        "c2_u64": (8, native.gen_rlev2_column(3 * CH // 8 - 45, 201, 8).view(np.uint64)),
        "c2_u32": (4, native.gen_rlev2_column(3 * CH // 4 - 13, 202, 4).view(np.uint32)),
        "mix_u64": (8, mixed_column(2 * CH // 8, 8, 203, rand_bits=40)),
        "wide_u64": (8, mixed_column(2 * CH // 8, 8, 209)),
        "mix_u32": (4, mixed_column(2 * CH // 4 - 7, 4, 204)),
        "mix_u16": (2, mixed_column(CH // 2 + 999, 2, 205)),
        "mix_u8": (1, mixed_column(CH + 4097, 1, 206)),
        "zeros_u64": (8, mixed_column(CH // 8 + 300, 8, 207, zero_run=300)),
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE))
    ap.add_argument("--ref", default=os.environ.get("CODAG_REFERENCE_DIR"), help="CODAG source tree")
    a = ap.parse_args()
    if not a.ref:
        sys.exit("give the CODAG source tree with --ref or CODAG_REFERENCE_DIR")
    subprocess.run(["sh", str(REPO / "oracle" / "build_ref.sh"), a.ref], check=True)
    exe = REPO / "oracle" / "_ref" / "ref_rlev2_host"
    out = Path(a.out)
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        subprocess.run([str(exe), "tables", str(t / "tables.bin")], check=True)
        tb = np.fromfile(t / "tables.bin", np.uint8)
        np.savez_compressed(out / "ref_rlev2_tables.npz", decode=tb[:32], encode=tb[32:97], closest=tb[97:162],
                            closest_aligned=tb[162:227])
        for name, (elem, col) in cases().items():
            col.tofile(t / "col.bin")
            subprocess.run([str(exe), "encode", str(elem), str(t / "col.bin"), str(t / "r")], check=True,
                           capture_output=True)
            comp = np.fromfile(t / "r_comp.bin", np.uint8)
            blk_off = np.fromfile(t / "r_blk_off.bin", np.uint64)
            col_len = np.fromfile(t / "r_col_len.bin", np.uint64)
            # header kinds on the chunks that CODAG's decoder reads as they were written
            walks = [walk(comp[int(blk_off[i]):int(blk_off[i] + col_len[i])]) for i in range(col_len.size)]
            clean = [w for w in walks if not (w["zero_run"] or w["wide_patch"])]
            kinds = np.array([sum(w[k] for w in clean) for k in KINDS], np.int64)
            np.savez_compressed(out / f"ref_rlev2_{name}.npz", src=col.view(np.uint8), elem=np.int64(elem),
                                comp=comp, blk_off=blk_off, col_len=col_len, kinds=kinds)
            print(name, "elem", elem, "chunks", col_len.size, "bytes", comp.size, "chunks read as written",
                  len(clean), "headers", dict(zip(KINDS, kinds.tolist())))
        for name, (elem, ru, col) in transposed_cases().items():
            col.tofile(t / "col.bin")
            subprocess.run([str(exe), "transposed", str(elem), str(ru), str(t / "col.bin"), str(t / "r")], check=True,
                           capture_output=True)
            comp = np.fromfile(t / "r_comp.bin", np.uint8)
            blk_off = np.fromfile(t / "r_blk_off.bin", np.uint64)
            col_len = np.fromfile(t / "r_col_len.bin", np.uint64)
            np.savez_compressed(out / f"ref_rlev2t_{name}.npz", src=col.view(np.uint8), elem=np.int64(elem),
                                read_unit=np.int64(ru), comp=comp, blk_off=blk_off, col_len=col_len)
            print("transposed", name, "elem", elem, "read_unit", ru, "chunks", blk_off.size - 1, "bytes", comp.size)


if __name__ == "__main__":
    main()
