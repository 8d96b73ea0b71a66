"""Regenerates tests/golden/ref_*.npz: outputs of CODAG's own GPU decoders.

Runs on a machine with a GPU, after `oracle/build_ref.sh` has compiled CODAG's decoders
into oracle/_ref/ (oracle/ref_harness.cu).  For each case it makes a seeded RLE v1 column with
this project's generator, compresses it with this project's producer (which restates
CODAG's encoder and file layout), decodes it with CODAG's kernel and stores the compressed
chunks with a SHA-256 per decoded chunk.  The tests decode the same chunks with the oracle
and with the CUDA decoders and compare the digests.  Only whole, well-formed chunks go to
CODAG's decoders: they stop when a chunk is full, so a malformed stream could keep them
running.

    python tests/golden/make_ref_golden.py [--out tests/golden]
"""
from __future__ import annotations

import argparse
import hashlib
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

CH = 131072
# Only CODAG's RLE v1 decoder is run.  Its RLE v2 decoder (inflate_orig_rdw of
# include/rlev2/decoder_new.h) did not finish within 600 s on six well-formed chunks, so it
# is not run again, and its Deflate decoder, which reads through the same input stream
# class, is not run either.
CASES = {
    # name: (codec, elem, chunks, seed)
    "rlev1_u64": ("rlev1", 8, 6, 101),
    "rlev1_u32": ("rlev1", 4, 4, 102),
}


def digests(buf: np.ndarray, n: int) -> np.ndarray:
    return np.frombuffer(b"".join(hashlib.sha256(buf[i * CH:(i + 1) * CH].tobytes()).digest() for i in range(n)),
                         np.uint8).reshape(n, 32)


def make_case(name: str, tmp: Path) -> dict:
    from codag_b200 import native
    codec, elem, chunks, seed = CASES[name]
    ref = REPO / "oracle" / "_ref" / f"ref_{codec}"
    src = native.gen_rlev1_column(chunks * CH // elem - 37, seed, elem)
    blob, off, ln = native.encode_rlev1(src, CH, elem)
    streams = blob[8:]
    n = chunks
    streams.tofile(tmp / "s.bin")
    off[:n].astype(np.uint64).tofile(tmp / "off.bin")
    ln[:n].astype(np.uint64).tofile(tmp / "len.bin")
    subprocess.run([str(ref), codec, str(elem), str(tmp / "s.bin"), str(tmp / "off.bin"), str(tmp / "len.bin"),
                    str(n), str(tmp / "o.bin")], check=True, timeout=600)
    out = np.fromfile(tmp / "o.bin", np.uint8)
    want = np.zeros(n * CH, np.uint8)
    want[:src.size] = src.view(np.uint8)
    return dict(comp=streams[:int(off[n])], off=off[:n], ln=ln[:n], elem=np.int64(elem), n=np.int64(n),
                ref_sha=digests(out[:n * CH], n), src_sha=digests(want, n),
                ref_equals_source=np.bool_(np.array_equal(out[:n * CH], want)))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        for name in CASES:
            d = make_case(name, Path(td))
            np.savez_compressed(out / f"ref_{name}.npz", **d)
            print(name, "chunks", int(d["n"]), "reference decoder equals source:", bool(d["ref_equals_source"]))


if __name__ == "__main__":
    main()
