"""Parity pinned to CODAG's own RLE v1 decoder.

tests/golden/ref_rlev1_*.npz hold RLE v1 chunks written by this project's producer and the
SHA-256 of every chunk as CODAG's GPU decoder (compiled from CODAG's sources,
oracle/ref_harness.cu) decoded it (tests/golden/make_ref_golden.py).  The oracle (CPU) and
the CUDA decoder (GPU) must give the same digests."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("ref_rlev1_*.npz"))
CH = 131072


def _load(name):
    d = np.load(GOLDEN / f"{name}.npz")
    return {k: d[k] for k in d.files}


def _sha(buf, n):
    return np.stack([np.frombuffer(hashlib.sha256(buf[i * CH:(i + 1) * CH].tobytes()).digest(), np.uint8)
                     for i in range(n)])


def test_golden_files_present():
    assert CASES == ["ref_rlev1_u32", "ref_rlev1_u64"]


@pytest.mark.parametrize("name", CASES)
def test_reference_decoder_agrees_with_source(name):
    g = _load(name)
    assert bool(g["ref_equals_source"])
    assert np.array_equal(g["ref_sha"], g["src_sha"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_decoder(oracle, name):
    g = _load(name)
    n, e = int(g["n"]), int(g["elem"])
    out = np.zeros(n * CH, np.uint8)
    st = oracle.decode_batch(g["comp"], g["off"], g["ln"], out, np.arange(n, dtype=np.uint64) * CH, [CH] * n, [CH] * n,
                             [0] * n, [e] * n, [0] * n)
    assert not st.any()
    assert np.array_equal(_sha(out, n), g["ref_sha"])


@pytest.mark.gpu
@pytest.mark.parametrize("two_pass", [False, True])
@pytest.mark.parametrize("name", CASES)
def test_cuda_decoder_matches_reference_decoder(cuda, name, two_pass):
    from codag_b200 import api
    g = _load(name)
    n, e = int(g["n"]), int(g["elem"])
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a).astype(np.uint64).view(np.int64)).to("cuda")
    out = cuda.zeros(n * CH, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_rlev1(cuda.from_numpy(g["comp"]).to("cuda"), t(g["off"]), t(g["ln"]), CH, e, out, None, st,
                         ws=api.AUTO_WORKSPACE if two_pass else None)
    cuda.cuda.synchronize()
    assert not st.cpu().numpy().any()
    assert np.array_equal(_sha(out.cpu().numpy(), n), g["ref_sha"])
