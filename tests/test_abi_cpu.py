"""The C ABI library loads and exports every symbol include/codag.h declares; argument
checks that need no GPU return CODAG_EINVAL.  No decode calls here (no GPU)."""
import ctypes as C
import re
from pathlib import Path

HEADER = Path(__file__).resolve().parents[1] / "include" / "codag.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(codag_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(native):
    names = declared_functions()
    assert len(names) >= 18
    lib = native.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(native.EXPORTS)


def test_argument_validation_without_gpu(native):
    lib = native.lib()
    # null pointers / bad element widths are rejected before any CUDA call
    assert lib.codag_decompress_rlev1(None, 0, None, None, 1, 131072, 8, None, 0, None, None, 0, None) == native.EINVAL
    assert lib.codag_decompress_rlev2(1, 1, 1, 1, 1, 131072, 3, 1, 1, None, None, 0, None) == native.EINVAL
    assert lib.codag_decompress_rlev2(1, 1, 1, 1, 1, 131071, 8, 1, 1, None, None, 0, None) == native.EINVAL
    assert lib.codag_decompress_deflate(1, 1, 1, 1, 131072, -1, 1, 1, None, None) == native.EINVAL
    bad = native.Tune(0, 4, 10, 0)
    assert lib.codag_set_tune(0, C.byref(bad)) == native.EINVAL
    bad = native.Tune(4, 3, 10, 0)
    assert lib.codag_set_tune(0, C.byref(bad)) == native.EINVAL
    assert lib.codag_set_wait_limit(0) == native.EINVAL
    # zero chunks is a no-op
    assert lib.codag_decompress_rlev1(1, 1, 1, 1, 0, 131072, 8, 1, 1, None, None, 0, None) == native.OK
    assert lib.codag_workspace_bytes(native.RLEV2, 8192) >= 8192 * 512 * 32
    assert lib.codag_workspace_bytes(native.DEFLATE, 8192) == 0


def test_tune_round_trip(native):
    old = native.get_tune(native.RLEV2)
    try:
        native.set_tune(native.RLEV2, 4, 8, 11)
        t = native.get_tune(native.RLEV2)
        assert (t.warps_per_cta, t.ring_slots, t.lut_bits) == (4, 8, 11)
    finally:
        native.set_tune(native.RLEV2, old.warps_per_cta, old.ring_slots, old.lut_bits)
