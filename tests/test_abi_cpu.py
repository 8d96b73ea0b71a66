"""The C ABI libraries load and export every symbol their headers declare (include/codag.h:
libcodag_b200.so; include/codag_format.h: libcodag_fmt.so), the decoder library holds no
format producer and the format library no CUDA; argument checks that need no GPU return
CODAG_EINVAL.  No decode calls here (no GPU)."""
import ctypes as C
import re
from pathlib import Path

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_functions(header):
    text = re.sub(r"/\*.*?\*/", "", (INCLUDE / header).read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(codag_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(native):
    names = declared_functions("codag.h")
    assert len(names) >= 13
    lib = native.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(native.EXPORTS)


def test_format_library_exports_every_declared_symbol(native):
    names = declared_functions("codag_format.h")
    assert len(names) >= 9
    lib = native.fmt_lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(native.FMT_EXPORTS)


def test_libraries_are_separate(native):
    """The format library loads without CUDA (a CPU-only caller, such as the timed CPU
    decoder, never maps the decoders), and the decoder library carries no producer."""
    import subprocess
    deps = subprocess.run(["ldd", str(native.FMT_LIB_PATH)], capture_output=True, text=True).stdout
    assert "libcudart" not in deps and "libcuda." not in deps
    dec = subprocess.run(["nm", "-D", "--defined-only", str(native.LIB_PATH)], capture_output=True, text=True).stdout
    assert "codag_encode_set" not in dec and "codag_gen_text" not in dec


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
