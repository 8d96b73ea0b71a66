"""ctypes bindings of the two in-tree libraries.

libcodag_b200.so (include/codag.h) is the product: every decode call goes to its CUDA
kernels.  libcodag_fmt.so (include/codag_format.h) holds the host-side format producers and
seeded generators, and loads without the decoders.  Loading fails loudly when a library has
not been built; there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libcodag_b200.so"
FMT_LIB_PATH = Path(__file__).resolve().parent / "libcodag_fmt.so"

OK, EINVAL, ECORRUPT, ETIMEOUT, ECUDA, ENOMEM, ELIMIT = 0, 1, 2, 3, 4, 5, 6
STATUS_NAMES = {OK: "OK", EINVAL: "EINVAL", ECORRUPT: "ECORRUPT", ETIMEOUT: "ETIMEOUT", ECUDA: "ECUDA", ENOMEM: "ENOMEM",
                ELIMIT: "ELIMIT"}
NOALLOC_MAX_CHUNKS = 512  # CODAG_NOALLOC_MAX_CHUNKS
RLEV1, RLEV2, DEFLATE = 0, 1, 2

# every symbol declared in include/codag.h (libcodag_b200.so)
EXPORTS = (
    "codag_decompress_rlev1", "codag_decompress_rlev2", "codag_decompress_deflate", "codag_workspace_bytes",
    "codag_decompress_rlev2_noalloc", "codag_decompress_rlev2_transposed",
    "codag_set_tune", "codag_get_tune", "codag_set_wait_limit", "codag_selftest_wait_timeout",
    "codag_batch_plan", "codag_batch_run", "codag_batch_destroy", "codag_batch_launch",
    "codag_compress_chunks", "codag_compress_bound", "codag_compress_workspace_bytes",
    "codag_compress_rlev1", "codag_compress_rlev2",
)
# every symbol declared in include/codag_format.h (libcodag_fmt.so)
FMT_EXPORTS = (
    "codag_hbuf_free", "codag_encode_rlev1", "codag_encode_rlev2", "codag_encode_deflate", "codag_encode_one",
    "codag_encode_set", "codag_encode_cudf_deflate", "codag_cudf_deflate_layout", "codag_encode_rlev2_transposed",
    "codag_gen_rlev1_column", "codag_gen_rlev2_column", "codag_gen_text",
)


class CodagError(RuntimeError):
    def __init__(self, where: str, status: int):
        super().__init__(f"{where} failed: {STATUS_NAMES.get(status, status)}")
        self.status = status


class HBuf(C.Structure):
    _fields_ = [("data", C.c_void_p), ("bytes", C.c_uint64)]


class Tune(C.Structure):
    _fields_ = [("warps_per_cta", C.c_int32), ("ring_slots", C.c_int32), ("lut_bits", C.c_int32),
                ("cta_per_chunk", C.c_int32), ("table_global", C.c_int32)]


class ChunkDesc(C.Structure):
    _fields_ = [("comp_off", C.c_uint64), ("out_off", C.c_uint64), ("comp_len", C.c_uint32), ("out_len", C.c_uint32),
                ("codec", C.c_uint8), ("elem_bytes", C.c_uint8), ("wrapper_bytes", C.c_uint8), ("reserved", C.c_uint8 * 5)]


CHUNK_DESC_DTYPE = np.dtype([("comp_off", "<u8"), ("out_off", "<u8"), ("comp_len", "<u4"), ("out_len", "<u4"),
                             ("codec", "u1"), ("elem_bytes", "u1"), ("wrapper_bytes", "u1"), ("reserved", "u1", (5,))])
assert CHUNK_DESC_DTYPE.itemsize == C.sizeof(ChunkDesc) == 32

_lib = None
_fmt = None


def lib() -> C.CDLL:
    """The loaded native library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m codag_b200.build` (the decoders have no fallback)")
    L = C.CDLL(str(LIB_PATH))
    u64, i32, vp = C.c_uint64, C.c_int32, C.c_void_p
    rle = [vp, u64, vp, vp, u64, u64, C.c_int, vp, u64, vp, vp, u64, vp]
    L.codag_workspace_bytes.argtypes = [C.c_int, u64]
    L.codag_workspace_bytes.restype = u64
    for name in ("codag_decompress_rlev1", "codag_decompress_rlev2"):
        getattr(L, name).argtypes = rle
        getattr(L, name).restype = i32
    L.codag_decompress_rlev2_noalloc.argtypes = [vp, u64, vp, vp, u64, u64, C.c_int, vp, u64, vp, vp]
    L.codag_decompress_rlev2_noalloc.restype = i32
    L.codag_decompress_deflate.argtypes = [vp, u64, vp, u64, u64, C.c_int, vp, u64, vp, vp]
    L.codag_decompress_rlev2_transposed.argtypes = [vp, u64, vp, vp, u64, u64, C.c_int, C.c_int, vp, u64, vp, vp]
    L.codag_decompress_rlev2_transposed.restype = i32
    L.codag_decompress_deflate.restype = i32
    L.codag_set_tune.argtypes = [C.c_int, C.POINTER(Tune)]
    L.codag_get_tune.argtypes = [C.c_int, C.POINTER(Tune)]
    L.codag_set_wait_limit.argtypes = [u64]
    L.codag_selftest_wait_timeout.argtypes = [vp, vp]
    L.codag_batch_plan.argtypes = [vp, u64, C.POINTER(Tune), C.POINTER(vp)]
    L.codag_batch_run.argtypes = [vp, vp, u64, vp, u64, vp, C.c_int, vp]
    L.codag_batch_destroy.argtypes = [vp]
    L.codag_batch_launch.argtypes = [vp, vp, u64, vp, C.POINTER(Tune), vp, u64, vp, u64, vp, vp]
    L.codag_compress_chunks.argtypes = [u64, u64]
    L.codag_compress_chunks.restype = u64
    for name in ("codag_compress_bound", "codag_compress_workspace_bytes"):
        getattr(L, name).argtypes = [C.c_int, u64, u64, C.c_int]
        getattr(L, name).restype = u64
    for name in ("codag_compress_rlev1", "codag_compress_rlev2"):
        getattr(L, name).argtypes = [vp, u64, u64, C.c_int, vp, u64, vp, vp, vp, vp, vp, u64, vp]
        getattr(L, name).restype = i32
    for name in ("codag_set_tune", "codag_get_tune", "codag_set_wait_limit", "codag_selftest_wait_timeout",
                 "codag_batch_plan", "codag_batch_run", "codag_batch_destroy", "codag_batch_launch"):
        getattr(L, name).restype = i32
    _lib = L
    return L


def fmt_lib() -> C.CDLL:
    """The loaded format library (raises if it was not built)."""
    global _fmt
    if _fmt is not None:
        return _fmt
    if not FMT_LIB_PATH.exists():
        raise RuntimeError(f"{FMT_LIB_PATH} is missing: run `python -m codag_b200.build`")
    L = C.CDLL(str(FMT_LIB_PATH))
    u64, i32, vp = C.c_uint64, C.c_int32, C.c_void_p
    L.codag_hbuf_free.argtypes = [C.POINTER(HBuf)]
    L.codag_hbuf_free.restype = None
    enc = [vp, u64, u64, C.c_int, C.POINTER(HBuf), C.POINTER(HBuf), C.POINTER(HBuf)]
    L.codag_encode_rlev1.argtypes = enc
    L.codag_encode_rlev2.argtypes = enc
    L.codag_encode_deflate.argtypes = [vp, u64, u64, C.c_int, C.c_int, C.c_int, C.POINTER(HBuf), C.POINTER(HBuf),
                                       C.POINTER(HBuf)]
    L.codag_encode_one.argtypes = [C.c_int, vp, u64, C.c_int, C.c_int, C.POINTER(HBuf)]
    L.codag_encode_set.argtypes = [vp, vp, vp, vp, vp, u64, C.c_int, vp, C.POINTER(HBuf), C.POINTER(u64)]
    L.codag_encode_cudf_deflate.argtypes = [vp, u64, u64, C.c_int, C.POINTER(HBuf)]
    L.codag_encode_rlev2_transposed.argtypes = [vp, u64, u64, C.c_int, C.c_int, C.POINTER(HBuf), C.POINTER(HBuf),
                                                C.POINTER(HBuf)]
    L.codag_cudf_deflate_layout.argtypes = [vp, u64, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64), vp]
    for name in ("codag_encode_rlev1", "codag_encode_rlev2", "codag_encode_deflate", "codag_encode_one",
                 "codag_encode_set", "codag_encode_cudf_deflate", "codag_cudf_deflate_layout",
                 "codag_encode_rlev2_transposed"):
        getattr(L, name).restype = i32
    for name in ("codag_gen_rlev1_column", "codag_gen_rlev2_column"):
        getattr(L, name).argtypes = [u64, u64, C.c_int, vp]
        getattr(L, name).restype = None
    L.codag_gen_text.argtypes = [u64, u64, vp]
    L.codag_gen_text.restype = None
    _fmt = L
    return L


def check(where: str, status: int) -> None:
    if status != OK:
        raise CodagError(where, status)


def _take(b: HBuf, dtype=np.uint8) -> np.ndarray:
    """Copy a library-owned host buffer into numpy and release it."""
    try:
        a = np.empty(b.bytes, dtype=np.uint8)
        if b.bytes:
            C.memmove(a.ctypes.data, b.data, b.bytes)
        return a.view(dtype)
    finally:
        fmt_lib().codag_hbuf_free(C.byref(b))


def _ptr(a: np.ndarray) -> int:
    if not a.flags.c_contiguous:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


# --- format producers ---------------------------------------------------------------------
def encode_rlev1(data: np.ndarray, chunk_bytes: int = 131072, elem_bytes: int = 8):
    """CODAG RLE v1 layout: (blob=[u64 size][streams], blk_off[n+1], col_len[n])."""
    raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    b1, b2, b3 = HBuf(), HBuf(), HBuf()
    check("codag_encode_rlev1", fmt_lib().codag_encode_rlev1(_ptr(raw), raw.nbytes, chunk_bytes, elem_bytes,
                                                        C.byref(b1), C.byref(b2), C.byref(b3)))
    return _take(b1), _take(b2, np.uint64), _take(b3, np.uint64)


def encode_rlev2(data: np.ndarray, chunk_bytes: int = 131072, elem_bytes: int = 8):
    """CODAG RLE v2 layout: (comp, blk_off[n+1] with blk_off[n] = size, col_len[n])."""
    raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    b1, b2, b3 = HBuf(), HBuf(), HBuf()
    check("codag_encode_rlev2", fmt_lib().codag_encode_rlev2(_ptr(raw), raw.nbytes, chunk_bytes, elem_bytes,
                                                        C.byref(b1), C.byref(b2), C.byref(b3)))
    return _take(b1), _take(b2, np.uint64), _take(b3, np.uint64)


def encode_deflate(data: np.ndarray, chunk_bytes: int = 131072, level: int = 6, zlib_wrapper: bool = True,
                   require_no_stored: bool = True):
    """CODAG Deflate layout: (comp, blk_offset[n+2] = [size, 0, cum...], col_len[n])."""
    raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    b1, b2, b3 = HBuf(), HBuf(), HBuf()
    check("codag_encode_deflate", fmt_lib().codag_encode_deflate(_ptr(raw), raw.nbytes, chunk_bytes, level,
                                                            int(zlib_wrapper), int(require_no_stored),
                                                            C.byref(b1), C.byref(b2), C.byref(b3)))
    return _take(b1), _take(b2, np.uint64), _take(b3, np.uint64)


def encode_rlev2_transposed(data: np.ndarray, chunk_bytes: int = 131072, elem_bytes: int = 8, read_unit: int = 4):
    """CODAG's transposed RLE v2 layout (codag_encode_rlev2_transposed): (comp, blk_off[n+1], col_len[n*32])."""
    raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    comp, off, ln = HBuf(), HBuf(), HBuf()
    check("codag_encode_rlev2_transposed", fmt_lib().codag_encode_rlev2_transposed(
        _ptr(raw), raw.nbytes, chunk_bytes, elem_bytes, read_unit, C.byref(comp), C.byref(off), C.byref(ln)))
    return _take(comp), _take(off, np.uint64), _take(ln, np.uint64)


def encode_cudf_deflate(data: np.ndarray, chunk_bytes: int = 65536, level: int = 9) -> np.ndarray:
    """CODAG's cuDF-comparison file (codag_encode_cudf_deflate) as one byte array."""
    raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    b = HBuf()
    check("codag_encode_cudf_deflate", fmt_lib().codag_encode_cudf_deflate(_ptr(raw), raw.nbytes, chunk_bytes, level,
                                                                           C.byref(b)))
    return _take(b)


def cudf_deflate_layout(file: np.ndarray):
    """(chunk_bytes, data_offset, blk_off[n+1] relative to data_offset) of a cuDF-comparison file."""
    raw = np.ascontiguousarray(file).view(np.uint8).reshape(-1)
    ch, n, off = C.c_uint64(), C.c_uint64(), C.c_uint64()
    check("codag_cudf_deflate_layout", fmt_lib().codag_cudf_deflate_layout(_ptr(raw), raw.nbytes, C.byref(ch), C.byref(n),
                                                                           C.byref(off), None))
    blk = np.zeros(n.value + 1, np.uint64)
    check("codag_cudf_deflate_layout", fmt_lib().codag_cudf_deflate_layout(_ptr(raw), raw.nbytes, C.byref(ch), C.byref(n),
                                                                           C.byref(off), _ptr(blk)))
    return int(ch.value), int(off.value), blk


def encode_one(codec: int, data: np.ndarray, elem_bytes: int = 8, level: int = 6) -> np.ndarray:
    raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    b = HBuf()
    check("codag_encode_one", fmt_lib().codag_encode_one(codec, _ptr(raw), raw.nbytes, elem_bytes, level, C.byref(b)))
    return _take(b)


def encode_set(src: np.ndarray, in_off: np.ndarray, in_len: np.ndarray, codecs: np.ndarray, elem_bytes: np.ndarray,
               level: int = 6):
    """Encodes independent files (slices of src) one stream each and packs them for a batch plan:
    returns (comp, descs, out_bytes)."""
    src = np.ascontiguousarray(src).view(np.uint8).reshape(-1)
    in_off = np.ascontiguousarray(in_off, dtype=np.uint64)
    in_len = np.ascontiguousarray(in_len, dtype=np.uint64)
    codecs = np.ascontiguousarray(codecs, dtype=np.uint8)
    elem_bytes = np.ascontiguousarray(elem_bytes, dtype=np.uint8)
    n = in_off.size
    if not (in_len.size == codecs.size == elem_bytes.size == n) or np.any(in_off + in_len > src.size):
        raise ValueError("encode_set: inconsistent file table")
    descs = np.zeros(n, dtype=CHUNK_DESC_DTYPE)
    b = HBuf()
    ob = C.c_uint64()
    check("codag_encode_set", fmt_lib().codag_encode_set(_ptr(src), _ptr(in_off), _ptr(in_len), _ptr(codecs),
                                                    _ptr(elem_bytes), n, level, descs.ctypes.data, C.byref(b),
                                                    C.byref(ob)))
    return _take(b), descs, int(ob.value)


def gen_rlev1_column(n: int, seed: int, elem_bytes: int = 8) -> np.ndarray:
    out = np.empty(n * elem_bytes, dtype=np.uint8)
    fmt_lib().codag_gen_rlev1_column(n, seed, elem_bytes, _ptr(out))
    return out


def gen_rlev2_column(n: int, seed: int, elem_bytes: int = 8) -> np.ndarray:
    out = np.empty(n * elem_bytes, dtype=np.uint8)
    fmt_lib().codag_gen_rlev2_column(n, seed, elem_bytes, _ptr(out))
    return out


def gen_text(nbytes: int, seed: int) -> np.ndarray:
    out = np.empty(nbytes, dtype=np.uint8)
    fmt_lib().codag_gen_text(nbytes, seed, _ptr(out))
    return out


# --- tuning ---------------------------------------------------------------------------------
def set_tune(codec: int, warps_per_cta: int, ring_slots: int, lut_bits: int = 10, cta_per_chunk: int = 0) -> None:
    t = Tune(warps_per_cta, ring_slots, lut_bits, cta_per_chunk)
    check("codag_set_tune", lib().codag_set_tune(codec, C.byref(t)))


def get_tune(codec: int) -> Tune:
    t = Tune()
    check("codag_get_tune", lib().codag_get_tune(codec, C.byref(t)))
    return t


def set_wait_limit(cycles: int) -> None:
    check("codag_set_wait_limit", lib().codag_set_wait_limit(cycles))
