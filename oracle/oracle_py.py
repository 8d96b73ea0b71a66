"""ctypes binding of oracle/liboracle.so.  TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, as the
checker or as the timed CPU baseline -- never by the product.  See oracle.c for what it
restates from CODAG and how its parity is pinned.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
OK, EINVAL, ECORRUPT = 0, 1, 2
RLEV1, RLEV2, DEFLATE = 0, 1, 2

_lib = None


def build() -> Path:
    src = HERE / "oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["bash", str(HERE / "build.sh")], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        u64, vp, ci = C.c_uint64, C.c_void_p, C.c_int
        L.oracle_rlev1_decode_chunk.argtypes = [vp, u64, vp, u64, u64, ci]
        L.oracle_rlev2_decode_chunk.argtypes = [vp, u64, vp, u64, u64, ci, C.POINTER(u64)]
        L.oracle_deflate_decode_chunk.argtypes = [vp, u64, ci, vp, u64, u64, C.POINTER(u64)]
        L.oracle_deflate_rfc_chunk.argtypes = [vp, u64, ci, vp, u64, C.POINTER(u64), C.POINTER(C.c_uint32)]
        L.oracle_decode_batch.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int64, ci]
        L.oracle_decode_batch.restype = C.c_int64
        L.oracle_zlib_version.restype = C.c_char_p
        L.oracle_max_threads.restype = ci
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    assert a.flags.c_contiguous
    return a.ctypes.data


def rlev1_chunk(stream: np.ndarray, chunk_bytes: int, elem_bytes: int, store_bytes: int | None = None):
    out = np.zeros(chunk_bytes, np.uint8)
    st = lib().oracle_rlev1_decode_chunk(_p(stream), stream.size, _p(out), chunk_bytes,
                                         chunk_bytes if store_bytes is None else store_bytes, elem_bytes)
    return st, out


def rlev2_chunk(stream: np.ndarray, chunk_bytes: int, elem_bytes: int, store_bytes: int | None = None):
    out = np.zeros(chunk_bytes, np.uint8)
    produced = C.c_uint64()
    st = lib().oracle_rlev2_decode_chunk(_p(stream), stream.size, _p(out), chunk_bytes,
                                         chunk_bytes if store_bytes is None else store_bytes, elem_bytes,
                                         C.byref(produced))
    return st, out


def deflate_chunk(stream: np.ndarray, chunk_bytes: int, wrapper: int = 2, store_bytes: int | None = None):
    out = np.zeros(chunk_bytes, np.uint8)
    produced = C.c_uint64()
    st = lib().oracle_deflate_decode_chunk(_p(stream), stream.size, wrapper, _p(out), chunk_bytes,
                                           chunk_bytes if store_bytes is None else store_bytes, C.byref(produced))
    return st, out


def deflate_rfc_chunk(stream: np.ndarray, cap: int, wrapper: int = 2):
    out = np.zeros(cap, np.uint8)
    produced = C.c_uint64()
    types = C.c_uint32()
    st = lib().oracle_deflate_rfc_chunk(_p(stream), stream.size, wrapper, _p(out), cap, C.byref(produced),
                                        C.byref(types))
    return st, out[:produced.value], types.value


def decode_batch(comp: np.ndarray, comp_off, comp_len, out: np.ndarray, out_off, chunk_len, store_len, codec,
                 elem, wrapper, nthreads: int = 0):
    """Decodes n independent chunks with OpenMP; returns the per-chunk status array."""
    n = len(comp_off)
    a = [np.ascontiguousarray(x, dtype=np.uint64) for x in (comp_off, comp_len, out_off, chunk_len, store_len)]
    b = [np.ascontiguousarray(x, dtype=np.uint8) for x in (codec, elem, wrapper)]
    status = np.zeros(n, np.int32)
    lib().oracle_decode_batch(_p(comp), _p(a[0]), _p(a[1]), _p(out), _p(a[2]), _p(a[3]), _p(a[4]), _p(b[0]),
                              _p(b[1]), _p(b[2]), _p(status), n, nthreads)
    return status


def zlib_version() -> str:
    return lib().oracle_zlib_version().decode()


def max_threads() -> int:
    return lib().oracle_max_threads()
