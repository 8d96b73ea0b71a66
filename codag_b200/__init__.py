"""codag_b200 -- B200-native (sm_100a) chunked decompressors for ORC RLE v1, ORC RLE v2 and
Deflate with CODAG's drop-in surface: the C ABI of include/codag.h, CODAG's on-disk chunk
layout, and the rlev1/rlev2/zlib command lines (build/exe/src/<codec>/<codec>.cu.exe).

    native   ctypes binding of libcodag_b200.so (decoders, format producers, generators)
    api      device calls on torch CUDA tensors, CODAG-style host calls, batched plans
    formats  CODAG's metadata files (blk_offset / col_len) on disk
    serving  continuous-batching request loop over the persistent batched kernel
    tuning   autotuner for warps per CTA, TMA ring depth and Huffman table width
"""
from . import native  # noqa: F401
from .native import CodagError, DEFLATE, RLEV1, RLEV2  # noqa: F401

__all__ = ["native", "CodagError", "RLEV1", "RLEV2", "DEFLATE"]
