"""Mixed sets of independently compressed files, and the two ways of decoding them.

A mixed set is many small files of uneven size and mixed codec, each compressed as ONE
stream (a chunk whose size is the file's size).  CODAG's kernels take one uniform chunk size
per launch (include/rlev1/rlev1.h:419-424, include/rlev2/decoder_trans.h:57-61,
include/zlib/zlib.h:1585-1587), so with CODAG such a set can only be decoded file by file:
`decode_per_file` does exactly that through the C ABI (one call per file, one stream).
`BatchPlan` (codag_batch_plan/run) decodes the whole set in one persistent launch.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import native

DEFLATE, RLEV1, RLEV2 = native.DEFLATE, native.RLEV1, native.RLEV2


@dataclass
class MixedSet:
    src: np.ndarray        # u8: all source data the files are slices of
    in_off: np.ndarray     # u64 per file: slice start in src
    in_len: np.ndarray     # u64 per file: decompressed size
    codecs: np.ndarray     # u8 per file
    elem: np.ndarray       # u8 per file (1 for Deflate)
    comp: np.ndarray       # packed streams (16-byte aligned)
    descs: np.ndarray      # native.CHUNK_DESC_DTYPE per file
    out_bytes: int         # output buffer size (outputs 256-byte aligned)

    @property
    def n(self) -> int:
        return int(self.in_len.size)

    def expected(self) -> np.ndarray:
        """The decoded output buffer the set must produce (zeros between files)."""
        out = np.zeros(self.out_bytes, np.uint8)
        for d, o, ln in zip(self.descs, self.in_off, self.in_len):
            out[int(d["out_off"]):int(d["out_off"]) + int(ln)] = self.src[int(o):int(o) + int(ln)]
        return out


def make_mixed_set(n_files: int = 20_000, seed: int = 20260104, min_bytes: int = 4096, max_bytes: int = 1 << 20,
                   mix=(0.4, 0.3, 0.3), source_bytes: int = 128 << 20, level: int = 6) -> MixedSet:
    """Seeded mixed set: sizes log-uniform in [min_bytes, max_bytes] rounded down to a multiple
    of 8; codec Deflate/RLE v1/RLE v2 with probabilities `mix`; RLE files u32 or u64 (50/50).
    Deflate files are slices of Zipf text, RLE files slices of the RLE v1/v2 column
    generators; every file is compressed on its own."""
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(min_bytes), np.log(max_bytes), n_files))).astype(np.int64)
    sizes = np.maximum(sizes // 8 * 8, 8)
    codec = rng.choice([DEFLATE, RLEV1, RLEV2], size=n_files, p=list(mix)).astype(np.uint8)
    elem = np.where(codec == DEFLATE, 1, np.where(rng.random(n_files) < 0.5, 4, 8)).astype(np.uint8)
    src_bytes = max(source_bytes, int(sizes.max()) * 2)
    # five sources: text, RLE v1 u32/u64, RLE v2 u32/u64
    parts = [native.gen_text(src_bytes, seed + 1),
             native.gen_rlev1_column(src_bytes // 4, seed + 2, 4), native.gen_rlev1_column(src_bytes // 8, seed + 3, 8),
             native.gen_rlev2_column(src_bytes // 4, seed + 4, 4), native.gen_rlev2_column(src_bytes // 8, seed + 5, 8)]
    base = np.cumsum([0] + [p.size for p in parts])
    src = np.concatenate(parts)
    which = np.where(codec == DEFLATE, 0, np.where(codec == RLEV1, 1, 3) + (elem == 8))
    room = src_bytes - sizes
    start = (rng.integers(0, room + 1) // 8) * 8
    in_off = (base[which] + start).astype(np.uint64)
    in_len = sizes.astype(np.uint64)
    comp, descs, out_bytes = native.encode_set(src, in_off, in_len, codec, elem, level)
    return MixedSet(src, in_off, in_len, codec, elem, comp, descs, out_bytes)


class PerFileDecoder:
    """One C-ABI call per file (CODAG's only way for a mixed set): chunk_bytes = the file's
    size, one stream per call, calls issued in order on one stream."""

    def __init__(self, ms: MixedSet, d_comp, d_out, device):
        import torch
        self.ms = ms
        self.d_comp, self.d_out = d_comp, d_out
        d = ms.descs
        # per-file metadata on the device: RLE [comp_off], [comp_len]; Deflate [comp_off, comp_off+len]
        self.d_off = torch.from_numpy(d["comp_off"].astype(np.int64)).to(device)
        self.d_len = torch.from_numpy(d["comp_len"].astype(np.int64)).to(device)
        pairs = np.stack([d["comp_off"], d["comp_off"] + d["comp_len"]], 1).astype(np.int64).reshape(-1)
        self.d_pairs = torch.from_numpy(pairs).to(device)
        self.d_st = torch.zeros(ms.n, dtype=torch.int32, device=device)

    def run(self, files, stream) -> None:
        lib = native.lib()
        d = self.ms.descs
        comp, cb = self.d_comp.data_ptr(), self.d_comp.numel()
        out = self.d_out.data_ptr()
        off, ln, pairs, st = self.d_off.data_ptr(), self.d_len.data_ptr(), self.d_pairs.data_ptr(), self.d_st.data_ptr()
        s = stream.cuda_stream or None
        for i in files:
            i = int(i)
            c, e, L, oo = int(d["codec"][i]), int(d["elem_bytes"][i]), int(d["out_len"][i]), int(d["out_off"][i])
            if c == DEFLATE:
                rc = lib.codag_decompress_deflate(comp, cb, pairs + 16 * i, 1, L, 2, out + oo, L, st + 4 * i, s)
            else:
                fn = lib.codag_decompress_rlev1 if c == RLEV1 else lib.codag_decompress_rlev2
                rc = fn(comp, cb, off + 8 * i, ln + 8 * i, 1, L, e, out + oo, L, st + 4 * i, None, 0, s)
            native.check("per-file decode", rc)


def stratified_sample(ms: MixedSet, k: int, seed: int = 7) -> np.ndarray:
    """k file indices spread over the size order and the codecs (for timing the per-file path,
    whose full run takes minutes)."""
    if k >= ms.n:
        return np.arange(ms.n)
    order = np.lexsort((ms.in_len, ms.codecs))
    pick = order[np.linspace(0, ms.n - 1, k).astype(np.int64)]
    return np.sort(pick)
