"""Python front end of the decompressors: device calls on torch CUDA tensors, the host-buffer
calls that mirror CODAG's host templates, and batched plans.

Device memory and streams come from PyTorch; every decode runs in libcodag_b200.so.

Mapping onto CODAG's host API (all host pointers in, a host buffer out):
  rle_v1::decompress_gpu_orig  (include/rlev1/rlev1.h:419-592)      -> decompress_rlev1_host
  rlev2::decompress_gpu_orig   (include/rlev2/decoder_trans.h:57-133) -> decompress_rlev2_host
  deflate::decompress_gpu      (include/zlib/zlib.h:1583-1700)      -> decompress_deflate_host
Unlike CODAG's templates these never print, never exit and never pick a device; errors
raise CodagError with the per-chunk status attached.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import native
from .native import CodagError, check

_U64 = torch.int64  # torch has no uint64 for most ops; offsets are < 2^63


def _dptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def _stream(stream: torch.cuda.Stream | None) -> int | None:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None


def _status_error(where: str, status: torch.Tensor) -> None:
    st = status.cpu().numpy()
    bad = np.nonzero(st)[0]
    if bad.size:
        err = CodagError(where, int(st[bad[0]]))
        err.chunk_status = st
        raise err


# --- device calls (C ABI, caller-owned device buffers) ----------------------------------------
def workspace(codec: int, n_chunks: int, device="cuda") -> torch.Tensor:
    """A device workspace for the two-pass RLE decode of n_chunks chunks."""
    nbytes = int(native.lib().codag_workspace_bytes(codec, n_chunks))
    return torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)


AUTO_WORKSPACE = object()  # ws=AUTO_WORKSPACE: allocate a workspace for this call (two-pass decode)


def _ws(codec, n, ws):
    if ws is AUTO_WORKSPACE:
        ws = workspace(codec, n)
    return (_dptr(ws), ws.numel()) if ws is not None else (None, 0)


def decompress_rlev1(comp: torch.Tensor, blk_off: torch.Tensor, col_len: torch.Tensor, chunk_bytes: int,
                     elem_bytes: int, out: torch.Tensor, out_bytes: int | None = None,
                     status: torch.Tensor | None = None, stream=None, ws=None) -> None:
    """codag_decompress_rlev1: comp is the stream base (blob+8), blk_off/col_len have n entries.
    ws: None (default) decodes each chunk in one pass; a workspace tensor (see workspace()) or
    AUTO_WORKSPACE selects the two-pass decode (header walk, then descriptor-driven expansion)."""
    n = col_len.numel()
    wp, wb = _ws(native.RLEV1, n, ws)
    check("codag_decompress_rlev1", native.lib().codag_decompress_rlev1(
        _dptr(comp), comp.numel(), _dptr(blk_off), _dptr(col_len), n, chunk_bytes, elem_bytes, _dptr(out),
        out.numel() if out_bytes is None else out_bytes, _dptr(status), wp, wb, _stream(stream)))


def decompress_rlev2(comp: torch.Tensor, blk_off: torch.Tensor, col_len: torch.Tensor, chunk_bytes: int,
                     elem_bytes: int, out: torch.Tensor, out_bytes: int | None = None,
                     status: torch.Tensor | None = None, stream=None, ws=None) -> None:
    """codag_decompress_rlev2: blk_off/col_len have n entries (the size entry is not passed).
    ws as for decompress_rlev1."""
    n = col_len.numel()
    wp, wb = _ws(native.RLEV2, n, ws)
    check("codag_decompress_rlev2", native.lib().codag_decompress_rlev2(
        _dptr(comp), comp.numel(), _dptr(blk_off), _dptr(col_len), n, chunk_bytes, elem_bytes, _dptr(out),
        out.numel() if out_bytes is None else out_bytes, _dptr(status), wp, wb, _stream(stream)))


def decompress_deflate(comp: torch.Tensor, blk_off: torch.Tensor, chunk_bytes: int, out: torch.Tensor,
                       wrapper_bytes: int = 2, out_bytes: int | None = None, status: torch.Tensor | None = None,
                       stream=None) -> None:
    """codag_decompress_deflate: blk_off has n+1 relative offsets (blk_offset file without entry 0)."""
    n = blk_off.numel() - 1
    check("codag_decompress_deflate", native.lib().codag_decompress_deflate(
        _dptr(comp), comp.numel(), _dptr(blk_off), n, chunk_bytes, wrapper_bytes, _dptr(out),
        out.numel() if out_bytes is None else out_bytes, _dptr(status), _stream(stream)))


def compress_rle(codec: int, col: torch.Tensor, chunk_bytes: int = 131072, elem_bytes: int = 8, stream=None,
                 ws: torch.Tensor | None = None):
    """GPU encoder (codag_compress_rlev1/_rlev2) of a device column (uint8 view): returns
    (file, blk_off, col_len) as device tensors in CODAG's layout, the same bytes as
    native.encode_rlev1/encode_rlev2 write on the host (the RLE v1 file is the blob
    [u64 size][streams]).  The output buffers (and the workspace unless given) are allocated
    here; the C ABI itself allocates nothing."""
    lib = native.lib()
    n_bytes = col.numel()
    n = int(lib.codag_compress_chunks(n_bytes, chunk_bytes))
    cap = int(lib.codag_compress_bound(codec, n_bytes, chunk_bytes, elem_bytes))
    need = int(lib.codag_compress_workspace_bytes(codec, n_bytes, chunk_bytes, elem_bytes))
    dev = col.device
    if ws is None or ws.numel() < need:
        ws = torch.empty(need + 256, dtype=torch.uint8, device=dev)
    wsp = (ws.data_ptr() + 255) // 256 * 256
    out = torch.empty(cap, dtype=torch.uint8, device=dev)
    blk_off = torch.empty(n + 1, dtype=torch.int64, device=dev)
    col_len = torch.empty(n, dtype=torch.int64, device=dev)
    meta = torch.zeros(2, dtype=torch.int64, device=dev)  # [file bytes, status]
    fn = lib.codag_compress_rlev1 if codec == native.RLEV1 else lib.codag_compress_rlev2
    check("codag_compress", fn(_dptr(col), n_bytes, chunk_bytes, elem_bytes, _dptr(out), cap, _dptr(blk_off),
                               _dptr(col_len), _dptr(meta), _dptr(meta) + 8, wsp, need, _stream(stream)))
    nbytes, status = (int(x) for x in meta.cpu())
    check("codag_compress (device status)", status & 0xffffffff)
    return out[:nbytes], blk_off, col_len


def decompress_rlev2_transposed(comp: torch.Tensor, blk_off: torch.Tensor, col_len: torch.Tensor, chunk_bytes: int,
                                elem_bytes: int, read_unit: int, out: torch.Tensor, out_bytes: int | None = None,
                                status: torch.Tensor | None = None, stream=None) -> None:
    """codag_decompress_rlev2_transposed: CODAG's transposed RLE v2 layout (blk_off: n chunk
    offsets, col_len: 32 substream lengths per chunk) into `out`."""
    n = blk_off.numel()
    check("codag_decompress_rlev2_transposed", native.lib().codag_decompress_rlev2_transposed(
        _dptr(comp), comp.numel(), _dptr(blk_off), _dptr(col_len), n, chunk_bytes, elem_bytes, read_unit, _dptr(out),
        out.numel() if out_bytes is None else out_bytes, _dptr(status), _stream(stream)))


def selftest_wait_timeout(wait_cycles: int = 2_000_000) -> int:
    """Runs the bounded-wait self test and returns the status it reports (expect ETIMEOUT)."""
    native.set_wait_limit(wait_cycles)
    try:
        st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        check("codag_selftest_wait_timeout", native.lib().codag_selftest_wait_timeout(_dptr(st), _stream(None)))
        torch.cuda.synchronize()
        return int(st.item())
    finally:
        native.set_wait_limit(2_000_000_000)


# --- host-buffer calls mirroring CODAG's templates ----------------------------------------------
def _h2d(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", non_blocking=False)


def decompress_rlev1_host(blob: np.ndarray, blk_off: np.ndarray, col_len: np.ndarray, chunk_bytes: int = 131072,
                          elem_bytes: int = 8) -> np.ndarray:
    """Host blob [u64 size][streams] in, original bytes out (rle_v1::decompress_gpu_orig)."""
    size = int(blob[:8].view(np.uint64)[0])
    n = col_len.size
    d_comp = _h2d(blob[8:])
    d_off = _h2d(blk_off[:n].astype(np.uint64).view(np.int64))
    d_len = _h2d(col_len[:n].astype(np.uint64).view(np.int64))
    out = torch.empty(size, dtype=torch.uint8, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    decompress_rlev1(d_comp, d_off, d_len, chunk_bytes, elem_bytes, out, size, st)
    _status_error("rlev1", st)
    return out.cpu().numpy()


def decompress_rlev2_host(comp: np.ndarray, blk_off: np.ndarray, col_len: np.ndarray, chunk_bytes: int = 131072,
                          elem_bytes: int = 8) -> np.ndarray:
    """Host streams in, original bytes out; blk_off[n] holds the size (rlev2::decompress_gpu_orig)."""
    n = col_len.size
    size = int(blk_off[n])
    d_comp = _h2d(comp)
    d_off = _h2d(blk_off[:n].astype(np.uint64).view(np.int64))
    d_len = _h2d(col_len.astype(np.uint64).view(np.int64))
    out = torch.empty(size, dtype=torch.uint8, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    decompress_rlev2(d_comp, d_off, d_len, chunk_bytes, elem_bytes, out, size, st)
    _status_error("rlev2", st)
    return out.cpu().numpy()


def decompress_deflate_host(comp: np.ndarray, blk_offset: np.ndarray, chunk_bytes: int = 131072,
                            wrapper_bytes: int = 2) -> np.ndarray:
    """comp.bin + blk_offset.bin ([size, 0, cum...]) in, original bytes out (deflate::decompress_gpu)."""
    size = int(blk_offset[0])
    rel = blk_offset[1:].astype(np.uint64)
    n = rel.size - 1
    d_comp = _h2d(comp)
    d_off = _h2d(rel.view(np.int64))
    out = torch.empty(size, dtype=torch.uint8, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    decompress_deflate(d_comp, d_off, chunk_bytes, out, wrapper_bytes, size, st)
    _status_error("deflate", st)
    return out.cpu().numpy()


def decompress_cudf_deflate_host(file: np.ndarray) -> np.ndarray:
    """A file in CODAG's cuDF-comparison layout (rapids_compressor.py:222-275) in, the n chunks
    decoded out (n x chunk size bytes, as CODAG's base_deflate tool writes them,
    include/base_deflate.h:20-130): the layout is parsed on the host and the streams go to
    codag_decompress_deflate."""
    chunk, data, rel = native.cudf_deflate_layout(file)
    n = rel.size - 1
    d_comp = _h2d(np.ascontiguousarray(file[data:]))
    d_off = _h2d(rel.view(np.int64))
    out = torch.empty(n * chunk, dtype=torch.uint8, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    decompress_deflate(d_comp, d_off, chunk, out, 2, n * chunk, st)
    _status_error("cudf deflate", st)
    return out.cpu().numpy()


# --- host buffers in, host buffer out, with copies and decode overlapped -------------------------
class HostPipeline:
    """Decodes a chunked file from pinned host memory into pinned host memory.

    The chunks are split into `groups`; group g's compressed bytes go up, its chunks are
    decoded and its output comes down on stream g % streams, so the host-to-device copy of
    one group, the decode of another and the device-to-host copy of a third overlap (the
    two copy directions run on separate copy engines).  Device buffers are kept between
    calls and grow as needed.  The streams of a chunk must be laid out in chunk order (as in
    every CODAG layout), so each group's compressed bytes are one contiguous range.
    """

    def __init__(self, codec: int, chunk_bytes: int = 131072, elem_bytes: int = 8, wrapper_bytes: int = 2,
                 groups: int = 8, streams: int = 3, device="cuda"):
        self.codec, self.chunk, self.elem, self.wrapper = codec, chunk_bytes, elem_bytes, wrapper_bytes
        self.groups, self.dev = groups, torch.device(device)
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(streams)]
        self.d_comp = self.d_out = self.d_off = self.d_len = self.d_st = None

    def _grow(self, name, n, dtype):
        t = getattr(self, name)
        if t is None or t.numel() < n:
            t = torch.empty(max(n, 1), dtype=dtype, device=self.dev)
            setattr(self, name, t)
        return t

    def run(self, h_comp: torch.Tensor, h_off: torch.Tensor, h_len: torch.Tensor | None, out_bytes: int,
            h_out: torch.Tensor, off_np: np.ndarray, len_np: np.ndarray | None) -> None:
        """h_comp/h_out pinned uint8; h_off/h_len pinned int64 (RLE: n offsets and lengths;
        Deflate: n+1 offsets, h_len None); off_np/len_np the same metadata on the host, used to
        find each group's byte range.  Returns after the output is in h_out; raises CodagError
        with the per-chunk status attached if a chunk failed."""
        deflate = self.codec == native.DEFLATE
        n = h_off.numel() - 1 if deflate else h_len.numel()
        ch = self.chunk
        d_comp = self._grow("d_comp", h_comp.numel(), torch.uint8)
        d_out = self._grow("d_out", n * ch, torch.uint8)
        d_off = self._grow("d_off", h_off.numel(), torch.int64)
        d_len = self._grow("d_len", 0 if deflate else h_len.numel(), torch.int64)
        d_st = self._grow("d_st", n, torch.int32)
        main = torch.cuda.current_stream(self.dev)
        s0 = self.streams[0]
        s0.wait_stream(main)
        with torch.cuda.stream(s0):
            d_off[:h_off.numel()].copy_(h_off, non_blocking=True)
            if not deflate:
                d_len[:h_len.numel()].copy_(h_len, non_blocking=True)
        meta = torch.cuda.Event()
        meta.record(s0)
        lib = native.lib()
        bounds = np.linspace(0, n, min(self.groups, n) + 1).astype(np.int64)
        for g in range(bounds.size - 1):
            a, b = int(bounds[g]), int(bounds[g + 1])
            s = self.streams[g % len(self.streams)]
            s.wait_event(meta)
            lo = int(off_np[a])
            hi = int(off_np[b]) if deflate else int(off_np[b - 1] + len_np[b - 1])
            hi = min(max(hi, lo), h_comp.numel())
            ob = min(out_bytes, b * ch) - a * ch
            with torch.cuda.stream(s):
                if hi > lo:
                    d_comp[lo:hi].copy_(h_comp[lo:hi], non_blocking=True)
                sp = s.cuda_stream
                if deflate:
                    rc = lib.codag_decompress_deflate(d_comp.data_ptr(), h_comp.numel(), d_off.data_ptr() + 8 * a, b - a,
                                                      ch, self.wrapper, d_out.data_ptr() + a * ch, max(ob, 0),
                                                      d_st.data_ptr() + 4 * a, sp)
                else:
                    fn = lib.codag_decompress_rlev1 if self.codec == native.RLEV1 else lib.codag_decompress_rlev2
                    rc = fn(d_comp.data_ptr(), h_comp.numel(), d_off.data_ptr() + 8 * a, d_len.data_ptr() + 8 * a,
                            b - a, ch, self.elem, d_out.data_ptr() + a * ch, max(ob, 0), d_st.data_ptr() + 4 * a, None,
                            0, sp)
                check("HostPipeline decode", rc)
                if ob > 0:
                    h_out[a * ch:a * ch + ob].copy_(d_out[a * ch:a * ch + ob], non_blocking=True)
        for s in self.streams:
            main.wait_stream(s)
        main.synchronize()
        _status_error("HostPipeline", d_st[:n])


# --- batched persistent plans --------------------------------------------------------------------
class BatchPlan:
    """codag_batch_plan/run/destroy: one persistent launch over many independent chunks."""

    def __init__(self, descs: np.ndarray, warps_per_cta: int | None = None, ring_slots: int | None = None,
                 lut_bits: int | None = None, cta_per_chunk: int = 0, table_global: int = 0):
        """cta_per_chunk=k in 1..4 (warps_per_cta even): Deflate files of k x 256 KiB or more are
        decoded first, each by a pair of warps (symbol decoder and byte expander).  table_global=1:
        the Huffman lookup tables in global memory (read through L1) instead of shared memory."""
        descs = np.ascontiguousarray(descs, dtype=native.CHUNK_DESC_DTYPE)
        self.n = descs.size
        tune = None
        if warps_per_cta is not None:
            d = native.get_tune(native.DEFLATE)
            tune = native.Tune(warps_per_cta, ring_slots or d.ring_slots, lut_bits or d.lut_bits, cta_per_chunk,
                               table_global)
        p = C.c_void_p()
        check("codag_batch_plan", native.lib().codag_batch_plan(descs.ctypes.data, self.n,
                                                                C.byref(tune) if tune is not None else None,
                                                                C.byref(p)))
        self._p = p

    def run(self, comp: torch.Tensor, out: torch.Tensor, status: torch.Tensor | None = None, use_graph: bool = False,
            stream=None) -> None:
        check("codag_batch_run", native.lib().codag_batch_run(self._p, _dptr(comp), comp.numel(), _dptr(out),
                                                              out.numel(), _dptr(status), int(use_graph),
                                                              _stream(stream)))

    def close(self) -> None:
        if self._p:
            native.lib().codag_batch_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchHostPipeline:
    """Decodes a packed set of independent files (codag_batch_plan descriptors) from pinned host
    memory into pinned host memory, one set per step, with the steps pipelined.

    Two device buffer pairs alternate between steps, and three streams carry the stages: step
    i's host-to-device copy runs while step i-1 decodes (one persistent launch, replayed from a
    CUDA graph captured per buffer pair) and step i-2's output goes back to the host, so a
    stream of steps runs at the pace of the slowest stage rather than the sum of the three.
    Events order the reuse of a buffer pair: its input is overwritten only after the launch
    that read it, its output only after the copy that read it.  Bytes between and after the
    files' outputs come back as zeros."""

    def __init__(self, descs: np.ndarray, comp_bytes: int, out_bytes: int, shape: tuple | None = None,
                 device="cuda", buffers: int = 2):
        descs = np.ascontiguousarray(descs, dtype=native.CHUNK_DESC_DTYPE)
        self.n = descs.size
        self.dev = torch.device(device)
        self.comp_bytes, self.out_bytes = comp_bytes, out_bytes
        # one plan per buffer pair, so that each keeps the graph captured for its pointers
        self.bufs = [dict(plan=BatchPlan(descs, *(shape or ())),
                          comp=torch.empty(max(comp_bytes, 1), dtype=torch.uint8, device=self.dev),
                          out=torch.zeros(max(out_bytes, 1), dtype=torch.uint8, device=self.dev),
                          st=torch.zeros(max(self.n, 1), dtype=torch.int32, device=self.dev),
                          decoded=None, copied=None) for _ in range(buffers)]
        self.s_in, self.s_dec, self.s_out = (torch.cuda.Stream(device=self.dev) for _ in range(3))

    h2d_bytes = property(lambda self: self.comp_bytes)
    d2h_bytes = property(lambda self: self.out_bytes)

    def run(self, steps, use_graph: bool = True) -> None:
        """steps: (h_comp, h_out) pairs of pinned uint8 tensors, one per step.  Returns after
        every output is in its h_out; raises CodagError with the per-file status if a file
        failed in any step."""
        main = torch.cuda.current_stream(self.dev)
        for s in (self.s_in, self.s_dec, self.s_out):
            s.wait_stream(main)
        bad = []
        for i, (h_comp, h_out) in enumerate(steps):
            b = self.bufs[i % len(self.bufs)]
            if b["decoded"] is not None:
                self.s_in.wait_event(b["decoded"])   # the previous launch on this pair read its input
            with torch.cuda.stream(self.s_in):
                b["comp"].copy_(h_comp[:self.comp_bytes], non_blocking=True)
            ready = torch.cuda.Event()
            ready.record(self.s_in)
            self.s_dec.wait_event(ready)
            if b["copied"] is not None:
                self.s_dec.wait_event(b["copied"])   # the previous copy-out of this pair is done
            with torch.cuda.stream(self.s_dec):
                b["plan"].run(b["comp"], b["out"], b["st"], use_graph=use_graph, stream=self.s_dec)
                bad.append((b["st"] != 0).any())
            b["decoded"] = torch.cuda.Event()
            b["decoded"].record(self.s_dec)
            self.s_out.wait_event(b["decoded"])
            with torch.cuda.stream(self.s_out):
                h_out[:self.out_bytes].copy_(b["out"], non_blocking=True)
            b["copied"] = torch.cuda.Event()
            b["copied"].record(self.s_out)
        for s in (self.s_in, self.s_dec, self.s_out):
            main.wait_stream(s)
        main.synchronize()
        if any(bool(x) for x in bad):
            for b in self.bufs:
                _status_error("BatchHostPipeline", b["st"])

    def close(self) -> None:
        for b in self.bufs:
            b["plan"].close()


@dataclass
class ChunkSet:
    """Independent compressed chunks packed into one buffer, with their descriptors."""
    comp: np.ndarray         # all streams, each starting on a 16-byte boundary
    descs: np.ndarray        # CHUNK_DESC_DTYPE
    out_bytes: int           # output buffer size (outputs start on 256-byte boundaries)


def pack_chunks(streams: list[np.ndarray], codecs: list[int], elem_bytes: list[int], out_lens: list[int],
                wrapper_bytes: int = 2) -> ChunkSet:
    """Packs independently compressed streams into one buffer and builds their descriptors."""
    n = len(streams)
    descs = np.zeros(n, dtype=native.CHUNK_DESC_DTYPE)
    comp_off = 0
    out_off = 0
    offs = []
    for i, s in enumerate(streams):
        offs.append(comp_off)
        descs[i]["comp_off"] = comp_off
        descs[i]["comp_len"] = s.size
        descs[i]["out_off"] = out_off
        descs[i]["out_len"] = out_lens[i]
        descs[i]["codec"] = codecs[i]
        descs[i]["elem_bytes"] = elem_bytes[i]
        descs[i]["wrapper_bytes"] = wrapper_bytes if codecs[i] == native.DEFLATE else 0
        comp_off += (s.size + 15) // 16 * 16
        out_off += (out_lens[i] + 255) // 256 * 256
    comp = np.zeros(comp_off, dtype=np.uint8)
    for o, s in zip(offs, streams):
        comp[o:o + s.size] = s
    return ChunkSet(comp=comp, descs=descs, out_bytes=out_off)
