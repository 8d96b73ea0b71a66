"""Autotuner for the decoders' launch shape.

Per codec it times every supported combination of
  warps_per_cta  chunks decoded by one CTA (one warp per chunk): 1, 2, 4, 8
  ring_slots     depth of the TMA input ring in 1 KiB slots: 4, 8 (2 also for Deflate)
  lut_bits       primary Huffman table width (Deflate only): 9, 10, 11
  cta_per_chunk  RLE only: a whole CTA of 4 or 8 warps per chunk instead of one warp
on a resident sample of the caller's chunks, keeps the fastest, installs it with
codag_set_tune and caches it in a JSON file keyed by GPU name and codec, so later runs
on the same kind of GPU skip the search.  Batched plans take their shape the same way
(codag_batch_plan's tune argument), searched over a sample of the batch.
"""
from __future__ import annotations

import itertools
import json
import os
from pathlib import Path

import torch

from . import native

CACHE = Path(os.environ.get("CODAG_TUNE_CACHE", Path(__file__).resolve().parent / "tune_cache.json"))


def candidates(codec: int):
    warps = (1, 2, 4, 8)
    if codec == native.DEFLATE:
        # one warp per chunk, or a decoder and an expander warp per chunk (1, 2 or 4 pairs per CTA)
        return (list(itertools.product(warps, (2, 4, 8), (9, 10, 11), (0,))) +
                list(itertools.product((2, 4, 8), (4,), (9, 10), (1,))))
    # one warp per chunk, or one CTA of 4 or 8 warps per chunk
    return list(itertools.product(warps, (4, 8), (10,), (0,))) + [(4, 4, 10, 1), (8, 4, 10, 1)]


def batch_candidates():
    """Launch shapes of the batched kernel: (warps_per_cta, ring_slots, lut_bits, cta_per_chunk,
    table_global).  RLE files need rings of at least 4 slots; with cta_per_chunk = k the Deflate
    files of at least k x 256 KiB go to warp pairs (so the warp count is even); table_global
    places the Huffman lookup tables in global memory (through L1) rather than shared memory."""
    return (list(itertools.product((2, 4, 8), (4, 8), (9, 10, 11), (0,), (0, 1))) +
            list(itertools.product((4, 8), (4,), (9, 10, 11), (1, 2, 3), (0,))))


def _key(codec: int, tag: str) -> str:
    return f"{torch.cuda.get_device_name()}|codec{codec}|{tag}"


def load_cached(codec: int, tag: str = "plain"):
    try:
        return json.loads(CACHE.read_text()).get(_key(codec, tag))
    except (OSError, ValueError):
        return None


def store_cached(codec: int, tag: str, shape) -> None:
    try:
        data = json.loads(CACHE.read_text())
    except (OSError, ValueError):
        data = {}
    data[_key(codec, tag)] = list(shape)
    # written whole and renamed into place: ranks of one job may store at the same time
    tmp = CACHE.with_name(f"{CACHE.name}.{os.getpid()}.tmp")
    try:
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        os.replace(tmp, CACHE)
    except OSError:
        pass


def time_call(fn, reps: int = 3) -> float:
    """Median device time (s) of fn() on the current stream after one warm-up call."""
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b) / 1e3)
    ts.sort()
    return ts[len(ts) // 2]


def autotune(codec: int, run, tag: str = "plain", use_cache: bool = True, verbose: bool = False):
    """Search the launch shape of `codec` with `run()` (one decode of a resident sample),
    install the winner and return (shape, {shape: seconds})."""
    if use_cache:
        hit = load_cached(codec, tag)
        if hit:
            native.set_tune(codec, *hit)
            return tuple(hit), {}
    results = {}
    for shape in candidates(codec):
        native.set_tune(codec, *shape)
        results[shape] = time_call(run)
        if verbose:
            print(f"codec {codec} shape {shape}: {results[shape] * 1e3:.3f} ms", flush=True)
    best = min(results, key=results.get)
    native.set_tune(codec, *best)
    store_cached(codec, tag, best)
    return best, results
