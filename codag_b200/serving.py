"""Serving loop: decompression requests of different sizes arrive over time; the loop keeps
their compressed files and output buffers resident in HBM, admits requests while an output
budget has room, and decodes admitted requests in persistent launches that overlap on the
device (continuous batching).

CODAG itself has no serving layer: its host templates decode one file per call and
synchronise the device (include/rlev1/rlev1.h:419-592, include/rlev2/decoder_trans.h:57-133,
include/zlib/zlib.h:1583-1700).  This module builds the request path on the chunk
descriptors of codag_batch_launch:

  arrival -> waiting (FIFO) -> admitted (output region granted by the Arena)
          -> launched (its chunks join the next launch, on one of `slots` streams)
          -> decoded (the launch's event completed: latency = now - arrival)
          -> verified (device compare with the expected bytes) -> output region freed.

A launch takes every admitted request that has not been launched yet, so requests that
arrive while earlier launches run join the next launch as soon as a stream slot and output
memory are free, and up to `slots` launches overlap on the GPU.
"""
from __future__ import annotations

import bisect
import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import native

CH = 131072
DEFLATE, RLEV1, RLEV2 = native.DEFLATE, native.RLEV1, native.RLEV2


class Arena:
    """First-fit allocator of output regions in [0, capacity), 256-byte aligned."""

    ALIGN = 256

    def __init__(self, capacity: int):
        self.capacity = capacity // self.ALIGN * self.ALIGN
        self.free_list = [(0, self.capacity)]  # sorted, disjoint, coalesced (start, size)
        self.used = {}

    def alloc(self, nbytes: int):
        n = max(self.ALIGN, (nbytes + self.ALIGN - 1) // self.ALIGN * self.ALIGN)
        for k, (s, z) in enumerate(self.free_list):
            if z >= n:
                if z == n:
                    del self.free_list[k]
                else:
                    self.free_list[k] = (s + n, z - n)
                self.used[s] = n
                return s
        return None

    def free(self, off: int) -> None:
        n = self.used.pop(off)
        fl = self.free_list
        k = bisect.bisect_left(fl, (off, 0))
        fl.insert(k, (off, n))
        if k + 1 < len(fl) and fl[k][0] + fl[k][1] == fl[k + 1][0]:  # merge with the next
            fl[k] = (fl[k][0], fl[k][1] + fl[k + 1][1])
            del fl[k + 1]
        if k > 0 and fl[k - 1][0] + fl[k - 1][1] == fl[k][0]:  # merge with the previous
            fl[k - 1] = (fl[k - 1][0], fl[k - 1][1] + fl[k][1])
            del fl[k]

    @property
    def in_use(self) -> int:
        return sum(self.used.values())


@dataclass
class PoolFile:
    """One compressed file of the request pool, in CODAG's chunk layout (128 KiB chunks)."""
    codec: int
    elem: int
    size: int              # original bytes
    descs: np.ndarray      # per chunk: comp_off absolute in the pool buffer, out_off relative
    src_off: int           # where the original bytes sit in the pool's source buffer

    @property
    def out_alloc(self) -> int:
        return int(self.descs.size) * CH

    @property
    def cost(self) -> np.ndarray:
        d = self.descs
        w = np.where(d["codec"] == DEFLATE, 8, 1).astype(np.int64)
        return w * d["comp_len"].astype(np.int64) + d["out_len"].astype(np.int64) // np.where(w == 8, 1, 4)


@dataclass
class Pool:
    comp: np.ndarray       # all compressed files
    src: np.ndarray        # all original files (the expected outputs)
    files: list


def build_pool(n_files: int, seed: int, min_bytes: int = 64 << 10, max_bytes: int = 256 << 20,
               mix=(0.4, 0.3, 0.3)) -> Pool:
    """Seeded request files: size log-uniform in [min_bytes, max_bytes] (multiple of 8);
    Deflate (Zipf text, zlib level 6) / RLE v1 (u64) / RLE v2 (int64) with probabilities `mix`;
    each compressed in CODAG's layout with 128 KiB chunks."""
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(min_bytes), np.log(max_bytes), n_files))).astype(np.int64) // 8 * 8
    codecs = rng.choice([DEFLATE, RLEV1, RLEV2], size=n_files, p=list(mix))
    comps, srcs, files = [], [], []
    c_base = s_base = 0
    for k in range(n_files):
        size, codec = int(sizes[k]), int(codecs[k])
        fseed = seed * 1000 + k
        n = (size + CH - 1) // CH
        d = np.zeros(n, dtype=native.CHUNK_DESC_DTYPE)
        if codec == DEFLATE:
            data = native.gen_text(size, fseed)
            comp, bo, _ = native.encode_deflate(data, CH, 6)
            d["comp_off"] = c_base + bo[1:1 + n]
            d["comp_len"] = np.diff(bo[1:2 + n])
            d["wrapper_bytes"] = 2
            d["elem_bytes"] = 1
        else:
            gen = native.gen_rlev1_column if codec == RLEV1 else native.gen_rlev2_column
            data = gen(size // 8, fseed, 8)
            if codec == RLEV1:
                blob, off, ln = native.encode_rlev1(data, CH, 8)
                comp, base = blob, 8
            else:
                comp, off, ln = native.encode_rlev2(data, CH, 8)
                base = 0
            d["comp_off"] = c_base + base + off[:n]
            d["comp_len"] = ln[:n]
            d["elem_bytes"] = 8
        d["codec"] = codec
        d["out_off"] = np.arange(n, dtype=np.uint64) * CH
        d["out_len"] = CH  # the tail chunk decodes to a whole chunk (CODAG pads the input)
        pad = (-comp.size) % 16
        comps.append(comp)
        if pad:
            comps.append(np.zeros(pad, np.uint8))
        srcs.append(data)
        files.append(PoolFile(codec, 1 if codec == DEFLATE else 8, size, d, s_base))
        c_base += comp.size + pad
        s_base += data.size
    return Pool(np.concatenate(comps), np.concatenate(srcs), files)


@dataclass
class Request:
    rid: int
    file: int
    t_arrival: float
    out_off: int = -1
    t_admit: float = 0.0
    t_launch: float = 0.0
    t_done: float = 0.0
    ok: bool | None = None


def poisson_arrivals(rate: float, duration: float, n_files: int, seed: int):
    """(t_arrival, file index) pairs of a Poisson process of `rate` per second."""
    rng = np.random.default_rng(seed)
    n = int(rate * duration * 1.5) + 16
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    t = t[t < duration]
    return list(zip(t.tolist(), rng.integers(0, n_files, t.size).tolist()))


# Launch shapes (warps_per_cta, ring_slots, lut_bits, cta_per_chunk) tried by tune_server.  The
# per-file Deflate default (2 warps per CTA) holds too few warps per SM for a loop whose launches
# carry thousands of 128 KiB chunks: 36.6 GB/s against 60.0 GB/s with 8 warps per CTA at
# 2000 requests per second on one B200.
SERVE_SHAPES = [(w, 4, lb, 0) for w in (2, 4, 8) for lb in (9, 10)]


def tune_server(srv: "Server", n_requests: int = 96, seed: int = 7, use_cache: bool = True):
    """Times a burst of n_requests requests that all arrive at once (the loop saturated) for each
    shape of SERVE_SHAPES, installs the fastest on `srv` and returns it; the result is cached per
    GPU model next to the decoders' (codag_b200.tuning)."""
    from . import tuning
    hit = tuning.load_cached(-1, "serve") if use_cache else None
    if hit:
        srv.tune = native.Tune(*hit, 0)
        return tuple(hit)
    rng = np.random.default_rng(seed)
    burst = [(0.0, int(f)) for f in rng.integers(0, len(srv.pool.files), n_requests)]
    best, best_t = None, None
    for shape in SERVE_SHAPES:
        srv.tune = native.Tune(*shape, 0)
        t0 = time.perf_counter()
        reqs = srv.run(burst)
        t = time.perf_counter() - t0
        if not all(r.ok for r in reqs):
            raise RuntimeError(f"serving shape {shape}: a request did not decode exactly")
        if best_t is None or t < best_t:
            best, best_t = shape, t
    srv.tune = native.Tune(*best, 0)
    tuning.store_cached(-1, "serve", best)
    return best


def admission_capacity(budget_bytes: int, free_bytes: int, reserve_bytes: int) -> int:
    """Output bytes the server may hold for admitted requests: the configured budget, but no
    more than the device memory that is free once the request pool is resident, less a
    reserve for the per-launch buffers and the verification copies."""
    return max(0, min(int(budget_bytes), int(free_bytes) - int(reserve_bytes)))


class Server:
    """The request loop on one GPU (see the module docstring).

    Requests are admitted by free device memory: the output arena is sized, after the pool
    is resident, to the smaller of the budget and the device's free memory less a reserve
    (admission_capacity), and a request waits until the arena grants its output region."""

    RESERVE = 2 << 30  # per-launch descriptor/status buffers and allocator slack

    def __init__(self, pool: Pool, budget_bytes: int, slots: int = 4, tune=None, device="cuda",
                 keep_outputs: bool = False, max_chunks_per_launch: int | None = None):
        import torch
        self.torch = torch
        self.pool = pool
        self.dev = torch.device(device)
        self.d_comp = torch.from_numpy(pool.comp).to(self.dev)
        self.d_src = torch.from_numpy(pool.src).to(self.dev)
        free, _ = torch.cuda.mem_get_info(self.dev)
        self.budget = budget_bytes
        self.arena = Arena(admission_capacity(budget_bytes, free, self.RESERVE))
        if self.arena.capacity < CH:
            raise MemoryError(f"no device memory left for request outputs ({free} bytes free)")
        self.d_out = torch.empty(self.arena.capacity, dtype=torch.uint8, device=self.dev)
        self.tune = native.Tune(*tune, 0) if tune else None
        cap = max_chunks_per_launch or max(1, self.arena.capacity // CH)
        self.cap = cap
        self.slots = []
        for _ in range(slots):
            self.slots.append(dict(
                stream=torch.cuda.Stream(device=self.dev),
                d_descs=torch.empty(cap * 32, dtype=torch.uint8, device=self.dev),
                d_order=torch.empty(cap, dtype=torch.int32, device=self.dev),
                d_queue=torch.zeros(1, dtype=torch.int32, device=self.dev),
                d_status=torch.zeros(cap, dtype=torch.int32, device=self.dev),
                h_descs=torch.empty(cap * 32, dtype=torch.uint8).pin_memory(),
                h_order=torch.empty(cap, dtype=torch.int32).pin_memory(),
                busy=None))
        self.verify_stream = torch.cuda.Stream(device=self.dev)
        self.keep_outputs = keep_outputs
        self.outputs = {}
        self.launches = 0
        self.chunks_launched = 0

    # -- one launch over the given requests on a free slot ----------------------------------
    def _launch(self, slot, reqs) -> None:
        torch = self.torch
        parts = []
        for r in reqs:
            d = self.pool.files[r.file].descs.copy()
            d["out_off"] += np.uint64(r.out_off)
            parts.append(d)
        descs = np.concatenate(parts)
        n = descs.size
        cost = np.concatenate([self.pool.files[r.file].cost for r in reqs])
        order = np.argsort(-cost, kind="stable").astype(np.int32)
        hd = slot["h_descs"].numpy()[:n * 32]
        hd[:] = descs.view(np.uint8)
        slot["h_order"].numpy()[:n] = order
        s = slot["stream"]
        with torch.cuda.stream(s):
            slot["d_descs"][:n * 32].copy_(slot["h_descs"][:n * 32], non_blocking=True)
            slot["d_order"][:n].copy_(slot["h_order"][:n], non_blocking=True)
            native.check("codag_batch_launch", native.lib().codag_batch_launch(
                slot["d_descs"].data_ptr(), slot["d_order"].data_ptr(), n, slot["d_queue"].data_ptr(),
                None if self.tune is None else native.C.byref(self.tune), self.d_comp.data_ptr(),
                self.d_comp.numel(), self.d_out.data_ptr(), self.d_out.numel(), slot["d_status"].data_ptr(),
                s.cuda_stream))
            ev = torch.cuda.Event()
            ev.record(s)
        slot["busy"] = (ev, reqs, n)
        self.launches += 1
        self.chunks_launched += n

    def _verify(self, slot, reqs, n):
        """Queues the checks of a finished launch; returns (event, flags, reqs)."""
        torch = self.torch
        vs = self.verify_stream
        vs.wait_stream(slot["stream"])
        flags = []
        with torch.cuda.stream(vs):
            bad_status = (slot["d_status"][:n] != 0).any()
            for r in reqs:
                f = self.pool.files[r.file]
                got = self.d_out[r.out_off:r.out_off + f.size]
                want = self.d_src[f.src_off:f.src_off + f.size]
                flags.append((got != want).any())
                if self.keep_outputs:
                    self.outputs[r.rid] = got.to("cpu", non_blocking=False)
            ev = torch.cuda.Event()
            ev.record(vs)
        return ev, bad_status, flags, reqs

    def run(self, arrivals, time_limit: float | None = None):
        """Serves `arrivals` ((t, file) pairs, t in seconds from now) and returns the requests."""
        reqs = [Request(i, f, t) for i, (t, f) in enumerate(arrivals)]
        waiting = collections.deque()
        admitted = []
        verifying = []
        done = []
        nxt = 0
        t0 = time.perf_counter()
        while len(done) < len(reqs):
            now = time.perf_counter() - t0
            if time_limit is not None and now > time_limit:
                break
            progressed = False
            while nxt < len(reqs) and reqs[nxt].t_arrival <= now:
                waiting.append(reqs[nxt])
                nxt += 1
            while waiting:  # FIFO admission while the output budget has room
                r = waiting[0]
                off = self.arena.alloc(self.pool.files[r.file].out_alloc)
                if off is None:
                    break
                r.out_off, r.t_admit = off, now
                admitted.append(waiting.popleft())
                progressed = True
            for slot in self.slots:  # completed launches
                if slot["busy"] is not None and slot["busy"][0].query():
                    ev, rs, n = slot["busy"]
                    t = time.perf_counter() - t0
                    for r in rs:
                        r.t_done = t
                    verifying.append(self._verify(slot, rs, n))
                    slot["busy"] = None
                    progressed = True
            for slot in self.slots:  # launch the admitted requests on a free slot
                if not admitted:
                    break
                if slot["busy"] is None:
                    take, total = [], 0
                    while admitted and total + self.pool.files[admitted[0].file].descs.size <= self.cap:
                        total += self.pool.files[admitted[0].file].descs.size
                        take.append(admitted.pop(0))
                    if not take:
                        raise RuntimeError("request larger than one launch's capacity")
                    t = time.perf_counter() - t0
                    for r in take:
                        r.t_launch = t
                    self._launch(slot, take)
                    progressed = True
            still = []
            for item in verifying:  # finished checks free their output regions
                ev, bad_status, flags, rs = item
                if ev.query():
                    bad = bool(bad_status.item())
                    for r, f in zip(rs, flags):
                        r.ok = (not bad) and not bool(f.item())
                        self.arena.free(r.out_off)
                        done.append(r)
                    progressed = True
                else:
                    still.append(item)
            verifying = still
            if not progressed:
                time.sleep(20e-6)
        self.torch.cuda.synchronize(self.dev)
        return reqs


def summarize(reqs, pool: Pool, duration: float):
    """Throughput and latency of the completed requests."""
    fin = [r for r in reqs if r.t_done > 0]
    lat = np.array([r.t_done - r.t_arrival for r in fin]) if fin else np.zeros(1)
    nbytes = sum(pool.files[r.file].size for r in fin)
    span = max((r.t_done for r in fin), default=duration)
    return {"requests": len(reqs), "completed": len(fin), "bit_exact": all(r.ok for r in fin) and len(fin) == len(reqs),
            "gbs": nbytes / max(span, 1e-9) / 1e9, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
            "bytes": int(nbytes)}
