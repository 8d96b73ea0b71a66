"""`bench.py --workload batched` (driver module beside bench.py): CODAG's batched configuration on one GPU per rank.

Workload: 20,000 independently compressed files, decompressed size log-uniform 4 KiB-1 MiB
(multiple of 8), 40% Deflate (Zipf text, zlib level 6), 30% RLE v1, 30% RLE v2, RLE values
u32 or u64 (50/50); about 3.8 GB decompressed.  Seeded per rank (weak scaling).

Two ways of decoding the same resident set are timed:
  batched   one persistent launch over all files (codag_batch_run, replayed from a CUDA
            graph), launch shape from the autotuner;
  per-file  one C-ABI call per file, in order on one stream -- the only way CODAG's kernels,
            which take one uniform chunk size per launch, can decode such a set.  Its full
            run takes minutes (each Deflate file is decoded by one warp), so it is timed on a
            stratified sample of the files; its GB/s is the sample's bytes over its time.
Both outputs are checked byte for byte against the source slices.
"""
from __future__ import annotations

import json
import time

import numpy as np

from bench import METRIC, ncu_traffic

SEED = 20260104


def _alg_bytes(ms) -> int:
    return int(ms.descs["comp_len"].astype(np.int64).sum() + ms.in_len.astype(np.int64).sum())


def _cpu(ms, files):
    """Oracle (OpenMP over files) on the given files; returns (GB/s, threads)."""
    from oracle import oracle_py
    d = ms.descs[files]
    out_off = np.cumsum(np.concatenate([[0], d["out_len"].astype(np.uint64)[:-1]])).astype(np.uint64)
    out = np.empty(int(d["out_len"].astype(np.int64).sum()), np.uint8)
    a = (ms.comp, d["comp_off"], d["comp_len"], out, out_off, d["out_len"], d["out_len"], d["codec"], d["elem_bytes"],
         d["wrapper_bytes"])
    oracle_py.decode_batch(*a)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        st = oracle_py.decode_batch(*a)
        ts.append(time.perf_counter() - t0)
        assert not st.any()
    return out.size / float(np.median(ts)) / 1e9, oracle_py.max_threads()


def _desc(n_files: int) -> str:
    return (f"{n_files} files, log-uniform 4 KiB-1 MiB, 40/30/30 Deflate/RLE v1/RLE v2, RLE u32/u64 50/50, "
            "each file one stream")


def _config(ms, args, world: int) -> dict:
    """The workload description shared by both arms."""
    by_codec = {name: int((ms.codecs == c).sum()) for name, c in (("deflate", 2), ("rlev1", 0), ("rlev2", 1))}
    return {"workload": "batched: " + _desc(ms.n), "files_by_codec": by_codec,
            "out_bytes": int(ms.in_len.astype(np.int64).sum()), "comp_bytes": int(ms.descs["comp_len"].astype(np.int64).sum()),
            "l2": "inputs larger than L2 (no flush)", "parallelism": f"{world} GPU(s), one set per GPU"}


def run_reference(args) -> None:
    """CPU decoder of the path (the oracle, OpenMP over files) on the whole set per step: the
    same files, codecs and bytes as our arm.  Loads the format library and the oracle only."""
    from codag_b200 import batched
    ms = batched.make_mixed_set(args.n_files or 20_000, seed=SEED)
    files = np.arange(ms.n)
    from oracle import oracle_py
    d = ms.descs[files]
    out_off = np.cumsum(np.concatenate([[0], d["out_len"].astype(np.uint64)[:-1]])).astype(np.uint64)
    out = np.empty(int(d["out_len"].astype(np.int64).sum()), np.uint8)
    a = (ms.comp, d["comp_off"], d["comp_len"], out, out_off, d["out_len"], d["out_len"], d["codec"], d["elem_bytes"],
         d["wrapper_bytes"])
    for _ in range(args.warmup):
        oracle_py.decode_batch(*a)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = oracle_py.decode_batch(*a)
    dt = time.perf_counter() - t0
    assert not st.any()
    ok = all(np.array_equal(out[int(o):int(o) + int(ln)], ms.src[int(s):int(s) + int(ln)])
             for o, ln, s in zip(out_off, d["out_len"], ms.in_off[files]))
    gbs = args.steps * out.size / dt / 1e9
    threads = oracle_py.max_threads()
    sample = f"all {ms.n} files per step, {out.size / 1e6:.0f} MB decompressed"
    print(json.dumps({
        "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generators standing in for CODAG's datasets)",
        "config": _config(ms, args, 1),
        "bit_exact": bool(ok),
        "impl": "reference",
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
        flush=True)


def main(args, rank: int, world: int, local: int):
    """Times the batched and the per-file path on this rank's set; returns the JSON line on
    rank 0 (None elsewhere)."""
    import torch
    import torch.distributed as dist
    from codag_b200 import api, batched, tuning
    from bench import Clocks, peaks

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    ms = batched.make_mixed_set(args.n_files or 20_000, seed=SEED + rank)
    total_out = int(ms.in_len.astype(np.int64).sum())
    alg = _alg_bytes(ms)
    d_comp = torch.from_numpy(ms.comp).to(dev)
    d_out = torch.zeros(ms.out_bytes, dtype=torch.uint8, device=dev)
    d_st = torch.zeros(ms.n, dtype=torch.int32, device=dev)
    want = torch.from_numpy(ms.expected()).to(dev)

    # launch shape: autotuner over (warps_per_cta, ring_slots, lut_bits), cached per GPU
    shape = None
    if args.tune:
        shape = tuple(int(x) for x in args.tune.split(","))
    elif args.autotune:
        hit = tuning.load_cached(-1, "batch") if args.autotune == "cached" else None
        if hit:
            shape = tuple(hit)
        else:
            res = {}
            for cand in tuning.batch_candidates():
                p = api.BatchPlan(ms.descs, *cand)
                res[cand] = tuning.time_call(lambda: p.run(d_comp, d_out, d_st, use_graph=False), reps=2)
                p.close()
                if rank == 0 and args.verbose:
                    print(f"batch shape {cand}: {res[cand] * 1e3:.2f} ms", flush=True)
            shape = min(res, key=res.get)
            tuning.store_cached(-1, "batch", shape)
    plan = api.BatchPlan(ms.descs, *shape) if shape else api.BatchPlan(ms.descs)

    for _ in range(max(args.warmup, 3)):
        plan.run(d_comp, d_out, d_st, use_graph=True)
    torch.cuda.synchronize()
    ok = int((d_st != 0).sum().item()) == 0 and bool(torch.equal(d_out, want))

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(local) if rank == 0 else None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        plan.run(d_comp, d_out, d_st, use_graph=True)
        ev[i][1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    elapsed = t0.elapsed_time(t1) / 1e3
    per_launch = float(np.mean([a.elapsed_time(b) for a, b in ev])) / 1e3
    if world > 1:
        t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())

    # per-file path on a stratified sample (same resident buffers)
    sample = batched.stratified_sample(ms, args.per_file_sample)
    pf = batched.PerFileDecoder(ms, d_comp, d_out, dev)
    d_out.zero_()
    pf.run(sample[:8], stream)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    pf.run(sample, stream)
    p1.record(stream)
    torch.cuda.synchronize()
    pf_t = p0.elapsed_time(p1) / 1e3
    pf_bytes = int(ms.in_len[sample].astype(np.int64).sum())
    for i in sample:
        o, ln = int(ms.descs["out_off"][i]), int(ms.in_len[i])
        ok = ok and bool(torch.equal(d_out[o:o + ln], want[o:o + ln]))
    ok = ok and int((pf.d_st[torch.from_numpy(sample).to(dev)] != 0).sum().item()) == 0

    # e2e: pinned host streams in, decoded files out, every step, through the public host-to-host
    # API (api.BatchHostPipeline: each step's H2D copy, launch and D2H copy, with consecutive
    # steps overlapped on three streams over two device buffer pairs); every copy is inside
    # the timed region
    h_comp = torch.from_numpy(ms.comp).pin_memory()
    h_outs = [torch.empty(ms.out_bytes, dtype=torch.uint8).pin_memory() for _ in range(2)]
    pipe = api.BatchHostPipeline(ms.descs, ms.comp.size, ms.out_bytes, shape=shape, device=dev)
    e_steps = max(4, min(args.steps, 8))
    pipe.run([(h_comp, h_outs[k % 2]) for k in range(2)])  # captures the graphs of both buffer pairs
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pipe.run([(h_comp, h_outs[k % 2]) for k in range(e_steps)])
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_t = e0.elapsed_time(e1) / 1e3
    if world > 1:
        t = torch.tensor([e2e_t], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
    want_h = want.cpu()
    ok = ok and all(bool(torch.equal(h, want_h)) for h in h_outs)
    e2e_h2d, e2e_d2h = pipe.h2d_bytes, pipe.d2h_bytes
    pipe.close()
    del pipe
    # whole-job bytes: every rank decodes its own seeded set, so sizes differ between ranks
    job_out, job_h2d, job_d2h = total_out, int(e2e_h2d), int(e2e_d2h)
    if world > 1:
        okt = torch.tensor([0 if ok else 1], dtype=torch.int32, device=dev)
        dist.all_reduce(okt)
        ok = int(okt.item()) == 0
        jt = torch.tensor([total_out, job_h2d, job_d2h], dtype=torch.int64, device=dev)
        dist.all_reduce(jt)
        job_out, job_h2d, job_d2h = (int(x) for x in jt.tolist())
    if rank != 0:
        plan.close()
        return None

    peak, peak_kind = peaks()
    achieved = alg / per_launch / 1e9
    value = job_out * args.steps / elapsed / 1e9
    pf_gbs = pf_bytes / pf_t / 1e9
    cpu = None
    if world == 1:
        gbs, threads = _cpu(ms, batched.stratified_sample(ms, 2000))
        cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": "2000 of the files (stratified by codec and size), median of 3"}
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(elapsed / args.steps * 1e3, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generators standing in for CODAG's datasets)",
        "config": {**_config(ms, args, world), "graph": True, "tune": list(shape) if shape else None},
        "bit_exact": ok,
        "plain_per_file": {"value": round(pf_gbs, 4), "unit": "GB/s", "files_timed": int(sample.size),
                           "bytes_timed": pf_bytes, "seconds": round(pf_t, 4),
                           "how": "one C-ABI call per file, in order on one stream, stratified sample"},
        "batched_over_plain": round(total_out * args.steps / elapsed / 1e9 / pf_gbs, 1),
        "e2e": {"value": round(job_out * e_steps / e2e_t / 1e9, 2), "unit": "GB/s",
                "h2d_bytes_per_step": job_h2d, "d2h_bytes_per_step": job_d2h,
                "how": f"api.BatchHostPipeline, {e_steps} steps, H2D/launch/D2H of consecutive steps overlapped, "
                       "pinned host buffers"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": ncu_traffic("batched") if (args.n_files or 20_000) == 20_000 else None,
                     "peak_kind": peak_kind, "kernel": "k_batch", "alg_bytes_per_launch": alg, "launch_ms": round(per_launch * 1e3, 4)},
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    plan.close()
    del d_comp, d_out, d_st, want, pf
    torch.cuda.empty_cache()
    return line
