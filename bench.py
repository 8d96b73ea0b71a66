#!/usr/bin/env python
"""Benchmark of the chunked decompressors on one node (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|rlev2|rlev1|rlev1x128|deflate|serving] [--no-extras]

Default workload (batched): CODAG's batched configuration -- 20,000 independently compressed
files, decompressed size log-uniform 4 KiB-1 MiB, 40% Deflate / 30% RLE v1 / 30% RLE v2, RLE
values u32 or u64 (50/50), about 3.8 GB decompressed -- decoded per step by one persistent
launch replayed from a CUDA graph (`value`), and compared with the plain per-file path (one
C-ABI call per file, the only way CODAG's kernels can decode such a set): `plain_per_file`
and `batched_over_plain`.  With one GPU the same line also carries, under `configs`, the
per-codec configurations (RLE v2 1 GiB, RLE v1 8 MiB and 1 GiB, Deflate 1 GiB text) with
their own roofline, e2e and CPU baseline, and a short serving sweep (Poisson arrivals at two
rates, p50/p99 latency).  Inputs exceed the 126 MB L2, so no flush is needed between steps.
N>1: every rank decodes its own instance (weak scaling, no collective on the data path;
timing is the max over ranks); the extra configurations run at N=1 only.

`value` is decompressed GB/s with inputs resident in HBM; `e2e` is the same metric through the
host-buffer API with every host-to-device copy of the inputs and device-to-host copy of the
outputs in the timed region; `roofline` relates the decode kernel's algorithmic bytes
(compressed bytes read + decompressed bytes written) to the measured HBM copy bandwidth;
`cpu_baseline` is the CPU decoder (OpenMP over chunks or files) on a bounded sample.
--impl reference times that CPU decoder on the whole workload as the reference arm (CODAG's
own decoders exist only as GPU kernels; the oracle restates them on the CPU).  The reference
arm loads only the format library (libcodag_fmt.so) and the oracle, never the decoders.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CH = 131072
SEED = 20260101
METRIC = "decompressed GB/s on 1 B200, batched vs plain per-file; p50/p99 request latency"
DATA = "synthetic (seeded generators standing in for CODAG's datasets)"
WORKLOADS = {
    "rlev2": dict(codec=1, n=134_217_728, elem=8, desc="ORC RLE v2, 134,217,728 int64 (1 GiB), 8192 x 128 KiB chunks"),
    "rlev1": dict(codec=0, n=1_048_576, elem=8, desc="ORC RLE v1, 1,048,576 uint64 (8 MiB), 64 x 128 KiB chunks"),
    "rlev1x128": dict(codec=0, n=134_217_728, elem=8, desc="ORC RLE v1, 134,217,728 uint64 (1 GiB), 8192 x 128 KiB chunks"),
    "deflate": dict(codec=2, n=1 << 30, elem=1, desc="Deflate (zlib level 6), 1 GiB Zipf text, 8192 x 128 KiB chunks"),
}
KERNEL_NAMES = {0: "k_rle_plain<.., RLEV1>", 1: "k_rle_plain<.., RLEV2>", 2: "k_inflate_plain"}


def _kernel_name(codec: int, t) -> str:
    if codec != 2:
        return "k_rle_cta<RLEV1/RLEV2, E>" if t.cta_per_chunk else KERNEL_NAMES[codec]
    return "k_inflate_cta" if t.cta_per_chunk else KERNEL_NAMES[codec]


EXTRA_CONFIGS = ("rlev2", "rlev1", "rlev1x128", "deflate")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload: str):
    """DRAM bytes per launch of the decode kernel from the committed ncu summary, if any."""
    f = ROOT / "profiles" / "ncu_traffic.md"
    if not f.exists():
        return None
    m = re.search(rf"^\|\s*{re.escape(workload)}\s*\|\s*([0-9]+)\s*\|", f.read_text(), re.M)
    return int(m.group(1)) if m else None


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# --- workload construction (format library only) ------------------------------------------------
def make_file(workload: str, rank: int, n_values: int | None = None):
    from codag_b200 import native as nat
    w = dict(WORKLOADS[workload])
    if n_values:
        w["n"] = n_values
    seed = SEED + 1000 * rank + w["codec"]
    if w["codec"] == 0:
        col = nat.gen_rlev1_column(w["n"], seed, w["elem"])
        blob, off, ln = nat.encode_rlev1(col, CH, w["elem"])
        return dict(col=col, comp=blob[8:], off=off[:ln.size], ln=ln)
    if w["codec"] == 1:
        col = nat.gen_rlev2_column(w["n"], seed, w["elem"])
        comp, off, ln = nat.encode_rlev2(col, CH, w["elem"])
        return dict(col=col, comp=comp, off=off[:ln.size], ln=ln)
    txt = nat.gen_text(w["n"], seed)
    comp, bo, cl = nat.encode_deflate(txt, CH, 6)
    return dict(col=txt, comp=comp, off=bo[1:], ln=cl)


def _oracle_args(f, codec: int, elem: int, n: int):
    if codec == 2:
        comp_off, comp_len, wrapper = f["off"][:n], np.diff(f["off"][:n + 1]), [2] * n
    else:
        comp_off, comp_len, wrapper = f["off"][:n], f["ln"][:n], [0] * n
    out = np.empty(n * CH, np.uint8)
    return (f["comp"], comp_off, comp_len, out, np.arange(n, dtype=np.uint64) * CH, [CH] * n, [CH] * n,
            [codec] * n, [elem] * n, wrapper)


def cpu_sample(f, codec: int, elem: int, max_chunks: int):
    """CPU decoder (the oracle, OpenMP over chunks) on the first max_chunks chunks with all host
    threads; returns (GB/s, threads, description)."""
    from oracle import oracle_py
    n = min(max_chunks, f["ln"].size)
    args = _oracle_args(f, codec, elem, n)
    oracle_py.decode_batch(*args)  # warm-up
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        st = oracle_py.decode_batch(*args)
        times.append(time.perf_counter() - t0)
        assert not st.any()
    t = float(np.median(times))
    return n * CH / t / 1e9, oracle_py.max_threads(), f"{n} chunks x 128 KiB ({n * CH / 2**20:.0f} MiB), median of 3"


# --- reference arm (CPU decoder of the path, whole workload per step) -----------------------------
def run_reference(args):
    from oracle import oracle_py
    w = WORKLOADS[args.workload]
    f = make_file(args.workload, 0, args.n_values)
    n = f["ln"].size
    a = _oracle_args(f, w["codec"], w["elem"], n)
    for _ in range(args.warmup):
        oracle_py.decode_batch(*a)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = oracle_py.decode_batch(*a)
    dt = time.perf_counter() - t0
    assert not st.any()
    out_bytes = f["col"].size
    ok = bool(np.array_equal(a[3][:out_bytes], f["col"].view(np.uint8)))
    gbs = args.steps * out_bytes / dt / 1e9
    threads = oracle_py.max_threads()
    desc = f"all {n} chunks of the workload per step ({out_bytes / 2**20:.0f} MiB decompressed)"
    line = {"metric": "decompressed GB/s", "value": round(gbs, 3), "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8" if w["codec"] == 2 else "int64", "data": DATA,
            "config": {"workload": w["desc"], "chunk_bytes": CH, "n_chunks": n, "out_bytes": out_bytes},
            "bit_exact": ok, "impl": "reference",
            "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --- our arm, one codec configuration -----------------------------------------------------------
def measure_codec(workload: str, args, rank: int, world: int, local: int, steps: int, warmup: int,
                  clocks_on: bool = True):
    """Times one per-codec configuration; returns its JSON line (rank 0) or None."""
    import torch
    import torch.distributed as dist
    from codag_b200 import api, native as nat

    torch.cuda.set_device(local)
    w = WORKLOADS[workload]
    codec, e = w["codec"], w["elem"]
    f = make_file(workload, rank, args.n_values)
    n = f["ln"].size
    out_bytes = f["col"].size
    comp_bytes = f["comp"].size
    alg_bytes = int(f["ln"].sum()) + n * CH  # compressed stream bytes read + decompressed bytes written
    dev = torch.device("cuda", local)

    def t64(a):
        return torch.from_numpy(np.ascontiguousarray(a).astype(np.uint64).view(np.int64)).to(dev)

    d_comp = torch.from_numpy(f["comp"]).to(dev)
    d_off, d_len = t64(f["off"]), t64(f["ln"])
    d_out = torch.empty(n * CH, dtype=torch.uint8, device=dev)
    d_st = torch.zeros(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    d_ws = api.workspace(codec, n, dev) if codec != 2 and args.rle_passes == 2 else None

    def launch():
        if codec == 0:
            api.decompress_rlev1(d_comp, d_off, d_len, CH, e, d_out, None, d_st, stream, ws=d_ws)
        elif codec == 1:
            api.decompress_rlev2(d_comp, d_off, d_len, CH, e, d_out, None, d_st, stream, ws=d_ws)
        else:
            api.decompress_deflate(d_comp, d_off, CH, d_out, 2, None, d_st, stream)

    if args.tune:
        nat.set_tune(codec, *[int(x) for x in args.tune.split(",")])
    elif args.autotune:
        from codag_b200 import tuning
        # the best shape depends on the chunk count (few chunks favour a CTA per chunk)
        tuning.autotune(codec, launch, tag=f"plain-{n}chunks", use_cache=args.autotune == "cached",
                        verbose=rank == 0 and args.verbose)
    for _ in range(max(warmup, 3)):
        launch()
    torch.cuda.synchronize()
    # correctness of the timed configuration (outside the timed region)
    ok = int((d_st != 0).sum().item()) == 0 and bool(torch.equal(d_out[:out_bytes], torch.from_numpy(f["col"]).to(dev)))

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    clocks = Clocks(local) if rank == 0 and clocks_on else None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    t_all0, t_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_all0.record(stream)
    for i in range(steps):
        ev[i][0].record(stream)
        launch()
        ev[i][1].record(stream)
    t_all1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    elapsed = t_all0.elapsed_time(t_all1) / 1e3
    per_launch = float(np.mean([a.elapsed_time(b) for a, b in ev])) / 1e3
    if world > 1:
        t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
        okt = torch.tensor([0 if ok else 1], dtype=torch.int32, device=dev)
        dist.all_reduce(okt)
        ok = int(okt.item()) == 0

    # e2e: host buffers in pinned memory through the public host-to-host API (api.HostPipeline:
    # H2D of the streams and metadata, decode and D2H of the output, overlapped by chunk
    # groups on three streams); every copy is inside the timed region
    h_comp = torch.from_numpy(f["comp"]).pin_memory()
    off_np = f["off"].astype(np.uint64)
    len_np = f["ln"].astype(np.uint64)
    h_off = torch.from_numpy(off_np.view(np.int64)).pin_memory()
    h_len = torch.from_numpy(len_np.view(np.int64)).pin_memory() if codec != 2 else None
    h_out = torch.empty(out_bytes, dtype=torch.uint8).pin_memory()
    pipe = api.HostPipeline(codec, CH, e, 2, groups=args.e2e_groups, device=dev)
    e_steps = max(2, min(steps, 5))
    h2d_bytes = h_comp.numel() + 8 * h_off.numel() + (8 * h_len.numel() if codec != 2 else 0)
    pipe.run(h_comp, h_off, h_len, out_bytes, h_out, off_np, len_np)  # sizes the device buffers
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e_steps):
        pipe.run(h_comp, h_off, h_len, out_bytes, h_out, off_np, len_np)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_t = e0.elapsed_time(e1) / 1e3
    if world > 1:
        t = torch.tensor([e2e_t], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
    ok = ok and bool(torch.equal(h_out, torch.from_numpy(f["col"])))
    del d_comp, d_off, d_len, d_out, d_st, d_ws, pipe
    torch.cuda.empty_cache()

    if rank != 0:
        return None
    peak, peak_kind = peaks()
    achieved = alg_bytes / per_launch / 1e9
    value = world * out_bytes * steps / elapsed / 1e9
    cpu = None
    if world == 1:
        gbs, threads, desc = cpu_sample(f, codec, e, 1024 if codec != 2 else 256)
        cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port", "sample": desc}
    t = nat.get_tune(codec)
    return {
        "metric": "decompressed GB/s", "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": round(elapsed / steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8" if codec == 2 else "int64", "data": DATA,
        "config": {"workload": w["desc"] if not args.n_values else f"{w['desc']} resized to {args.n_values} values",
                   "chunk_bytes": CH, "n_chunks": n, "comp_bytes": comp_bytes,
                   "out_bytes": out_bytes, "l2": "inputs larger than L2 (no flush)",
                   "parallelism": f"{world} GPU(s), chunks per GPU independent",
                   "tune": {k: getattr(t, k) for k in ("warps_per_cta", "ring_slots", "lut_bits", "cta_per_chunk")}},
        "bit_exact": ok,
        "e2e": {"value": round(world * out_bytes * e_steps / e2e_t / 1e9, 2), "unit": "GB/s",
                "h2d_bytes_per_step": int(h2d_bytes), "d2h_bytes_per_step": int(out_bytes)},
        "gpu_launches": steps * (2 if codec != 2 and args.rle_passes == 2 else 1),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": ncu_traffic(workload), "peak_kind": peak_kind,
                     "kernel": _kernel_name(codec, t),
                     "alg_bytes_per_launch": alg_bytes,
                     "note": ("launch = header walk + expansion kernels of one call" if codec != 2 and args.rle_passes == 2
                              else "one kernel"),
                     "launch_ms": round(per_launch * 1e3, 4)},
        "cpu_baseline": cpu,
        "clocks": clk,
    }


def measure_encode(workload: str, local: int, steps: int = 5) -> dict:
    """GPU encoder (codag_compress_rlev1/_rlev2) on a per-codec column resident in HBM: input
    GB/s, and whether the file equals the host producer's byte for byte."""
    import torch
    from codag_b200 import api, native as nat
    w = WORKLOADS[workload]
    codec, e = w["codec"], w["elem"]
    f = make_file(workload, 0)
    dev = torch.device("cuda", local)
    d_col = torch.from_numpy(f["col"]).to(dev)
    need = int(nat.lib().codag_compress_workspace_bytes(codec, d_col.numel(), CH, e))
    ws = torch.empty(need + 256, dtype=torch.uint8, device=dev)
    out = api.compress_rle(codec, d_col, CH, e, ws=ws)  # warm-up
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        out = api.compress_rle(codec, d_col, CH, e, ws=ws)
    t1.record()
    torch.cuda.synchronize()
    dt = t0.elapsed_time(t1) / 1e3 / steps
    blob = out[0].cpu().numpy()
    want = np.concatenate([np.frombuffer(np.uint64(f["col"].size).tobytes(), np.uint8), f["comp"]]) if codec == 0 \
        else f["comp"]
    ok = bool(np.array_equal(blob, want))
    del d_col, ws, out
    torch.cuda.empty_cache()
    return {"workload": "GPU encode of " + w["desc"], "value": round(f["col"].size / dt / 1e9, 2), "unit": "GB/s",
            "ms_per_step": round(dt * 1e3, 3), "bit_exact_vs_host_producer": ok,
            "how": f"codag_compress_rlev{codec + 1}: one warp per chunk, scan, gather; input bytes per second"}


def measure_transposed(local: int, steps: int = 10, read_unit: int = 1) -> dict:
    """CODAG's transposed RLE v2 layout (32 interleaved substreams per chunk) of the RLE v2
    workload's 1 GiB int64 column, written by the host producer and decoded resident in HBM by
    codag_decompress_rlev2_transposed: decompressed GB/s, its HBM roofline, byte equality."""
    import torch
    from codag_b200 import api, native as nat
    f = make_file("rlev2", 0)
    col = f["col"]
    comp, off, ln = nat.encode_rlev2_transposed(col, CH, 8, read_unit)
    n = ln.size // 32
    dev = torch.device("cuda", local)
    d_comp = torch.from_numpy(comp).to(dev)
    d_off = torch.from_numpy(off[:n].view(np.int64)).to(dev)
    d_len = torch.from_numpy(ln.view(np.int64)).to(dev)
    out = torch.empty(col.nbytes, dtype=torch.uint8, device=dev)
    st = torch.zeros(n, dtype=torch.int32, device=dev)
    run = lambda: api.decompress_rlev2_transposed(d_comp, d_off, d_len, CH, 8, read_unit, out, col.nbytes, st)
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        run()
    t1.record()
    torch.cuda.synchronize()
    dt = t0.elapsed_time(t1) / 1e3 / steps
    ok = int((st != 0).sum().item()) == 0 and bool(torch.equal(out, torch.from_numpy(col.view(np.uint8)).to(dev)))
    peak, peak_kind = peaks()
    alg = int(comp.size) + int(col.nbytes)
    del d_comp, d_off, d_len, out, st
    torch.cuda.empty_cache()
    return {"workload": f"transposed RLE v2 (read unit {read_unit}), {WORKLOADS['rlev2']['desc']}",
            "value": round(col.nbytes / dt / 1e9, 2), "unit": "GB/s", "ms_per_step": round(dt * 1e3, 4),
            "bit_exact": ok, "roofline": {"bound": "hbm", "achieved": round(alg / dt / 1e9, 1), "peak": peak,
                                          "unit": "GB/s", "frac": round(alg / dt / 1e9 / peak, 4), "traffic": None,
                                          "peak_kind": peak_kind, "kernel": "k_rlev2_transposed<8>",
                                          "alg_bytes_per_launch": alg, "launch_ms": round(dt * 1e3, 4)}}


def _summary(line: dict) -> dict:
    """The figures of a per-codec line kept under the headline's `configs`."""
    keep = ("value", "unit", "ms_per_step", "bit_exact", "e2e", "roofline", "cpu_baseline", "clocks")
    return {"workload": line["config"]["workload"], **{k: line[k] for k in keep}, "tune": line["config"]["tune"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched"] + sorted(WORKLOADS) + ["serving"])
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="batched: skip the per-codec configurations and the short serving sweep")
    ap.add_argument("--autotune", default="cached", choices=["cached", "search", ""],
                    help="pick the launch shape with the autotuner (cached result or a fresh search)")
    ap.add_argument("--rle-passes", type=int, default=1, choices=[1, 2],
                    help="RLE: 2 = header walk + expansion (with workspace), 1 = single pass")
    ap.add_argument("--tune", default="", help="explicit launch shape warps_per_cta,ring_slots,lut_bits[,cta_per_chunk]")
    ap.add_argument("--n-values", type=int, default=None,
                    help="override a codec workload's element count (profiling cases; not a bench line)")
    ap.add_argument("--n-files", type=int, default=None, help="batched: number of files (default 20,000)")
    ap.add_argument("--e2e-groups", type=int, default=8, help="e2e: chunk groups overlapped by the host pipeline")
    ap.add_argument("--per-file-sample", type=int, default=600,
                    help="batched: files timed through the per-file path (stratified sample)")
    ap.add_argument("--rates", default="50,100,200,500,1000,2000", help="serving: request rates (per second)")
    ap.add_argument("--duration", type=float, default=60.0, help="serving: seconds of arrivals per rate")
    ap.add_argument("--pool-files", type=int, default=48, help="serving: distinct request files")
    ap.add_argument("--budget-gb", type=int, default=64, help="serving: output memory budget")
    ap.add_argument("--slots", type=int, default=4, help="serving: launches in flight")
    ap.add_argument("--extra-steps", type=int, default=10, help="batched: timed steps of each extra configuration")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            if args.workload == "batched":
                import bench_batched
                bench_batched.run_reference(args)
            elif args.workload == "serving":
                print(json.dumps({"impl": "reference", "unavailable": "the serving loop has no CPU counterpart; "
                                  "the per-codec workloads time the CPU decoders"}), flush=True)
            else:
                run_reference(args)
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    try:
        if args.workload == "batched":
            import bench_batched
            line = bench_batched.main(args, rank, world, local)
            if rank == 0 and line is not None and world == 1 and args.extras:
                import bench_serving
                configs = {}
                for wl in EXTRA_CONFIGS:
                    configs[wl] = _summary(measure_codec(wl, args, rank, world, local, args.extra_steps, 3,
                                                         clocks_on=False))
                configs["encode_rlev2"] = measure_encode("rlev2", local)
                configs["encode_rlev1"] = measure_encode("rlev1x128", local)
                configs["rlev2_transposed"] = measure_transposed(local)
                configs["serving"] = bench_serving.short_sweep(args, local)
                line["configs"] = configs
                line["configs_note"] = ("per-codec configurations and a short serving sweep, timed in the same run "
                                        f"({args.extra_steps} steps each; serving: 2 rates x 10 s)")
            if line is not None:
                print(json.dumps(line), flush=True)
        elif args.workload == "serving":
            import bench_serving
            bench_serving.main(args, rank, world, local)
        else:
            line = measure_codec(args.workload, args, rank, world, local, args.steps, args.warmup)
            if line is not None:
                print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
