"""`bench.py --workload serving` (driver module beside bench.py): CODAG's serving configuration on one GPU.

A pool of request files (log-uniform 64 KiB-256 MiB, 40/30/30 Deflate/RLE v1/RLE v2, CODAG's
128 KiB chunk layout) is made resident in HBM; requests drawn uniformly from the pool arrive
as a Poisson process at each rate for `--duration` seconds; outputs live in a 64 GB budget.
One JSON line reports, per rate, decompressed GB/s and p50/p99 latency (arrival to decoded),
and every request is checked byte for byte on the device.
"""
from __future__ import annotations

import json

SEED = 20260105


def _shape(args, srv):
    """The serving loop's launch shape: --tune if given, else the serving tuner (cached per GPU
    model unless --autotune search), else the library default (--autotune '')."""
    from codag_b200 import native, serving
    if args.tune:
        shape = tuple(int(x) for x in args.tune.split(","))[:4]
        srv.tune = native.Tune(*shape, 0)
        return shape
    if args.autotune:
        return serving.tune_server(srv, use_cache=args.autotune == "cached")
    return None


def short_sweep(args, local: int, rates=(500.0, 2000.0), duration: float = 10.0, pool_files: int = 24) -> dict:
    """A short sweep for the default bench line: `rates` for `duration` seconds each over a
    pool of `pool_files` files; returns decompressed GB/s and p50/p99 latency per rate."""
    import torch
    from codag_b200 import serving

    torch.cuda.set_device(local)
    pool = serving.build_pool(pool_files, SEED)
    srv = serving.Server(pool, args.budget_gb << 30, slots=args.slots, device=f"cuda:{local}")
    srv.run(serving.poisson_arrivals(50, 0.5, len(pool.files), 1))
    shape = _shape(args, srv)
    rows = []
    for k, rate in enumerate(rates):
        arr = serving.poisson_arrivals(rate, duration, len(pool.files), SEED + 17 * k)
        reqs = srv.run(arr, time_limit=duration * 3 + 30)
        s = serving.summarize(reqs, pool, duration)
        rows.append({"rate": rate, **{k2: (round(v, 3) if isinstance(v, float) else v) for k2, v in s.items()}})
    sizes = [f.size for f in pool.files]
    out = {"workload": f"serving: Poisson arrivals, {duration:g} s per rate, pool of {len(pool.files)} files "
                       f"log-uniform 64 KiB-256 MiB (mean {sum(sizes) / len(sizes) / 1e6:.1f} MB), "
                       "40/30/30 Deflate/RLE v1/RLE v2, 128 KiB chunks",
           "budget_bytes": args.budget_gb << 30, "rates": rows, "bit_exact": all(r["bit_exact"] for r in rows),
           "launches": srv.launches, "tune": list(shape) if shape else None}
    del srv, pool
    torch.cuda.empty_cache()
    return out


def main(args, rank: int, world: int, local: int) -> None:
    import torch
    from codag_b200 import serving
    from bench import Clocks

    torch.cuda.set_device(local)
    pool = serving.build_pool(args.pool_files, SEED + rank)
    srv = serving.Server(pool, args.budget_gb << 30, slots=args.slots, device=f"cuda:{local}")
    warm = serving.poisson_arrivals(50, 0.5, len(pool.files), 1)
    srv.run(warm)
    shape = _shape(args, srv)
    rates = [float(x) for x in args.rates.split(",")]
    rows = []
    clocks = Clocks(local) if rank == 0 else None
    if clocks:
        clocks.start()
    for k, rate in enumerate(rates):
        arr = serving.poisson_arrivals(rate, args.duration, len(pool.files), SEED + 17 * k)
        reqs = srv.run(arr, time_limit=args.duration * 3 + 30)
        s = serving.summarize(reqs, pool, args.duration)
        s["rate"] = rate
        if world > 1:  # one replica per GPU: the job's throughput is the sum, its latency the worst
            import torch.distributed as dist
            t = torch.tensor([s["gbs"], s["p50_ms"], s["p99_ms"], 0.0 if s["bit_exact"] else 1.0],
                             dtype=torch.float64, device=f"cuda:{local}")
            tot = t.clone()
            dist.all_reduce(tot, op=dist.ReduceOp.SUM)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            s.update(gbs=float(tot[0]), p50_ms=float(t[1]), p99_ms=float(t[2]), bit_exact=float(t[3]) == 0.0,
                     replicas=world)
        rows.append(s)
        if rank == 0:
            print(json.dumps({"serving_rate": rate, **s}), flush=True)
    clk = clocks.stop() if clocks else None
    if rank != 0:
        return
    best = max(rows, key=lambda r: r["gbs"])
    sizes = [f.size for f in pool.files]
    line = {
        "metric": "decompressed GB/s and p50/p99 request latency under Poisson load", "value": round(best["gbs"], 2),
        "unit": "GB/s", "n_gpus": world, "steps": len(rates), "warmup": 1, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generators standing in for CODAG's datasets)",
        "config": {"workload": f"serving: Poisson arrivals, {args.duration:g} s per rate, pool of {len(pool.files)} files "
                               f"log-uniform 64 KiB-256 MiB (mean {sum(sizes) / len(sizes) / 1e6:.1f} MB), "
                               "40/30/30 Deflate/RLE v1/RLE v2, 128 KiB chunks",
                   "budget_bytes": args.budget_gb << 30, "slots": args.slots,
                   "tune": list(shape) if shape else None},
        "bit_exact": all(r["bit_exact"] for r in rows),
        "rates": rows, "launches": srv.launches, "gpu_launches": srv.launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
