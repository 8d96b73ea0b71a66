"""Serving loop: output arena, arrivals and the request pool on the CPU; on the GPU, every
request decoded in a mix of overlapping requests equals the same request decoded alone."""
import numpy as np
import pytest

from codag_b200 import serving


def test_arena_first_fit_and_coalescing():
    a = serving.Arena(1 << 20)
    x = a.alloc(1000)
    y = a.alloc(300_000)
    z = a.alloc(5000)
    assert x == 0 and y == 1024 and z % 256 == 0 and z >= y + 300_000
    assert a.alloc(1 << 20) is None
    a.free(y)
    assert a.alloc(200_000) == y  # first fit reuses the hole
    a.free(x)
    a.free(z)
    a.free(y)
    assert a.free_list == [(0, 1 << 20)] and a.in_use == 0


def test_arena_never_overlaps():
    rng = np.random.default_rng(3)
    a = serving.Arena(64 << 20)
    live = {}
    for _ in range(2000):
        if live and rng.random() < 0.45:
            off = list(live)[rng.integers(len(live))]
            a.free(off)
            del live[off]
        else:
            n = int(rng.integers(1, 4 << 20))
            off = a.alloc(n)
            if off is not None:
                live[off] = n
        spans = sorted(live.items())
        for (o1, n1), (o2, _) in zip(spans, spans[1:]):
            assert o1 + n1 <= o2
        assert all(o + n <= a.capacity for o, n in spans)


def test_poisson_arrivals_rate_and_order():
    arr = serving.poisson_arrivals(500, 4.0, 10, 1)
    t = np.array([x[0] for x in arr])
    assert np.all(np.diff(t) >= 0) and t[-1] < 4.0
    assert 1800 < t.size < 2200
    assert {f for _, f in arr} == set(range(10))


@pytest.fixture(scope="module")
def small_pool(native):
    return serving.build_pool(9, 5, min_bytes=64 << 10, max_bytes=2 << 20)


def test_pool_layout_decodes_with_oracle(small_pool, oracle):
    p = small_pool
    assert p.comp.size % 16 == 0
    for f in p.files:
        d = f.descs
        out = np.zeros(d.size * serving.CH, np.uint8)
        st = oracle.decode_batch(p.comp, d["comp_off"], d["comp_len"], out, d["out_off"], d["out_len"], d["out_len"],
                                 d["codec"], d["elem_bytes"], d["wrapper_bytes"])
        assert not st.any()
        assert np.array_equal(out[:f.size], p.src[f.src_off:f.src_off + f.size])
        assert not out[f.size:].any()  # CODAG pads the tail chunk's input with zeros


@pytest.mark.gpu
def test_mixed_requests_equal_alone(cuda, small_pool):
    p = small_pool
    # alone: one request in flight at a time
    alone_srv = serving.Server(p, 256 << 20, slots=1, keep_outputs=True)
    alone = {}
    for f in range(len(p.files)):
        reqs = alone_srv.run([(0.0, f)])
        assert reqs[0].ok
        alone[f] = alone_srv.outputs[0].numpy().copy()
        alone_srv.outputs.clear()
    # mixed: 60 overlapping requests, a small budget so that admission waits for memory
    arr = [(0.0005 * i, i % len(p.files)) for i in range(60)]
    srv = serving.Server(p, 24 << 20, slots=3, keep_outputs=True)
    reqs = srv.run(arr)
    assert all(r.ok for r in reqs)
    assert srv.launches >= 2
    for r in reqs:
        got = srv.outputs[r.rid].numpy()
        assert np.array_equal(got, alone[r.file])
        f = p.files[r.file]
        assert np.array_equal(got, p.src[f.src_off:f.src_off + f.size])
    s = serving.summarize(reqs, p, 0.03)
    assert s["bit_exact"] and s["completed"] == 60 and s["p99_ms"] >= s["p50_ms"] > 0


def test_admission_capacity_follows_free_memory():
    GiB = 1 << 30
    assert serving.admission_capacity(64 * GiB, 170 * GiB, 2 * GiB) == 64 * GiB  # the budget binds
    assert serving.admission_capacity(64 * GiB, 40 * GiB, 2 * GiB) == 38 * GiB   # free memory binds
    assert serving.admission_capacity(64 * GiB, 1 * GiB, 2 * GiB) == 0


@pytest.mark.gpu
def test_server_admits_by_free_device_memory(cuda, small_pool):
    """A budget far above the device's memory is cut to what is free: requests are still
    admitted and decoded, bit-exact."""
    free, _ = cuda.cuda.mem_get_info()
    pool = small_pool
    srv = serving.Server(pool, 1 << 50, slots=2)
    assert srv.arena.capacity <= free - serving.Server.RESERVE
    reqs = srv.run(serving.poisson_arrivals(400, 0.05, len(pool.files), 3))
    assert reqs and all(r.ok for r in reqs)
    del srv  # give the device memory back for the tests after this one
    import gc
    gc.collect()
    cuda.cuda.empty_cache()


@pytest.mark.gpu
def test_tune_server_picks_a_listed_shape(cuda, small_pool, monkeypatch, tmp_path):
    """The serving tuner times each listed launch shape on a saturating burst, keeps the fastest
    (every request exact under every shape) and caches it."""
    from codag_b200 import tuning
    monkeypatch.setattr(tuning, "CACHE", tmp_path / "tune.json")
    import gc
    gc.collect()
    cuda.cuda.empty_cache()
    srv = serving.Server(small_pool, 1 << 30, slots=2, device="cuda")
    shape = serving.tune_server(srv, n_requests=24, use_cache=False)
    assert shape in serving.SERVE_SHAPES
    assert tuple(tuning.load_cached(-1, "serve")) == shape
    assert serving.tune_server(srv) == shape  # from the cache
    reqs = srv.run([(0.0, f) for f in range(len(small_pool.files))])
    assert all(r.ok for r in reqs)
