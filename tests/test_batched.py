"""Mixed sets of independently compressed files: the set producer against the oracle (CPU),
and the batched persistent launch and the per-file path against the source data (GPU)."""
import numpy as np
import pytest

from codag_b200 import batched


@pytest.fixture(scope="module")
def small_set(native):
    return batched.make_mixed_set(400, seed=99, max_bytes=256 << 10, source_bytes=8 << 20)


def test_set_layout_and_oracle_round_trip(small_set, oracle):
    ms = small_set
    d = ms.descs
    assert np.all(d["comp_off"] % 16 == 0) and np.all(d["out_off"] % 256 == 0)
    assert np.all(d["out_len"] == ms.in_len) and np.all(ms.in_len % 8 == 0)
    assert set(np.unique(d["codec"]).tolist()) == {0, 1, 2}
    assert np.all((d["wrapper_bytes"] == 2) == (d["codec"] == 2))
    assert np.all(np.isin(d["elem_bytes"][d["codec"] != 2], [4, 8]))
    out = np.zeros(ms.out_bytes, np.uint8)
    st = oracle.decode_batch(ms.comp, d["comp_off"], d["comp_len"], out, d["out_off"], d["out_len"], d["out_len"],
                             d["codec"], d["elem_bytes"], d["wrapper_bytes"])
    assert not st.any()
    assert np.array_equal(out, ms.expected())


def test_stratified_sample_covers_codecs(small_set):
    s = batched.stratified_sample(small_set, 30)
    assert s.size == 30 and np.all(np.diff(s) > 0)
    assert set(small_set.codecs[s].tolist()) == {0, 1, 2}


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [False, True])
@pytest.mark.parametrize("shape", [None, (1, 4, 9), (4, 8, 11), (8, 4, 10), (2, 4, 9, 0, 1), (8, 8, 11, 0, 1)])
def test_batched_matches_source(cuda, small_set, shape, use_graph):
    """Shapes (warps_per_cta, ring_slots, lut_bits[, cta_per_chunk, table_global]); the last two
    keep the Huffman lookup tables in global memory."""
    from codag_b200 import api
    ms = small_set
    d_comp = cuda.from_numpy(ms.comp).to("cuda")
    d_out = cuda.full((ms.out_bytes,), 0x77, dtype=cuda.uint8, device="cuda")
    st = cuda.full((ms.n,), -1, dtype=cuda.int32, device="cuda")
    plan = api.BatchPlan(ms.descs, *shape) if shape else api.BatchPlan(ms.descs)
    try:
        for _ in range(2):  # second run replays the graph over the first run's output
            plan.run(d_comp, d_out, st, use_graph=use_graph)
        cuda.cuda.synchronize()
    finally:
        plan.close()
    assert not st.cpu().numpy().any()
    got = d_out.cpu().numpy()
    want = ms.expected()
    for d, ln in zip(ms.descs, ms.in_len):
        o = int(d["out_off"])
        assert np.array_equal(got[o:o + int(ln)], want[o:o + int(ln)])


@pytest.mark.gpu
@pytest.mark.parametrize("how", ["base", "offsets"])
def test_batched_unaligned_outputs(cuda, small_set, how):
    """Outputs that are not element aligned: the batch kernel stores their RLE values byte by
    byte.  Either the output base is off 8-byte alignment, or every output offset is shifted by
    one byte."""
    from codag_b200 import api
    ms = small_set
    descs = ms.descs.copy()
    shift = 0
    if how == "offsets":
        descs["out_off"] = descs["out_off"] + 1
    else:
        shift = 3
    d_comp = cuda.from_numpy(ms.comp).to("cuda")
    buf = cuda.full((ms.out_bytes + 16,), 0x77, dtype=cuda.uint8, device="cuda")
    d_out = buf[shift:]
    st = cuda.full((ms.n,), -1, dtype=cuda.int32, device="cuda")
    plan = api.BatchPlan(descs)
    try:
        plan.run(d_comp, d_out, st, use_graph=False)
        cuda.cuda.synchronize()
    finally:
        plan.close()
    assert not st.cpu().numpy().any()
    got = d_out.cpu().numpy()
    want = ms.expected()
    for d0, d1, ln in zip(ms.descs, descs, ms.in_len):
        o0, o1 = int(d0["out_off"]), int(d1["out_off"])
        assert np.array_equal(got[o1:o1 + int(ln)], want[o0:o0 + int(ln)])


@pytest.mark.gpu
def test_per_file_path_matches_source(cuda, small_set):
    ms = small_set
    d_comp = cuda.from_numpy(ms.comp).to("cuda")
    d_out = cuda.zeros((ms.out_bytes,), dtype=cuda.uint8, device="cuda")
    pf = batched.PerFileDecoder(ms, d_comp, d_out, "cuda")
    files = batched.stratified_sample(ms, 60)
    pf.run(files, cuda.cuda.current_stream())
    cuda.cuda.synchronize()
    assert not pf.d_st.cpu().numpy()[files].any()
    got = d_out.cpu().numpy()
    for i in files:
        o, ln, s = int(ms.descs["out_off"][i]), int(ms.in_len[i]), int(ms.in_off[i])
        assert np.array_equal(got[o:o + ln], ms.src[s:s + ln])


@pytest.mark.gpu
def test_batched_reports_corrupt_file_and_decodes_the_rest(cuda, small_set):
    from codag_b200 import api
    ms = small_set
    comp = ms.comp.copy()
    bad = int(np.nonzero(ms.codecs == 2)[0][0])
    d = ms.descs[bad]
    comp[int(d["comp_off"]) + 2:int(d["comp_off"]) + int(d["comp_len"])] = 0xFF  # invalid block type 3
    d_comp = cuda.from_numpy(comp).to("cuda")
    d_out = cuda.zeros((ms.out_bytes,), dtype=cuda.uint8, device="cuda")
    st = cuda.full((ms.n,), -1, dtype=cuda.int32, device="cuda")
    plan = api.BatchPlan(ms.descs)
    try:
        plan.run(d_comp, d_out, st, use_graph=False)
        cuda.cuda.synchronize()
    finally:
        plan.close()
    s = st.cpu().numpy()
    assert s[bad] == 2 and np.count_nonzero(s) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [1, 2, 5])
def test_batch_host_pipeline_matches_source(cuda, small_set, steps):
    """Host-to-host decode of a mixed set over consecutive pipelined steps (graphs captured,
    then replayed), each step into its own host buffer."""
    from codag_b200 import api
    ms = small_set
    h_comp = cuda.from_numpy(ms.comp).pin_memory()
    outs = [cuda.full((ms.out_bytes,), 0x5A, dtype=cuda.uint8).pin_memory() for _ in range(steps)]
    pipe = api.BatchHostPipeline(ms.descs, ms.comp.size, ms.out_bytes)
    try:
        assert pipe.h2d_bytes == ms.comp.size and pipe.d2h_bytes == ms.out_bytes
        pipe.run([(h_comp, h) for h in outs])
        pipe.run([(h_comp, h) for h in outs])
        for h in outs:
            assert np.array_equal(h.numpy(), ms.expected())
    finally:
        pipe.close()


@pytest.fixture(scope="module")
def large_set(native):
    return batched.make_mixed_set(160, seed=101, max_bytes=1 << 20, source_bytes=16 << 20)


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [False, True])
@pytest.mark.parametrize("shape", [(2, 4, 9, 1), (4, 4, 10, 1), (8, 4, 11, 1), (4, 4, 10, 1, 1), (4, 4, 10, 2),
                                   (8, 4, 9, 3)])
def test_batched_warp_pairs_match_source(cuda, large_set, shape, use_graph):
    """Plans made with cta_per_chunk = k: Deflate files of k x 256 KiB or more decoded by warp
    pairs (symbol decoder and byte expander), everything else by single warps."""
    from codag_b200 import api
    ms = large_set
    big = (ms.codecs == 2) & (ms.in_len >= shape[3] * (256 << 10))
    assert big.sum() >= 2
    plan = api.BatchPlan(ms.descs, *shape)
    try:
        out = cuda.zeros(ms.out_bytes, dtype=cuda.uint8, device="cuda")
        st = cuda.full((ms.n,), -1, dtype=cuda.int32, device="cuda")
        for _ in range(2):
            out.zero_()
            plan.run(cuda.from_numpy(ms.comp).to("cuda"), out, st, use_graph=use_graph)
            cuda.cuda.synchronize()
            assert int((st != 0).sum().item()) == 0
            assert np.array_equal(out.cpu().numpy(), ms.expected())
    finally:
        plan.close()


@pytest.mark.gpu
def test_batched_warp_pairs_report_damage_like_single_warps(cuda, large_set):
    from codag_b200 import api
    ms = large_set
    comp = ms.comp.copy()
    rng = np.random.default_rng(3)
    for i in np.flatnonzero(ms.codecs == 2)[::2]:  # damage every other Deflate file
        d = ms.descs[i]
        comp[int(d["comp_off"]) + 2 + rng.integers(0, int(d["comp_len"]) - 2, 4)] ^= 0x5A
    res = []
    for shape in ((4, 4, 10, 0), (4, 4, 10, 1)):
        plan = api.BatchPlan(ms.descs, *shape)
        try:
            out = cuda.zeros(ms.out_bytes, dtype=cuda.uint8, device="cuda")
            st = cuda.full((ms.n,), -1, dtype=cuda.int32, device="cuda")
            plan.run(cuda.from_numpy(comp).to("cuda"), out, st)
            cuda.cuda.synchronize()
            res.append((st.cpu().numpy(), out.cpu().numpy()))
        finally:
            plan.close()
    (s1, o1), (s2, o2) = res
    assert np.array_equal(s1, s2) and (s1 != 0).any()
    for i in np.flatnonzero(s1 == 0):
        a, ln = int(ms.descs[i]["out_off"]), int(ms.in_len[i])
        assert np.array_equal(o1[a:a + ln], o2[a:a + ln]), i


def test_pair_threshold_range(native, small_set):
    """cta_per_chunk in a plan: 0..4 (multiples of 256 KiB) with an even warp count; checked
    before anything touches the device."""
    import ctypes as C
    d = np.ascontiguousarray(small_set.descs, dtype=native.CHUNK_DESC_DTYPE)
    p = C.c_void_p()
    for shape in ((4, 4, 10, 5), (4, 4, 10, -1), (3, 4, 10, 2)):
        t = native.Tune(*shape)
        assert native.lib().codag_batch_plan(d.ctypes.data, d.size, C.byref(t), C.byref(p)) == native.EINVAL, shape


def test_table_placement_is_a_plan_option(native):
    """Global-memory lookup tables need the plan's scratch: the per-file calls refuse them."""
    import ctypes as C
    t = native.Tune(2, 2, 9, 0, 1)
    assert native.lib().codag_set_tune(native.DEFLATE, C.byref(t)) == native.EINVAL
    assert native.get_tune(native.DEFLATE).table_global == 0


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [False, True])
def test_plans_sharing_a_kernel_at_different_warp_counts(cuda, small_set, use_graph):
    """Plans of 8 and of 2 warps per CTA with the same ring depth and table width launch the same
    kernel with different shared-memory sizes: making the small plan after the large one (and a
    small unplanned launch in between) must leave the large plan launchable."""
    from codag_b200 import api
    ms = small_set
    d_comp = cuda.from_numpy(ms.comp).to("cuda")
    want = cuda.from_numpy(ms.expected()).to("cuda")
    big = api.BatchPlan(ms.descs, 8, 4, 10)
    small = api.BatchPlan(ms.descs, 2, 4, 10)
    try:
        for plan in (small, big, small, big):
            out = cuda.zeros(ms.out_bytes, dtype=cuda.uint8, device="cuda")
            st = cuda.full((ms.n,), -1, dtype=cuda.int32, device="cuda")
            plan.run(d_comp, out, st, use_graph=use_graph)
            cuda.cuda.synchronize()
            assert int((st != 0).sum().item()) == 0 and bool(cuda.equal(out, want))
    finally:
        big.close()
        small.close()
