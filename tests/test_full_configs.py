"""The benchmark configurations at their full sizes, decoded on the GPU and checked byte for
byte: against the source (every configuration) and against the oracle (C1, whose 64 chunks
the oracle decodes in well under a second).  C2 (RLE v2, 1 GiB) is in test_gpu_parity.py.

  C1     ORC RLE v1, 1,048,576 uint64 (8 MiB), 64 chunks of 128 KiB
  C1x128 the same generator at 134,217,728 uint64 (1 GiB), 8192 chunks
  C3     Deflate (zlib level 6), 1 GiB of Zipf text, 8192 chunks
  C4     20,000 independently compressed files through the batched persistent launch,
         replayed from a CUDA graph, and a sample of them through the per-file path"""
import numpy as np
import pytest

CH = 131072
pytestmark = pytest.mark.gpu


def _t(cuda, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    return cuda.from_numpy(a.copy() if not a.flags.writeable else a).to("cuda")


@pytest.mark.parametrize("n_values", [1_048_576, 134_217_728], ids=["C1_8MiB", "C1x128_1GiB"])
def test_rlev1_configs(native, oracle, cuda, n_values):
    from codag_b200 import api
    col = native.gen_rlev1_column(n_values, 20260101, 8)
    blob, off, ln = native.encode_rlev1(col, CH, 8)
    n = ln.size
    out = cuda.empty(col.size, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_rlev1(_t(cuda, blob[8:]), _t(cuda, off[:n]), _t(cuda, ln), CH, 8, out, col.size, st)
    cuda.cuda.synchronize()
    assert int((st != 0).sum().item()) == 0
    assert bool(cuda.equal(out, _t(cuda, col)))
    if n <= 64:
        ref = np.zeros(n * CH, np.uint8)
        ost = oracle.decode_batch(blob[8:], off[:n], ln, ref, np.arange(n, dtype=np.uint64) * CH, [CH] * n, [CH] * n,
                                  [0] * n, [8] * n, [0] * n)
        assert not ost.any() and np.array_equal(out.cpu().numpy(), ref[:col.size])


def test_deflate_config_1gib(native, cuda):
    from codag_b200 import api
    txt = native.gen_text(1 << 30, 20260103)
    comp, bo, cl = native.encode_deflate(txt, CH, 6)
    n = cl.size
    assert n == 8192
    out = cuda.empty(txt.size, dtype=cuda.uint8, device="cuda")
    st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
    api.decompress_deflate(_t(cuda, comp), _t(cuda, bo[1:]), CH, out, 2, txt.size, st)
    cuda.cuda.synchronize()
    assert int((st != 0).sum().item()) == 0
    assert bool(cuda.equal(out, _t(cuda, txt)))


def test_batched_config_20000_files(native, cuda):
    from codag_b200 import api, batched
    ms = batched.make_mixed_set(20_000, seed=20260104)
    assert ms.n == 20_000 and set(np.unique(ms.codecs).tolist()) == {0, 1, 2}
    d_comp = _t(cuda, ms.comp)
    want = _t(cuda, ms.expected())
    out = cuda.zeros(ms.out_bytes, dtype=cuda.uint8, device="cuda")
    st = cuda.full((ms.n,), -1, dtype=cuda.int32, device="cuda")
    plan = api.BatchPlan(ms.descs)
    try:
        for _ in range(2):  # captured on the first call, replayed on the second
            out.zero_()
            st.fill_(-1)
            plan.run(d_comp, out, st, use_graph=True)
            cuda.cuda.synchronize()
            assert int((st != 0).sum().item()) == 0
            assert bool(cuda.equal(out, want))
    finally:
        plan.close()
    # the per-file path on a stratified sample of the same resident set
    sample = batched.stratified_sample(ms, 300)
    out.zero_()
    pf = batched.PerFileDecoder(ms, d_comp, out, "cuda")
    pf.run(sample, cuda.cuda.current_stream())
    cuda.cuda.synchronize()
    assert int((pf.d_st[cuda.from_numpy(sample).to("cuda")] != 0).sum().item()) == 0
    for i in sample:
        o, ln = int(ms.descs["out_off"][i]), int(ms.in_len[i])
        assert bool(cuda.equal(out[o:o + ln], want[o:o + ln])), i
