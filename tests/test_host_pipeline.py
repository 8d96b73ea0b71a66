"""api.HostPipeline: pinned host buffers in and out, copies and decode overlapped by chunk
groups; the output must equal the source for every codec, group count and a file whose
size is not a multiple of the chunk size."""
import numpy as np
import pytest

CH = 131072


def _file(native, codec, size, seed):
    if codec == 2:
        src = native.gen_text(size, seed)
        comp, bo, _ = native.encode_deflate(src, CH, 6)
        return src, comp, bo[1:], None
    gen = native.gen_rlev1_column if codec == 0 else native.gen_rlev2_column
    src = gen(size // 8, seed, 8)
    if codec == 0:
        blob, off, ln = native.encode_rlev1(src, CH, 8)
        return src, blob[8:], off[:ln.size], ln
    comp, off, ln = native.encode_rlev2(src, CH, 8)
    return src, comp, off[:ln.size], ln


@pytest.mark.gpu
@pytest.mark.parametrize("groups", [1, 3, 64])
@pytest.mark.parametrize("codec", [0, 1, 2])
def test_host_pipeline_round_trip(cuda, native, codec, groups):
    from codag_b200 import api
    src, comp, off, ln = _file(native, codec, 21 * CH + 8 * 1234, 40 + codec)
    h_comp = cuda.from_numpy(comp).pin_memory()
    off = off.astype(np.uint64)
    h_off = cuda.from_numpy(off.view(np.int64)).pin_memory()
    h_len = cuda.from_numpy(ln.astype(np.uint64).view(np.int64)).pin_memory() if ln is not None else None
    h_out = cuda.zeros(src.size, dtype=cuda.uint8).pin_memory()
    pipe = api.HostPipeline(codec, CH, 8, 2, groups=groups)
    for _ in range(2):
        pipe.run(h_comp, h_off, h_len, src.size, h_out, off, ln)
        assert np.array_equal(h_out.numpy(), src.view(np.uint8))
        h_out.zero_()
