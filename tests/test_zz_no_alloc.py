"""codag_decompress_rlev2_noalloc: the RLE v2 decode for callers that cannot allocate device
memory (an engine plugin whose device memory is all held by the engine's own pool, or a path
that must not allocate), which uses a fixed scratch array inside the library instead of a
caller workspace.

Its output must equal codag_decompress_rlev2's on the same input, byte for byte, over two
calls in a row with different inputs: the second call reuses the scratch the first one
left behind.  The entry point returns an error rather than decoding in one pass when its
scratch could not be used, so a match here is a match of the two-pass decode.  This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from codag_b200 import native

CHUNK = 131072


def _column(n_values, seed, e):
    return native.gen_rlev2_column(n_values, seed, e)


def test_rejects_more_chunks_than_the_scratch_holds(native):
    lib = native.lib()
    n = native.NOALLOC_MAX_CHUNKS + 1
    # the argument and size checks come before any CUDA call, so they run without a GPU too
    assert lib.codag_decompress_rlev2_noalloc(1, 1, 1, 1, n, CHUNK, 8, 1, 1, None, None) == native.ELIMIT
    assert lib.codag_decompress_rlev2_noalloc(1, 1, 1, 1, 0, CHUNK, 8, 1, 1, None, None) == native.OK


def test_checks_arguments_like_the_workspace_call(native):
    """Bad pointers and element widths give CODAG_EINVAL before the chunk-count limit is
    looked at, and with no chunks at all, as codag_decompress_rlev2 does."""
    lib = native.lib()
    for n in (0, 1, native.NOALLOC_MAX_CHUNKS + 1):
        assert lib.codag_decompress_rlev2_noalloc(None, 1, 1, 1, n, CHUNK, 8, 1, 1, None, None) == native.EINVAL
        assert lib.codag_decompress_rlev2_noalloc(1, 1, 1, 1, n, CHUNK, 3, 1, 1, None, None) == native.EINVAL
        assert lib.codag_decompress_rlev2_noalloc(1, 1, 1, 1, n, CHUNK + 4, 8, 1, 1, None, None) == native.EINVAL
        assert lib.codag_decompress_rlev2(None, 1, 1, 1, n, CHUNK, 8, 1, 1, None, None, 0, None) == native.EINVAL


def _decode_both(cuda, data, e):
    """Decodes `data` encoded as RLE v2 with the existing entry point and the no-alloc one."""
    lib = native.lib()
    comp, off, ln = native.encode_rlev2(data, CHUNK, e)
    n = ln.size
    assert 0 < n <= native.NOALLOC_MAX_CHUNKS
    size = int(off[n])
    d_comp = cuda.from_numpy(comp).to("cuda")
    d_off = cuda.from_numpy(off[:n].view(np.int64)).to("cuda")
    d_len = cuda.from_numpy(ln.view(np.int64)).to("cuda")
    outs, sts = [], []
    for noalloc in (False, True):
        out = cuda.full((n * CHUNK,), 0x5A, dtype=cuda.uint8, device="cuda")
        st = cuda.full((n,), -1, dtype=cuda.int32, device="cuda")
        args = (d_comp.data_ptr(), d_comp.numel(), d_off.data_ptr(), d_len.data_ptr(), n, CHUNK, e,
                out.data_ptr(), size, st.data_ptr())
        if noalloc:
            rc = lib.codag_decompress_rlev2_noalloc(*args, None)
        else:
            ws = cuda.empty(int(lib.codag_workspace_bytes(native.RLEV2, n)), dtype=cuda.uint8, device="cuda")
            rc = lib.codag_decompress_rlev2(*args, ws.data_ptr(), ws.numel(), None)
        assert rc == native.OK
        cuda.cuda.synchronize()
        outs.append(out.cpu().numpy())
        sts.append(st.cpu().numpy())
    return size, outs, sts


@pytest.mark.gpu
def test_noalloc_matches_workspace_decode_two_calls(cuda):
    # first call: 300 chunks of 64-bit values; second: fewer chunks of 32-bit values, so the
    # second call runs over scratch that still holds the first call's descriptors
    cases = [(_column(300 * CHUNK // 8, 11, 8), 8), (_column(77 * CHUNK // 4 - 5, 12, 4), 4)]
    for data, e in cases:
        size, (ref, got), (st_ref, st_got) = _decode_both(cuda, data, e)
        assert np.all(st_ref == 0) and np.all(st_got == 0)
        assert np.array_equal(got[:size], ref[:size])
        assert np.array_equal(got[:size], np.ascontiguousarray(data).view(np.uint8))
        assert np.all(got[size:] == 0x5A)
