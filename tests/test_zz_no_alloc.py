"""The allocation-free COMPRESS_16 entry point (rtm_c16_compress_noalloc).

It serves callers that cannot allocate GPU memory (a host program that carves
all of HBM up front with its own pool allocator, or a thread that must not
wait on the allocator): they pass device buffers and the entry point's scratch
lives in a fixed array of the library.  Its codes must equal those of the allocating
entry point rtm_c16_compress bit for bit, on two calls in a row (the second
call reuses the scratch the first one left behind).  This file is collected
last so a run that stops at the first failure has run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_compress_matches_allocating_entry_point():
    import torch
    from konglong_b200 import _lib
    from konglong_b200.propagator import c16_compress
    from tests.golden_inputs import codec_input

    L = _lib.lib()
    cases = list(codec_input().values())
    rng = np.random.default_rng(99)
    a2 = (rng.standard_normal((30, 20, 16)) * np.exp(-np.arange(30))[:, None, None]).astype(np.float32)
    cases.append((a2, 20, 30, 16))
    for a, nx, ny, nz in cases:                      # consecutive calls share the scratch
        want = c16_compress(a, nx, ny, nz)
        d_in = torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).cuda()
        d_out = torch.zeros(want.size, dtype=torch.int16, device="cuda")
        rc = L.rtm_c16_compress_noalloc(d_in.data_ptr(), d_out.data_ptr(), nx, ny, nz, None)
        assert rc == 0, _lib.lib().rtm_last_error(None)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(np.uint16)
        np.testing.assert_array_equal(got, want)


def test_noalloc_at_the_slab_limit_matches_allocating_entry_point():
    """ny = RTM_NOALLOC_MAX_SLABS (65535, the largest y extent a launch grid
    row count allows) with one cell per slab runs and equals the allocating
    entry point; one slab more is refused before anything is launched."""
    import torch
    from konglong_b200 import _lib
    from konglong_b200.propagator import c16_compress

    L = _lib.lib()
    ny = 65535
    rng = np.random.default_rng(7)
    a = (rng.standard_normal(ny) * np.exp(rng.uniform(-20, 5, ny))).astype(np.float32)
    want = c16_compress(a, 1, ny, 1)
    d_in = torch.from_numpy(a).cuda()
    for _ in range(2):
        d_out = torch.zeros(want.size, dtype=torch.int16, device="cuda")
        assert L.rtm_c16_compress_noalloc(d_in.data_ptr(), d_out.data_ptr(), 1, ny, 1, None) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint16), want)
    err = _lib.STATUS_CODE["RTM_ERR_ARG"]
    assert L.rtm_c16_compress_noalloc(d_in.data_ptr(), d_out.data_ptr(), 1, ny + 1, 1, None) == err
    assert L.rtm_c16_compress_noalloc(1, 1, 4, 65537, 4, None) == err


def test_noalloc_compress_replayed_from_a_captured_graph():
    """The stated use: a warm-up call, then the call recorded on the caller's own
    (non-default) stream into a CUDA graph and replayed; every replay writes
    the allocating entry point's codes."""
    import torch
    from konglong_b200 import _lib
    from konglong_b200.propagator import c16_compress
    from tests.golden_inputs import codec_input

    L = _lib.lib()
    a, nx, ny, nz = codec_input()["wave"]
    want = c16_compress(a, nx, ny, nz)
    d_in = torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).cuda()
    d_out = torch.zeros(want.size, dtype=torch.int16, device="cuda")
    s = torch.cuda.Stream()
    assert L.rtm_c16_compress_noalloc(d_in.data_ptr(), d_out.data_ptr(), nx, ny, nz, s.cuda_stream) == 0  # warm-up
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        rc = L.rtm_c16_compress_noalloc(d_in.data_ptr(), d_out.data_ptr(), nx, ny, nz, s.cuda_stream)
        g.capture_end()
    assert rc == 0
    for _ in range(2):
        d_out.zero_()
        g.replay()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint16), want)
