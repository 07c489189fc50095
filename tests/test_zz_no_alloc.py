"""The allocation-free window filter (epb_window_filter_noalloc) against epb_window_filter.

Some callers cannot let a library allocate device memory: their memory belongs to a caching
allocator (a Julia CUDA.jl or PyTorch pool), or their hot loop must not pay an allocation's latency
or failure. The allocation-free entry point serves them with a fixed device scratch array and a
plain stream. This file is collected last so that a run stopping at the first failure has already
run every other test; it also passes on its own in a fresh process.

The filter is integer/index work, so results must be identical (bit-exact), on two calls in a row.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(L, fn, stream_or_ctx, E, wmin, wmax):
    import torch

    nw, nk = E.shape[1], E.shape[0]
    bmin = torch.full((nk,), -7, dtype=torch.int32, device="cuda")
    bmax = torch.full((nk,), -7, dtype=torch.int32, device="cuda")
    keep = torch.full((max(nk, 1),), -7, dtype=torch.int32, device="cuda")
    nkeep = torch.full((1,), -7, dtype=torch.int64, device="cuda")
    nbelow = torch.full((nk,), -7.0, dtype=torch.float64, device="cuda")
    st = fn(stream_or_ctx, E.data_ptr(), nw, nk, wmin, wmax, bmin.data_ptr(), bmax.data_ptr(), keep.data_ptr(),
            nkeep.data_ptr(), nbelow.data_ptr())
    torch.cuda.synchronize()
    assert st == 0, L.epb_last_error()
    n = int(nkeep.item())
    return bmin.cpu().numpy(), bmax.cpu().numpy(), keep[:n].cpu().numpy(), nbelow.cpu().numpy()


def test_window_filter_noalloc_matches(gpu_lib):
    import ctypes

    import torch
    from epb200 import _lib

    L = gpu_lib
    ctx = _lib.default_context()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(77)
    # two calls in a row with different inputs: the second must not see the first's scratch
    for nk, nw, (wmin, wmax) in [(300001, 16, (-0.5, 0.25)), (5000, 8, (-2.0, -1.0))]:
        e = np.sort(rng.standard_normal((nk, nw)) * 3, axis=1)  # (nk, nw) C order == Julia (nw, nk)
        e[7, :] = 0.25
        E = torch.from_numpy(e).cuda()
        ref = _run(L, L.epb_window_filter, ctx.h, E, wmin, wmax)
        got = _run(L, L.epb_window_filter_noalloc, stream, E, wmin, wmax)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b)
        assert ref[2].size > 0


def test_window_filter_noalloc_rejects_oversize(gpu_lib):
    import ctypes

    import torch

    L = gpu_lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    nk = 16384 * 1024 + 1
    st = L.epb_window_filter_noalloc(stream, 1, 16, nk, 0.0, 1.0, 1, 1, 1, 1, None)
    assert st == 1  # EPB_ERR_ARG, nothing launched
    assert b"exceeds the fixed scratch" in L.epb_last_error()
