"""sgi_interpolate_noalloc: the forward pass for callers that must not allocate
device memory (a solver whose device memory is all in its own arena, a loop
that cannot take cudaMalloc's implicit synchronization).  Its work counters
live in a fixed array of the library's device image instead of a workspace
allocated on first use.

Checked through the C ABI against sgi_interpolate, the entry point that
allocates its workspace, on two calls in a row (the shared counter array keeps
the previous call's contents, so the second call shows it is cleared).  The
FP64 form must match bit for bit, as every FP64 test here does.  The FP32C
form must match sgi_interpolate's FP32C bits on a large batch; on a small one
sgi_interpolate adds the kept terms' FP64 rows in its two-phase kernels,
which this entry cannot use (they need scratch), so there both stay within
1e-7 of FP64 instead.

Named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

import hddm_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu

_fn = H.lib.sgi_interpolate_noalloc
_fn.restype = ctypes.c_int
_fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_int, ctypes.c_void_p]
SGI_E_RANGE = -4
MAX_LAUNCHES = 64


def _noalloc(grids, x, counts, precision, out):
    import torch
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    arr = (ctypes.c_void_p * len(grids))(*[g.handle.value for g in grids])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _fn(len(grids), arr, offs.ctypes.data, x.data_ptr(), out.data_ptr(), precision, stream)


@pytest.mark.parametrize("counts", [[700, 0, 13, 1500], [5, 0, 3, 9]])
def test_noalloc_matches_allocating_entry_point(cuda, counts):
    """A batch of 2,213 points, and one of 17 (small batches take their own
    kernels), through both entry points."""
    import torch
    hosts = [H.HostGrid.adaptive(30, n, 300, seed=40 + k) for k, n in enumerate((3000, 9000, 500, 6000))]
    grids = [H.Grid(h, flags=H.BUILD_FP32) for h in hosts]
    X = H.gen_points(30, sum(counts), kind=2, seed=12)
    x = torch.from_numpy(X).cuda()
    ref64 = H.interpolate(grids, x, counts=counts, precision=H.FP64).cpu().numpy()
    ref32 = H.interpolate(grids, x, counts=counts, precision=H.FP32C).cpu().numpy()
    small = sum(counts) < 1000
    for precision, ref in ((H.FP64, ref64), (H.FP32C, ref32)):
        for call in range(2):
            out = torch.full((x.shape[0], 300), float("nan"), dtype=torch.float64, device="cuda")
            rc = _noalloc(grids, x, counts, precision, out)
            assert rc == 0, H.lib.sgi_last_error().decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            if precision == H.FP32C and small:
                assert O.rel_error(got, ref64)[0] <= 1e-7, call
            else:
                assert np.array_equal(got, ref), (precision, call)
    assert O.rel_error(ref32, ref64)[0] <= 1e-7


def test_noalloc_unchunked_matches_chunked_allocating_entry_point(cuda):
    """sgi_interpolate walks large grids in node chunks, carrying the outputs
    between launches; this entry launches every grid whole.  FP64 keeps gold's
    order either way: the bits agree with a forced chunking of 1,000 nodes,
    on two calls in a row.  FP32C stays within 1e-7 of FP64."""
    import torch
    hg = H.HostGrid.adaptive(59, 20000, 256, seed=45)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    X = H.gen_points(59, 6000, kind=2, seed=46)
    x = torch.from_numpy(X).cuda()
    prev = H.set_chunk_rows(1000)
    try:
        ref64 = H.interpolate(g, x, precision=H.FP64)
        assert H.last_launch().kernels > 1        # node-chunked
        ref64 = ref64.cpu().numpy()
    finally:
        H.set_chunk_rows(prev)
    for precision in (H.FP64, H.FP32C):
        for call in range(2):
            out = torch.full((x.shape[0], 256), float("nan"), dtype=torch.float64, device="cuda")
            assert _noalloc([g], x, [x.shape[0]], precision, out) == 0, H.lib.sgi_last_error().decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            if precision == H.FP64:
                assert np.array_equal(got, ref64), call
            else:
                assert O.rel_error(got, ref64)[0] <= 1e-7, call


def test_noalloc_rejects_requests_beyond_its_scratch(cuda):
    import torch
    td = 256 * (MAX_LAUNCHES + 1)   # one launch per 256 outputs: 65 launches
    idx = np.zeros((2, 4), np.int32)
    idx[1, 0] = 2
    hg = H.HostGrid.from_dense(idx, np.ones((2, td)))
    g = H.Grid(hg)
    x = torch.full((3, 2), 0.25, dtype=torch.float64, device="cuda")
    out = torch.zeros((3, td), dtype=torch.float64, device="cuda")
    rc = _noalloc([g], x, [3], H.FP64, out)
    assert rc == SGI_E_RANGE
    assert "at most 64" in H.lib.sgi_last_error().decode()
    # the same grid through the allocating entry point works
    assert float(H.interpolate(g, x).sum()) == pytest.approx(3 * td * 1.5)
