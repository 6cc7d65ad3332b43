"""The configurations the benchmark and the measurements are quoted on, at
their full sizes, checked against the oracle (gold restatement, pinned to the
reference's known answers and to the reference's own gold kernel) on seeded
subsamples the oracle finishes in seconds:

* d=59 adaptive grid of 1M nodes, TotalDof 256, 1M points (half uniform, half
  N(0.5, 0.05^2)): the benchmark workload, node-chunked, on a 4,096-point
  subsample (seed 40);
* d=59 adaptive grid of 300k nodes, TotalDof 128, 32,768 points kept 1e-6
  from every kink: dL/dx and dL/dsurplus of L = sum c * f on a 1,024-point
  subsample against the oracle's gold-path gradient, and central differences;
* 8 adaptive d=30 grids (20k-200k nodes), TotalDof 64, ragged batches of
  1-100k points per grid in one call, 256 points per grid.

Plus FP32C on surpluses that stress its per-output bound: output columns of
very different scales, and a zero root row (outputs small next to the
grid's largest surplus).

FP64 form: bit-identical to gold.  FP32C form: max relative error <= 1e-7,
max_o |a - b| / max(|b_o|, 1e-3 * max_o |b_o|) per point.
"""
import os

import numpy as np
import pytest

import hddm_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu

FP32C_TOL = 1e-7
THREADS = os.cpu_count() or 1


def _dev(X):
    import torch
    return torch.from_numpy(np.ascontiguousarray(X)).cuda()


def test_c4_workload_subsample_against_oracle(cuda):
    """1M nodes, 1M points, TotalDof 256: both forms over every point (node
    chunks as the library picks them), checked on the 4,096-point subsample."""
    import torch
    hg = H.HostGrid.adaptive(59, 1_000_000, 256, seed=4)
    X = H.gen_points(59, 1_000_000, kind=2, seed=40)
    sub = np.sort(np.random.Generator(np.random.PCG64(40)).choice(len(X), 4096, replace=False))
    g = H.Grid(hg, flags=H.BUILD_FP32)
    x = _dev(X)
    o64 = H.interpolate(g, x, precision=H.FP64)
    o32 = H.interpolate(g, x, precision=H.FP32C)
    torch.cuda.synchronize()
    assert H.last_launch().kernels > 1          # node-chunked
    o64 = o64.cpu().numpy()[sub]
    o32 = o32.cpu().numpy()[sub]
    del x
    ref = O.Gold(*hg.arrays()).interpolate(X[sub], nthreads=THREADS)
    assert np.array_equal(o64, ref)
    e = O.rel_error(o32, ref)
    assert e[0] <= FP32C_TOL, e


def test_c3_backward_subsample_against_oracle(cuda):
    """300k nodes, TotalDof 128: dL/dx of the full 32,768-point batch on a
    1,024-point subsample, dL/dsurplus of the subsample's own loss, both
    against the oracle's gradient; and central differences (h = 1e-6) at 24
    coordinates."""
    import torch
    hg = H.HostGrid.adaptive(59, 300_000, 128, seed=3)
    X = H.gen_points(59, 32768, kind=0, seed=3, kink_reject=1e-6)
    C = np.random.Generator(np.random.PCG64(3)).standard_normal((32768, 128))
    sub = np.sort(np.random.Generator(np.random.PCG64(30)).choice(len(X), 1024, replace=False))
    g = H.Grid(hg)
    gx, _ = H.backward(g, _dev(X), _dev(C), want_surplus=False)
    gx_s, gs_s = H.backward(g, _dev(X[sub]), _dev(C[sub]))
    torch.cuda.synchronize()
    gx = gx.cpu().numpy()[sub]
    gx_s, gs_s = gx_s.cpu().numpy(), gs_s.cpu().numpy()
    ox, os_ = O.Gold(*hg.arrays()).gradient(X[sub], C[sub])
    assert np.array_equal(gx, gx_s)            # per-point: the batch does not change it
    assert np.abs(gx - ox).max() <= 1e-10 * np.abs(ox).max()
    assert np.abs(gs_s - os_).max() <= 1e-12 * np.abs(os_).max()

    def loss(p, xp):
        return float(H.interpolate(g, _dev(xp[None, :])).cpu().numpy()[0] @ C[p])

    rng = np.random.default_rng(33)
    h = 1e-6
    for p, k in zip(rng.choice(sub, 24), rng.integers(0, 59, 24)):
        xp, xm = X[p].copy(), X[p].copy()
        xp[k] += h
        xm[k] -= h
        fd = (loss(p, xp) - loss(p, xm)) / (2 * h)
        row = int(np.searchsorted(sub, p))
        assert abs(fd - gx[row, k]) <= 1e-5 * max(1.0, abs(fd)), (p, k, fd, gx[row, k])


def test_c2_multistate_subsample_against_oracle(cuda):
    """8 adaptive d=30 grids, TotalDof 64, ragged batches in one call: 256
    points of every grid (all of them below that)."""
    rng = np.random.Generator(np.random.PCG64(2))
    nnos = np.exp(rng.uniform(np.log(20_000), np.log(200_000), 8)).astype(int)
    counts = [int(c) for c in rng.integers(1, 100_001, 8)]
    hosts = [H.HostGrid.adaptive(30, int(n), 64, seed=200 + k) for k, n in enumerate(nnos)]
    grids = [H.Grid(h, flags=H.BUILD_FP32) for h in hosts]
    X = H.gen_points(30, sum(counts), kind=0, seed=2)
    x = _dev(X)
    o64 = H.interpolate(grids, x, counts=counts, precision=H.FP64).cpu().numpy()
    o32 = H.interpolate(grids, x, counts=counts, precision=H.FP32C).cpu().numpy()
    off = np.concatenate([[0], np.cumsum(counts)])
    pick = np.random.default_rng(22)
    for k, hgk in enumerate(hosts):
        rows = np.arange(off[k], off[k + 1])
        if len(rows) > 256:
            rows = np.sort(pick.choice(rows, 256, replace=False))
        ref = O.Gold(*hgk.arrays()).interpolate(X[rows], nthreads=THREADS)
        assert np.array_equal(o64[rows], ref), k
        e = O.rel_error(o32[rows], ref)
        assert e[0] <= FP32C_TOL, (k, e)


def _stressed(case, td):
    idx, sur = H.HostGrid.adaptive(59, 40_000, td, seed=71).arrays()
    sur = sur.copy()
    if case in ("columns", "both"):
        sur *= np.array([1.0, 1e-3, 1e-6, 1e-9])[np.arange(td) % 4]
    if case in ("zero_root", "both"):
        root = np.flatnonzero((idx == 0).all(axis=1))
        assert len(root) == 1
        sur[root] = 0.0
    return idx, sur


@pytest.mark.parametrize("td", [64, 256])
@pytest.mark.parametrize("npts", [64, 12_000])
@pytest.mark.parametrize("case", ["columns", "zero_root", "both"])
def test_fp32c_per_output_bound_on_stressed_surpluses(cuda, case, npts, td):
    """Output columns scaled by 1, 1e-3, 1e-6 and 1e-9, and a zero root row, so
    that a point's outputs are small next to the grid's largest surplus.
    12,000 points take the large-batch kernels, 64 the small-batch ones; rows
    of 256 outputs also read FP16 rows for their smallest fine terms."""
    idx, sur = _stressed(case, td)
    hg = H.HostGrid.from_dense(idx, sur)
    X = H.gen_points(59, npts, kind=2, seed=72)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    x = _dev(X)
    o64 = H.interpolate(g, x, precision=H.FP64).cpu().numpy()
    o32 = H.interpolate(g, x, precision=H.FP32C).cpu().numpy()
    rows = np.arange(npts) if npts <= 2048 else np.sort(np.random.default_rng(73).choice(npts, 2048, replace=False))
    ref = O.Gold(idx, sur).interpolate(X[rows], nthreads=THREADS)
    assert np.array_equal(o64[rows], ref)
    e = O.rel_error(o32[rows], ref)
    assert e[0] <= FP32C_TOL, e
