"""Small FP64 calls through the host-pointer entry replay a CUDA graph kept per
call shape (device, grids, point offsets).  The kept graphs must give gold's
bits on every call, follow a grid that was destroyed and replaced by another
(possibly at the same address) with the same shape, and survive the staging
buffers being replaced by larger ones in between."""
import gc

import numpy as np
import pytest

import hddm_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu


def _gold(hg, X):
    return O.Gold(*hg.arrays()).interpolate(X)


def test_repeated_small_calls_stay_gold_exact(cuda):
    hosts = [H.HostGrid.adaptive(12, 4000, 40, seed=70 + k) for k in range(3)]
    grids = [H.Grid(h) for h in hosts]
    X = H.gen_points(12, 3, kind=2, seed=73)
    ref = np.stack([_gold(hosts[k], X[k:k + 1])[0] for k in range(3)])
    for _ in range(4):                                 # first call records, later ones replay
        got = H.interpolate_host(grids, X, counts=[1, 1, 1])
        assert np.array_equal(got, ref)
        assert np.array_equal(H.interpolate_host(grids[1], X[1:2])[0], ref[1])
    # another point set of the same shape reuses the graph with the new coordinates
    X2 = H.gen_points(12, 3, kind=0, seed=74)
    ref2 = np.stack([_gold(hosts[k], X2[k:k + 1])[0] for k in range(3)])
    assert np.array_equal(H.interpolate_host(grids, X2, counts=[1, 1, 1]), ref2)


def test_replaced_grid_and_grown_staging_buffers(cuda):
    X = H.gen_points(10, 5, kind=2, seed=80)
    for k in range(4):
        hg = H.HostGrid.adaptive(10, 3000, 24, seed=81 + k)
        g = H.Grid(hg)
        for _ in range(2):
            assert np.array_equal(H.interpolate_host(g, X), _gold(hg, X))
        # a large call between two small ones replaces the staging buffers
        big = H.gen_points(10, 70_000, kind=0, seed=90 + k)
        out = H.interpolate_host(g, big)
        sub = slice(0, 70_000, 997)
        assert np.array_equal(out[sub], _gold(hg, big[sub]))
        assert np.array_equal(H.interpolate_host(g, X), _gold(hg, X))
        del g
        gc.collect()                                   # the next grid may reuse the address
