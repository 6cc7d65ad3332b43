"""Host layer of the product (no GPU): grid files, generators, the reference's
xps/chains form, and the containment tree the kernels walk."""
import json
import os
import struct

import numpy as np
import pytest

import hddm_b200 as H
import oracle as O
from conftest import GOLDEN

PLT = os.path.join(GOLDEN, "interpolate_array_surplus.plt")


def test_reader_matches_oracle_reader_on_reference_fixture():
    hg = H.HostGrid.read_plt(PLT, 59)
    idx, sur = hg.arrays()
    og = O.Gold.read_plt(PLT, 59)
    assert np.array_equal(idx, og.index) and np.array_equal(sur, og.surplus)
    assert hg.shape() == (59, 119, 118)


def test_reader_errors(tmp_path):
    with pytest.raises(H.SgiError) as e:
        H.HostGrid.read_plt(PLT, 60)
    assert e.value.code == -2 and "mismatches config" in str(e.value)
    with pytest.raises(H.SgiError) as e:
        H.HostGrid.read_plt(str(tmp_path / "missing.plt"), 59)
    assert e.value.code == -3
    data = open(PLT, "rb").read()
    for cut in (5, 30, 200, len(data) - 3):
        p = tmp_path / f"cut{cut}.plt"
        p.write_bytes(data[:cut])
        with pytest.raises(H.SgiError) as e:
            H.HostGrid.read_plt(str(p), 59)
        assert e.value.code in (-3, -2)
    # corrupt the index block's IA[0] (first row delta after the pairs)
    nnz = struct.unpack_from("<I", data, 31)[0]
    bad = bytearray(data)
    bad[35 + 4 * nnz] = 7
    p = tmp_path / "ia0.plt"
    p.write_bytes(bytes(bad))
    with pytest.raises(H.SgiError, match="IA"):
        H.HostGrid.read_plt(str(p), 59)


def _levels_form(index, dim):
    """Dense (i, j) back to the uncompressed layouts' (level, 1-based index)."""
    i = index[:, :dim]
    j = index[:, dim:]
    lev = np.where(i == 0, 1, np.log2(np.maximum(i, 1)).astype(np.int64) + 1)
    ind = np.where(i == 0, 1, j + 1)
    return lev.astype(np.int32), ind.astype(np.int32)


@pytest.mark.parametrize("layout", ["binary", "text"])
def test_uncompressed_layouts_read_like_oracle(tmp_path, layout):
    g = H.HostGrid.regular(5, 3, 3, seed=4)
    idx, sur = g.arrays()
    lev, ind = _levels_form(idx, 5)
    p = tmp_path / f"g.{layout}"
    if layout == "binary":
        with open(p, "wb") as f:
            f.write(struct.pack("<4i", 5, g.nno, 3, 2))
            for n in range(g.nno):
                f.write(lev[n].tobytes() + ind[n].tobytes() + sur[n].tobytes())
    else:
        with open(p, "w") as f:
            f.write(f"5 {g.nno} 3 2\n")
            for n in range(g.nno):
                f.write(" ".join(map(str, lev[n])) + " " + " ".join(map(str, ind[n])) + " " +
                        " ".join(repr(float(v)) for v in sur[n]) + "\n")
    h2 = H.HostGrid.read_plt(str(p), 5)
    i2, s2 = h2.arrays()
    assert np.array_equal(i2, idx) and np.array_equal(s2, sur)
    og = O.Gold.read_plt(str(p), 5)
    assert np.array_equal(og.index, idx) and np.array_equal(og.surplus, sur)


def test_writer_round_trip(tmp_path):
    for g, d in ((H.HostGrid.regular(4, 4, 8, 0), 4), (H.HostGrid.adaptive(30, 3000, 64, 2), 30)):
        p = tmp_path / "rt.plt"
        g.write_plt(str(p))
        g2 = H.HostGrid.read_plt(str(p), d)
        a, b = g.arrays(), g2.arrays()
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        og = O.Gold.read_plt(str(p), d)
        assert np.array_equal(og.index, a[0]) and np.array_equal(og.surplus, a[1])


def test_generators():
    # regular grids: node counts of sum(l-1) <= L-1 (C0: 137, C1: 51137)
    assert H.HostGrid.regular(4, 4, 8, 0).nno == 137
    assert H.HostGrid.regular(16, 5, 32, 1).nno == 51137
    assert H.HostGrid.regular(59, 2, 118, 0).nno == 119
    # deterministic per seed, different across seeds
    a = H.HostGrid.adaptive(59, 5000, 8, 3).arrays()
    b = H.HostGrid.adaptive(59, 5000, 8, 3).arrays()
    c = H.HostGrid.adaptive(59, 5000, 8, 4).arrays()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])
    idx = a[0]
    # levels <= 7 (i <= 64), distinct nodes, surplus scale 2^(-2 |l|_1)
    assert idx[:, :59].max() <= 64
    assert len({r.tobytes() for r in idx}) == 5000
    i = idx[:, :59]
    depth = np.where(i > 0, np.log2(np.maximum(i, 1)), 0).sum(axis=1)
    assert np.all(np.abs(a[1]) <= 2.0 ** (-2 * depth)[:, None])
    X = H.gen_points(59, 1000, kind=2, seed=1, kink_reject=1e-6)
    assert X.min() >= 0 and X.max() <= 1
    r = X * 64
    assert np.abs(r - np.round(r)).min() * (1 / 64) >= 1e-6
    assert abs(X[500:].mean() - 0.5) < 0.01 and X[500:].std() < 0.06


def _check_xps_chains_vs_reference(g, dim, tmp_path):
    p = tmp_path / "x.plt"
    g.write_plt(str(p))
    r = O.RefGrid(str(p), dim, "x86")
    xr, cr = r.xps_chains()
    xm, cm, perm = g.xps_chains()
    assert np.array_equal(xr, xm)
    assert np.array_equal(cr, cm)
    assert np.array_equal(r.surplus(), g.arrays()[1][perm])


@pytest.mark.skipif(not O.ref_available("x86"), reason="reference not compiled here")
def test_xps_chains_bit_identical_to_reference_x86_loader(tmp_path):
    # the reference's fixture, C1's regular grid, an adaptive d=59 grid
    hg = H.HostGrid.read_plt(PLT, 59)
    r = O.RefGrid(PLT, 59, "x86")
    xr, cr = r.xps_chains()
    xm, cm, perm = hg.xps_chains()
    assert np.array_equal(xr, xm) and np.array_equal(cr, cm)
    _check_xps_chains_vs_reference(H.HostGrid.regular(16, 5, 32, 1), 16, tmp_path)
    _check_xps_chains_vs_reference(H.HostGrid.adaptive(59, 20000, 4, 3), 59, tmp_path)
    _check_xps_chains_vs_reference(H.HostGrid.adaptive(30, 8000, 4, 9, max_level=7, p_dim=0.3), 30, tmp_path)


def _supports(index, dim):
    i = index[:, :dim].astype(np.float64)
    j = index[:, dim:].astype(np.float64)
    lo = np.where(i > 0, (j - 1) / np.maximum(i, 1), -np.inf)
    hi = np.where(i > 0, (j + 1) / np.maximum(i, 1), np.inf)
    return lo, hi


@pytest.mark.parametrize("kind", ["regular", "adaptive", "shuffled", "fixture"])
def test_containment_tree_invariants(kind):
    if kind == "regular":
        g, dim = H.HostGrid.regular(6, 4, 2, 0), 6
    elif kind == "adaptive":
        g, dim = H.HostGrid.adaptive(20, 4000, 2, 5), 20
    elif kind == "shuffled":
        idx, sur = H.HostGrid.adaptive(20, 2000, 2, 6).arrays()
        perm = np.random.default_rng(0).permutation(len(idx))
        g, dim = H.HostGrid.from_dense(idx[perm], sur[perm]), 20
    else:
        g, dim = H.HostGrid.read_plt(PLT, 59), 59
    skip, parent = g.tree()
    idx, _ = g.arrays()
    lo, hi = _supports(idx, dim)
    n = len(skip)
    assert np.all(skip > np.arange(n)) and np.all(skip <= n)
    for c in range(n):
        p = parent[c]
        if p < 0:
            continue
        assert p < c and skip[p] >= skip[c] and c < skip[p]          # nested ranges
        assert np.all(lo[p] <= lo[c]) and np.all(hi[c] <= hi[p])     # nested supports
    if kind in ("regular", "adaptive", "fixture"):
        assert (parent < 0).sum() == 1                               # one root: depth-first order


def test_grid_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    with pytest.raises(H.SgiError) as e:
        H.Grid(H.HostGrid.regular(4, 2, 2, 0))
    assert e.value.code == -7
