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


def _hat(x, ij):
    i = np.float64(int(ij) & 0xFFFF)
    j = np.float64(int(ij) >> 16)
    return 1.0 - abs(x * i - j)


def _descend(desc, x, lo, hi, starts, act, wfull):
    """The FP32C descent over the exported child groups for one point: from
    the start segments (group range, parent weight), every group yields at
    most one active child; hits outside [lo, hi) are not kept or expanded."""
    a, b, first, count, _ = desc
    hits = {}
    stack = list(starts)
    while stack:
        gb, ge, wp = stack.pop()
        for g in range(gb, ge):
            kind, d = (int(a[g, 2]) >> 16) & 3, int(a[g, 2]) & 0xFFFF
            c, w = None, None
            if kind == 0:
                h = _hat(x[d], b[g, 0])
                if h > 0:
                    c = int(a[g, 0])
                elif a[g, 1] != 0xFFFFFFFF:
                    h = _hat(x[d], b[g, 1])
                    if h > 0:
                        c = int(a[g, 1])
                if c is not None:
                    w = wp * h / (_hat(x[d], a[g, 3]) if a[g, 3] else 1.0)
            elif kind == 1:
                # several changed dimensions: every component is checked
                c = int(a[g, 0])
                c, w = (c, wfull[c]) if act[c] else (None, None)
            else:
                c, w = int(a[g, 0]), wp
            if c is None or not (lo <= c < hi):
                continue
            assert c not in hits
            hits[c] = w
            if count[c] and c + 1 < hi:
                stack.append((int(first[c]), int(first[c] + count[c]), w))
    return hits


@pytest.mark.parametrize("kind", ["regular", "adaptive", "shuffled", "fixture"])
def test_descent_groups_reach_exactly_the_active_nodes(kind):
    """Every node whose hats are all positive is reached exactly once, from
    the roots or from the active ancestors of a node-range start, with the
    weight of the full product; no other node is reached."""
    if kind == "regular":
        g, dim = H.HostGrid.regular(6, 4, 2, 0), 6
    elif kind == "adaptive":
        g, dim = H.HostGrid.adaptive(20, 3000, 2, 5), 20
    elif kind == "shuffled":
        idx, sur = H.HostGrid.adaptive(12, 1500, 2, 6).arrays()
        perm = np.random.default_rng(0).permutation(len(idx))
        g, dim = H.HostGrid.from_dense(idx[perm], sur[perm]), 12
    else:
        g, dim = H.HostGrid.read_plt(PLT, 59), 59
    desc = g.descent()
    a, b, first, count, npairs = desc
    idx, _ = g.arrays()
    skip, parent = g.tree()
    n = len(skip)
    assert len(first) == n + 1 and a.shape[0] == count.sum()
    if kind != "shuffled":
        assert npairs > 0
    i = idx[:, :dim].astype(np.float64)
    j = idx[:, dim:].astype(np.float64)
    X = H.gen_points(dim, 12, kind=2, seed=7)
    rng = np.random.default_rng(1)
    ranges = [(0, n)] + [tuple(sorted(rng.choice(n + 1, 2, replace=False))) for _ in range(4)]
    for x in X:
        h = 1.0 - np.abs(x[None, :] * i - j)
        nz = (i != 0) | (j != 0)
        act = np.all(np.where(nz, h > 0, True), axis=1)
        wfull = np.prod(np.where(nz, h, 1.0), axis=1)
        for lo, hi in ranges:
            starts = [(int(first[n]), int(first[n] + count[n]), 1.0)]
            if lo > 0:
                # the strict ancestors of lo: the groups of the active ones start the range
                q = lo - 1
                while q >= 0 and skip[q] <= lo:
                    q -= 1
                chain = []
                while q >= 0:
                    if skip[q] > lo:
                        chain.append(q)
                    q = parent[q]
                # activity along the ancestor path is monotone (nested
                # supports): the active ones are the shallowest
                starts += [(int(first[c]), int(first[c] + count[c]), wfull[c]) for c in chain if act[c]]
            hits = _descend(desc, x, lo, hi, starts, act, wfull)
            want = {c for c in range(lo, hi) if act[c]}
            assert set(hits) == want, (kind, lo, hi)
            for c, w in hits.items():
                assert abs(w - wfull[c]) <= 1e-13 * max(1.0, abs(wfull[c]))


SCAP = 96  # descent stack entries per warp (fwd_f32d_kernel)


def _stack_peak(desc, x, depth, lo=0, hi=None):
    """Largest stack size of the descent kernel's stepping rule for one point:
    each step takes min(32, SCAP - depth - size) groups (at least one) from
    the top ranges, ranges taken whole are popped, the range taken in part
    keeps its remainder, and every hit with children pushes a range."""
    a, b, first, count, _ = desc
    n = len(first) - 1
    hi = n if hi is None else hi
    stack = [[int(first[n]), int(first[n] + count[n])]]
    peak = len(stack)
    while stack:
        B = max(1, min(32, SCAP - depth - len(stack)))
        taken, take = [], B
        while take and stack:
            gb, ge = stack[-1]
            k = min(take, ge - gb)
            taken += range(gb, gb + k)
            take -= k
            if gb + k == ge:
                stack.pop()
            else:
                stack[-1][0] = gb + k
        for g in taken:
            kind, d = (int(a[g, 2]) >> 16) & 3, int(a[g, 2]) & 0xFFFF
            c = None
            if kind == 0:
                if _hat(x[d], b[g, 0]) > 0:
                    c = int(a[g, 0])
                elif a[g, 1] != 0xFFFFFFFF and _hat(x[d], b[g, 1]) > 0:
                    c = int(a[g, 1])
            else:
                c = int(a[g, 0])
            if c is not None and lo <= c < hi and count[c] and c + 1 < hi:
                stack.append([int(first[c]), int(first[c] + count[c])])
        peak = max(peak, len(stack))
    return peak


@pytest.mark.parametrize("kind", ["regular_wide", "adaptive", "fixture"])
def test_descent_stack_stays_within_capacity(kind):
    """The descent kernel's stack bound (depth <= SCAP - 32): replaying its
    stepping rule on grids with many children per node never needs more than
    SCAP entries."""
    if kind == "regular_wide":
        g, dim = H.HostGrid.regular(40, 3, 1, 0), 40
    elif kind == "adaptive":
        g, dim = H.HostGrid.adaptive(59, 20000, 1, 4), 59
    else:
        g, dim = H.HostGrid.read_plt(PLT, 59), 59
    desc = g.descent()
    _, parent = g.tree()
    depth = 1
    dep = np.zeros(len(parent), np.int64)
    for c in range(len(parent)):
        dep[c] = 1 if parent[c] < 0 else dep[parent[c]] + 1
    depth = int(dep.max())
    assert depth <= SCAP - 32
    for x in H.gen_points(dim, 8, kind=2, seed=3):
        assert _stack_peak(desc, x, depth) <= SCAP


def test_layout_cache_file(tmp_path):
    """The layout cache without a GPU: written deterministically, valid for
    its own .plt, flags and nagents, invalid once the .plt changes (size or
    modification time) or the file is damaged."""
    import os
    p = str(tmp_path / "g.plt")
    H.HostGrid.adaptive(30, 3000, 40, seed=5).write_plt(p)
    c1, c2 = str(tmp_path / "a.cache"), str(tmp_path / "b.cache")
    assert not H.cache_valid(p, 30, H.BUILD_FP32, c1)
    H.cache_write(p, 30, H.BUILD_FP32, c1)
    H.cache_write(p, 30, H.BUILD_FP32, c2)
    assert open(c1, "rb").read() == open(c2, "rb").read()
    assert H.cache_valid(p, 30, H.BUILD_FP32, c1)
    assert not H.cache_valid(p, 30, 0, c1)          # other build flags
    assert not H.cache_valid(p, 29, H.BUILD_FP32, c1)
    # the default name sits beside the .plt
    H.cache_write(p, 30, 0)
    assert os.path.exists(p + ".sgi-layout") and H.cache_valid(p, 30, 0)
    # damage: one flipped byte in the middle, or a truncated file
    b = bytearray(open(c1, "rb").read())
    b[len(b) // 2] ^= 0x40
    open(c2, "wb").write(bytes(b))
    assert not H.cache_valid(p, 30, H.BUILD_FP32, c2)
    open(c2, "wb").write(bytes(b[: len(b) - 100]))
    assert not H.cache_valid(p, 30, H.BUILD_FP32, c2)
    # a rewritten .plt (new modification time) makes the cache stale
    st = os.stat(p)
    os.utime(p, ns=(st.st_atime_ns, st.st_mtime_ns + 1000))
    assert not H.cache_valid(p, 30, H.BUILD_FP32, c1)
    with pytest.raises(H.SgiError):
        H.cache_write(str(tmp_path / "missing.plt"), 30, 0)
