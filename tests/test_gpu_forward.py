"""Forward kernels on the GPU against the oracle (gold restatement, pinned to
the reference's known answers and to the reference's own gold kernel).

FP64 form: bit-identical to gold (same node order, same multiplies and adds).
FP32C form: max relative error <= 1e-7 against gold, with the error metric
max_o |a - b| / max(|b_o|, 1e-3 * max_o |b_o|) per point.
"""
import json
import os

import numpy as np
import pytest

import hddm_b200 as H
import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

PLT = os.path.join(GOLDEN, "interpolate_array_surplus.plt")
DOC = json.load(open(os.path.join(GOLDEN, "interpolate_array.json")))
FP32C_TOL = 1e-7


def _run(grid, X, precision=H.FP64, counts=None):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    out = H.interpolate(grid, x, counts=counts, precision=precision)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_reference_known_answer_fixture_bit_exact(cuda):
    hg = H.HostGrid.read_plt(PLT, 59)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    x = np.array(DOC["x"])[None, :]
    v = _run(g, x)[0]
    assert np.array_equal(v, np.array(DOC["ref_gold"]))
    assert np.abs(v - np.array(DOC["expected_test_cpp"])).max() < DOC["epsilon_test_cpp"]
    v32 = _run(g, x, H.FP32C)
    assert O.rel_error(v32, np.array(DOC["ref_gold"])[None])[0] <= FP32C_TOL
    # the host-pointer entry point gives the same bits
    assert np.array_equal(H.interpolate_host(g, x)[0], v)


def test_config0_regular_d4_bit_exact(cuda):
    hg = H.HostGrid.regular(4, 4, 8, seed=0)
    assert hg.nno == 137
    X = H.gen_points(4, 1024, kind=0, seed=0)
    ref = O.Gold(*hg.arrays()).interpolate(X)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    assert np.array_equal(_run(g, X), ref)
    assert O.rel_error(_run(g, X, H.FP32C), ref)[0] <= FP32C_TOL


def test_config1_regular_d16_bit_exact(cuda):
    hg = H.HostGrid.regular(16, 5, 32, seed=1)
    assert hg.nno == 51137
    X = H.gen_points(16, 65536, kind=0, seed=1)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    out = _run(g, X)
    sub = np.random.default_rng(11).choice(len(X), 2048, replace=False)
    ref = O.Gold(*hg.arrays()).interpolate(X[sub])
    assert np.array_equal(out[sub], ref)
    e32 = O.rel_error(_run(g, X, H.FP32C), out)
    assert e32[0] <= FP32C_TOL, e32


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_adaptive_d59_bit_exact(cuda, kind):
    hg = H.HostGrid.adaptive(59, 30000, 64, seed=3)
    X = H.gen_points(59, 512, kind=kind, seed=kind + 20)
    ref = O.Gold(*hg.arrays()).interpolate(X)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    assert np.array_equal(_run(g, X), ref)
    assert O.rel_error(_run(g, X, H.FP32C), ref)[0] <= FP32C_TOL


def test_td256_multi_pass_and_ragged_td(cuda):
    for td in (118, 256, 300, 5):
        hg = H.HostGrid.adaptive(12, 3000, td, seed=td)
        X = H.gen_points(12, 300, kind=2, seed=td)
        ref = O.Gold(*hg.arrays()).interpolate(X)
        g = H.Grid(hg, flags=H.BUILD_FP32)
        assert np.array_equal(_run(g, X), ref), td
        assert O.rel_error(_run(g, X, H.FP32C), ref)[0] <= FP32C_TOL, td


def test_multistate_ragged_batch_one_launch(cuda):
    """8 grids of uneven size, ragged point counts (including 0 and 1), one call."""
    rng = np.random.default_rng(2)
    hosts = [H.HostGrid.adaptive(30, int(n), 64, seed=100 + k)
             for k, n in enumerate(np.exp(rng.uniform(np.log(2000), np.log(20000), 8)).astype(int))]
    grids = [H.Grid(h, flags=H.BUILD_FP32) for h in hosts]
    counts = [37, 0, 1, 500, 3, 1200, 64, 9]
    X = H.gen_points(30, sum(counts), kind=0, seed=7)
    out = _run(grids, X, counts=counts)
    out32 = _run(grids, X, H.FP32C, counts=counts)
    off = np.concatenate([[0], np.cumsum(counts)])
    for k, h in enumerate(hosts):
        seg = slice(off[k], off[k + 1])
        if counts[k] == 0:
            continue
        ref = O.Gold(*h.arrays()).interpolate(X[seg])
        assert np.array_equal(out[seg], ref), k
        assert O.rel_error(out32[seg], ref)[0] <= FP32C_TOL, k
        assert np.array_equal(_run(grids[k], X[seg]), ref)
    # the reference's multistate call shape: one point per state
    X1 = H.gen_points(30, 8, kind=0, seed=8)
    out1 = _run(grids, X1, counts=[1] * 8)
    for k, h in enumerate(hosts):
        assert np.array_equal(out1[k], O.Gold(*h.arrays()).interpolate(X1[k])[0])


def test_edge_cases(cuda):
    import torch
    # root-only grid, a never-active node, duplicated node, points outside [0, 1]
    dim = 3
    index = np.array([[0, 0, 0, 0, 0, 0],
                      [2, 0, 0, 0, 0, 0],
                      [0, 0, 0, 5, 0, 0],     # i = 0, j = 5: weight 1 - 5 < 0 everywhere
                      [2, 0, 0, 0, 0, 0],     # duplicate of node 1
                      [4, 2, 0, 1, 0, 0],
                      [4, 2, 0, 1, 2, 0]], np.int32)
    sur = np.arange(6 * 3, dtype=np.float64).reshape(6, 3) / 7.0 - 1.0
    hg = H.HostGrid.from_dense(index, sur)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    X = np.array([[0.1, 0.2, 0.3], [0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.5, 0.5, 0.5],
                  [0.25, 0.25, 0.25], [-0.3, 1.7, 0.5], [0.125, 0.5 - 1e-17, 0.99]])
    ref = O.Gold(index, sur).interpolate(X)
    assert np.array_equal(_run(g, X), ref)
    assert O.rel_error(_run(g, X, H.FP32C), ref)[0] <= FP32C_TOL
    # root-only grid
    g1 = H.Grid(H.HostGrid.from_dense(index[:1], sur[:1]))
    assert np.array_equal(_run(g1, X), np.repeat(sur[:1], len(X), axis=0))
    # non-finite coordinates: gold multiplies NaN into every node
    Xn = np.array([[np.nan, 0.1, 0.2], [0.1, np.inf, 0.2]])
    assert np.isnan(_run(g, Xn)).all() and np.isnan(O.Gold(index, sur).interpolate(Xn)).all()
    # empty batch
    out = H.interpolate(g, torch.zeros((0, dim), dtype=torch.float64, device="cuda"))
    assert out.shape == (0, 3)


def test_grid_points_and_kinks_exact(cuda):
    """Points on grid nodes and hat kinks (hats exactly 0 there)."""
    hg = H.HostGrid.regular(5, 5, 16, seed=9)
    r = np.random.default_rng(4)
    X = r.integers(0, 17, size=(400, 5)) / 16.0
    ref = O.Gold(*hg.arrays()).interpolate(X)
    g = H.Grid(hg)
    assert np.array_equal(_run(g, X), ref)


def test_file_order_not_depth_first_still_exact(cuda):
    """Rows in random order: the tree degrades (many roots), results stay exact."""
    idx, sur = H.HostGrid.adaptive(16, 4000, 32, seed=5).arrays()
    perm = np.random.default_rng(1).permutation(len(idx))
    hg = H.HostGrid.from_dense(idx[perm], sur[perm])
    g = H.Grid(hg)
    assert g.info.tree_roots > 1
    X = H.gen_points(16, 256, kind=0, seed=3)
    assert np.array_equal(_run(g, X), O.Gold(idx[perm], sur[perm]).interpolate(X))


@pytest.mark.parametrize("rows", [1, 2, 3, 5, 17, 64])
def test_chunk_boundaries_everywhere(cuda, rows):
    """Tiny node chunks put a boundary inside every subtree: chunk roots are
    decided from the boundary's ancestor chain.  Depth-first grids, a grid
    in random order (many tree roots) and never-active nodes between live
    ones; FP64 stays bit-exact, FP32C within tolerance."""
    idx, sur = H.HostGrid.adaptive(8, 600, 16, seed=7).arrays()
    dead_i = np.zeros((3, idx.shape[1]), np.int32)
    dead_i[:, 8:] = 3                      # i = 0, j = 3 in every dimension: never active
    cases = [(idx, sur)]
    ins = np.insert(idx, [0, 1, 40, 41, 300], dead_i[[0, 1, 2, 0, 1]], axis=0)
    cases.append((ins, np.insert(sur, [0, 1, 40, 41, 300], 0.5, axis=0)))
    perm = np.random.default_rng(2).permutation(len(idx))
    cases.append((idx[perm], sur[perm]))
    X = H.gen_points(8, 300, kind=2, seed=9)
    prev = H.set_chunk_rows(rows)
    try:
        for ci, (i_, s_) in enumerate(cases):
            g = H.Grid(H.HostGrid.from_dense(i_, s_), flags=H.BUILD_FP32)
            ref = O.Gold(i_, s_).interpolate(X)
            assert np.array_equal(_run(g, X), ref), ci
            assert O.rel_error(_run(g, X, H.FP32C), ref)[0] <= FP32C_TOL, ci
    finally:
        H.set_chunk_rows(prev)


def test_active_count_matches_oracle(cuda):
    import torch
    hg = H.HostGrid.adaptive(59, 20000, 4, seed=3)
    X = H.gen_points(59, 64, kind=2, seed=6)
    g = H.Grid(hg)
    cnt = H.active_count(g, torch.from_numpy(X).cuda()).cpu().numpy()
    og = O.Gold(*hg.arrays())
    assert np.array_equal(cnt, [og.active_count(x) for x in X])


def test_errors(cuda):
    import torch
    a = H.Grid(H.HostGrid.regular(4, 3, 8, 0))
    b = H.Grid(H.HostGrid.regular(4, 3, 9, 0))
    x = torch.zeros((2, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(H.SgiError) as e:
        H.interpolate([a, b], x, counts=[1, 1])
    assert e.value.code == -2 and "TotalDof" in str(e.value)
    with pytest.raises(H.SgiError) as e:
        H.interpolate(a, x, precision=H.FP32C)   # built without BUILD_FP32
    assert e.value.code == -1


@pytest.mark.parametrize("rows", [37, 1000, 4096])
def test_chunked_walk_bit_exact(cuda, rows):
    """Node-range chunks (outputs carried across launches in FP64) keep gold's bits."""
    hosts = [H.HostGrid.adaptive(59, 12000, 64, seed=30), H.HostGrid.adaptive(59, 3000, 64, seed=31)]
    grids = [H.Grid(h, flags=H.BUILD_FP32) for h in hosts]
    counts = [300, 200]
    X = H.gen_points(59, 500, kind=2, seed=33)
    prev = H.set_chunk_rows(rows)
    try:
        out = _run(grids, X, counts=counts)
        out32 = _run(grids, X, H.FP32C, counts=counts)
        n = H.last_launch().kernels
    finally:
        H.set_chunk_rows(prev)
    assert n == -(-12000 // rows)
    for k, (h, sl) in enumerate(zip(hosts, (slice(0, 300), slice(300, 500)))):
        ref = O.Gold(*h.arrays()).interpolate(X[sl])
        assert np.array_equal(out[sl], ref), k
        assert O.rel_error(out32[sl], ref)[0] <= FP32C_TOL, k


@pytest.mark.parametrize("chunk_rows", [-1, 0, 777])
def test_graph_plan_bit_exact_and_replayable(cuda, chunk_rows):
    """A forward call recorded into a CUDA graph (autotuned or fixed chunks)
    replays to the bits of the direct call with the same node chunks; the FP64
    form also to gold's bits, whatever the chunks."""
    import torch
    hosts = [H.HostGrid.adaptive(59, 9000, 128, seed=50), H.HostGrid.adaptive(59, 4000, 128, seed=51)]
    grids = [H.Grid(h, flags=H.BUILD_FP32) for h in hosts]
    counts = [4000, 1000]
    X = H.gen_points(59, 5000, kind=2, seed=52)
    x = torch.from_numpy(X).cuda()
    for precision in (H.FP64, H.FP32C):
        out = torch.full((5000, 128), float("nan"), dtype=torch.float64, device="cuda")
        plan = H.Plan(grids, x, out, counts=counts, precision=precision, chunk_rows=chunk_rows)
        if chunk_rows >= 0:
            assert plan.chunk_rows == chunk_rows
        prev = H.set_chunk_rows(plan.chunk_rows)
        prev_v = H.set_fp32c_variant(plan.variant)
        try:
            direct = H.interpolate(grids, x, counts=counts, precision=precision).cpu().numpy()
        finally:
            H.set_chunk_rows(prev)
            H.set_fp32c_variant(prev_v)
        for _ in range(3):
            out.fill_(float("nan"))
            plan.launch()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.array_equal(got, direct), precision
        for k, (h, sl) in enumerate(zip(hosts, (slice(0, 4000), slice(4000, 5000)))):
            sub = np.arange(sl.start, sl.stop)[::37]
            ref = O.Gold(*h.arrays()).interpolate(X[sub])
            if precision == H.FP64:
                assert np.array_equal(got[sub], ref), k
            else:
                assert O.rel_error(got[sub], ref)[0] <= FP32C_TOL, k


@pytest.mark.parametrize("variant", [0, 1, 2, 4])
@pytest.mark.parametrize("td,rows", [(256, 0), (256, 1500), (128, 0), (300, 2000), (64, 0), (20, 0)])
def test_fp32c_variants_within_tolerance(cuda, variant, td, rows):
    """Every FP32C kernel variant (E = 1, 2 and 4 output layouts, one and two
    output passes, chunked or not; 0-2 walk by descent, 4 forces the window
    walk) stays within the FP32C tolerance of gold, and the FP64 form stays
    bit-exact under the same settings.  The FP32C grid keeps no FP64 rows, so
    that this small batch runs the FP32C kernels (with FP64 rows it would run
    the two-phase small-batch kernels)."""
    h = H.HostGrid.adaptive(59, 6000, td, seed=60 + td)
    g = H.Grid(h, flags=H.BUILD_FP32)
    g32 = H.Grid(h, flags=H.BUILD_FP32 | H.BUILD_NO_FP64)
    X = H.gen_points(59, 700, kind=2, seed=61)
    prev, prev_v = H.set_chunk_rows(rows), H.set_fp32c_variant(variant)
    try:
        out32 = _run(g32, X, H.FP32C)
        out64 = _run(g, X, H.FP64)
    finally:
        H.set_chunk_rows(prev)
        H.set_fp32c_variant(prev_v)
    ref = O.Gold(*h.arrays()).interpolate(X)
    assert np.array_equal(out64, ref)
    e = O.rel_error(out32, ref)
    assert e[0] <= FP32C_TOL, (variant, td, rows, e)


def test_wide_component_form_bit_exact(cuda):
    """Grids whose hat scales are not powers of two (or exceed the 32-bit
    packed form) use the wide components; still gold-exact."""
    rng = np.random.default_rng(8)
    dim = 6
    idx = np.zeros((300, 2 * dim), np.int32)
    for n in range(1, 300):
        for k in rng.choice(dim, rng.integers(1, 4), replace=False):
            idx[n, k] = int(rng.integers(1, 9))          # i = 3, 5, 6, ... too
            idx[n, dim + k] = int(rng.integers(0, idx[n, k] + 1))
    sur = rng.uniform(-1, 1, (300, 16))
    hg = H.HostGrid.from_dense(idx, sur)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    X = rng.random((400, dim))
    ref = O.Gold(idx, sur).interpolate(X)
    assert np.array_equal(_run(g, X), ref)
    assert O.rel_error(_run(g, X, H.FP32C), ref)[0] <= FP32C_TOL


def test_host_entry_pipelined_sub_batches(cuda):
    """Pinned host buffers with 192k points or more go through overlapped
    copy-in / kernel / copy-out sub-batches on two alternating compute
    streams (here five, of 75k and 150k points, one of them spanning both
    grids); FP64 stays gold-exact."""
    import ctypes
    import torch
    hosts = [H.HostGrid.adaptive(8, 3000, 40, seed=60), H.HostGrid.adaptive(8, 1500, 40, seed=61)]
    grids = [H.Grid(h, flags=H.BUILD_FP32) for h in hosts]
    counts = [450_000, 150_000]
    X = H.gen_points(8, sum(counts), kind=2, seed=62)
    xh = torch.from_numpy(X).pin_memory()
    outh = torch.zeros((sum(counts), 40), dtype=torch.float64).pin_memory()
    offs = np.array([0, counts[0], sum(counts)], np.int64)
    arr = (ctypes.c_void_p * 2)(grids[0].handle.value, grids[1].handle.value)
    for precision in (H.FP64, H.FP32C):
        rc = H.lib.sgi_interpolate_host(2, arr, offs.ctypes.data, xh.data_ptr(), outh.data_ptr(), precision)
        assert rc == 0, H.lib.sgi_last_error().decode()
        dev = _run(grids, X, precision, counts=counts)
        if precision == H.FP64:
            assert np.array_equal(outh.numpy(), dev)
            sub = np.r_[0:450_000:1997, 450_000:600_000:997]
            for k, sl in ((0, sub[sub < 450_000]), (1, sub[sub >= 450_000])):
                assert np.array_equal(dev[sl], O.Gold(*hosts[k].arrays()).interpolate(X[sl]))
        else:
            assert O.rel_error(outh.numpy(), dev)[0] <= 1e-9


def _deep_chain_grid(dim, depth, td, seed):
    """Nodes c_0 .. c_{depth-1}: c_k has the level-2 half hat at 0 (i=2, j=0)
    in dimensions 0 .. k-1, so each holds the next (a chain of containment);
    beside each c_k (k >= 1) a sibling with the half hat at 1 (i=2, j=2) in
    dimension k-1 forms a pair with it.  Depth-first order: the chain, then the
    siblings from the deepest up."""
    rows = []
    for k in range(depth):
        r = np.zeros(2 * dim, np.int32)
        r[:k] = 2
        rows.append(r)
    for k in range(depth - 1, 0, -1):
        r = np.zeros(2 * dim, np.int32)
        r[:k] = 2
        r[dim + k - 1] = 2
        rows.append(r)
    idx = np.array(rows)
    lev = np.where(idx[:, :dim] > 0, 1, 0).sum(axis=1)
    sur = np.random.default_rng(seed).uniform(-1, 1, (len(idx), td)) * 4.0 ** (-lev[:, None])
    return idx, sur


@pytest.mark.parametrize("rows", [0, 7])
def test_deep_tree_descent_and_fallback(cuda, rows):
    """A containment tree of depth 46: the FP32C descent handles it whole
    (depth <= 64); in node chunks (chains must be complete, depth <= 32) the
    window walk takes over.  FP64 bit-exact, FP32C within tolerance (on a
    grid without FP64 rows, so that this small batch runs the FP32C kernels)."""
    dim, depth = 48, 46
    idx, sur = _deep_chain_grid(dim, depth, 64, seed=3)
    hg = H.HostGrid.from_dense(idx, sur)
    g = H.Grid(hg)
    g32 = H.Grid(hg, flags=H.BUILD_FP32 | H.BUILD_NO_FP64)
    assert g.info.tree_depth == depth
    rng = np.random.default_rng(4)
    X = rng.uniform(0.0, 0.5, (400, dim))          # deep in the chain ...
    X[::3, rng.integers(0, dim, 400)[::3]] = 0.75  # ... and points that leave it early
    ref = O.Gold(idx, sur).interpolate(X)
    prev = H.set_chunk_rows(rows)
    try:
        assert np.array_equal(_run(g, X), ref)
        assert O.rel_error(_run(g32, X, H.FP32C), ref)[0] <= FP32C_TOL
    finally:
        H.set_chunk_rows(prev)


def _term_bounds(index, surplus, X):
    """|w_n(x)| * max_o |surplus[n][o]| for every point and node (FP64)."""
    dim = index.shape[1] // 2
    i, j = index[:, :dim].astype(np.float64), index[:, dim:].astype(np.float64)
    rowmax = np.abs(surplus).max(axis=1)
    out = np.zeros((len(X), len(index)))
    for p, x in enumerate(X):
        t = np.where(i != 0, 1.0 - np.abs(x[None, :] * i - j), 1.0)
        out[p] = np.where((t > 0).all(axis=1), np.clip(t, 0, None).prod(axis=1), 0.0) * rowmax
    return out


@pytest.mark.parametrize("variant,flags", [(H.FP32C_AUTO, H.BUILD_FP32),
                                           (H.FP32C_AUTO, H.BUILD_FP32 | H.BUILD_NO_FP64),
                                           (4, H.BUILD_FP32 | H.BUILD_NO_FP64)])
def test_surplus_cutoff_error_bound(cuda, variant, flags):
    """A surplus cutoff moves each FP32C output from gold by at most the sum of
    the skipped terms' bounds (plus the form's own 1e-7); cutoff <= 0 restores
    the default bits, and a plan made before the cutoff keeps the default.
    With FP64 rows kept, this small batch runs the two-phase kernels; without
    them the descent (automatic variant) or the window walk (variant 4)."""
    import torch
    hg = H.HostGrid.adaptive(59, 30000, 64, seed=3)
    index, surplus = hg.arrays()
    X = H.gen_points(59, 256, kind=2, seed=31)
    ref = O.Gold(index, surplus).interpolate(X)
    g = H.Grid(hg, flags=flags)
    prev = H.set_fp32c_variant(variant)
    try:
        x = torch.from_numpy(X).cuda()
        base = _run(g, X, H.FP32C)
        out_plan = torch.zeros(len(X), 64, dtype=torch.float64, device="cuda")
        plan = H.Plan(g, x, out_plan, precision=H.FP32C)
        plan.launch()
        torch.cuda.synchronize()
        plan_base = out_plan.cpu().numpy()
        floor = g.set_surplus_cutoff(0.0)
        assert floor == pytest.approx(np.abs(surplus).max() * 2.0 ** -42, rel=1e-6)
        assert g.set_surplus_cutoff(floor / 4) == floor
        smax = np.abs(surplus).max()
        bounds = _term_bounds(index, surplus, X)
        for k in (40, 30, 24):
            eff = g.set_surplus_cutoff(smax * 2.0 ** -k)
            assert eff == pytest.approx(smax * 2.0 ** -k, rel=1e-6)
            got = _run(g, X, H.FP32C)
            skipped = np.where(bounds < eff * (1 + 1e-5), bounds, 0.0).sum(axis=1)
            scale = np.maximum(np.abs(ref), 1e-3 * np.abs(ref).max(axis=1, keepdims=True))
            excess = np.abs(got - ref) - skipped[:, None] - FP32C_TOL * scale
            assert excess.max() <= 0, (k, excess.max())
            if k == 24:
                assert not np.array_equal(got, base)
        out_plan.zero_()
        plan.launch()
        torch.cuda.synchronize()
        assert np.array_equal(out_plan.cpu().numpy(), plan_base)
        assert g.set_surplus_cutoff(-1.0) == floor
        assert np.array_equal(_run(g, X, H.FP32C), base)
        if not flags & H.BUILD_NO_FP64:
            # the FP64 form ignores it
            g.set_surplus_cutoff(smax * 2.0 ** -10)
            assert np.array_equal(_run(g, X), ref)
        del plan
    finally:
        H.set_fp32c_variant(prev)


def test_surplus_cutoff_needs_fp32_form(cuda):
    g = H.Grid(H.HostGrid.regular(4, 3, 8, seed=0))
    with pytest.raises(H.SgiError):
        g.set_surplus_cutoff(1e-3)


def _deep_subtree_grid(td, seed):
    """A containment chain of depth 46 (_deep_chain_grid over 52 dimensions)
    whose deepest node holds a regular level-5 grid over dimensions 45-51
    (2,464 nodes at depths 47 to 51), placed right after it: the node chunk
    starting at 2,048 then lies below the 31 stored chain levels."""
    dim = 52
    idx, _ = _deep_chain_grid(dim, 46, td, seed)
    sub, _ = H.HostGrid.regular(7, 5, 1, seed=0).arrays()
    sub = sub[(sub[:, :7] != 0).any(axis=1)]          # the subtree root is the chain's last node
    rows = np.zeros((len(sub), 2 * dim), np.int32)
    rows[:, :45] = 2                                   # inside the last chain node (i = 2, j = 0, dims 0-44)
    rows[:, 45:52] = sub[:, :7]
    rows[:, dim + 45:dim + 52] = sub[:, 7:]
    idx = np.concatenate([idx[:46], rows, idx[46:]])
    lev = np.where(idx[:, :dim] > 0, 1, 0).sum(axis=1)
    sur = np.random.default_rng(seed).uniform(-1, 1, (len(idx), td)) * 2.0 ** (-lev[:, None])
    return idx, sur


@pytest.mark.parametrize("case", ["adaptive", "permuted", "dead", "deep"])
def test_small_batch_two_phase_exact(cuda, case):
    """Small FP64 batches walk node chunks of 2,048 in parallel and then add
    the listed hits in order: bit-identical to gold across chunk boundaries
    (grids in random order with many tree roots, never-active nodes between
    live ones, chunk starts deeper than the stored ancestor chains), through
    direct calls, a graph plan and the host-pointer entry, for one point and
    for a few hundred."""
    import torch
    if case == "deep":
        idx, sur = _deep_subtree_grid(40, seed=5)
        rng = np.random.default_rng(6)
        X = rng.uniform(0.0, 1.0, (300, 52))
        X[:, :45] *= 0.5                                # inside the chain ...
        X[::4, rng.integers(0, 45, 75)] = 0.8           # ... or leaving it
    else:
        idx, sur = H.HostGrid.adaptive(8, 9000, 40, seed=7).arrays()
        if case == "permuted":
            perm = np.random.default_rng(1).permutation(len(idx))
            idx, sur = idx[perm], sur[perm]
        elif case == "dead":
            dead = np.zeros((5, idx.shape[1]), np.int32)
            dead[:, 8:] = 3                             # i = 0, j = 3: never active
            at = [0, 2047, 2048, 4000, 8999]
            idx = np.insert(idx, at, dead, axis=0)
            sur = np.insert(sur, at, np.ones((5, sur.shape[1])), axis=0)
        X = H.gen_points(8, 300, kind=2, seed=9)
    hg = H.HostGrid.from_dense(idx, sur)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    assert g.nno > 2048
    if case == "deep":
        assert g.info.tree_depth > 32
    ref = O.Gold(idx, sur).interpolate(X)
    assert np.array_equal(_run(g, X), ref)
    assert np.array_equal(_run(g, X[:1]), ref[:1])
    # FP32C: the same kernels add the FP64 rows of the terms FP32C keeps
    # (dropped: bound below 2^-42 of the largest surplus)
    assert O.rel_error(_run(g, X, H.FP32C), ref)[0] <= FP32C_TOL
    assert np.array_equal(H.interpolate_host(g, X), ref)
    x = torch.from_numpy(X).cuda()
    out = torch.zeros(len(X), sur.shape[1], dtype=torch.float64, device="cuda")
    plan = H.Plan(g, x, out, precision=H.FP64)
    plan.launch()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
    del plan


@pytest.mark.parametrize("td", [64, 256])
def test_term_classes_partition_the_active_pairs(cuda, td):
    """sgi_term_classes: big + fine (FP32 rows) + fine (FP16 rows) + dropped =
    the active count per point; FP16 rows exist for 256-output rows only; a
    higher surplus cutoff only moves fine terms to dropped; an FP64-only grid
    is refused."""
    import torch
    hg = H.HostGrid.adaptive(59, 20000, td, seed=8)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    x = torch.from_numpy(H.gen_points(59, 700, kind=2, seed=9)).cuda()
    cnt = H.active_count(g, x).cpu().numpy()
    c0 = H.term_classes(g, x).cpu().numpy()
    assert np.array_equal(c0.sum(axis=1), cnt)
    assert c0[:, 0].sum() > 0 and c0[:, 1].sum() > 0 and c0[:, 3].sum() > 0
    assert (c0[:, 2].sum() > 0) == (td == 256)
    smax = g.set_surplus_cutoff(0.0) * 2.0 ** 42
    g.set_surplus_cutoff(smax * 2.0 ** -28)
    c1 = H.term_classes(g, x).cpu().numpy()
    g.set_surplus_cutoff(0.0)
    assert np.array_equal(c1[:, 0], c0[:, 0]) and np.array_equal(c1.sum(axis=1), cnt)
    assert c1[:, 2].sum() == 0          # the cutoff lies above the FP16 rows' bound
    assert (c1[:, 3] >= c0[:, 3]).all() and c1[:, 3].sum() > c0[:, 3].sum()
    with pytest.raises(H.SgiError):
        H.term_classes(H.Grid(hg), x)
