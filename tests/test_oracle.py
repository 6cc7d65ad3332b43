"""The oracle pinned against the reference's own known answers."""
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN

PLT = os.path.join(GOLDEN, "interpolate_array_surplus.plt")
DOC = json.load(open(os.path.join(GOLDEN, "interpolate_array.json")))


def test_oracle_reproduces_reference_known_answers():
    """LinearBasis/tests/InterpolateArray/test.cpp: surplus.plt at init()'s x, check() at 1e-3."""
    g = O.Gold.read_plt(PLT, DOC["nagents"])
    assert (g.dim, g.total_dof) == (59, 118)
    v = g.interpolate(np.array(DOC["x"]))[0]
    assert np.abs(v - np.array(DOC["expected_test_cpp"])).max() < DOC["epsilon_test_cpp"]


def test_oracle_bit_identical_to_reference_gold_outputs():
    """The committed outputs of the reference's gold kernel (compiled in place) match bit for bit."""
    g = O.Gold.read_plt(PLT, DOC["nagents"])
    v = g.interpolate(np.array(DOC["x"]))[0]
    assert np.array_equal(v, np.array(DOC["ref_gold"]))
    # the other reference variants sum in another order: equal to ~1e-13
    for k in ("ref_x86", "ref_avx2"):
        assert np.abs(v - np.array(DOC[k])).max() < 1e-12


@pytest.mark.skipif(not O.ref_available("gold"), reason="reference not compiled here")
def test_oracle_matches_reference_gold_on_random_points():
    g = O.Gold.read_plt(PLT, 59)
    r = O.RefGrid(PLT, 59, "gold")
    X = np.random.default_rng(0).random((200, 59))
    assert np.array_equal(g.interpolate(X), r.interpolate(X))
    assert np.array_equal(g.index, r.index()) and np.array_equal(g.surplus, r.surplus())


@pytest.mark.skipif(not O.ref_available("gold"), reason="reference not compiled here")
@pytest.mark.parametrize("dim,nno,td,seed", [(59, 20000, 64, 3), (30, 8000, 32, 2), (16, 51137, 32, 1)])
def test_oracle_bit_identical_to_reference_gold_on_generated_grids(tmp_path, dim, nno, td, seed):
    """Generated grids (adaptive d=59 and d=30, regular d=16 level 5) written
    as .plt and read back by the reference's own gold loader: the oracle's
    reader gives the same arrays, and the oracle's kernel the reference gold
    kernel's bits, on points of both distributions."""
    import hddm_b200 as H
    hg = H.HostGrid.regular(16, 5, 32, seed=seed) if dim == 16 else H.HostGrid.adaptive(dim, nno, td, seed=seed)
    p = str(tmp_path / "grid.plt")
    hg.write_plt(p)
    g = O.Gold.read_plt(p, dim)
    r = O.RefGrid(p, dim, "gold")
    assert np.array_equal(g.index, r.index()) and np.array_equal(g.surplus, r.surplus())
    X = H.gen_points(dim, 256, kind=2, seed=seed + 50)
    assert np.array_equal(g.interpolate(X), r.interpolate(X))


@pytest.mark.parametrize("dim,nno,td,seed", [(59, 30000, 16, 4), (30, 5000, 64, 203), (3, 40, 2, 9)])
def test_oracle_generator_matches_product_generator(tmp_path, dim, nno, td, seed):
    """The oracle's restatement of the seeded workload (used by the CPU
    reference arm, which must not load the product library) gives the product
    generator's grid and points array for array, and its .plt file reads back
    to the same arrays."""
    import hddm_b200 as H
    og = O.Gold.adaptive(dim, nno, td, seed)
    pi, ps = H.HostGrid.adaptive(dim, nno, td, seed=seed).arrays()
    assert np.array_equal(og.index, pi) and np.array_equal(og.surplus, ps)
    for kind, kr in ((0, 0.0), (1, 0.0), (2, 0.0), (0, 1e-6)):
        assert np.array_equal(O.gen_points(dim, 301, kind, seed, kr), H.gen_points(dim, 301, kind, seed, kr)), kind
    p = str(tmp_path / "g.plt")
    og.write_plt(p)
    back = O.Gold.read_plt(p, dim)
    assert np.array_equal(back.index, pi) and np.array_equal(back.surplus, ps)
    q = str(tmp_path / "h.plt")
    H.HostGrid.adaptive(dim, nno, td, seed=seed).write_plt(q)
    assert open(p, "rb").read() == open(q, "rb").read()


def test_oracle_reader_rejects_bad_input(tmp_path):
    with pytest.raises(ValueError, match="mismatches config"):
        O.Gold.read_plt(PLT, 58)
    bad = tmp_path / "trunc.plt"
    bad.write_bytes(open(PLT, "rb").read()[:1000])
    with pytest.raises(ValueError):
        O.Gold.read_plt(str(bad), 59)
    with pytest.raises(ValueError, match="opening"):
        O.Gold.read_plt(str(tmp_path / "none.plt"), 59)


def test_oracle_gradient_matches_finite_differences():
    g = O.Gold.read_plt(PLT, 59)
    rng = np.random.default_rng(3)
    X = rng.random((4, 59))
    X = np.where(np.abs(X - 0.5) < 1e-3, X + 0.01, X)
    C = rng.standard_normal((4, 118))
    dx, ds = g.gradient(X, C)
    h = 1e-6
    for p in range(4):
        for k in (0, 7, 58):
            xp = X[p].copy(); xm = X[p].copy()
            xp[k] += h; xm[k] -= h
            fd = (C[p] @ (g.interpolate(xp)[0] - g.interpolate(xm)[0])) / (2 * h)
            assert abs(fd - dx[p, k]) <= 1e-5 * max(1.0, abs(fd))
    # dL/dsurplus is linear: sum_p c[p,o] * w_n(x_p)
    assert np.isfinite(ds).all()


@pytest.mark.parametrize("variant", ["x86", "avx2"])
def test_reference_simd_kernels_agree_with_oracle_on_a_generated_grid(tmp_path, variant):
    """The reference's own sparse CPU kernels (compiled in place) on an
    adaptive d=59 grid: within 1e-12 of the oracle's gold restatement, which
    sums in another order."""
    import bench
    if not O.ref_available(variant):
        pytest.skip("reference not compiled here")
    if variant == "avx2" and not bench.ref_variants():
        pytest.skip("this host cannot run the avx2 kernel")
    import hddm_b200 as H
    hg = H.HostGrid.adaptive(59, 12000, 48, seed=17)
    p = str(tmp_path / "grid.plt")
    hg.write_plt(p)
    X = H.gen_points(59, 300, kind=2, seed=18)
    ref = O.Gold(*hg.arrays()).interpolate(X)
    got = O.RefGrid(p, 59, variant).interpolate(X, nthreads=4)
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
