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
