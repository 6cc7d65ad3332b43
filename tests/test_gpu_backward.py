"""Backward kernel: dL/dx and dL/dsurplus for L = sum_p sum_o c[p,o] f_o(x_p),
checked against the oracle's gold-path gradient and central finite differences
(h = 1e-6, FP64) at points kept 1e-6 away from every hat kink."""
import numpy as np
import pytest

import hddm_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu


def _grad(g, X, C):
    import torch
    x = torch.from_numpy(X).cuda()
    c = torch.from_numpy(C).cuda()
    gx, gs = H.backward(g, x, c)
    torch.cuda.synchronize()
    return gx.cpu().numpy(), gs.cpu().numpy()


@pytest.mark.parametrize("dim,nno,td", [(59, 20000, 128), (16, 6000, 32), (8, 2000, 256)])
def test_backward_matches_oracle_gradient(cuda, dim, nno, td):
    hg = H.HostGrid.adaptive(dim, nno, td, seed=dim)
    X = H.gen_points(dim, 256, kind=0, seed=1, kink_reject=1e-6)
    C = np.random.default_rng(2).standard_normal((256, td))
    g = H.Grid(hg)
    gx, gs = _grad(g, X, C)
    ox, os_ = O.Gold(*hg.arrays()).gradient(X, C)
    sx = np.abs(ox).max() + 1e-300
    ss = np.abs(os_).max() + 1e-300
    assert np.abs(gx - ox).max() <= 1e-10 * sx
    assert np.abs(gs - os_).max() <= 1e-12 * ss


def test_backward_matches_finite_differences(cuda):
    import torch
    hg = H.HostGrid.adaptive(59, 20000, 128, seed=3)
    g = H.Grid(hg)
    X = H.gen_points(59, 64, kind=0, seed=4, kink_reject=1e-6)
    C = np.random.default_rng(5).standard_normal((64, 128))
    gx, gs = _grad(g, X, C)
    h = 1e-6

    def L(Xe):
        x = torch.from_numpy(np.ascontiguousarray(Xe)).cuda()
        return float((H.interpolate(g, x).cpu().numpy() * C).sum())

    rng = np.random.default_rng(6)
    for p, k in zip(rng.integers(0, 64, 24), rng.integers(0, 59, 24)):
        Xp = X.copy(); Xm = X.copy()
        Xp[p, k] += h; Xm[p, k] -= h
        fd = (L(Xp) - L(Xm)) / (2 * h)
        assert abs(fd - gx[p, k]) <= 1e-5 * max(1.0, abs(fd)), (p, k, fd, gx[p, k])
    # dL/dsurplus: L is linear in the surplus, so a finite difference along a
    # random direction equals the inner product with the gradient.
    idx, sur = hg.arrays()
    D = rng.standard_normal(sur.shape)
    hp = H.Grid(H.HostGrid.from_dense(idx, sur + 1e-3 * D))
    hm = H.Grid(H.HostGrid.from_dense(idx, sur - 1e-3 * D))
    x = torch.from_numpy(X).cuda()
    fd = ((H.interpolate(hp, x).cpu().numpy() - H.interpolate(hm, x).cpu().numpy()) * C).sum() / 2e-3
    assert abs(fd - (gs * D).sum()) <= 1e-5 * max(1.0, abs(fd))


def test_backward_deterministic_and_autograd(cuda):
    import torch
    hg = H.HostGrid.adaptive(20, 5000, 64, seed=8)
    g = H.Grid(hg)
    X = H.gen_points(20, 500, kind=2, seed=9, kink_reject=1e-6)
    C = np.random.default_rng(10).standard_normal((500, 64))
    a = _grad(g, X, C)
    b = _grad(g, X, C)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    F = H.make_function()
    x = torch.from_numpy(X).cuda().requires_grad_(True)
    token = torch.zeros((g.nno, g.total_dof), dtype=torch.float64, device="cuda", requires_grad=True)
    y = F.apply(x, token, g)
    (y * torch.from_numpy(C).cuda()).sum().backward()
    assert np.array_equal(x.grad.cpu().numpy(), a[0])
    assert np.array_equal(token.grad.cpu().numpy(), a[1])


def test_backward_empty_and_no_outputs(cuda):
    import torch
    g = H.Grid(H.HostGrid.regular(4, 3, 8, 0))
    x = torch.zeros((0, 4), dtype=torch.float64, device="cuda")
    gx, gs = H.backward(g, x, torch.zeros((0, 8), dtype=torch.float64, device="cuda"))
    assert gx.shape == (0, 4) and float(gs.abs().sum()) == 0.0


def test_sharded_backward_single_rank_is_the_kernel(cuda):
    """Without a process group, backward_sharded is the GPU backward itself."""
    import torch
    from hddm_b200.shard import backward_sharded
    hg = H.HostGrid.adaptive(16, 3000, 32, seed=8)
    g = H.Grid(hg)
    X = H.gen_points(16, 128, kind=0, seed=9, kink_reject=1e-6)
    C = np.random.default_rng(3).standard_normal((128, 32))
    x, c = torch.from_numpy(X).cuda(), torch.from_numpy(C).cuda()
    gx, gs = backward_sharded(g, x, c)
    rx, rs = H.backward(g, x, c)
    assert torch.equal(gx, rx) and torch.equal(gs, rs)
