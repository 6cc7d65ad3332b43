"""The device-layout cache (sgi_grid_load): a grid loaded from the cache is
the grid sgi_grid_create builds from the same .plt, computing the same bits
in both forms; a changed .plt is rebuilt; the plugin's Data::load uses the
cache when SGI_LAYOUT_CACHE asks for it."""
import os
import subprocess

import numpy as np
import pytest

import hddm_b200 as H
import oracle as O
from conftest import GOLDEN, PKG
from test_plugin_cpu import _build_plugin_host

pytestmark = pytest.mark.gpu


def _out(g, X, precision):
    import torch
    return H.interpolate(g, torch.from_numpy(X).cuda(), precision=precision).cpu().numpy()


def test_cached_grid_is_the_built_grid(cuda, tmp_path):
    p = str(tmp_path / "g.plt")
    hg = H.HostGrid.adaptive(59, 30000, 96, seed=12)
    hg.write_plt(p)
    X = H.gen_points(59, 6000, kind=2, seed=13)
    ref = H.Grid(H.HostGrid.read_plt(p, 59), flags=H.BUILD_FP32)
    first = H.Grid.load(p, 59, flags=H.BUILD_FP32)
    assert not first.cache_hit and os.path.exists(p + ".sgi-layout")
    second = H.Grid.load(p, 59, flags=H.BUILD_FP32)
    assert second.cache_hit
    assert ref.info.as_dict() == second.info.as_dict()
    for prec in (H.FP64, H.FP32C):
        a = _out(ref, X, prec)
        assert np.array_equal(a, _out(first, X, prec)) and np.array_equal(a, _out(second, X, prec)), prec
    gold = O.Gold(*hg.arrays()).interpolate(X[:256])
    assert np.array_equal(_out(second, X[:256], H.FP64), gold)
    # an FP64-only load does not take the FP32 cache, and makes its own
    third = H.Grid.load(p, 59, flags=0, cache_path=str(tmp_path / "f64.cache"))
    assert not third.cache_hit and np.array_equal(_out(third, X, H.FP64), _out(ref, X, H.FP64))
    # a rewritten file (another grid under the same name) is rebuilt
    H.HostGrid.adaptive(59, 20000, 96, seed=14).write_plt(p)
    st = os.stat(p)
    os.utime(p, ns=(st.st_atime_ns, st.st_mtime_ns + 1))
    fourth = H.Grid.load(p, 59, flags=H.BUILD_FP32)
    assert not fourth.cache_hit and fourth.nno == 20000


def test_plugin_load_through_the_cache(cuda, tmp_path):
    exe = _build_plugin_host(tmp_path)
    (tmp_path / "hddm-solver.cfg").write_text("n_agents 59\npriorityCUDA 2\n")
    plt = str(tmp_path / "fixture.plt")
    open(plt, "wb").write(open(os.path.join(GOLDEN, "interpolate_array_surplus.plt"), "rb").read())
    import json
    x = json.load(open(os.path.join(GOLDEN, "interpolate_array.json")))["x"]
    gold = O.Gold.read_plt(plt, 59).interpolate(np.array([x]))[0]
    cdir = tmp_path / "caches"
    cdir.mkdir()
    for run in range(2):
        r = subprocess.run([exe, os.path.join(PKG, "lib", "libsgi_b200.so"), plt, "2"] + [repr(float(v)) for v in x],
                           cwd=tmp_path, capture_output=True, text=True, timeout=300,
                           env=dict(os.environ, SGI_LAYOUT_CACHE=str(cdir)))
        assert r.returncode == 0, r.stderr
        single = np.array([float(v) for v in r.stdout.splitlines()[1].split()[1:]])
        assert np.array_equal(single, gold), run
        assert (cdir / "fixture.plt.sgi-layout").exists()
