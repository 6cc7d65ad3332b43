"""The plugin surface as the HDDM solver binds it: a C++ host (tests/
plugin_host.cpp) dlopens the library, takes the extern "C" entry points with
dlsym and calls Data::load and both Interpolator::interpolate overloads
through the vtables of include/sgi_plugin.h, on the reference's known-answer
fixture. The plugin computes in the FP64 form, so its values equal the
oracle's gold path bit for bit, and the reference test's own check (1e-3)
holds."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, PKG
from test_plugin_cpu import _build_plugin_host

pytestmark = pytest.mark.gpu

PLT = os.path.join(GOLDEN, "interpolate_array_surplus.plt")
DOC = json.load(open(os.path.join(GOLDEN, "interpolate_array.json")))


def test_plugin_host_single_and_multistate(cuda, tmp_path):
    exe = _build_plugin_host(tmp_path)
    (tmp_path / "hddm-solver.cfg").write_text("n_agents 59\npriorityCUDA 2\n")
    x = DOC["x"]
    r = subprocess.run([exe, os.path.join(PKG, "lib", "libsgi_b200.so"), PLT, "3"] + [repr(float(v)) for v in x],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0] == "priority 2"
    single = np.array([float(v) for v in lines[1].split()[1:]])
    gold = O.Gold.read_plt(PLT, 59).interpolate(np.array([x]))[0]
    assert np.array_equal(single, gold)
    assert np.abs(single - np.array(DOC["expected_test_cpp"])).max() <= DOC["epsilon_test_cpp"]
    multi = [l for l in lines[2:] if l.startswith("multi")]
    assert len(multi) == 3
    assert all(np.array_equal(np.array([float(v) for v in l.split()[2:]]), gold) for l in multi)


def test_plugin_batch_entry_over_states(cuda, tmp_path):
    """sgi_plugin_interpolate_batch: (state, point) pairs in any order over
    states holding different grids, one call; every pair equals the oracle's
    gold value of its own state's grid bit for bit."""
    import hddm_b200 as H
    exe = _build_plugin_host(tmp_path)
    (tmp_path / "hddm-solver.cfg").write_text("n_agents 59\npriorityCUDA 2\n")
    files = [PLT]
    for k in range(2):
        p = str(tmp_path / f"g{k}.plt")
        H.HostGrid.adaptive(59, 20000 + 7000 * k, 118, seed=60 + k).write_plt(p)
        files.append(p)
    nstates = 5
    x = np.array(DOC["x"])
    r = subprocess.run([exe, os.path.join(PKG, "lib", "libsgi_b200.so"), ",".join(files), str(nstates)]
                       + [repr(float(v)) for v in x], cwd=tmp_path, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, PLUGIN_HOST_TOTALDOF="118"))
    assert r.returncode == 0, r.stderr
    golds = [O.Gold.read_plt(f, 59) for f in files]
    rows = [l.split() for l in r.stdout.splitlines() if l.startswith("batch")]
    assert len(rows) == 2 * nstates
    for f in rows:
        k, s = int(f[1]), int(f[2])
        assert s == (3 * k + 1) % nstates
        xk = np.mod(x + 0.01 * k, 1.0)
        ref = golds[s % len(files)].interpolate(xk[None])[0]
        assert np.array_equal(np.array([float(v) for v in f[3:]]), ref), (k, s)
    lat = [l for l in r.stdout.splitlines() if l.startswith("latency")]
    assert len(lat) == 1
