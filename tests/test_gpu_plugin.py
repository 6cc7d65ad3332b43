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
    r = subprocess.run([exe, os.path.join(PKG, "lib", "libsgi_b200.so"), PLT, "3"] + [repr(v) for v in x],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0] == "priority 2"
    single = np.array([float(v) for v in lines[1].split()[1:]])
    multi = [np.array([float(v) for v in l.split()[2:]]) for l in lines[2:]]
    gold = O.Gold.read_plt(PLT, 59).interpolate(np.array([x]))[0]
    assert np.array_equal(single, gold)
    assert np.abs(single - np.array(DOC["expected_test_cpp"])).max() <= DOC["epsilon_test_cpp"]
    assert len(multi) == 3 and all(np.array_equal(m, gold) for m in multi)
