"""A process whose first call goes through the host-pointer entry (the
plugin's path, holding the device workspace while it launches): the scratch
pool of the small-batch kernels is created inside that call.  Run in a child
process so that nothing earlier in the test session has created it."""
import subprocess
import sys

import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import sys
sys.path[:0] = [{root!r}, {pkg!r}]
import numpy as np
import hddm_b200 as H
import oracle as O
hg = H.HostGrid.adaptive(20, 6000, 24, seed=3)
g = H.Grid(hg)
X = H.gen_points(20, 5, kind=0, seed=1)
got = H.interpolate_host(g, X)
ref = O.Gold(*hg.arrays()).interpolate(X)
sys.exit(0 if np.array_equal(got, ref) else 3)
"""


def test_first_call_through_host_entry(cuda):
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, pkg=PKG)],
                       timeout=180, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
