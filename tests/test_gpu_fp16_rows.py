"""FP32C's FP16 rows checked on their own: with the FP16 threshold raised to
the whole largest surplus (SGI_F16_REL=1, read once per process, so the check
runs in a child process), every fine term reads its row from the FP16 copy.
Each output must then stay within the FP16 rounding bound of gold: 2^-11 of
the summed bounds |w| * max|s_row| of the point's fine terms, plus the FP32C
tolerance for the rest.  A wrong lane layout, row scale or decode of the
FP16 rows would miss that by orders of magnitude.  The same holds for rows
whose values span 2^-40 of their maximum (subnormal and zero halves), and
for a grid whose largest |surplus| is 2^-58, near the low end at which FP16
rows are still built (2^-60, where the weight scale 2^(floor(log2 rowmax) -
14) stays a normal FP32 number); at 2^-70 no FP16 rows are built and the
FP32 rows serve.  The default threshold is checked by every other FP32C
test on rows of 256 outputs."""
import os
import subprocess
import sys

import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import sys
import numpy as np
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import torch
import hddm_b200 as H
import oracle as O
from test_gpu_forward import _term_bounds
hg0 = H.HostGrid.adaptive(59, 8000, 256, seed=91)
idx, sur0 = hg0.arrays()
rng = np.random.default_rng(94)
wide = sur0 * np.exp2(-rng.integers(0, 41, size=sur0.shape).astype(np.float64))
wide[:, 5] = 0.0
wide[:, 6] = -0.0
smax0 = np.abs(sur0).max()
cases = [("as built", sur0, (600, 40)), ("wide rows", wide, (300,)),
         ("largest 2^-58", sur0 * (2.0 ** -58 / smax0), (300,)), ("largest 2^-70", sur0 * (2.0 ** -70 / smax0), (300,))]
for name, sur, sizes in cases:
  hg = H.HostGrid.from_dense(idx, sur)
  for npts, seed in zip(sizes, (92, 93)):
    X = H.gen_points(59, npts, kind=2, seed=seed)
    g = H.Grid(hg, flags=H.BUILD_FP32 | H.BUILD_NO_FP64)
    x = torch.from_numpy(X).cuda()
    classes = H.term_classes(g, x).cpu().numpy()
    if name == "largest 2^-70":
        assert classes[:, 2].sum() == 0 and classes[:, 1].sum() > 0, (name, classes.sum(axis=0))
    else:
        assert classes[:, 1].sum() == 0 and classes[:, 2].sum() > 0, (name, classes.sum(axis=0))
    got = H.interpolate(g, x, precision=H.FP32C).cpu().numpy()
    ref = O.Gold(idx, sur).interpolate(X)
    b = _term_bounds(idx, sur, X)
    smax = np.abs(sur).max()
    fine = np.where(b < smax * 2.0 ** -16, b, 0.0).sum(axis=1)
    scale = np.maximum(np.abs(ref), 1e-3 * np.abs(ref).max(axis=1, keepdims=True))
    excess = np.abs(got - ref) - 2.0 ** -11 * fine[:, None] - 1e-7 * scale
    assert excess.max() <= 0, (name, excess.max())
print("ok")
"""


def test_all_fine_terms_through_fp16_rows(cuda):
    r = subprocess.run([sys.executable, "-c", CHILD, PKG, os.path.join(ROOT, "tests")], cwd=ROOT,
                       capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, SGI_F16_REL="1.0", PYTHONPATH=ROOT))
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]
