"""Regenerate the golden fixtures under tests/golden/ from the reference tree.

Run in a container that has the reference checked out (default
/root/reference, or $HDDM_REF_TREE, or --ref) after `make -C oracle`:

    python tests/golden/make_golden.py

It writes
  * interpolate_array_surplus.plt: the reference's single-state known-answer
    grid (LinearBasis/tests/InterpolateArray/surplus.plt), copied verbatim;
  * interpolate_array.json: the query point of init()
    (LinearBasis/tests/InterpolateArray/test.cpp:24-87), the 118 expected values
    of check() (:89-215, tolerance EPSILON=0.001 at :10), the n_agents value of
    the test's hddm-solver.cfg, and the full-precision outputs of the
    reference's own gold, x86 and avx2 kernels run on that grid and point
    (oracle/_ref, compiled in place from the reference sources).

The reference's multistate known-answer tables
(LinearBasis/tests/InterpolateArrayManyMultistate/{medium,large}/test.cpp) are
not turned into fixtures: their grids are absent from the reference tree
(medium is missing, large holds git-LFS pointers only).
"""
import argparse
import ctypes
import json
import os
import re
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def parse_test_cpp(path):
    src = open(path).read()
    xs = {int(k): float(v) for k, v in re.findall(r"input\[(\d+)\]\s*=\s*([-0-9.eE+]+);", src)}
    ex = {int(k): float(v) for k, v in re.findall(r"expected\[(\d+)\]\s*=\s*([-0-9.eE+]+);", src)}
    eps = float(re.search(r"#define EPSILON\s+([0-9.eE+-]+)", src).group(1))
    x = [xs[k] for k in range(len(xs))]
    e = [ex[k] for k in range(len(ex))]
    return x, e, eps


def parse_cfg(path):
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] in ("n_agents", "nagents"):
            return int(parts[1])
    raise RuntimeError("no n_agents in " + path)


def run_ref(variant, plt, nagents, x):
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", f"libref_{variant}.so"))
    lib.ref_load.restype = ctypes.c_void_p
    lib.ref_load.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int]
    paths = (ctypes.c_char_p * 1)(plt.encode())
    h = lib.ref_load(paths, 1, nagents)
    info = (ctypes.c_int * 6)()
    lib.ref_info(ctypes.c_void_p(h), 0, info)
    td = info[2]
    X = np.ascontiguousarray(np.array(x, dtype=np.float64)[None, :])
    out = np.zeros((1, td))
    lib.ref_interpolate_batch(ctypes.c_void_p(h), 0, ctypes.c_long(1),
                              X.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p), 1)
    lib.ref_free(ctypes.c_void_p(h))
    return out[0].tolist()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("HDDM_REF_TREE", "/root/reference"))
    a = ap.parse_args()
    tdir = os.path.join(a.ref, "LinearBasis", "tests", "InterpolateArray")
    plt_src = os.path.join(tdir, "surplus.plt")
    plt_dst = os.path.join(HERE, "interpolate_array_surplus.plt")
    shutil.copyfile(plt_src, plt_dst)
    x, expected, eps = parse_test_cpp(os.path.join(tdir, "test.cpp"))
    nagents = parse_cfg(os.path.join(tdir, "hddm-solver.cfg"))
    doc = {
        "source": "LinearBasis/tests/InterpolateArray/{surplus.plt,test.cpp,hddm-solver.cfg}",
        "nagents": nagents,
        "x": x,
        "expected_test_cpp": expected,
        "epsilon_test_cpp": eps,
    }
    for v in ("gold", "x86", "avx2"):
        doc[f"ref_{v}"] = run_ref(v, plt_dst, nagents, x)
    with open(os.path.join(HERE, "interpolate_array.json"), "w") as f:
        json.dump(doc, f, indent=1)
    err = max(abs(a - b) for a, b in zip(doc["ref_gold"], expected))
    print(f"wrote fixtures; ref gold vs test.cpp max abs diff {err:.3g} (tolerance {eps})")
    return 0


if __name__ == "__main__":
    sys.exit(main())
