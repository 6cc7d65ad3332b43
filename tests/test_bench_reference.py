"""bench.py's reference arm: the reference's own CPU kernel (built from its
sources into oracle/_ref) timed on a bounded sample of the benchmark
workload, printed as one JSON line with the benchmark contract's keys, in a
process that never loads the product library.  And bench.py's multi-rank
launcher on CPU."""
import json
import subprocess
import sys

import pytest

import oracle as O
from conftest import ROOT


def test_reference_arm_prints_contract_line():
    if not O.ref_available("avx2"):
        pytest.skip("the reference's CPU kernels are not built")
    # run the arm, then report whether the product library was mapped into the process
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3', "
            "'--ref-sample', '4']; runpy.run_path('bench.py', run_name='__main__'); "
            "print('MAPS', sum('libsgi_b200' in l for l in open('/proc/self/maps')))")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, timeout=900, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MAPS 0" in r.stdout, r.stdout[-500:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "points/s" and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_launcher_runs_one_process_per_rank():
    """`bench.py --gpus 2` started directly launches two ranks (torchrun),
    which form a process group, meet at a barrier and reduce their times to
    the maximum; rank 0 alone prints the line (gloo, no GPU work)."""
    r = subprocess.run([sys.executable, "bench.py", "--gpus", "2", "--launch-check"], cwd=ROOT, timeout=300,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d == {"launch_check": "ok", "n_gpus": 2, "max_over_ranks_ms": 2.0}
