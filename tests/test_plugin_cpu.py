"""Plugin surface behaviour that needs no GPU: config parsing, priority,
isSupported, and the reference's abort-on-error contract (in subprocesses)."""
import os
import subprocess
import sys
import textwrap

import pytest

from conftest import PKG

LIB = os.path.join(PKG, "lib", "libsgi_b200.so")


def _run(code, cwd):
    src = textwrap.dedent(f"""
        import ctypes, sys
        lib = ctypes.CDLL({LIB!r})
        lib.getPriority.restype = ctypes.c_int
        lib.isSupported.restype = ctypes.c_bool
        lib.getInterpolator.restype = ctypes.c_void_p
        lib.getData.restype = ctypes.c_void_p
        lib.getData.argtypes = [ctypes.c_int]
        lib.sgi_plugin_interpolate.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.sgi_plugin_data_load.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    """) + textwrap.dedent(code)
    return subprocess.run([sys.executable, "-c", src], cwd=cwd, capture_output=True, text=True, timeout=120)


def test_config_priority_and_nagents(tmp_path):
    (tmp_path / "hddm-solver.cfg").write_text(
        "n_agents                  59            !number of grid dimensions\n"
        "priorityCPU               3             !CPU interpolator priority\n"
        "priorityCUDA              2             !GPU interpolator priority\n")
    r = _run("print(lib.getPriority()); assert lib.getInterpolator()", tmp_path)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "2"


def test_missing_config_aborts_with_reference_message(tmp_path):
    r = _run("lib.getPriority()", tmp_path)
    assert r.returncode != 0
    assert 'Cannot open config file "hddm-solver.cfg"' in r.stderr


def test_missing_parameter_value_aborts(tmp_path):
    (tmp_path / "hddm-solver.cfg").write_text("priorityCUDA 2\nn_agents !oops\n")
    r = _run("lib.getPriority()", tmp_path)
    assert r.returncode != 0 and 'Missing "n_agents" parameter value' in r.stderr


def test_undefined_required_parameter_aborts(tmp_path):
    (tmp_path / "hddm-solver.cfg").write_text("priorityCUDA 2\n")
    r = _run("lib.getPriority()", tmp_path)
    assert r.returncode != 0 and 'Required parameter "nagents" is undefined' in r.stderr


def test_is_supported_without_gpu(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    r = _run("print(lib.isSupported())", tmp_path)
    assert r.returncode == 0 and r.stdout.strip() == "False"


def test_load_checks_nagents_and_state_range(tmp_path):
    """Data::load aborts on a dim mismatch and on an out-of-range state, as the
    reference's DataDense::load does (LinearBasis/gold/src/Data.cpp:328-344, 400-405)."""
    from conftest import GOLDEN
    plt = os.path.join(GOLDEN, "interpolate_array_surplus.plt")
    (tmp_path / "hddm-solver.cfg").write_text("priorityCUDA 2\nn_agents 58\n")
    r = _run(f"d = lib.getData(1); lib.sgi_plugin_data_load(d, {plt!r}.encode(), 0)", tmp_path)
    assert r.returncode != 0 and "mismatches config (58)" in r.stderr
    (tmp_path / "hddm-solver.cfg").write_text("priorityCUDA 2\nn_agents 59\n")
    r = _run(f"d = lib.getData(1); lib.sgi_plugin_data_load(d, {plt!r}.encode(), 3)", tmp_path)
    assert r.returncode != 0 and "State 3 index out of range 0 .. 0" in r.stderr


def _build_plugin_host(out_dir):
    """Compiles tests/plugin_host.cpp, the parent-loader stand-in (dlopen +
    dlsym + virtual calls through include/sgi_plugin.h); returns its path."""
    root = os.path.dirname(PKG)
    exe = os.path.join(str(out_dir), "plugin_host")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "plugin_host.cpp"), "-o", exe, "-ldl"],
                   check=True, capture_output=True, text=True)
    return exe


def test_plugin_host_compiles_against_the_plugin_header(tmp_path):
    """The reference-side binding a maintainer adds compiles against the
    plugin header alone (no link against the library)."""
    assert os.path.exists(_build_plugin_host(tmp_path))
