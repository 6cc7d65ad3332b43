"""The C-ABI library loads and exports every function declared in include/*.h."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import PKG, ROOT

LIB = os.path.join(PKG, "lib", "libsgi_b200.so")


def _declared_functions():
    names = set()
    for h in ("sgi.h", "sgi_plugin.h", "sgi_kernels.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        if h in ("sgi_plugin.h", "sgi_kernels.h"):
            src = src[src.index('extern "C"'):]
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{}]*\)\s*;", src):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return names


def test_header_declares_expected_entry_points():
    names = _declared_functions()
    for must in ("sgi_interpolate", "sgi_interpolate_host", "sgi_backward", "sgi_grid_create",
                 "getInterpolator", "getData", "isSupported", "getPriority", "resetInterpolator",
                 "tryAcquireDevice", "releaseDevice", "getDeviceProperties",
                 "LinearBasis_b200_Generic_InterpolateArray",
                 "LinearBasis_b200_Generic_InterpolateArrayManyMultistate"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in sorted(_declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    assert _declared_functions() <= exported


def test_library_links_no_oracle():
    out = subprocess.run(["ldd", LIB], capture_output=True, text=True).stdout
    assert "oracle" not in out and "libref_" not in out
    nm = subprocess.run(["nm", "-D", LIB], capture_output=True, text=True).stdout
    assert "oracle_" not in nm and "ref_interpolate" not in nm


def test_surplus_cutoff_rejects_null_grid():
    lib = ctypes.CDLL(LIB)
    f = lib.sgi_grid_set_surplus_cutoff
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    assert f(None, 1e-3, None) == -1
