"""The kernel-level entry points with the reference's x86 signatures
(include/sgi_kernels.h), fed the reference's own x86 loader's containers
(oracle/_ref, compiled from the reference tree) exactly as the reference's
test hands them to LinearBasis_x86_Generic_InterpolateArray
(LinearBasis/tests/InterpolateArray/test.cpp:285-313).

CPU: the container layouts include/sgi_kernels.h mirrors match the objects
the reference's loader builds (sizes read through the mirrored layout equal
the loader's own).  GPU: values within 1e-12 of the reference x86 kernel and
of the oracle's gold restatement, single state and multistate."""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, PKG

PLT = os.path.join(GOLDEN, "interpolate_array_surplus.plt")
DOC = json.load(open(os.path.join(GOLDEN, "interpolate_array.json")))
needs_ref = pytest.mark.skipif(not O.ref_available("x86"), reason="reference not compiled here")


class _Vec(ctypes.Structure):           # std::vector<T>: begin, end, end of storage
    _fields_ = [("b", ctypes.c_void_p), ("e", ctypes.c_void_p), ("c", ctypes.c_void_p)]


class _Mat(ctypes.Structure):           # sgi_x86::Matrix<double>
    _fields_ = [("data", _Vec), ("dimY", ctypes.c_int), ("dimX", ctypes.c_int), ("dimX_aligned", ctypes.c_int)]


def _grid_file(tmp_path, nno, td, seed):
    import hddm_b200 as H
    p = str(tmp_path / f"g{seed}.plt")
    H.HostGrid.adaptive(59, nno, td, seed=seed).write_plt(p)
    return p


@needs_ref
def test_mirrored_layouts_match_the_reference_loader(tmp_path):
    for path in (PLT, _grid_file(tmp_path, 3000, 40, 5)):
        r = O.RefGrid(path, 59, "x86")
        info = r.info()
        xps_p, chains_p, sur_p, nfreqs = r.containers()
        xps = _Vec.from_address(xps_p)
        chains = _Vec.from_address(chains_p)
        mat = _Mat.from_address(sur_p)
        assert (xps.e - xps.b) // 4 == info["szxps"]              # Index<uint16_t>: 4 bytes
        assert (chains.e - chains.b) // 2 >= info["nno"] * nfreqs
        assert nfreqs == info["nfreqs"]
        assert (mat.dimY, mat.dimX) == (info["nno"], info["TotalDof"])
        assert mat.dimX_aligned >= mat.dimX
        assert (mat.data.e - mat.data.b) // 8 >= mat.dimY * mat.dimX_aligned
        # the surplus read through the mirrored layout is the loader's
        rows = np.ctypeslib.as_array((ctypes.c_double * (mat.dimY * mat.dimX_aligned)).from_address(mat.data.b))
        rows = rows.reshape(mat.dimY, mat.dimX_aligned)[:, :mat.dimX]
        assert np.array_equal(rows, r.surplus())


def _symbols():
    import hddm_b200 as H
    lib = ctypes.CDLL(H.LIB_PATH)
    one = lib.LinearBasis_b200_Generic_InterpolateArray
    one.restype = None
    one.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    many = lib.LinearBasis_b200_Generic_InterpolateArrayManyMultistate
    many.restype = None
    many.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return one, many


@needs_ref
@pytest.mark.gpu
def test_x86_signature_single_state(cuda, tmp_path):
    import hddm_b200 as H
    one, _ = _symbols()
    for path in (PLT, _grid_file(tmp_path, 20000, 118, 61)):
        r = O.RefGrid(path, 59, "x86")
        td = r.info()["TotalDof"]
        xps_p, chains_p, sur_p, nfreqs = r.containers()
        X = np.concatenate([np.array(DOC["x"])[None], H.gen_points(59, 40, kind=2, seed=62)])
        got = np.zeros((len(X), td))
        for k in range(len(X)):           # one call per point, the containers' grid built once
            xk = np.ascontiguousarray(X[k])
            one(None, 59, td, xk.ctypes.data, nfreqs, xps_p, chains_p, sur_p, got[k].ctypes.data)
        ref86 = r.interpolate(X, nthreads=4)
        gold = O.Gold.read_plt(path, 59).interpolate(X)
        scale = max(1.0, np.abs(gold).max())
        assert np.abs(got - ref86).max() <= 1e-12 * scale
        assert np.abs(got - gold).max() <= 1e-12 * scale
        if path == PLT:
            assert np.abs(got[0] - np.array(DOC["expected_test_cpp"])).max() <= DOC["epsilon_test_cpp"]


@needs_ref
@pytest.mark.gpu
def test_x86_signature_multistate(cuda, tmp_path):
    import hddm_b200 as H
    _, many = _symbols()
    paths = [PLT, _grid_file(tmp_path, 8000, 118, 63), _grid_file(tmp_path, 12000, 118, 64)]
    grids = [O.RefGrid(p, 59, "x86") for p in paths]
    cont = [g.containers() for g in grids]
    # the reference passes arrays of containers: XPS xps[count] etc.; here the
    # containers live in separate loaders, so they are copied into contiguous
    # arrays of the mirrored objects (shallow: the vectors' buffers are shared)
    n = len(paths)
    xps_arr = (_Vec * n)(*[_Vec.from_address(c[0]) for c in cont])
    chains_arr = (_Vec * n)(*[_Vec.from_address(c[1]) for c in cont])
    sur_arr = (_Mat * n)(*[_Mat.from_address(c[2]) for c in cont])
    nfreqs = (ctypes.c_int * n)(*[c[3] for c in cont])
    X = H.gen_points(59, n, kind=0, seed=65)
    xs = [np.ascontiguousarray(X[k]) for k in range(n)]
    vals = [np.zeros(118) for _ in range(n)]
    xptr = (ctypes.c_void_p * n)(*[v.ctypes.data for v in xs])
    vptr = (ctypes.c_void_p * n)(*[v.ctypes.data for v in vals])
    many(None, 59, 118, n, xptr, nfreqs, ctypes.addressof(xps_arr), ctypes.addressof(chains_arr),
         ctypes.addressof(sur_arr), vptr)
    for k in range(n):
        gold = O.Gold.read_plt(paths[k], 59).interpolate(X[k][None])[0]
        ref86 = grids[k].interpolate(X[k][None], nthreads=1)[0]
        scale = max(1.0, np.abs(gold).max())
        assert np.abs(vals[k] - gold).max() <= 1e-12 * scale, k
        assert np.abs(vals[k] - ref86).max() <= 1e-12 * scale, k
