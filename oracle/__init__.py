"""ORACLE — test infrastructure only.

ctypes bindings to
  * oracle/liboracle.so: a C restatement of the reference's FP64 gold kernel
    and .plt reader (oracle/gold.c), and
  * oracle/_ref/libref_{gold,x86,avx2}.so: the reference's own CPU loaders and
    kernels, compiled in place from the reference tree by oracle/Makefile.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, as the checker; the product never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


class OracleGrid(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("nno", ctypes.c_int), ("TotalDof", ctypes.c_int),
                ("Level", ctypes.c_int), ("index", ctypes.POINTER(ctypes.c_int)),
                ("surplus", ctypes.POINTER(ctypes.c_double))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C {HERE}`")
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.oracle_plt_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(OracleGrid), ctypes.c_char_p,
                                      ctypes.c_size_t]
        L.oracle_grid_free.argtypes = [ctypes.POINTER(OracleGrid)]
        L.oracle_interpolate.argtypes = [ctypes.POINTER(OracleGrid), P, P]
        L.oracle_interpolate_batch.argtypes = [ctypes.POINTER(OracleGrid), ctypes.c_long, P, P, ctypes.c_int]
        L.oracle_gradient.argtypes = [ctypes.POINTER(OracleGrid), ctypes.c_long, P, P, P, P]
        L.oracle_active_count.argtypes = [ctypes.POINTER(OracleGrid), P]
        L.oracle_active_count.restype = ctypes.c_long
        L.oracle_gen_adaptive.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_ulonglong, ctypes.POINTER(OracleGrid)]
        L.oracle_gen_points.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_int, ctypes.c_ulonglong,
                                        ctypes.c_double, ctypes.c_int, P]
        L.oracle_plt_write.argtypes = [ctypes.POINTER(OracleGrid), ctypes.c_char_p]
        _lib = L
    return _lib


class Gold:
    """The oracle's view of one grid: dense index [nno, 2*dim] and surplus [nno, TD]."""

    def __init__(self, index, surplus):
        self.index = np.ascontiguousarray(index, dtype=np.int32)
        self.surplus = np.ascontiguousarray(surplus, dtype=np.float64)
        self.g = OracleGrid()
        self.g.nno, two_dim = self.index.shape
        self.g.dim = two_dim // 2
        self.g.TotalDof = self.surplus.shape[1]
        self.g.index = self.index.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        self.g.surplus = self.surplus.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    @property
    def dim(self):
        return self.g.dim

    @property
    def total_dof(self):
        return self.g.TotalDof

    @classmethod
    def read_plt(cls, path, nagents):
        g = OracleGrid()
        err = ctypes.create_string_buffer(1024)
        rc = lib().oracle_plt_read(os.fsencode(path), nagents, ctypes.byref(g), err, 1024)
        if rc:
            raise ValueError(err.value.decode())
        index = np.ctypeslib.as_array(g.index, shape=(g.nno, 2 * g.dim)).copy() if g.nno else \
            np.zeros((0, 2 * g.dim), np.int32)
        surplus = np.ctypeslib.as_array(g.surplus, shape=(g.nno, g.TotalDof)).copy() if g.nno else \
            np.zeros((0, g.TotalDof))
        lib().oracle_grid_free(ctypes.byref(g))
        return cls(index, surplus)

    def interpolate(self, X, nthreads=0):
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        out = np.zeros((X.shape[0], self.total_dof))
        lib().oracle_interpolate_batch(ctypes.byref(self.g), X.shape[0], X.ctypes.data, out.ctypes.data, nthreads)
        return out

    def gradient(self, X, C):
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        C = np.ascontiguousarray(C, dtype=np.float64)
        dx = np.zeros_like(X)
        ds = np.zeros_like(self.surplus)
        lib().oracle_gradient(ctypes.byref(self.g), X.shape[0], X.ctypes.data, C.ctypes.data, dx.ctypes.data,
                              ds.ctypes.data)
        return dx, ds

    @classmethod
    def adaptive(cls, dim, nno, total_dof, seed, max_level=7, p_dim=0.125):
        """The seeded adaptive grid, generated by the oracle's restatement
        (the same arrays as the product's generator)."""
        g = OracleGrid()
        if lib().oracle_gen_adaptive(dim, nno, total_dof, max_level, p_dim, seed, ctypes.byref(g)):
            raise ValueError("bad adaptive-grid arguments")
        index = np.ctypeslib.as_array(g.index, shape=(g.nno, 2 * g.dim)).copy()
        surplus = np.ctypeslib.as_array(g.surplus, shape=(g.nno, g.TotalDof)).copy()
        level = g.Level
        lib().oracle_grid_free(ctypes.byref(g))
        out = cls(index, surplus)
        out.g.Level = level
        return out

    def write_plt(self, path):
        """The compressed .plt layout the reference's loaders read."""
        if lib().oracle_plt_write(ctypes.byref(self.g), os.fsencode(path)):
            raise OSError(f"cannot write {path}")

    def active_count(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        return lib().oracle_active_count(ctypes.byref(self.g), x.ctypes.data)


def gen_points(dim, npts, kind=0, seed=0, kink_reject=0.0, max_level=7):
    """The seeded query points, generated by the oracle's restatement."""
    out = np.zeros((npts, dim), np.float64)
    if lib().oracle_gen_points(dim, npts, kind, seed, kink_reject, max_level, out.ctypes.data):
        raise ValueError("bad point arguments")
    return out


def ref_available(variant="gold"):
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}.so"))


class RefGrid:
    """The reference's own loader + kernel (oracle/_ref/libref_<variant>.so)."""

    _libs = {}

    def __init__(self, paths, nagents, variant="gold"):
        self.variant = variant
        L = self._lib(variant)
        if isinstance(paths, (str, bytes, os.PathLike)):
            paths = [paths]
        arr = (ctypes.c_char_p * len(paths))(*[os.fsencode(p) for p in paths])
        self.nstates = len(paths)
        self.h = ctypes.c_void_p(L.ref_load(arr, len(paths), nagents))
        self.L = L

    @classmethod
    def _lib(cls, variant):
        if variant not in cls._libs:
            path = os.path.join(REF_DIR, f"libref_{variant}.so")
            if not os.path.exists(path):
                raise ImportError(f"{path} missing: run `make -C {HERE}` where the reference tree exists")
            L = ctypes.CDLL(path)
            L.ref_load.restype = ctypes.c_void_p
            L.ref_load.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int]
            L.ref_free.argtypes = [ctypes.c_void_p]
            L.ref_info.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            L.ref_get_surplus.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            L.ref_get_index.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            L.ref_interpolate_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_int]
            if variant == "x86":
                L.ref_get_xps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
                L.ref_get_chains.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
                L.ref_containers.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.POINTER(ctypes.c_int)]
            cls._libs[variant] = L
        return cls._libs[variant]

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.ref_free(self.h)
            self.h = None

    def info(self, istate=0):
        v = (ctypes.c_int * 6)()
        self.L.ref_info(self.h, istate, v)
        return dict(dim=v[0], nno=v[1], TotalDof=v[2], nfreqs=v[3], szxps=v[4], ld=v[5])

    def interpolate(self, X, istate=0, nthreads=0):
        inf = self.info(istate)
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        out = np.zeros((X.shape[0], inf["TotalDof"]))
        self.L.ref_interpolate_batch(self.h, istate, X.shape[0], X.ctypes.data, out.ctypes.data, nthreads)
        return out

    def surplus(self, istate=0):
        inf = self.info(istate)
        out = np.zeros((inf["nno"], inf["TotalDof"]))
        self.L.ref_get_surplus(self.h, istate, out.ctypes.data)
        return out

    def index(self, istate=0):
        inf = self.info(istate)
        out = np.zeros((inf["nno"], 2 * inf["dim"]), np.int32)
        self.L.ref_get_index(self.h, istate, out.ctypes.data)
        return out

    def containers(self, istate=0):
        """x86 only: addresses of the loaded state's XPS, Chains and surplus
        Matrix objects (valid while this RefGrid lives) and its nfreqs."""
        out = (ctypes.c_void_p * 3)()
        nf = ctypes.c_int(0)
        self.L.ref_containers(self.h, istate, out, ctypes.byref(nf))
        return out[0], out[1], out[2], nf.value

    def xps_chains(self, istate=0):
        inf = self.info(istate)
        xps = np.zeros((inf["szxps"], 3), np.int32)
        chains = np.zeros((inf["nno"], inf["nfreqs"]), np.int32)
        self.L.ref_get_xps(self.h, istate, xps.ctypes.data)
        self.L.ref_get_chains(self.h, istate, chains.ctypes.data)
        return xps, chains


def rel_error(a, b):
    """Per-point relative error max_o |a-b| / max(|b_o|, 1e-3 ||b||_inf); returns (max, rms) over points."""
    a = np.atleast_2d(a)
    b = np.atleast_2d(b)
    den = np.maximum(np.abs(b), 1e-3 * np.abs(b).max(axis=1, keepdims=True))
    den = np.where(den > 0, den, 1.0)
    e = (np.abs(a - b) / den).max(axis=1)
    return float(e.max()) if e.size else 0.0, float(np.sqrt((e ** 2).mean())) if e.size else 0.0
