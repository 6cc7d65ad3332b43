"""Python harness over the C ABI of libsgi_b200.so (include/sgi.h).

Thin plumbing for tests and benchmarks: numpy for host arrays, torch CUDA
tensors for device memory and streams.  All compute happens in the library's
CUDA kernels; there is no Python or CPU fallback — if the library is missing
or was built without CUDA support, importing this module raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libsgi_b200.so")

FP64 = 0
FP32C = 1
BUILD_FP32 = 0x1
BUILD_NO_FP64 = 0x2

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_double_p = ctypes.POINTER(ctypes.c_double)


class SgiError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"sgi error {code}: {msg}")
        self.code = code


class GridInfo(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("nno", ctypes.c_int), ("TotalDof", ctypes.c_int),
                ("ld", ctypes.c_int), ("max_comps", ctypes.c_int), ("tree_depth", ctypes.c_int),
                ("tree_roots", ctypes.c_int), ("multi_delta", ctypes.c_int), ("ncoarse", ctypes.c_int),
                ("comps", ctypes.c_longlong), ("device_bytes", ctypes.c_longlong),
                ("coarse_threshold", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LaunchStats(ctypes.Structure):
    _fields_ = [("kernels", ctypes.c_int), ("grid_blocks", ctypes.c_int),
                ("block_threads", ctypes.c_int), ("points", ctypes.c_longlong)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {PKG_ROOT}` "
                          "(or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, LL, D, U64, U = (ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double,
                           ctypes.c_uint64, ctypes.c_uint)
    sig = {
        "sgi_last_error": (ctypes.c_char_p, []),
        "sgi_device_count": (I, []),
        "sgi_host_grid_read_plt": (I, [ctypes.c_char_p, I, ctypes.POINTER(P)]),
        "sgi_host_grid_write_plt": (I, [P, ctypes.c_char_p]),
        "sgi_host_grid_from_dense": (I, [I, I, I, P, P, ctypes.POINTER(P)]),
        "sgi_host_grid_view": (I, [P, _c_int_p, _c_int_p, _c_int_p, ctypes.POINTER(P), ctypes.POINTER(P)]),
        "sgi_host_grid_free": (None, [P]),
        "sgi_host_grid_xps_chains": (I, [P, _c_int_p, _c_int_p, P, P, P]),
        "sgi_host_grid_tree": (I, [P, P, P]),
        "sgi_host_grid_descent": (I, [P, _c_int_p, _c_int_p, P, P, P, P]),
        "sgi_gen_regular": (I, [I, I, I, U64, ctypes.POINTER(P)]),
        "sgi_gen_adaptive": (I, [I, I, I, I, D, U64, ctypes.POINTER(P)]),
        "sgi_gen_points": (I, [I, ctypes.c_long, I, U64, D, I, P]),
        "sgi_grid_create": (I, [P, I, U, ctypes.POINTER(P)]),
        "sgi_grid_info_get": (I, [P, ctypes.POINTER(GridInfo)]),
        "sgi_grid_destroy": (None, [P]),
        "sgi_grid_load": (I, [ctypes.c_char_p, I, I, U, ctypes.c_char_p, ctypes.POINTER(P), _c_int_p]),
        "sgi_grid_cache_write": (I, [ctypes.c_char_p, I, U, ctypes.c_char_p]),
        "sgi_grid_cache_valid": (I, [ctypes.c_char_p, I, U, ctypes.c_char_p]),
        "sgi_grid_set_surplus_cutoff": (I, [P, D, ctypes.POINTER(D)]),
        "sgi_interpolate": (I, [I, P, P, P, P, I, P]),
        "sgi_interpolate_host": (I, [I, P, P, P, P, I]),
        "sgi_backward": (I, [P, LL, P, P, P, P, P]),
        "sgi_active_count": (I, [P, LL, P, P, P]),
        "sgi_term_classes": (I, [P, LL, P, P, P]),
        "sgi_last_launch": (I, [ctypes.POINTER(LaunchStats)]),
        "sgi_set_chunk_rows": (I, [I]),
        "sgi_set_fp32c_variant": (I, [I]),
        "sgi_plan_create": (I, [I, P, P, P, P, I, I, P, ctypes.POINTER(P)]),
        "sgi_plan_launch": (I, [P, P]),
        "sgi_plan_info": (I, [P, _c_int_p, _c_int_p, _c_int_p, ctypes.POINTER(ctypes.c_float)]),
        "sgi_plan_destroy": (None, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def _check(rc):
    if rc != 0:
        raise SgiError(rc, lib.sgi_last_error().decode())


def device_count():
    return lib.sgi_device_count()


# ------------------------------------------------------------------ host grids
class HostGrid:
    """A grid in the reference's dense form, owned by the library."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.sgi_host_grid_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @classmethod
    def read_plt(cls, path, nagents):
        h = ctypes.c_void_p()
        _check(lib.sgi_host_grid_read_plt(os.fsencode(path), nagents, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_dense(cls, index, surplus):
        index = np.ascontiguousarray(index, dtype=np.int32)
        surplus = np.ascontiguousarray(surplus, dtype=np.float64)
        nno, two_dim = index.shape
        h = ctypes.c_void_p()
        _check(lib.sgi_host_grid_from_dense(two_dim // 2, nno, surplus.shape[1],
                                            index.ctypes.data, surplus.ctypes.data, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def regular(cls, dim, level, total_dof, seed):
        h = ctypes.c_void_p()
        _check(lib.sgi_gen_regular(dim, level, total_dof, seed, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def adaptive(cls, dim, nno, total_dof, seed, max_level=7, p_dim=0.125):
        h = ctypes.c_void_p()
        _check(lib.sgi_gen_adaptive(dim, nno, total_dof, max_level, p_dim, seed, ctypes.byref(h)))
        return cls(h.value)

    def write_plt(self, path):
        _check(lib.sgi_host_grid_write_plt(self._h, os.fsencode(path)))

    def shape(self):
        d, n, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib.sgi_host_grid_view(self._h, ctypes.byref(d), ctypes.byref(n), ctypes.byref(t), None, None))
        return d.value, n.value, t.value

    @property
    def dim(self):
        return self.shape()[0]

    @property
    def nno(self):
        return self.shape()[1]

    @property
    def total_dof(self):
        return self.shape()[2]

    def arrays(self):
        """(index [nno, 2*dim] int32, surplus [nno, TotalDof] float64) copies."""
        d, n, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ip, sp = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib.sgi_host_grid_view(self._h, ctypes.byref(d), ctypes.byref(n), ctypes.byref(t),
                                      ctypes.byref(ip), ctypes.byref(sp)))
        nno, dim, td = n.value, d.value, t.value
        if nno == 0:
            return np.zeros((0, 2 * dim), np.int32), np.zeros((0, td))
        index = np.ctypeslib.as_array(ctypes.cast(ip, _c_int_p), shape=(nno, 2 * dim)).copy()
        surplus = np.ctypeslib.as_array(ctypes.cast(sp, _c_double_p), shape=(nno, td)).copy()
        return index, surplus

    def xps_chains(self):
        """The reference x86 loader's (xps [szxps,3], chains [nno,nfreqs], row_perm [nno])."""
        nf, sz = ctypes.c_int(), ctypes.c_int()
        _check(lib.sgi_host_grid_xps_chains(self._h, ctypes.byref(nf), ctypes.byref(sz), None, None, None))
        nno = self.nno
        xps = np.zeros((sz.value, 3), np.int32)
        chains = np.zeros((nno, nf.value), np.int32)
        perm = np.zeros(nno, np.int32)
        _check(lib.sgi_host_grid_xps_chains(self._h, ctypes.byref(nf), ctypes.byref(sz), xps.ctypes.data,
                                            chains.ctypes.data, perm.ctypes.data))
        return xps, chains, perm

    def tree(self):
        """(skip [nno], parent [nno]) of the containment tree over grid order."""
        nno = self.nno
        skip = np.zeros(nno, np.int32)
        parent = np.zeros(nno, np.int32)
        _check(lib.sgi_host_grid_tree(self._h, skip.ctypes.data, parent.ctypes.data))
        return skip, parent


    def descent(self):
        """Child groups of the FP32C descent: (a [ngroups, 4], b [ngroups, 2],
        first [nno + 1], count [nno + 1], npairs), uint32."""
        ng, npr = ctypes.c_int(), ctypes.c_int()
        _check(lib.sgi_host_grid_descent(self._h, ctypes.byref(ng), ctypes.byref(npr), None, None, None, None))
        nno = self.nno
        a = np.zeros((ng.value, 4), np.uint32)
        b = np.zeros((ng.value, 2), np.uint32)
        first = np.zeros(nno + 1, np.uint32)
        count = np.zeros(nno + 1, np.uint32)
        _check(lib.sgi_host_grid_descent(self._h, ctypes.byref(ng), ctypes.byref(npr), a.ctypes.data,
                                         b.ctypes.data, first.ctypes.data, count.ctypes.data))
        return a, b, first, count, npr.value


def cache_write(path, nagents, flags=0, cache_path=None):
    """Build the layout of a .plt grid on the host and write its cache (no GPU)."""
    _check(lib.sgi_grid_cache_write(os.fsencode(path), nagents, flags,
                                    os.fsencode(cache_path) if cache_path else None))


def cache_valid(path, nagents, flags=0, cache_path=None):
    rc = lib.sgi_grid_cache_valid(os.fsencode(path), nagents, flags, os.fsencode(cache_path) if cache_path else None)
    if rc < 0:
        _check(rc)
    return rc == 1


def gen_points(dim, npts, kind=0, seed=0, kink_reject=0.0, max_level=7):
    out = np.zeros((npts, dim), np.float64)
    _check(lib.sgi_gen_points(dim, npts, kind, seed, kink_reject, max_level, out.ctypes.data))
    return out


# ---------------------------------------------------------------- device grids
def _stream_ptr(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


class Grid:
    """A grid resident on one GPU."""

    def __init__(self, host_grid, device=0, flags=0):
        h = ctypes.c_void_p()
        _check(lib.sgi_grid_create(host_grid.handle, device, flags, ctypes.byref(h)))
        self._h = h
        self.device = device
        self.info = self.get_info()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.sgi_grid_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @classmethod
    def load(cls, path, nagents, device=0, flags=0, cache_path=None):
        """A .plt grid through the layout cache (see sgi_grid_load); the
        grid's `cache_hit` tells whether the cache was used."""
        h = ctypes.c_void_p()
        hit = ctypes.c_int()
        _check(lib.sgi_grid_load(os.fsencode(path), nagents, device, flags,
                                 os.fsencode(cache_path) if cache_path else None, ctypes.byref(h), ctypes.byref(hit)))
        g = cls.__new__(cls)
        g._h = h
        g.device = device
        g.info = g.get_info()
        g.cache_hit = bool(hit.value)
        return g

    def get_info(self):
        info = GridInfo()
        _check(lib.sgi_grid_info_get(self._h, ctypes.byref(info)))
        return info

    def set_surplus_cutoff(self, cutoff):
        """FP32C only: skip terms whose bound |w| * max|surplus row| is below
        `cutoff` (absolute; <= 0 restores the form's own 2^-42 * max|surplus|).
        Returns the bound in use."""
        eff = ctypes.c_double()
        _check(lib.sgi_grid_set_surplus_cutoff(self._h, float(cutoff), ctypes.byref(eff)))
        return eff.value

    @property
    def dim(self):
        return self.info.dim

    @property
    def total_dof(self):
        return self.info.TotalDof

    @property
    def nno(self):
        return self.info.nno


def _grid_array(grids):
    arr = (ctypes.c_void_p * len(grids))()
    for k, g in enumerate(grids):
        arr[k] = g.handle.value
    return arr


def interpolate(grids, x, counts=None, precision=FP64, out=None, stream=None):
    """Forward over a set of grids. x: CUDA float64 tensor [npts, dim]; counts:
    points per grid (defaults to all points on a single grid)."""
    import torch
    if not isinstance(grids, (list, tuple)):
        grids = [grids]
    if counts is None:
        assert len(grids) == 1
        counts = [x.shape[0]]
    offs = np.zeros(len(grids) + 1, np.int64)
    offs[1:] = np.cumsum(counts)
    assert x.is_cuda and x.dtype == torch.float64 and x.is_contiguous()
    assert offs[-1] == x.shape[0]
    td = grids[0].total_dof
    if out is None:
        out = torch.empty((x.shape[0], td), dtype=torch.float64, device=x.device)
    _check(lib.sgi_interpolate(len(grids), _grid_array(grids), offs.ctypes.data, x.data_ptr(), out.data_ptr(),
                               precision, _stream_ptr(stream)))
    return out


def interpolate_host(grids, x, counts=None, precision=FP64):
    """Forward with host numpy arrays (copies in, launches, copies out, syncs)."""
    if not isinstance(grids, (list, tuple)):
        grids = [grids]
    x = np.ascontiguousarray(x, dtype=np.float64)
    if counts is None:
        counts = [x.shape[0]]
    offs = np.zeros(len(grids) + 1, np.int64)
    offs[1:] = np.cumsum(counts)
    out = np.zeros((x.shape[0], grids[0].total_dof), np.float64)
    _check(lib.sgi_interpolate_host(len(grids), _grid_array(grids), offs.ctypes.data, x.ctypes.data,
                                    out.ctypes.data, precision))
    return out


def active_count(grid, x, stream=None):
    import torch
    out = torch.empty(x.shape[0], dtype=torch.int64, device=x.device)
    _check(lib.sgi_active_count(grid.handle, x.shape[0], x.data_ptr(), out.data_ptr(), _stream_ptr(stream)))
    return out


def term_classes(grid, x, stream=None):
    """FP32C terms per point by class: int64 [npts, 4] = (big: FP64 row, fine:
    FP32 row, fine: FP16 row, dropped)."""
    import torch
    out = torch.empty((x.shape[0], 4), dtype=torch.int64, device=x.device)
    _check(lib.sgi_term_classes(grid.handle, x.shape[0], x.data_ptr(), out.data_ptr(), _stream_ptr(stream)))
    return out


def backward(grid, x, gout, want_x=True, want_surplus=True, stream=None):
    import torch
    gx = torch.empty_like(x) if want_x else None
    gs = torch.empty((grid.nno, grid.total_dof), dtype=torch.float64, device=x.device) if want_surplus else None
    _check(lib.sgi_backward(grid.handle, x.shape[0], x.data_ptr(), gout.data_ptr(),
                            gx.data_ptr() if gx is not None else None,
                            gs.data_ptr() if gs is not None else None, _stream_ptr(stream)))
    return gx, gs


class Plan:
    """A forward call recorded into a CUDA graph (see sgi_plan_create); x and out
    are fixed at creation, every launch() recomputes out from x."""

    def __init__(self, grids, x, out, counts=None, precision=FP64, chunk_rows=-1, stream=None):
        if not isinstance(grids, (list, tuple)):
            grids = [grids]
        if counts is None:
            counts = [x.shape[0]]
        self.offs = np.zeros(len(grids) + 1, np.int64)
        self.offs[1:] = np.cumsum(counts)
        self.grids, self.x, self.out = list(grids), x, out   # keep buffers alive
        self._arr = _grid_array(grids)
        h = ctypes.c_void_p()
        _check(lib.sgi_plan_create(len(grids), self._arr, self.offs.ctypes.data, x.data_ptr(), out.data_ptr(),
                                   precision, chunk_rows, _stream_ptr(stream), ctypes.byref(h)))
        self._h = h
        c, v, n, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        _check(lib.sgi_plan_info(h, ctypes.byref(c), ctypes.byref(v), ctypes.byref(n), ctypes.byref(t)))
        self.chunk_rows, self.variant, self.launches, self.tuned_ms = c.value, v.value, n.value, t.value

    def launch(self, stream=None):
        _check(lib.sgi_plan_launch(self._h, _stream_ptr(stream)))
        return self.out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.sgi_plan_destroy(h)
            self._h = None


def set_chunk_rows(rows):
    """-1 automatic, 0 never chunk, n > 0 chunks of n nodes; returns the previous setting."""
    return lib.sgi_set_chunk_rows(rows)


FP32C_AUTO = 255


def set_fp32c_variant(variant):
    """FP32C kernel variant of interpolate/interpolate_host (-1 or FP32C_AUTO:
    automatic by batch size); returns the previous one (FP32C_AUTO when
    automatic), which restores it when passed back."""
    rc = lib.sgi_set_fp32c_variant(variant)
    if rc < 0:
        _check(rc)
    return rc


def last_launch():
    s = LaunchStats()
    _check(lib.sgi_last_launch(ctypes.byref(s)))
    return s


def make_function():
    """torch.autograd.Function over the FP64 forward and the backward kernel:
    y = f(x; surplus) with gradients for x and for the grid's surplus."""
    import torch

    class SparseGridInterp(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, surplus_token, grid):
            ctx.grid = grid
            ctx.save_for_backward(x)
            return interpolate(grid, x.contiguous())

        @staticmethod
        def backward(ctx, gout):
            (x,) = ctx.saved_tensors
            gx, gs = backward(ctx.grid, x.contiguous(), gout.contiguous(),
                              want_x=ctx.needs_input_grad[0], want_surplus=ctx.needs_input_grad[1])
            return gx, gs, None

    return SparseGridInterp
