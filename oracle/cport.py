"""ctypes access to the oracle's C restatement (test infrastructure only)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import build

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build.build())
        for sfx in ("f64", "f32"):
            fn = getattr(_LIB, f"lpo_apply_masked_{sfx}")
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_int] * 3 + [ctypes.c_void_p]
        _LIB.lpo_threads.restype = ctypes.c_int
        for name in ("lpo_coarse_residual_f32", "lpo_add_correction_f32"):
            f_ = getattr(_LIB, name)
            f_.restype = ctypes.c_int
            f_.argtypes = [ctypes.c_void_p] * (5 if name == "lpo_coarse_residual_f32" else 4) + [ctypes.c_int] * 6
        fn = _LIB.lpo_apply_weights_f32
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_int] * 3 + [ctypes.c_void_p] * 2 + [ctypes.c_longlong,
                                                                                           ctypes.c_void_p]
    return _LIB


def threads() -> int:
    return int(lib().lpo_threads())


class MaskedApply:
    """out = m K(e) (m u) + (1 - m) u with the reference's two-pass CPU scheme; keeps its
    (24, cells) product buffer like the reference's Cells.ft (loadpath/mgops.py:238-244)."""

    def __init__(self, ke, e, m, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        self.ke = np.ascontiguousarray(ke, np.float64)
        self.e = np.ascontiguousarray(e, self.dtype)
        self.m = np.ascontiguousarray(m, self.dtype)
        self.dims = self.e.shape
        self.ft = np.empty((24, int(np.prod(self.dims))), self.dtype)
        self.fn = getattr(lib(), "lpo_apply_masked_" + ("f64" if self.dtype == np.float64 else "f32"))

    def __call__(self, u, out=None):
        u = np.ascontiguousarray(u, self.dtype)
        out = np.empty_like(u) if out is None else out
        nx, ny, nz = self.dims
        self.fn(out.ctypes.data, u.ctypes.data, self.e.ctypes.data, self.m.ctypes.data, self.ke.ctypes.data,
                nx, ny, nz, self.ft.ctypes.data)
        return out


class WeightsApply:
    """The level-1 ("weights") operator out = m K1 (m u) + (1 - m) u of the reference's hierarchy
    in float32 (loadpath/mg.py:213-230, :251-276, :317-346), from an oracle Level of kind
    "weights" (its w, mcat, patch cells and mask)."""

    def __init__(self, level):
        assert level.kind == "weights"
        self.dims = tuple(level.dims)
        self.w = np.ascontiguousarray(level.w.reshape(8, -1), np.float32)
        self.mcat = np.ascontiguousarray(np.asarray(level.mcat, np.float64).reshape(8, 24, 24))
        self.m = np.ascontiguousarray(level.mask, np.float32)
        has_patch = level.patch_ijk is not None and len(level.patch_ijk)
        self.pidx = np.ascontiguousarray(level.patch_index() if has_patch else np.zeros((0, 24)), np.int64)
        self.pk = np.ascontiguousarray(level.patch_k if has_patch else np.zeros((0, 24, 24)), np.float32)
        self.ft = np.empty((24, int(np.prod(self.dims))), np.float32)

    def __call__(self, u, out=None):
        u = np.ascontiguousarray(u, np.float32)
        out = np.empty_like(u) if out is None else out
        nx, ny, nz = self.dims
        lib().lpo_apply_weights_f32(out.ctypes.data, u.ctypes.data, self.w.ctypes.data, self.mcat.ctypes.data,
                                    self.m.ctypes.data, nx, ny, nz, self.pidx.ctypes.data, self.pk.ctypes.data,
                                    len(self.pidx), self.ft.ctypes.data)
        return out


def coarse_residual(b, ax, m, cm, out=None):
    """rc = cm * R((b - ax) * m) in float32 (the C port of loadpath/mgops.py:753-763)."""
    b, ax, m, cm = (np.ascontiguousarray(a, np.float32) for a in (b, ax, m, cm))
    out = np.empty(cm.shape, np.float32) if out is None else out
    lib().lpo_coarse_residual_f32(out.ctypes.data, b.ctypes.data, ax.ctypes.data, m.ctypes.data, cm.ctypes.data,
                                  *b.shape[1:], *cm.shape[1:])
    return out


def add_correction(xc, cm, m, x):
    """x += m * P(cm * xc) in float32, in place (the C port of loadpath/mgops.py:766-773)."""
    xc, cm, m = (np.ascontiguousarray(a, np.float32) for a in (xc, cm, m))
    assert x.dtype == np.float32 and x.flags.c_contiguous
    lib().lpo_add_correction_f32(x.ctypes.data, xc.ctypes.data, cm.ctypes.data, m.ctypes.data, *x.shape[1:],
                                 *cm.shape[1:])
    return x
