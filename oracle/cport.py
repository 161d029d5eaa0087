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
