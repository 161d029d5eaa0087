"""ctypes binding of liblpb200.so, typed from include/loadpath_b200.h.

Every function the header declares is bound with its argument types; a declared symbol
missing from the library is an import error, and a nonzero status from any call raises
LpError. There is no fallback: without the built library (python -m loadpath_b200.build)
nothing in this package computes.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblpb200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "loadpath_b200.h")

_CTYPES = {
    "int": ctypes.c_int,
    "long long": ctypes.c_longlong,
    "float": ctypes.c_float,
    "double": ctypes.c_double,
    "void": None,
    "void*": ctypes.c_void_p,
}
_STATUS = {-1: "bad arguments", -2: "kernel launch failed", -3: "size beyond the kernel's limit"}
# kernels each entry point launches (1 when not listed; 0 for host-only entries)
_KERNELS = {"lpb_modal_ke": 0, "lpb_modal_g1": 0, "lpb_reduce_blocks": 0, "lpb_max_f64": 2, "lpb_max_abs_diff_f64": 2, "lpb_dot_f64": 2,
            "lpb_dot_f32": 2, "lpb_dot_f64_f32": 2, "lpb_cg_step": 2, "lpb_cg_step_r": 2, "lpb_apply_fine_dot_f64": 2, "lpb_oc_volumes": 2, "lpb_oc_apply": 2, "lpb_oc_apply_at": 2, "lpb_oc_walk_init": 2,
            "lpb_band_dims": 0, "lpb_band_inverse": 2, "lpb_band_solve_f32": 2, "lpb_band_solve_f64": 2,
            "lpb_count_positive_f64": 2, "lpb_count_active_weights_f32": 2, "lpb_count_active_weights_f64": 2,
            "lpb_count_active_explicit_f32": 2, "lpb_count_active_explicit_f64": 2, "lpb_count_ne_u8": 2,
            "lpb_memcpy_async": 0, "lpb_memset_async": 0, "lpb_event_record": 0, "lpb_capture_begin": 0,
            "lpb_capture_end": 0, "lpb_graph_launch": 0, "lpb_graph_free": 0, "lpb_while_begin": 0, "lpb_tune_set": 0, "lpb_tune_get": 0,
            "lpb_while_end": 0,
            "lpb_mma_part_len": 0, "lpb_mma_prepare": 2, "lpb_mma_newton_a": 2, "lpb_mma_newton_b": 2,
            "lpb_mma_trial": 2, "lpb_project": 2, "lpb_live_seed": 2, "lpb_live_outside": 2,
            "lpb_dead_loads": 2, "lpb_apply_rf_f32": 2, "lpb_apply_explicit_modal_f32": 2,
            "lpb_apply_explicit_modal_cheb_f32": 2, "lpb_modal_sym": 0, "lpb_hex8_ke": 0,
            "lpb_level1_products": 0, "lpb_uniform_numpy": 0, "lpb_layout_dims": 0, "lpb_layout_nodes_f64": 0,
            "lpb_unlayout_nodes_f64": 0, "lpb_layout_cells_f64": 0, "lpb_mg_levels": 0, "lpb_mg_strict": 0,
            "lpb_mg_destroy": 0,
            # the handle's entries launch on its own stream; their kernels are not counted here
            "lpb_mg_create": 0, "lpb_mg_set_moduli": 0, "lpb_mg_solve": 0}
# entries whose kernel count depends on their arguments
_VARIABLE = {"lpb_sensitivity": lambda a: 1 + (a[9] is not None), "lpb_stress_pass": lambda a: 1 + (a[0] < 2),
             "lpb_band_solve_cols_f32": lambda a: a[3] + (a[3] + 7) // 8,
             "lpb_band_solve_cols_f64": lambda a: a[3] + (a[3] + 7) // 8}
_COUNT = [0]


def launches() -> int:
    """Kernels launched through this binding so far (sensitivity with a compliance output counts
    as 2; a CUDA graph replay counts the kernels it holds, see add_launches)."""
    return _COUNT[0]


def add_launches(n: int) -> None:
    """Adjust the count: a graph capture subtracts the launches it recorded (they did not run)
    and each replay of the graph adds them back."""
    _COUNT[0] += n


class LpError(RuntimeError):
    pass


def parse_header(path: str = HEADER):
    """[(name, restype, [argtype, ...])] of every `lpb_*` declaration in the header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = []
    for m in re.finditer(r"\b(int|void\s*\*|void|long long)\s*(lpb_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, args = re.sub(r"\s+", "", m.group(1)) if "*" in m.group(1) else m.group(1), m.group(2), m.group(3).strip()
        types = []
        if args and args != "void":
            for a in args.split(","):
                a = a.strip()
                if "*" in a:
                    types.append(ctypes.c_void_p)
                    continue
                a = re.sub(r"\bconst\b", "", a).strip()
                base = " ".join(a.split()[:-1])
                if base not in _CTYPES:
                    raise LpError(f"{name}: unsupported argument type {a!r}")
                types.append(_CTYPES[base])
        out.append((name, _CTYPES[ret], types))
    return out


class _Lib:
    def __init__(self):
        if not os.path.exists(LIB_PATH):
            raise LpError(f"{LIB_PATH} is not built: run `python -m loadpath_b200.build` "
                          "(loadpath_b200 has no CPU fallback)")
        self.dll = ctypes.CDLL(LIB_PATH)
        self.decls = parse_header()
        self.fns = {}
        for name, ret, types in self.decls:
            try:
                fn = getattr(self.dll, name)
            except AttributeError as e:
                raise LpError(f"{LIB_PATH} does not export {name} declared in {HEADER}") from e
            fn.restype = ret
            fn.argtypes = types
            self.fns[name] = fn

    def __getattr__(self, name):
        fn = self.fns.get(name)
        if fn is None:
            raise AttributeError(name)

        nk = _KERNELS.get(name, 1)
        var = _VARIABLE.get(name)

        def call(*args):
            _COUNT[0] += var(args) if var is not None else nk
            st = fn(*args)
            if st is not None and st < 0:
                raise LpError(f"{name}: {_STATUS.get(st, 'error')} (status {st})")
            return st

        call.__name__ = name
        return call


_LIB = None


def lib() -> _Lib:
    global _LIB
    if _LIB is None:
        _LIB = _Lib()
    return _LIB
