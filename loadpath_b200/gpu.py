"""The reference's device seam (loadpath/gpu.py:56-80, :280-525): `resolve_device(name)` and
`TorchMG(grid, device)` with `load()` and `solve(b, x0) -> (x, iterations, converged)` on float64
numpy node grids, here over `mg.GridElasticity` (whose hierarchy already lives on the device).

loadpath builds `TorchMG(self, dev)` when `resolve_device` names a device (loadpath/mg.py:477-484);
with this package `GridElasticity` is the device solver itself, so the seam only forwards.
"""
from __future__ import annotations

import os

import numpy as np
import torch

__all__ = ["resolve_device", "TorchMG"]


def resolve_device(name: str | None = None):
    """The torch device to run on, or None for the reference's numpy path (LOADPATH_DEVICE:
    "auto", "b200", "cuda", "cuda:N"; "cpu" / "none" / "off" / "numpy" -> None). Raises when a
    CUDA device is asked for and there is none: this package has no host path."""
    name = (name if name is not None else os.environ.get("LOADPATH_DEVICE", "auto")).strip().lower()
    if name in ("", "cpu", "none", "off", "numpy"):
        return None
    if name in ("auto", "b200", "cuda") or name.startswith("cuda:"):
        if not torch.cuda.is_available():
            if name == "auto":
                return None
            raise RuntimeError(f"LOADPATH_DEVICE={name} but torch sees no CUDA device")
        return torch.device("cuda" if name in ("auto", "b200") else name)
    raise RuntimeError(f"LOADPATH_DEVICE={name}: this package runs on CUDA devices only")


class TorchMG:
    """The reference's device solve seam over a GridElasticity `grid` (already on the device)."""

    def __init__(self, grid, device):
        self.g = grid
        self.dev = device

    def load(self):
        """After every set_moduli in the reference; here the hierarchy is built on the device by
        set_moduli itself, so there is nothing to copy."""
        if not self.g.levels:
            raise RuntimeError("load() before set_moduli: the hierarchy is not built")

    def solve(self, b, x0):
        """float64 node grids (3, X+1, Y+1, Z+1), masked -> (x, iterations, converged)
        (loadpath/gpu.py:394-397); no exception on non-convergence, as the reference's."""
        g = self.g.g0
        bd = g.nodes_to_dev(np.asarray(b, np.float64), torch.float64)
        x0d = g.nodes_to_dev(np.asarray(x0, np.float64), torch.float64) if x0 is not None else None
        m = self.g.levels[0].mask
        from ._lib import lib
        from .grid import stream_handle

        L = lib()
        st = stream_handle()
        L.lpb_mask_field_f64(bd.data_ptr(), bd.data_ptr(), m.data_ptr(), *g.args, 0, st)
        if x0d is not None:
            L.lpb_mask_field_f64(x0d.data_ptr(), x0d.data_ptr(), m.data_ptr(), *g.args, 0, st)
        x, it, ok = self.g._solve_device(bd, x0d)
        self.g.last_iters = it
        return g.nodes_to_host(x), it, ok
