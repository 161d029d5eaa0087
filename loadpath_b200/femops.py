"""The reference's `femops.element_energy` (loadpath/femops.py:236-242) on the device.

`element_energy(u, v, edof, ke)`: per element u_e^T ke v_e with u_e = u[edof[e]] over a general
mesh's element dof table (v None: u), host arrays in, a float64 host array out. The SIMP loop on
the box grid uses `GridElasticity.strain_energy_device`, which reads the node fields in place.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import lib
from .grid import stream_handle

__all__ = ["element_energy"]


def element_energy(u, v, edof, ke):
    """einsum("ij,jk,ik->i", u[edof], ke, v[edof]) per element, float64, summed on the device
    (row by row of ke: the same value to rounding, not the reference's bits)."""
    u = np.ascontiguousarray(u, np.float64).reshape(-1)
    v = None if v is None else np.ascontiguousarray(v, np.float64).reshape(-1)
    edof = np.ascontiguousarray(edof, np.int64)
    ke = np.ascontiguousarray(ke, np.float64)
    if edof.ndim != 2 or edof.shape[1] != 24 or ke.shape != (24, 24):
        raise ValueError("edof is (elements, 24) and ke 24 x 24")
    if v is not None and v.shape != u.shape:
        raise ValueError("u and v differ in length")
    ne = len(edof)
    if ne and (edof.min() < 0 or edof.max() >= len(u)):
        raise IndexError("an element dof lies outside the vectors")
    dev = torch.device("cuda")
    ud = torch.from_numpy(u).to(dev)
    vd = torch.from_numpy(v).to(dev) if v is not None else None
    ed = torch.from_numpy(edof).to(dev)
    kd = torch.from_numpy(ke).to(dev)
    out = torch.empty(max(ne, 1), dtype=torch.float64, device=dev)
    lib().lpb_element_energy_edof(out.data_ptr(), ud.data_ptr(), None if vd is None else vd.data_ptr(),
                                  ed.data_ptr(), kd.data_ptr(), ne, stream_handle())
    return out[:ne].cpu().numpy()
