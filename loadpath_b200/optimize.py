"""SIMP with the MMA update and a penalty continuation, its sensitivities from the autograd path.

Each iteration: the penalty p_k = p0 + (p - p0) min(k, ramp) / ramp; compliance c(x) through
`autograd.Compliance` (filter, SIMP law, MG-PCG) and its gradient from the backward (element
energy, SIMP derivative, filter transpose); the volume constraint g(x) = mean(H x / hs) / vf - 1
with the constant gradient H (1 / hs) / (n vf); one step of `mma.MMA` (m = 1) on the objective
scaled by the first compliance. The reference drives its MMA (loadpath/mma.py:31-214) from
loadpath/simp.py's optimiser with the same objective and constraint forms; the penalty ramp and
the scaling are the loop's parameters.

The design lives in grid order (nx, ny, nz) as a float64 CUDA tensor; every n-sized pass
(filter, solve, sensitivities, the MMA's passes) runs on the device and the host reads scalars.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import lib
from .autograd import Compliance, SimpProblem
from .grid import stream_handle
from .mma import MMA

__all__ = ["MMALoop"]


class MMALoop:
    """dims: cells (even); fixed_grid: bool (3, nx+1, ny+1, nz+1); f_grid: float64 loads on the
    node grid; x0: initial design (default volfrac everywhere); dtype: the V-cycle precision."""

    def __init__(self, dims, volfrac, rmin, fixed_grid, f_grid, nu=0.3, element="im", emin=1e-9, penal=3.0,
                 penal0=1.0, ramp=20, move=0.2, rtol=1e-6, dtype=np.float32, coarse_cells=2000, maxiter=500,
                 x0=None, device="cuda"):
        self.dims = tuple(int(d) for d in dims)
        self.volfrac = float(volfrac)
        self.penal, self.penal0, self.ramp = float(penal), float(penal0), int(ramp)
        self.problem = SimpProblem(self.dims, fixed_grid, rmin=rmin, nu=nu, penal=penal0, emin=emin,
                                   element=element, dtype=dtype, rtol=rtol, maxiter=maxiter,
                                   coarse_cells=coarse_cells, device=device)
        p = self.problem
        g = p.grid
        self.n = int(np.prod(self.dims))
        self.f = p.node_load(f_grid)
        if x0 is None:
            self.x = torch.full(self.dims, self.volfrac, dtype=torch.float64, device=g.device)
        else:
            self.x = torch.as_tensor(np.asarray(x0, np.float64), device=g.device).reshape(self.dims).clone()
        # dg/dx = H (1 / hs) / (n vf): the filter's own volume weights, constant
        self.dg = (g.cell_grid(p.filter.gv) / (self.n * self.volfrac)).reshape(1, -1).contiguous()
        self.mma = MMA(self.n, 1, 0.0, 1.0, move, device=device)
        self._ones = g.set_cells(g.cell_field(torch.float64), 1.0)
        self._vol = torch.zeros(1, dtype=torch.float64, device=g.device)
        self.c0 = None
        self.loop = 0
        self.history = []        # (compliance, volume fraction, change, penalty, CG iterations)

    def penal_at(self, k):
        return self.penal0 + (self.penal - self.penal0) * min(k, self.ramp) / self.ramp

    def step(self):
        """One iteration; returns (compliance, volume fraction of the filtered design, change)."""
        p = self.problem
        p.penal = self.penal_at(self.loop)
        xt = self.x.clone().requires_grad_(True)
        c = Compliance.apply(xt, p, [self.f])
        c.backward()
        cval = float(c.detach())
        if self.c0 is None:
            self.c0 = abs(cval) if cval != 0 else 1.0
        # the filtered design's volume fraction (the padding of the cell field is zero)
        lib().lpb_dot_f64(p.xphys.data_ptr(), self._ones.data_ptr(), p.xphys.numel(), p._part.data_ptr(),
                          self._vol.data_ptr(), stream_handle())
        vol = float(self._vol.item()) / self.n
        g1 = vol / self.volfrac - 1.0
        xnew = self.mma.update(self.x.reshape(-1), cval / self.c0, (xt.grad / self.c0).reshape(-1),
                               np.array([g1]), self.dg)
        xnew = xnew.reshape(self.dims)
        change = float((xnew - self.x).abs().max())
        self.x = xnew
        self.loop += 1
        self.history.append((cval, vol, change, p.penal, p.ge.last_iters))
        return cval, vol, change

    def run(self, iters):
        for _ in range(iters):
            self.step()
        return self

    def xphys_host(self):
        """The last forward's filtered design (grid order)."""
        return self.problem.grid.cells_to_host(self.problem.xphys)
