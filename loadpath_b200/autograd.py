"""Compliance and a point-displacement objective of a SIMP design as torch.autograd.Functions.

The reference writes its sensitivities out by hand and has no autograd: compliance is
self-adjoint, dc/dE_e = -u_e^T k_e u_e (loadpath/simp.py:1901-1904), chained through the density
filter's transpose (loadpath/simp.py:2001); a point-displacement output l . u needs its own
adjoint solve K lam = l and has dJ/dE_e = -lam_e^T k_e u_e (loadpath/mechanism.py:13-22,
156-164). Here both are functions of the design x (cells, grid order (nx, ny, nz), float64 on the
device) through

    xphys = H x / hs,   E = emin + xphys^p (1 - emin),   K(E) u_k = f_k,

and their backward is the device pipeline the SIMP loop uses: the element-energy kernel on
(u, u) or (lam, u), the sensitivity kernel (the SIMP derivative), and the filter applied as its
own transpose (H is symmetric). A point displacement's backward runs the adjoint MG-PCG solve.

Saved displacements: the forward keeps each load case's u for the backward while they fit in
`save_bytes` (float64 node fields); the cases past that are solved again in the backward on the
same moduli (checkpointing), so many load cases need not hold all their fields at once.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import lib
from .grid import stream_handle
from .mg import BoxMesh, GridElasticity
from .simp import DeviceFilter

__all__ = ["SimpProblem", "Compliance", "PointDisplacement", "compliance", "point_displacement"]


class SimpProblem:
    """The solver, filter and SIMP law an objective differentiates through.

    dims: cells (even); fixed_grid: bool (3, nx+1, ny+1, nz+1), True on held dofs; dtype: the
    V-cycle's precision (np.float32: the mixed path, np.float64: the plain FP64 path); the outer
    CG is float64 in both. save_bytes: how many bytes of saved displacements the forward keeps."""

    def __init__(self, dims, fixed_grid, rmin=2.0, nu=0.3, penal=3.0, emin=1e-9, element="im", dtype=np.float32,
                 rtol=1e-10, maxiter=2000, coarse_cells=2000, pad=False, save_bytes=8 << 30, warm_start=True,
                 device="cuda"):
        dims = tuple(int(d) for d in dims)
        self.dims = dims
        self.penal, self.emin = float(penal), float(emin)
        self.mesh = BoxMesh(dims)
        flat = np.asarray(fixed_grid, bool).reshape(3, -1)
        fixed = np.empty(self.mesh.n_dof, bool)
        for i in range(3):
            fixed[i::3] = flat[i]
        self.ge = GridElasticity(self.mesh, nu, fixed, rtol=rtol, maxiter=maxiter, coarse_cells=coarse_cells,
                                 dtype=dtype, element=element, device=device)
        g = self.ge.g0
        self.grid = g
        self.filter = DeviceFilter(g, rmin, pad=pad)
        self.save_bytes = int(save_bytes)
        self.warm_start = warm_start
        self.x = g.cell_field(torch.float64)
        self.xphys = g.cell_field(torch.float64)
        self.e = g.cell_field(torch.float64)
        self.ce = g.cell_field(torch.float64)
        self.dc = g.cell_field(torch.float64)
        self.grad = g.cell_field(torch.float64)
        self._part = torch.zeros(4096, dtype=torch.float64, device=g.device)
        self._dot = torch.zeros(1, dtype=torch.float64, device=g.device)
        self._warm = {}          # load key -> the last displacement solved for it
        self.version = 0         # counts set_design calls: a backward re-sets its forward's design
        self.solves = 0
        self.iterations = 0

    # ---- the forward pieces ----------------------------------------------------------------
    def set_design(self, x):
        """x (nx, ny, nz) float64 device tensor -> xphys = H x / hs and E on the device, and the
        solver's moduli."""
        g = self.grid
        if tuple(x.shape) != self.dims:
            raise ValueError(f"design of shape {tuple(x.shape)}, expected {self.dims}")
        g.set_cells(self.x, x.detach())
        self.filter.apply(self.xphys, self.x, hs_out=self.filter.hs, e_out=self.e, penal=self.penal, emin=self.emin)
        self.ge.set_moduli_device(self.e)
        self.version += 1
        return self.version

    def ensure_design(self, x, version):
        """Make the design of a forward (x, the version set_design returned) current again."""
        if self.version != version:
            self.set_design(x)

    def solve(self, f, key=None):
        """K(E) u = f on the current moduli (f: float64 device node field); warm-started from the
        last solve of the same key."""
        x0 = self._warm.get(key) if (self.warm_start and key is not None) else None
        u = self.ge.solve_device(f, x0)
        self.solves += 1
        self.iterations += self.ge.last_iters
        if self.warm_start and key is not None:
            self._warm[key] = u
        return u

    def dot(self, a, b, out):
        """out (a device scalar) = a . b over float64 node fields, without a host sync."""
        lib().lpb_dot_f64(a.data_ptr(), b.data_ptr(), a.numel(), self._part.data_ptr(), out.data_ptr(),
                          stream_handle())
        return out

    # ---- the backward pieces ---------------------------------------------------------------
    def accumulate(self, pairs):
        """self.dc = -sum over (a, b) of p (1 - emin) xphys^(p-1) a_e^T k_e b_e (dJ/dxphys) on the
        current design, then self.grad = H (dc / hs) (dJ/dx, the filter's transpose); returns
        self.grad."""
        L = lib()
        g = self.grid
        st = stream_handle()
        for k, (a, b) in enumerate(pairs):
            self.ge.strain_energy_device(a, b, out=self.ce)
            L.lpb_sensitivity(self.dc.data_ptr(), self.xphys.data_ptr(), self.ce.data_ptr(), None, self.penal,
                              self.emin, 1.0, int(k > 0), self._part.data_ptr(), None, *g.args, st)
        self.filter.apply(self.grad, self.dc, hs_in=self.filter.hs)
        return self.grad

    def node_load(self, f_grid):
        """(3, nx+1, ny+1, nz+1) host array or device tensor -> a float64 device node field."""
        g = self.grid
        t = g.node_field(torch.float64)
        if isinstance(f_grid, torch.Tensor):
            return g.set_nodes(t, f_grid)
        return g.nodes_to_dev(np.asarray(f_grid, np.float64), torch.float64, out=t)

    def unit_load(self, node, comp):
        """The point-displacement functional l with l . u = u_comp(node), a device node field."""
        f = np.zeros((3,) + tuple(d + 1 for d in self.dims))
        f[(comp,) + tuple(node)] = 1.0
        return self.node_load(f)


class Compliance(torch.autograd.Function):
    """c(x) = sum_k f_k . u_k with K(E(x)) u_k = f_k; backward: -sum_k u_k^T dK u_k through the
    SIMP law and the filter."""

    @staticmethod
    def forward(ctx, x, problem: SimpProblem, loads):
        ctx.version = problem.set_design(x)
        c = torch.zeros(1, dtype=torch.float64, device=x.device)
        saved, budget = [], problem.save_bytes
        for k, f in enumerate(loads):
            u = problem.solve(f, key=("case", k))
            problem.dot(f, u, problem._dot)
            c += problem._dot
            nb = u.numel() * u.element_size()
            if nb <= budget:
                saved.append(u)
                budget -= nb
            else:
                saved.append(None)          # solved again in the backward
        ctx.problem, ctx.loads, ctx.saved = problem, loads, saved
        ctx.x = x.detach().clone()
        return c[0]

    @staticmethod
    def backward(ctx, gc):
        p = ctx.problem
        us = ctx.saved
        p.ensure_design(ctx.x, ctx.version)
        if any(u is None for u in us):
            us = [u if u is not None else p.solve(f, key=("case", k)) for k, (u, f) in enumerate(zip(us, ctx.loads))]
        grad = p.accumulate([(u, u) for u in us])
        return p.grid.cell_grid(grad) * gc, None, None


class PointDisplacement(torch.autograd.Function):
    """J(x) = l . u with K(E(x)) u = f and l the unit functional of one dof; backward: the
    adjoint solve K lam = l, then -lam^T dK u through the SIMP law and the filter."""

    @staticmethod
    def forward(ctx, x, problem: SimpProblem, f, l):
        ctx.version = problem.set_design(x)
        u = problem.solve(f, key="point_u")
        j = torch.zeros(1, dtype=torch.float64, device=x.device)
        problem.dot(l, u, j)
        ctx.problem, ctx.f, ctx.l, ctx.u = problem, f, l, u
        ctx.x = x.detach().clone()
        return j[0]

    @staticmethod
    def backward(ctx, gj):
        p = ctx.problem
        p.ensure_design(ctx.x, ctx.version)
        lam = p.solve(ctx.l, key="point_lam")
        grad = p.accumulate([(lam, ctx.u)])
        return p.grid.cell_grid(grad) * gj, None, None, None


def compliance(x, problem: SimpProblem, loads):
    """Differentiable total compliance of the design x over the load cases (device node fields)."""
    return Compliance.apply(x, problem, list(loads))


def point_displacement(x, problem: SimpProblem, f, node, comp):
    """Differentiable displacement component `comp` of `node` (grid indices) under the load f."""
    return PointDisplacement.apply(x, problem, f, problem.unit_load(node, comp))
