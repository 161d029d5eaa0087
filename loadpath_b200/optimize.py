"""The SIMP loops over the device pieces.

`OptimizeLoop`: loadpath's own SIMP loop (loadpath/simp.py:1640-2455, `simp.optimize` /
`_optimize_run`) for a plain compliance problem: blueprint and eroded projections of the filtered
design, the SIMP law on the eroded one, MG-PCG solves, sensitivities carried back through the
eroded projection and the filter, the volume's through the blueprint's, the measured step length,
the optimality-criteria step whose volume multiplier is solved to rounding, beta continuation and
the stopping rules. Described in its docstring.

`ConstrainedLoop`: loadpath's minimum-mass loop under stress and deflection limits
(loadpath/constrained.py:295-854, `optimize_constrained`) over the same pieces, with MMA.

`MMALoop`: SIMP with the MMA update and a penalty continuation, its sensitivities from the autograd path.

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

import math
import os
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import lib
from .autograd import Compliance, SimpProblem
from .fem import corner_stress_ops
from .grid import stream_handle
from .mg import BoxMesh, GridElasticity
from .mma import MMA
from .simp import MG_MIN_CELLS, SUB_REUSE, DeviceFilter, LiveCells, ProjectedDesign, _cells_touching

__all__ = ["MMALoop", "OptimizeLoop", "ConstrainedLoop", "Limits", "SimpOptions", "E_MIN", "PENALTY"]

E_MIN = 1e-6          # void modulus of loadpath's SIMP loop (loadpath/simp.py:42)
PENALTY = 3.0         # SIMP exponent (loadpath/simp.py:55)
STEP_SHRINK = 0.5     # the measured step's limits per iteration (loadpath/simp.py:1239-1240)
STEP_GROW = 1.2


@dataclass
class SimpOptions:
    """The options of loadpath's SIMP loop that `OptimizeLoop` runs, with the reference's names,
    meanings and defaults (loadpath/simp.py:899-1000). Options of terms this package does not run
    (build direction, access, extrusion, pattern, mirror, heat, buckling and the rest) are not
    listed; the delivered part's post-processing (opening, pruning) is not part of the loop."""
    volume_fraction: float
    filter_radius: float
    max_iterations: int = 120
    beta_max: float = 32.0
    beta_every: int = 10
    beta_schedule: tuple | None = None
    move: float = 0.2
    adaptive_move: bool = True
    tol: float = 0.01
    solve_rtol: float = 1e-4
    adaptive_rtol: bool = False
    stall_rtol: float = 2e-3
    stall_window: int = 6
    stiffness_bound: bool = False
    eta: float = 0.5
    erode: float = 0.15
    beta_start: float = 1.0
    pad_filter: bool | None = None
    x0: np.ndarray | None = None


def beta_hold(opts: SimpOptions, beta: float) -> int:
    """Most iterations at projection sharpness beta (loadpath/simp.py:1436-1440)."""
    s = opts.beta_schedule
    k = int(round(math.log2(max(beta, 1.0))))
    return s[k] if s is not None and k < len(s) else opts.beta_every


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


class OptimizeLoop:
    """loadpath's SIMP loop (loadpath/simp.py:1640-2455) on the device, for compliance under one or
    more weighted load cases at a volume fraction, with passive solid / void cells.

    Per iteration, as the reference's loop body: the blueprint xp = P(H x / hs, beta, eta) and the
    eroded xe = P(H x / hs, beta, eta + erode) (`physical`, `eroded`, :1775-1814); moduli
    E = E_MIN + xe^3 (1 - E_MIN); one MG-PCG solve per case, warm-started from the last one, on the
    cells the reference's analysis solves (`_Analysis`, :114-330: when fewer than 80 % of the cells
    are alive only the alive cells connected to a support, `LiveCells`, a reduced system reused
    while the alive cells stay in it on grids the reference solves directly); compliance sum_k w_k f_k.u_k;
    dc = min(H^T(dc_xe P'(xt, eta + erode) / hs), 0) and dv = max(H^T(w P'(xt, eta) / hs), 1e-12)
    (:1994-2204); the move limit measured from the slope of the Lagrangian along the last step
    (:2229-2243) or the fixed schedule (move, then move / 2 past beta 4); the optimality-criteria
    step with its volume multiplier bracketed in log space from the last one and found by
    false position with the Illinois halving (`ProjectedDesign.oc_step`, :2249-2376); then beta
    continuation and the stopping rules (:2418-2450). Every cell-sized pass runs on the device; the
    host reads the loop's scalars, as the reference's loop does.

    dims: cells (even); fixed_grid: bool (3, nx+1, ny+1, nz+1); loads: node-grid force arrays
    (3, nx+1, ny+1, nz+1), one per case; preserve / void: bool cell grids or None; pitch: the cell
    size (Ke and the filter scale with it as the reference's `_Analysis` and `density_filter` do);
    mirror: the mirror planes of a symmetric problem ('x', 'y', 'z' in the domain's order), whose
    sensitivities and trial designs are averaged across them (loadpath/simp.py:2222-2224, 2300);
    dtype: the V-cycle's precision (the CG is float64)."""

    def __init__(self, dims, fixed_grid, loads, nu, opts: SimpOptions, preserve=None, void=None,
                 case_weights=None, pitch=1.0, mirror=(), element="im", dtype=np.float32, coarse_cells=2000,
                 maxiter=2000, live_cells=True, device="cuda"):
        dims = tuple(int(d) for d in dims)
        if any(d % 2 for d in dims):
            raise ValueError("the device SIMP loop takes even cell counts")
        self.dims, self.opts, self.pitch = dims, opts, float(pitch)
        self.mesh = BoxMesh(dims)
        flat = np.asarray(fixed_grid, bool).reshape(3, -1)
        fixed = np.empty(self.mesh.n_dof, bool)
        for i in range(3):
            fixed[i::3] = flat[i]
        self.ge = GridElasticity(self.mesh, nu, fixed, rtol=opts.solve_rtol, maxiter=maxiter,
                                 coarse_cells=coarse_cells, dtype=dtype, element=element, device=device)
        g = self.ge.g0
        self.grid = g
        pad = True if opts.pad_filter is None else bool(opts.pad_filter)
        self.filter = DeviceFilter(g, opts.filter_radius, self.pitch, pad=pad)
        pres = np.zeros(dims, bool) if preserve is None else np.asarray(preserve, bool)
        vd = np.zeros(dims, bool) if void is None else np.asarray(void, bool)
        design = ~pres
        if not design.any():
            raise ValueError("nothing to optimize: every cell is preserved")
        self.n_design = int(design.sum())
        flags = (pres & ~vd).astype(np.uint8) | (vd.astype(np.uint8) << 1)
        self.flags = g.set_cells(g.cell_field(torch.uint8), torch.from_numpy(flags))
        self.w = g.cells_to_dev(design.astype(np.float64), torch.float64)
        axes = {"x": 0, "y": 1, "z": 2}
        self.mirror = tuple(axes.get(a, a) for a in mirror)
        self.pd = ProjectedDesign(self.filter, w=self.w, flags=self.flags, mirror=self.mirror)
        self.target = float(opts.volume_fraction) * float(design.sum())
        x = np.full(dims, float(opts.volume_fraction))
        if opts.x0 is not None:
            x = np.clip(np.asarray(opts.x0, np.float64).reshape(dims), 0.0, 1.0)
        x[pres] = 1.0
        x[vd] = 0.0
        self.x = g.cells_to_dev(x, torch.float64)
        cases = list(loads) if isinstance(loads, (list, tuple)) else [loads]
        self.fs = [g.nodes_to_dev(np.asarray(f, np.float64), torch.float64) for f in cases]
        self.weights = [1.0] * len(cases) if case_weights is None else [float(c) for c in case_weights]
        self.us = [None] * len(cases)
        self.live = None
        if live_cells:
            held = np.asarray(fixed_grid, bool).reshape(g.node_shape).any(axis=0)
            loaded = np.zeros(g.node_shape[1:], bool)
            for f in cases:
                loaded |= (np.asarray(f).reshape(g.node_shape) != 0).any(axis=0)
            # the reference's analysis reuses a reduced system on grids it solves directly
            reuse = SUB_REUSE if int(np.prod(dims)) < MG_MIN_CELLS else 0
            self.live = LiveCells(g, _cells_touching(held), _cells_touching(held | loaded) | pres, reuse=reuse)
        cf = lambda: g.cell_field(torch.float64)   # noqa: E731
        self.xp, self.dproj, self.xe, self.dproj_e, self.e, self.ce = cf(), cf(), cf(), cf(), cf(), cf()
        self.dc_xe, self.dc, self.dv, self.dx, self.gp, self._tmp = cf(), cf(), cf(), cf(), cf(), cf()
        self._part = torch.zeros(4096, dtype=torch.float64, device=g.device)
        self._s = torch.zeros(8, dtype=torch.float64, device=g.device)
        self.n = self.x.numel()
        self.beta = float(opts.beta_start)
        self.since_beta = 0
        self.step_prev = None     # the last step's multiplier while dx / gp hold its step and gradient
        self.move_k = float(opts.move)
        self.lam_last = None
        self.c0 = None
        self.it = 0
        self.history = []
        self.converged = False
        self.reduced = False
        self.measured = bool(opts.adaptive_move)
        self.scheduled = (self.measured and os.environ.get("LOADPATH_STOP", "hold") != "stall"
                          and not opts.stiffness_bound)

    # ---- device helpers ------------------------------------------------------------------------
    def _dot(self, a, b):
        lib().lpb_dot_f64(a.data_ptr(), b.data_ptr(), a.numel(), self._part.data_ptr(), self._s.data_ptr(),
                          stream_handle())
        return float(self._s[0].item())

    def _axpby(self, out, a, x, b, y):
        lib().lpb_axpby_f64(out.data_ptr(), float(a), x.data_ptr(), float(b), y.data_ptr(), out.numel(),
                            stream_handle())
        return out

    def _solve(self, rtol):
        """The cases' displacements on the moduli self.e (the reference's `_Analysis.solve`); returns
        sum_k w_k f_k.u_k and leaves dc_xe = -sum_k w_k p xe^(p-1) (1 - E_MIN) ce_k / pitch."""
        L = lib()
        g = self.grid
        st = stream_handle()
        self.ge.rtol = rtol
        self.reduced = False
        if self.live is not None:
            self.reduced = self.ge.set_moduli_live(self.e, self.live, self.xe, self.fs)
        else:
            self.ge.set_moduli_device(self.e)
        try:
            us = [self.ge.solve_device(f, u) for f, u in zip(self.fs, self.us)]
        except RuntimeError:
            if not self.reduced:
                raise
            # a reduced system the multigrid cannot hold: the full grid, void at E_MIN
            # (loadpath/simp.py:815-822), and no reduced system kept for reuse
            self.reduced = False
            self.live._cache = None
            self.ge.set_moduli_device(self.e)
            us = [self.ge.solve_device(f, None) for f in self.fs]
        self.us = us
        comp = 0.0
        # K scales with the pitch (loadpath/simp.py:159): u, its energies and f.u by 1 / pitch
        for k, (f, u, wk) in enumerate(zip(self.fs, us, self.weights)):
            self.ge.strain_energy_device(u, out=self.ce)
            L.lpb_sensitivity(self.dc_xe.data_ptr(), self.xe.data_ptr(), self.ce.data_ptr(), self.e.data_ptr(),
                              PENALTY, E_MIN, wk / self.pitch, int(k > 0), self._part.data_ptr(), None, *g.args, st)
            comp += wk * self._dot(f, u) / self.pitch
        return comp

    def step(self):
        """One iteration; returns its record (the reference's keys)."""
        L = lib()
        g = self.grid
        st = stream_handle()
        o = self.opts
        self.it += 1
        beta = self.beta
        eta, eta_e = o.eta, o.eta + o.erode
        pd = self.pd
        # blueprint (and its volume on the design cells) and eroded design, both from xt = H x / hs
        vol_b = pd.physical(self.x, beta, eta, xp=self.xp, dxp=self.dproj)
        L.lpb_project(self.xe.data_ptr(), self.dproj_e.data_ptr(), pd.xt.data_ptr(), beta, eta_e,
                      self.flags.data_ptr(), None, None, None, *g.args, st)
        L.lpb_simp_law(self.e.data_ptr(), self.xe.data_ptr(), PENALTY, E_MIN, *g.args, st)
        rtol = o.solve_rtol * (10.0 if beta <= 2 else 3.0 if beta <= 8 else 1.0) if o.adaptive_rtol \
            else o.solve_rtol
        comp = self._solve(rtol)
        if self.c0 is None:
            self.c0 = comp
        pd.chain(self.dc, self.dc_xe, self.dproj_e, clip=True)
        pd.chain(self.dv, self.w, self.dproj)
        L.lpb_cell_product(self.dv.data_ptr(), self.dv.data_ptr(), None, None, 2, *g.args, st)
        for ax in self.mirror:
            L.lpb_mirror_average(self.dc.data_ptr(), ax, *g.args, st)
            L.lpb_mirror_average(self.dv.data_ptr(), ax, *g.args, st)
        sec = None
        if self.measured:
            if self.step_prev is not None:
                a_s = self._dot(self.gp, self.dx)
                b_s = self._dot(self._axpby(self._tmp, 1.0, self.dc, self.step_prev, self.dv), self.dx)
                if a_s < 0:
                    t_s = a_s / (a_s - b_s) if b_s > a_s else math.inf
                    sec = t_s
                    self.move_k = min(self.move_k * min(max(t_s, STEP_SHRINK), STEP_GROW), o.move)
            move = self.move_k
        else:
            move = o.move if beta <= 4 else o.move / 2
        pd.lam_last = self.lam_last
        xn, lm, held = pd.oc_step(self.x, self.dc, self.dv, move, beta, eta, self.target)
        self.lam_last = lm
        L.lpb_max_abs_diff_f64(xn.data_ptr(), self.x.data_ptr(), self.n, self._part.data_ptr(),
                               self._s[1:].data_ptr(), st)
        change = float(self._s[1].item())
        if self.measured:
            self._axpby(self.dx, 1.0, xn, -1.0, self.x)
            self._axpby(self.gp, 1.0, self.dc, lm, self.dv)
            self.step_prev = lm
        L.lpb_memcpy_async(self.x.data_ptr(), xn.data_ptr(), self.n * 8, st)
        self.since_beta += 1
        its = self.ge.last_iters
        rec = {"iteration": self.it, "compliance": comp, "relative": comp / self.c0 if self.c0 else 1.0,
               "volume": vol_b / self.n_design, "beta": beta, "change": change,
               "cgIterations": max(its) if isinstance(its, (list, tuple)) else its,
               "reduced": self.reduced, "volumeSolves": pd.n_eval}
        if o.adaptive_move:
            rec["move"] = move
            if sec is not None:
                rec["stepFit"] = float(min(sec, 99.0))
        self.history.append(rec)
        self._continue(change, move, comp, held)
        return rec

    def _continue(self, change, move, comp, held):
        """beta continuation and the stopping rules (loadpath/simp.py:2418-2450)."""
        o = self.opts
        free_step = not self.measured or change < 0.999 * move
        if self.beta < o.beta_max and ((change < o.tol * 2 and free_step)
                                       or self.since_beta >= beta_hold(o, self.beta)):
            self.beta = min(self.beta * 2, o.beta_max)
            self.since_beta = 0
            # twice as steep a projection: half as long a step
            self.step_prev = None
            self.move_k = self.move_k / 2
        elif self.beta >= o.beta_max and self.it >= 3:
            if change < o.tol and free_step:
                self.converged = True
                return
            w = o.stall_window
            if self.scheduled and held:
                if self.since_beta >= beta_hold(o, self.beta):
                    self.converged = True
            elif self.since_beta >= w and len(self.history) > w:
                old = self.history[-1 - w]["compliance"]
                if abs(comp - old) <= o.stall_rtol * abs(old):
                    self.converged = True

    def run(self, on_iter=None):
        """Iterate until a stopping rule holds or max_iterations; returns the history."""
        while self.it < self.opts.max_iterations and not self.converged:
            rec = self.step()
            if on_iter is not None:
                on_iter(rec)
        return self.history

    def xphys_host(self):
        """The blueprint of the current design (grid order), as the loop delivers it before
        post-processing (loadpath/simp.py:2454)."""
        self.pd.physical(self.x, self.beta, self.opts.eta, xp=self._tmp)
        return self.grid.cells_to_host(self._tmp)

    def x_host(self):
        return self.grid.cells_to_host(self.x)


@dataclass
class Limits:
    """The limits of loadpath's minimum-mass loop (loadpath/constrained.py:117-144): the allowable
    peak von Mises stress (MPa) and deflection at the loads (mm), either None, and the modulus
    (MPa) that turns unit-modulus displacements into mm. The reference's buckling, layer-bond,
    contact-band and averaging-radius options are not run here."""
    stress: float | None
    deflection: float | None
    modulus: float


STRESS_P = 8.0        # the P-mean's exponent (loadpath/constrained.py:46)
STALL_GAIN = 5e-3     # the lightest feasible design's gain that ends the run (loadpath/constrained.py:66)


class ConstrainedLoop:
    """loadpath's minimum-mass loop under stress and deflection limits (loadpath/constrained.py:
    295-854, `optimize_constrained` with Limits(stress, deflection, modulus) and default options)
    on the device. Per iteration: the blueprint and eroded designs, the solves (as OptimizeLoop:
    live cells, warm starts); per case with a deflection limit, the deflection f.u / (sum_n |f_n| E)
    and its gradient -dE ce / (sum |f| E) through the eroded projection and the filter; per case,
    with a stress limit, the relaxed von Mises ratio xe vm / limit at the 8 corners of every cell
    that moved and touches no support or load (lpb_stress_pass), its P-mean (P = 8) scaled by
    Le et al.'s adaptive normalisation, the adjoint solve on the same system (the right-hand side
    gathered by lpb_cell_vectors_to_nodes) and its gradient; the objective 10 mean(xp) over the
    design cells; one MMA step on the free cells (move 0.1 capped; halved with the asymptotes
    tightened while the worst constraint grows above 0.02, grown by 1.2 up to the cap inside); the
    loop's own beta continuation (once feasible, or after three holds; the cap times 0.6) and, at
    beta_max, the lightest feasible design kept and the run stopped on a feasible small change or
    a stalled volume. Constraints come in the reference's order: deflections, then stresses.

    Arguments as OptimizeLoop's, with limits: Limits."""

    def __init__(self, dims, fixed_grid, loads, nu, opts: SimpOptions, limits: Limits, preserve=None,
                 pitch=1.0, mirror=(), element="im", dtype=np.float32, coarse_cells=2000, maxiter=2000,
                 live_cells=True, device="cuda"):
        if limits.stress is None and limits.deflection is None:
            raise ValueError("optimize_constrained needs a stress or deflection limit")
        base = OptimizeLoop(dims, fixed_grid, loads, nu, opts, preserve=preserve, pitch=pitch, mirror=mirror,
                            element=element, dtype=dtype, coarse_cells=coarse_cells, maxiter=maxiter,
                            live_cells=live_cells, device=device)
        self.base, self.opts, self.limits = base, opts, limits
        g = base.grid
        self.grid, self.dims, self.pitch = g, base.dims, float(pitch)
        cases = list(loads) if isinstance(loads, (list, tuple)) else [loads]
        f = [np.asarray(c, np.float64).reshape(g.node_shape) for c in cases]
        self.load_size = [float(np.linalg.norm(fk.reshape(3, -1), axis=0).sum()) for fk in f]
        self.defl_cases = [c for c in range(len(f)) if limits.deflection is not None and self.load_size[c] > 0]
        self.stress_cases = list(range(len(f))) if limits.stress is not None else []
        self.m = len(self.defl_cases) + len(self.stress_cases)
        # stress is not counted in the cells the loads and supports touch
        held = np.asarray(fixed_grid, bool).reshape(g.node_shape).any(axis=0)
        loaded = np.zeros(g.node_shape[1:], bool)
        for fk in f:
            loaded |= (fk != 0).any(axis=0)
        counted = ~_cells_touching(held | loaded)
        self.counted = g.set_cells(g.cell_field(torch.uint8), torch.from_numpy(counted.astype(np.uint8)))
        self.nc = float(max(int(counted.sum()), 1) * 8)
        # C B_k / pitch acts on the reference's displacement; the solver's is pitch times it
        self.cb = torch.tensor(corner_stress_ops(nu, self.pitch, element) / self.pitch, dtype=torch.float64,
                               device=g.device).reshape(-1).contiguous()
        pres = np.zeros(self.dims, bool) if preserve is None else np.asarray(preserve, bool)
        design = ~pres
        self.n_design = int(design.sum())
        # the design cells' positions in the padded cell layout, in grid (C) order as the reference's
        # flatnonzero(design)
        xs, ys, zs = np.nonzero(design)
        pos = (((zs >> 2) * g.ny + ys) * g.nx + xs) * 4 + (zs & 3)
        self.free = torch.from_numpy(pos.astype(np.int64)).to(g.device)
        self.mma = MMA(self.free.numel(), self.m, 0.0, 1.0, min(opts.move, 0.1), device=device)
        self.move_cap = self.mma.move
        self.worst_prev = math.inf
        self.kappa = [1.0] * len(f)
        self.lams = [None] * len(f)
        cf = lambda: g.cell_field(torch.float64)   # noqa: E731
        self.gxe, self.df0 = cf(), cf()
        self.grads = [cf() for _ in range(self.m)]
        self.g0 = g.cells_to_dev(10.0 * design / design.sum(), torch.float64)
        self.fe = torch.zeros(g.n_cell_field * 24, dtype=torch.float64, device=g.device)
        self.rhs = g.node_field(torch.float64)
        self._part = torch.zeros(4096, dtype=torch.float64, device=g.device)
        self._s = torch.zeros(4, dtype=torch.float64, device=g.device)
        self.beta = float(opts.beta_start)
        self.since_beta = 0
        self.it = 0
        self.history = []
        self.best = None
        self.trail = []
        self.converged = False

    def _stress(self, c, u, pos):
        """The stress constraint of case c (loadpath/constrained.py:597-652): its value g - 1 and its
        gradient in grads[pos] (before the filter chain), the adjoint solved on the last system."""
        L = lib()
        g = self.grid
        st = stream_handle()
        b = self.base
        lim = float(self.limits.stress)
        args = (u.data_ptr(), b.xe.data_ptr(), self.counted.data_ptr(), self.cb.data_ptr(), lim)
        L.lpb_stress_pass(0, *args, 0.0, 0.0, 0.0, self.nc, self._part.data_ptr(), self._s.data_ptr(), None, None,
                          *g.args, st)
        smax = float(self._s[0].item())
        sc = max(smax, 1e-30)
        L.lpb_stress_pass(1, *args, sc, 0.0, 0.0, self.nc, self._part.data_ptr(), self._s[1:].data_ptr(), None,
                          None, *g.args, st)
        pm = sc * (float(self._s[1].item()) / self.nc) ** (1.0 / STRESS_P)
        k = smax / max(pm, 1e-30)
        self.kappa[c] = 0.5 * (self.kappa[c] + k) if self.it > 1 else k
        L.lpb_stress_pass(2, *args, sc, pm, self.kappa[c], self.nc, None, None, self.gxe.data_ptr(),
                          self.fe.data_ptr(), *g.args, st)
        L.lpb_cell_vectors_to_nodes(self.rhs.data_ptr(), self.fe.data_ptr(), *g.args, st)
        lam = b.ge.solve_device(self.rhs, self.lams[c])
        self.lams[c] = lam
        # - dE lam_e . Ke u_e (loadpath/constrained.py:649-650): lam and u both the solver's
        b.ge.strain_energy_device(u, lam, out=b.ce)
        L.lpb_sensitivity(self.gxe.data_ptr(), b.xe.data_ptr(), b.ce.data_ptr(), b.e.data_ptr(), PENALTY, E_MIN, 1.0,
                          1, self._part.data_ptr(), None, *g.args, st)
        b.pd.chain(self.grads[pos], self.gxe, b.dproj_e)
        return self.kappa[c] * pm - 1.0, smax * lim

    def step(self):
        """One iteration; returns its record (the reference's keys; the readings per case in
        "deflection" and "stress" lists)."""
        L = lib()
        g = self.grid
        st = stream_handle()
        o, b, lim = self.opts, self.base, self.limits
        self.it += 1
        b.it = self.it
        beta = self.beta
        eta, eta_e = o.eta, o.eta + o.erode
        x_now = b.x.clone()
        vol_b = b.pd.physical(b.x, beta, eta, xp=b.xp, dxp=b.dproj)
        L.lpb_project(b.xe.data_ptr(), b.dproj_e.data_ptr(), b.pd.xt.data_ptr(), beta, eta_e, b.flags.data_ptr(),
                      None, None, None, *g.args, st)
        L.lpb_simp_law(b.e.data_ptr(), b.xe.data_ptr(), PENALTY, E_MIN, *g.args, st)
        b.ge.rtol = o.solve_rtol
        b._solve(o.solve_rtol)   # the cases' displacements in b.us (its compliance sums are not used here)
        cons, defl, stress = [], [], []
        pos = 0
        for c in self.defl_cases:
            u, fk = b.us[c], b.fs[c]
            d = b._dot(fk, u) / (self.load_size[c] * lim.modulus * self.pitch)
            b.ge.strain_energy_device(u, out=b.ce)
            L.lpb_sensitivity(self.gxe.data_ptr(), b.xe.data_ptr(), b.ce.data_ptr(), b.e.data_ptr(), PENALTY, E_MIN,
                              1.0 / (self.load_size[c] * lim.modulus * self.pitch * lim.deflection), 0,
                              self._part.data_ptr(), None, *g.args, st)
            b.pd.chain(self.grads[pos], self.gxe, b.dproj_e)
            cons.append(d / lim.deflection - 1.0)
            defl.append(d)
            pos += 1
        for c in self.stress_cases:
            v, smax = self._stress(c, b.us[c], pos)
            cons.append(v)
            stress.append(smax)
            pos += 1
        f0 = 10.0 * vol_b / self.n_design
        b.pd.chain(self.df0, self.g0, b.dproj)
        for ax in b.mirror:
            L.lpb_mirror_average(self.df0.data_ptr(), ax, *g.args, st)
            for gr in self.grads:
                L.lpb_mirror_average(gr.data_ptr(), ax, *g.args, st)
        worst = max(cons)
        if worst > 0.02 and worst > self.worst_prev:
            self.mma.move = max(0.02, 0.5 * self.mma.move)
            self.mma.tighten(0.5)
        elif worst <= 0.02:
            self.mma.move = min(self.move_cap, 1.2 * self.mma.move)
        self.worst_prev = worst
        xf = b.x.reshape(-1)[self.free]
        dfs = torch.stack([gr.reshape(-1)[self.free] for gr in self.grads])
        xnew = self.mma.update(xf, f0, self.df0.reshape(-1)[self.free], np.array(cons), dfs)
        b.xn = b.x.clone()
        b.xn.reshape(-1)[self.free] = xnew
        for ax in b.mirror:
            L.lpb_mirror_average(b.xn.data_ptr(), ax, *g.args, st)
        L.lpb_max_abs_diff_f64(b.xn.data_ptr(), b.x.data_ptr(), b.n, self._part.data_ptr(), self._s[2:].data_ptr(), st)
        change = float(self._s[2].item())
        b.x = b.xn
        self.since_beta += 1
        its = b.ge.last_iters
        rec = {"iteration": self.it, "volume": vol_b / self.n_design, "beta": beta, "change": change,
               "constraints": [float(v) for v in cons], "deflection": defl, "stress": stress,
               "cgIterations": max(its) if isinstance(its, (list, tuple)) else its, "reduced": b.reduced}
        self.history.append(rec)
        self._continue(rec, x_now)
        return rec

    def _continue(self, rec, x_now):
        """The loop's continuation, lightest-design record and stopping rules
        (loadpath/constrained.py:789-829)."""
        o = self.opts
        feasible = max(rec["constraints"]) <= 0.02
        change = rec["change"]
        if self.beta < o.beta_max and ((feasible and (self.since_beta >= o.beta_every or change < 2 * o.tol))
                                       or self.since_beta >= 3 * o.beta_every):
            self.beta = min(self.beta * 2, o.beta_max)
            self.since_beta = 0
            self.move_cap = max(0.02, self.move_cap * 0.6)
            self.mma.move = min(self.mma.move, self.move_cap)
        elif self.beta >= o.beta_max:
            if feasible and (self.best is None or rec["volume"] < self.best[1]["volume"]):
                self.best = (x_now, rec)
            self.trail.append(self.best[1]["volume"] if self.best is not None else math.inf)
            w = o.stall_window
            if self.best is not None and ((feasible and change < o.tol) or (
                    len(self.trail) > w and self.trail[-1] > (1.0 - STALL_GAIN) * self.trail[-1 - w])):
                self.converged = True

    def run(self, on_iter=None):
        """Iterate until a stopping rule holds or max_iterations; the design becomes the lightest
        feasible one checked at beta_max when there is one (loadpath/constrained.py:831-839)."""
        while self.it < self.opts.max_iterations and not self.converged:
            rec = self.step()
            if on_iter is not None:
                on_iter(rec)
        if self.best is not None:
            self.base.x = self.best[0]
        return self.history

    @property
    def x(self):
        return self.base.x

    def x_host(self):
        return self.grid.cells_to_host(self.base.x)

    @property
    def xp(self):
        """The blueprint the last iteration started from."""
        return self.base.xp
