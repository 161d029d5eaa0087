"""The SIMP loop on the device: density filter, SIMP law, solve, sensitivities, OC update.

Mirrors the reference pieces that sit on the hot path:
  - `density_filter(dims, radius, pad)` -> (H, hs) with H supporting `@` and `.T`
    (loadpath/simp.py:1143-1228: the cone stencil w = r - |d| pitch > 0 within floor(r / pitch)
    cells; H is symmetric; hs = full-kernel sum if padded, else row sums)
  - `_project` / `_dproject` (loadpath/simp.py:1443-1450)
  - `Top3dLoop`: the plain SIMP loop of the reference's top3d port
    (loadpath/benchmarks/reference.py:74-117): E = Emin + x^p (1 - Emin), compliance and
    sensitivities, density-filter chain rule, OC bisection on the multiplier with the volume
    measured on the filtered densities, stop on change <= 0.01 or the iteration cap.
Everything per iteration runs in this package's kernels on device-resident fields; the host
walks the bisection tree (a few doubles per pass) and reads the compliance and change.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from ._lib import add_launches, lib
from .grid import DevGrid, ptr, stream_handle
from .mg import BoxMesh, GridElasticity

__all__ = ["filter_taps", "DeviceFilter", "density_filter", "oc_bisection", "case_compliance", "adjoint_sensitivity",
           "LoadCaseShards",
           "LiveCells", "ProjectedDesign", "Top3dLoop",
           "_project", "_dproject"]


def filter_taps(radius: float, pitch: float = 1.0):
    """[(dx, dy, dz), w] of the cone filter (loadpath/simp.py:1148-1161)."""
    reach = int(np.floor(radius / pitch))
    out = []
    for dx in range(-reach, reach + 1):
        for dy in range(-reach, reach + 1):
            for dz in range(-reach, reach + 1):
                w = radius - math.sqrt(dx * dx + dy * dy + dz * dz) * pitch
                if w > 0:
                    out.append(((dx, dy, dz), float(w)))
    return out


class DeviceFilter:
    """H on a device cell grid (zeros outside the grid)."""

    def __init__(self, grid: DevGrid, radius: float, pitch: float = 1.0, pad: bool = False):
        self.grid = grid
        taps = filter_taps(radius, pitch)
        self.ntaps = len(taps)
        self.toff = torch.tensor([list(d) for d, _ in taps], dtype=torch.int32, device=grid.device).reshape(-1)
        self.tw = torch.tensor([w for _, w in taps], dtype=torch.float64, device=grid.device)
        self.full = float(sum(w for _, w in taps))
        ones = grid.set_cells(grid.cell_field(torch.float64), 1.0)
        self.rowsum = self.apply(grid.cell_field(torch.float64), ones)
        if pad:
            self.hs = grid.set_cells(grid.cell_field(torch.float64), self.full)
        else:
            self.hs = self.rowsum
        # H (1 / hs): the filtered volume's weights, and top3d's dv = H (1 / hs)
        self.gv = self.apply(grid.cell_field(torch.float64), ones, hs_in=self.hs)

    def apply(self, out, v, hs_in=None, hs_out=None, e_out=None, penal=3.0, emin=1e-9):
        """out = H (v / hs_in) / hs_out; with e_out also e_out = emin + out^p (1 - emin)."""
        lib().lpb_filter(out.data_ptr(), v.data_ptr(), self.toff.data_ptr(), self.tw.data_ptr(), self.ntaps,
                         ptr(hs_in), ptr(hs_out), ptr(e_out), float(penal), float(emin), *self.grid.args,
                         stream_handle())
        return out


class _HostFilter:
    """`H @ v` / `H.T @ v` on host vectors in the grid's C order, computed on the device."""

    def __init__(self, dev: DeviceFilter):
        self.dev = dev
        self.T = self
        n = dev.grid.nx * dev.grid.ny * dev.grid.nz
        self.shape = (n, n)

    def __matmul__(self, v):
        g = self.dev.grid
        vd = g.cells_to_dev(np.asarray(v, np.float64).reshape(g.cells), torch.float64)
        out = self.dev.apply(g.cell_field(torch.float64), vd)
        return g.cells_to_host(out).reshape(-1)

    def sum(self, axis=1):
        return self.dev.grid.cells_to_host(self.dev.rowsum).reshape(-1)


def density_filter(dims, radius, pad=True, pitch=1.0, device="cuda"):
    """(H, hs) of the cone filter on a full box of cells in C order (loadpath/simp.py:1181-1228).
    dims: the cell counts, or a domain with `.dims` and `.pitch` as the reference takes (a full
    box: every cell a design cell)."""
    if hasattr(dims, "dims"):
        pitch = float(getattr(dims, "pitch", pitch))
        dims = tuple(int(d) for d in dims.dims)
    g = DevGrid(dims, device)
    f = DeviceFilter(g, radius, pitch, pad)
    return _HostFilter(f), g.cells_to_host(f.hs).reshape(-1)


def _project(xt, beta, eta):
    """tanh Heaviside projection (loadpath/simp.py:1443-1446)."""
    den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
    return (np.tanh(beta * eta) + np.tanh(beta * (xt - eta))) / den


def _dproject(xt, beta, eta):
    """its derivative (loadpath/simp.py:1448-1450)."""
    den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
    return beta * (1 - np.tanh(beta * (xt - eta)) ** 2) / den


class LoadCaseShards:
    """Load cases split over the ranks of a torch.distributed group (one process per GPU): rank r
    solves cases r, r + world, ...; after each rank has summed its cases' compliance and
    sensitivity, one all-reduce (sum) gives every rank the totals, and every rank then takes the
    same design step, so the designs stay identical without being sent. The only exchange per
    SIMP iteration is that one reduction of a cell field plus one scalar (NCCL on CUDA tensors,
    gloo on CPU tensors)."""

    def __init__(self, n_cases, group=None):
        import torch.distributed as dist

        self.n_cases = int(n_cases)
        self.group = group
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.world = self.dist.get_world_size(group) if self.dist else 1

    def mine(self):
        """This rank's case indices."""
        return list(range(self.rank, self.n_cases, self.world))

    def reduce(self, dc, comp):
        """dc (a cell field, summed in place over the ranks) and comp (this rank's compliance
        sum) -> the total compliance."""
        if self.dist is None or self.world == 1:
            return float(comp)
        c = torch.tensor([float(comp)], dtype=dc.dtype, device=dc.device)
        self.dist.all_reduce(dc, group=self.group)
        self.dist.all_reduce(c, group=self.group)
        return float(c.item())


def case_compliance(f, u, part=None):
    """f . u on float64 device node fields: a load case's compliance, the single-direction case of
    loadpath/directions.py:167-180 (`collapse`, whose energy terms are then [(1.0, u)])."""
    L = lib()
    g_n = f.numel()
    part = part if part is not None else torch.zeros(2048, dtype=torch.float64, device=f.device)
    out = torch.zeros(1, dtype=torch.float64, device=f.device)
    L.lpb_dot_f64(f.data_ptr(), u.data_ptr(), g_n, part.data_ptr(), out.data_ptr(), stream_handle())
    return float(out.item())


def adjoint_sensitivity(ge, pairs, xp, dproj, out, modulus=1.0, penal=3.0, emin=1e-9):
    """The compliant-mechanism output's sensitivity (loadpath/mechanism.py:156-165):
    out = -sum over (u, lam) pairs of lam_e . k_e u_e, times modulus p (1 - emin) xp^(p - 1) and
    dproj, with K lam = l the adjoint solve of the output functional l (ge.solve_device(l)).
    pairs: [(u, lam)] float64 device node fields; xp, dproj, out: float64 cell fields of ge's fine
    grid."""
    L = lib()
    g = ge.g0
    st = stream_handle()
    ce = ge._tbuf("adj_ce", out.shape, torch.float64)
    part = ge._tbuf("adj_part", (4096,), torch.float64)
    for k, (u, lam) in enumerate(pairs):
        ge.strain_energy_device(lam, u, out=ce)
        L.lpb_sensitivity(out.data_ptr(), xp.data_ptr(), ce.data_ptr(), None, float(penal), float(emin),
                          float(modulus), int(k > 0), part.data_ptr(), None, *g.args, st)
    L.lpb_cell_product(out.data_ptr(), out.data_ptr(), dproj.data_ptr(), None, 0, *g.args, st)
    return out


ALIVE = 1e-3          # cells at or below this projected density leave the solve (loadpath/simp.py:59)
REDUCE_BELOW = 0.8    # ...once fewer than this share of the cells are alive (loadpath/simp.py:61)
MG_SLOW_ITERS = 60    # CG iterations past which the SIMP driver leaves the multigrid (loadpath/simp.py:85)
OC_TOL = 1e-3         # top3d's bisection stops at (l2 - l1) / (l1 + l2) <= 1e-3 (loadpath/benchmarks/reference.py:100)
MG_MAXITER = 2000     # the SIMP driver's CG cap for its multigrid (loadpath/simp.py:182)
MG_MIN_CELLS = 100_000  # grids the SIMP driver solves by multigrid from; smaller ones directly (loadpath/simp.py:69)
SUB_REUSE = 6         # solves the direct path keeps a reduced system for (loadpath/simp.py:288)


def _cells_touching(node_flags):
    """bool (nx, ny, nz): cells with any of their eight corner nodes set in node_flags
    (nx+1, ny+1, nz+1)."""
    n = np.asarray(node_flags, bool)
    out = np.zeros(tuple(d - 1 for d in n.shape), bool)
    for i in (0, 1):
        for j in (0, 1):
            for k in (0, 1):
                out |= n[i:i + out.shape[0], j:j + out.shape[1], k:k + out.shape[2]]
    return out


class LiveCells:
    """The solve's live-cell reduction on the device (loadpath/simp.py:725 the alive set, :263-289
    `_connected`, :795-826 `_solve_mg`): alive = projected density above ALIVE or an anchor cell
    (touching a support or a load, or preserved); when fewer than REDUCE_BELOW of the cells are
    alive, the solve keeps the alive cells 26-connected to an alive cell touching a support and
    the others get modulus 0 on the fixed grid. The components are found by a flood fill from
    those support cells (lp_live.cu), the union the reference's labelling keeps.

    support_touch, anchor: bool (nx, ny, nz) host arrays in grid order. reuse: 0 for the multigrid
    path's rule above (the kept cells found again every solve); n > 0 for the direct path's
    (loadpath/simp.py:288-315 `_subsystem`, grids under MG_MIN_CELLS cells): a reduced system is
    kept for up to n further solves while every alive cell stays inside it, its cells keeping their
    moduli (set_moduli_live records it once its loads are found held)."""

    def __init__(self, grid: DevGrid, support_touch, anchor, reuse=0):
        self.grid = grid
        self.reuse = int(reuse)
        self._cache = None       # the reduced system's kept cells (a flooded state), or None
        self._age = 0
        self.reused = False      # the last keep() handed back the cached system
        st = np.asarray(support_touch, bool)
        an = np.asarray(anchor, bool)
        bits = torch.from_numpy((st.astype(np.uint8) | (an.astype(np.uint8) << 1)))
        self.flags = grid.set_cells(grid.cell_field(torch.uint8), bits)
        self.state = grid.cell_field(torch.uint8)
        self._part = torch.zeros(592, dtype=torch.float64, device=grid.device)
        self._cnt = torch.zeros(1, dtype=torch.float64, device=grid.device)
        self._changed = torch.zeros(1, dtype=torch.int32, device=grid.device)
        self.n_cells = grid.nx * grid.ny * grid.nz
        self.alive_share = 1.0
        self.passes = 0

    def keep(self, xp, max_passes=1 << 20):
        """The kept cells (self.state == 2) for projected densities xp (float64 cell field), or
        None when REDUCE_BELOW or more of the cells are alive (the reference keeps them all)."""
        L = lib()
        g = self.grid
        st = stream_handle()
        L.lpb_live_seed(self.state.data_ptr(), xp.data_ptr(), self.flags.data_ptr(), ALIVE, self._part.data_ptr(),
                        self._cnt.data_ptr(), *g.args, st)
        self.alive_share = float(self._cnt.item()) / self.n_cells
        self.passes = 0
        self.reused = False
        if self.alive_share >= REDUCE_BELOW:
            return None
        if self.reuse and self._cache is not None and self._age < self.reuse:
            L.lpb_live_outside(self.state.data_ptr(), self._cache.data_ptr(), self._part.data_ptr(),
                               self._cnt.data_ptr(), *g.args, st)
            if float(self._cnt.item()) == 0.0:
                self._age += 1
                self.reused = True
                return self._cache
        while self.passes < max_passes:
            L.lpb_memset_async(self._changed.data_ptr(), 0, 4, st)
            for _ in range(4):   # a few passes between reads of the flag
                L.lpb_live_flood(self.state.data_ptr(), self._changed.data_ptr(), *g.args, st)
                self.passes += 1
            if int(self._changed.item()) == 0:
                return self.state
        raise RuntimeError("live-cell flood fill did not settle")

    def moduli(self, e, out):
        """out = e on the kept cells, 0 elsewhere (after keep())."""
        kept = self._cache if self.reused else self.state
        lib().lpb_live_moduli(out.data_ptr(), e.data_ptr(), kept.data_ptr(), *self.grid.args, stream_handle())
        return out

    def record(self, held):
        """After a fresh reduction (not a reused one): keep it for reuse when its loads are held,
        drop any cached one when they are not."""
        if not self.reuse or self.reused:
            return
        if held:
            self._cache = self.state.clone()
            self._age = 0
        else:
            self._cache = None


VOLUME_RTOL = 1e-13   # the volume multiplier's stopping tolerance (loadpath/simp.py:1234)


class ProjectedDesign:
    """loadpath's own design update on the device: the filtered and projected physical density
    (loadpath/simp.py:1775-1786 `physical`, :1809-1814 `eroded`), the filter chain rule of a
    gradient through the projection (loadpath/simp.py:1995-2001, :2077), and the optimality-
    criteria step whose volume multiplier is solved to rounding (loadpath/simp.py:2249-2376): bracket
    the root outward from the last step's multiplier in log space, then false position with the
    Illinois modification, every trial measured on the physical density's volume.

    flt: the grid's DeviceFilter (H symmetric, as the reference's cone filter); w: volume weight per
    cell (float64 cell field; None: 1 on every cell); flags: uint8 cell field, bit 0 passive solid
    (held at 1), bit 1 passive void (held at 0), or None; mirror: the axes (0 x, 1 y, 2 z, in the
    reference's order) whose mirror symmetry each trial design is averaged onto (loadpath/simp.py:
    2300-2301, `_symmetrize`; the pinned and void cells mirror-symmetric, as the reference's
    domains build them). The reference's column extrusion, printed-hook and blockage terms are not
    part of this step."""

    def __init__(self, flt: DeviceFilter, w=None, flags=None, mirror=()):
        g = flt.grid
        self.flt, self.grid, self.flags = flt, g, flags
        self.mirror = tuple(int(a) for a in mirror)
        self.w = w if w is not None else g.set_cells(g.cell_field(torch.float64), 1.0)
        self.xt = g.cell_field(torch.float64)
        self.xp = g.cell_field(torch.float64)
        self.xn = g.cell_field(torch.float64)
        self._tmp = g.cell_field(torch.float64)
        self._part = torch.zeros(592, dtype=torch.float64, device=g.device)
        self._vol = torch.zeros(1, dtype=torch.float64, device=g.device)
        self.lam_last = None
        self.n_eval = 0

    def physical(self, x, beta, eta, xp=None, dxp=None):
        """xt = H x / hs into self.xt, its projection into xp (default self.xp) and the derivative
        into dxp (if given); returns the projected volume sum xp w."""
        L = lib()
        g = self.grid
        self.flt.apply(self.xt, x, hs_out=self.flt.hs)
        xp = self.xp if xp is None else xp
        L.lpb_project(xp.data_ptr(), ptr(dxp), self.xt.data_ptr(), float(beta), float(eta), ptr(self.flags),
                      self.w.data_ptr(), self._part.data_ptr(), self._vol.data_ptr(), *g.args, stream_handle())
        return float(self._vol.item())

    def chain(self, out, grad, dxp, clip=False):
        """out = H^T (grad dxp / hs) (zero on held cells), then min(out, 0) with clip."""
        L = lib()
        g = self.grid
        st = stream_handle()
        L.lpb_cell_product(self._tmp.data_ptr(), grad.data_ptr(), ptr(dxp), ptr(self.flags), 0, *g.args, st)
        self.flt.apply(out, self._tmp, hs_in=self.flt.hs)
        if clip:
            L.lpb_cell_product(out.data_ptr(), out.data_ptr(), None, None, 1, *g.args, st)
        return out

    def oc_step(self, x, dc, dv, move, beta, eta, target):
        """The step x -> clip(x sqrt(-dc / dv / lm), x -+ move) with the multiplier lm that puts the
        physical volume on target (loadpath/simp.py:2320-2376). Returns (x_new, lm, held): x_new is
        self.xn (the last trial), held False when the move limits kept the volume off target."""
        L = lib()
        g = self.grid
        st = stream_handle()
        n_eval = [0]

        def stepped(lm_):
            n_eval[0] += 1
            L.lpb_oc_stepped(self.xn.data_ptr(), x.data_ptr(), dc.data_ptr(), dv.data_ptr(), float(lm_), float(move),
                             ptr(self.flags), *g.args, st)
            for ax in self.mirror:
                L.lpb_mirror_average(self.xn.data_ptr(), ax, *g.args, st)
            return self.physical(self.xn, beta, eta) - target

        l1, l2 = 1e-12, 1e12
        s_lo, s_hi = np.log(l1), np.log(l2)
        lam_last = self.lam_last
        sm = min(max(np.log(lam_last), s_lo), s_hi) if lam_last else 0.0
        f = stepped(float(np.exp(sm)))
        lm = float(np.exp(sm))
        s1 = s2 = sm
        f1 = f2 = None
        if f > 0:
            f1 = f
        else:
            f2 = f
        reach = 0.25
        while (f1 is None or f2 is None) and f != 0.0:
            if f1 is None:
                if s1 <= s_lo:
                    break
                s1 = max(s1 - reach, s_lo)
                sm = s1
            else:
                if s2 >= s_hi:
                    break
                s2 = min(s2 + reach, s_hi)
                sm = s2
            reach *= 4.0
            lm = float(np.exp(sm))
            f = stepped(lm)
            if f > 0:
                f1, s1 = f, sm
            else:
                f2, s2 = f, sm
        if f1 is not None and f2 is not None:
            side = 0
            for _ in range(60):
                if abs(f) <= VOLUME_RTOL * target or f2 == f1 or s2 - s1 <= 4e-16 * max(abs(s1), abs(s2), 1.0):
                    break
                sm = (s1 * f2 - s2 * f1) / (f2 - f1)
                if not s1 < sm < s2:
                    sm = 0.5 * (s1 + s2)
                lm = float(np.exp(sm))
                f = stepped(lm)
                if f > 0:
                    s1, f1 = sm, f
                    if side == 1:
                        f2 *= 0.5
                    side = 1
                else:
                    s2, f2 = sm, f
                    if side == -1:
                        f1 *= 0.5
                    side = -1
        self.lam_last = lm
        self.n_eval = n_eval[0]
        return self.xn, lm, f1 is not None and f2 is not None


def oc_bisection(volumes, target, l1=0.0, l2=1e9, tol=1e-3, width=31):
    """The reference's bisection (loadpath/benchmarks/reference.py:100-110):
        while (l2 - l1) / (l1 + l2) > tol: lmid = (l1 + l2) / 2; V(lmid) > target ? l1 = lmid : l2 = lmid
    with V evaluated in batches: `volumes(cands)` returns V at `width` multipliers at once.

    V is non-increasing in the multiplier (every cell's OC step is), so an evaluated
    V(lam) <= target decides every midpoint >= lam (l2 = lmid) and V(lam) > target every
    midpoint <= lam (l1 = lmid). The walk decides each midpoint from the evaluations so far and
    stops at the first one they leave open. While l1 = 0 a batch is the ladder l2 / 2^(2i+1) of
    the midpoints the walk visits next (exact halvings, so they equal the walk's own midpoints);
    otherwise it is the `width` midpoints of the next levels of the bisection tree below the
    open one, breadth first. Returns the last midpoint (the reference's lmid) and the
    number of batches."""
    below = math.inf    # smallest multiplier seen with V <= target
    above = -math.inf   # largest multiplier seen with V > target
    lmid = None
    passes = 0
    while (l2 - l1) / (l1 + l2) > tol:
        m = 0.5 * (l2 + l1)
        if m >= below:
            lmid = l2 = m
            continue
        if m <= above:
            lmid = l1 = m
            continue
        if l1 == 0.0:
            cands = [l2 * 2.0 ** -(2 * i + 1) for i in range(width)]
        else:
            nodes, cands = [(l1, l2)], []
            while len(cands) < width:
                nxt = []
                for a, b in nodes:
                    mm = 0.5 * (b + a)
                    cands.append(mm)
                    nxt += [(a, mm), (mm, b)]
                nodes = nxt
            cands = cands[:width]
        vols = volumes(cands)
        passes += 1
        for lam, v in zip(cands, vols):
            if v > target:
                above = max(above, lam)
            else:
                below = min(below, lam)
    return lmid, passes


class Top3dLoop:
    """top3d's SIMP loop with the density filter, on the device
    (loadpath/benchmarks/reference.py:74-117), solved by the device MG-PCG.

    dims: cells (even counts); fixed_grid: bool (3, nx+1, ny+1, nz+1); f_grid: float64 loads on
    the same grid, or a list of them (load cases: the objective is their equally weighted
    compliance sum, the cases solved as one block of right-hand sides); x0: optional initial
    density (cells), default volfrac everywhere.

    live_cells: solve the way loadpath's SIMP driver runs its multigrid (loadpath/simp.py:720-826,
    `_solve` / `_solve_mg`): once fewer than REDUCE_BELOW of the cells are alive (physical density
    above ALIVE, or touching a support or a load), only the alive cells 26-connected to a support
    keep their moduli; a load left on a dof without stiffness, or a reduced solve that fails, goes
    back to the full grid. Off (the default), every solve is on the full grid as top3d's direct
    solve. Either way a solve that takes more than slow_iters CG iterations (the driver's
    MG_SLOW_ITERS, loadpath/simp.py:85) is recorded in self.slow_solves as (iteration, CG count):
    the reference's driver then leaves the multigrid for a factorisation or AMG-CG, which this
    package does not build, so the answer is kept and the caller can see it. maxiter defaults to
    the driver's own cap (2000, loadpath/simp.py:182).

    shards: a LoadCaseShards over the ranks of a process group (one process per GPU): this
    rank solves only its cases, and one all-reduce per iteration sums the raw sensitivity and
    the compliance over the ranks before the filter, so every rank takes the same design step."""

    def __init__(self, dims, volfrac, rmin, fixed_grid, f_grid, nu=0.3, element=None, penal=3.0, emin=1e-9,
                 move=0.2, rtol=1e-8, dtype=np.float32, x0=None, coarse_cells=2000, maxiter=MG_MAXITER,
                 smoother="chebyshev", warm_start=True, block_cases=True, autotune=True, device="cuda",
                 live_cells=False, slow_iters=MG_SLOW_ITERS, shards=None):
        dims = tuple(int(d) for d in dims)
        if any(d % 2 for d in dims):
            raise ValueError("the device SIMP loop takes even cell counts (the multigrid pads odd ones)")
        self.dims = dims
        self.volfrac, self.penal, self.emin, self.move = float(volfrac), float(penal), float(emin), float(move)
        self.mesh = BoxMesh(dims)
        flat = np.asarray(fixed_grid, bool).reshape(3, -1)
        fixed = np.empty(self.mesh.n_dof, bool)
        for i in range(3):
            fixed[i::3] = flat[i]
        self.ge = GridElasticity(self.mesh, nu, fixed, rtol=rtol, maxiter=maxiter, coarse_cells=coarse_cells,
                                 dtype=dtype, element=element, smoother=smoother, device=device)
        g = self.ge.g0
        self.grid = g
        self.filter = DeviceFilter(g, rmin, pad=False)
        cases = f_grid if isinstance(f_grid, (list, tuple)) else [f_grid]
        self.shards = shards
        self.c_total = None
        mine = shards.mine() if shards is not None else range(len(cases))
        self.fs = [g.nodes_to_dev(np.asarray(cases[i], np.float64), torch.float64) for i in mine]
        self.f = self.fs[0] if self.fs else None
        self.x = g.cell_field(torch.float64)
        if x0 is None:
            g.set_cells(self.x, self.volfrac)
        else:
            g.cells_to_dev(np.asarray(x0, np.float64), torch.float64, out=self.x)
        self.xphys = self.x.clone()
        self._x_start = None     # restart(): the design the loop was constructed with
        self._x_stage = None     # step_host: the design in grid order on the device
        self.xnew = g.cell_field(torch.float64)
        self.e = g.cell_field(torch.float64)
        self.ce = g.cell_field(torch.float64)
        self.dc = g.cell_field(torch.float64)
        self.dcf = g.cell_field(torch.float64)
        self.u = None
        self.us = None           # the load cases' displacements (several cases)
        self.block_cases = block_cases   # False: the cases one solve after another
        self.autotune = autotune         # time the applies' launch geometry after the first build
        self.warm_start = warm_start
        self.ncell = dims[0] * dims[1] * dims[2]
        # [0] compliance, [1] change, [8 + k] case k's compliance
        self._scal = torch.zeros(8 + max(len(self.fs), 56), dtype=torch.float64, device=g.device)
        self._part = torch.zeros(31 * 592 + 1024, dtype=torch.float64, device=g.device)
        self._lam = torch.zeros(31, dtype=torch.float64, device=g.device)
        self._vols = torch.zeros(31, dtype=torch.float64, device=g.device)
        self._oc_state = torch.zeros(8, dtype=torch.float64, device=g.device)
        self.device_oc = True    # the bisection walked on the device (oc())
        self._oc_graph = None
        self.loop = 0
        self.history = []
        self.timing = None       # a list to collect per-phase CUDA events into, or None
        self.slow_iters = int(slow_iters)
        self.slow_solves = []    # (iteration, CG iterations) of solves above slow_iters
        self.live = None
        self.reduced = False     # the last solve ran on the live cells only
        if live_cells:
            held = np.asarray(fixed_grid, bool).reshape(g.node_shape).any(axis=0)
            loaded = np.zeros(g.node_shape[1:], bool)
            for fk in cases:
                loaded |= (np.asarray(fk).reshape(g.node_shape) != 0).any(axis=0)
            self.live = LiveCells(g, _cells_touching(held), _cells_touching(held | loaded))
            # the dead-load test looks at every case, so all ranks of a sharded loop decide alike
            self._loads_all = self.fs if shards is None else [
                g.nodes_to_dev(np.asarray(fk, np.float64), torch.float64) for fk in cases]
        lib().lpb_simp_law(self.e.data_ptr(), self.xphys.data_ptr(), self.penal, self.emin, *g.args, stream_handle())
        self._x_start = self.x.clone()

    def restart(self, x=None):
        """Put the loop back at a first iteration: the design x (a float64 device cell field in the
        padded layout; default: the design the loop was constructed with) becomes both the design
        and its physical density, as top3d starts (loadpath/benchmarks/reference.py:80-82,
        xPhys = x), the moduli are formed from it and the next solve starts from zero. Device work
        only: two cell-field copies and the SIMP law."""
        src = self._x_start if x is None else x
        L = lib()
        st = stream_handle()
        g = self.grid
        nb = src.numel() * 8
        for dst in (self.x, self.xphys):
            if dst.data_ptr() != src.data_ptr():
                L.lpb_memcpy_async(dst.data_ptr(), src.data_ptr(), nb, st)
        L.lpb_simp_law(self.e.data_ptr(), self.xphys.data_ptr(), self.penal, self.emin, *g.args, st)
        self.u = None
        self.us = None
        return self

    # ---- one iteration -------------------------------------------------------------------
    def _solve_cases(self):
        try:
            self._solve_cases_once()
        except RuntimeError:
            if not self.reduced:
                raise
            # the live cells hang on the rest by an edge or a corner, or a coarse level lost a
            # thin support: the full grid, void at Emin, holds it (loadpath/simp.py:815-822)
            self.reduced = False
            self.ge.set_moduli_device(self.e)
            self.u = self.us = None
            self._solve_cases_once()
        its = self.ge.last_iters
        worst = max(its) if isinstance(its, (list, tuple)) else its
        if worst > self.slow_iters:
            self.slow_solves.append((self.loop, int(worst)))

    def _solve_cases_once(self):
        if not self.fs:          # a rank with no load case of its own (more ranks than cases)
            self.u, self.us = None, []
            self.ge.last_iters = 0
            return
        if len(self.fs) == 1:
            x0 = self.u if (self.warm_start and self.u is not None) else None
            self.u = self.ge.solve_device(self.f, x0)
            self.us = [self.u]
        else:
            x0s = self.us if (self.warm_start and self.us is not None) else [None] * len(self.fs)
            if self.block_cases:
                self.us = self.ge.solve_block_device(self.fs, x0s)
            else:
                us, its = [], []
                for f, x0 in zip(self.fs, x0s):
                    us.append(self.ge.solve_device(f, x0))
                    its.append(self.ge.last_iters)
                self.us = us
                self.ge.last_iters = its
            self.u = self.us[0]

    def _set_moduli(self):
        if self.live is not None:
            self.reduced = self.ge.set_moduli_live(self.e, self.live, self.xphys, self._loads_all)
        else:
            self.ge.set_moduli_device(self.e)
        if self.autotune:
            from .tune import autotune

            autotune(self.ge)
            self.autotune = False

    def solve(self):
        self._set_moduli()
        self._solve_cases()
        return self.u

    def sensitivities(self):
        """ce, compliance (device scalar), dc = H (dc_raw / hs) (loadpath/benchmarks/reference.py:91-99);
        with several load cases the sums of the cases' compliances and raw sensitivities."""
        L = lib()
        st = stream_handle()
        g = self.grid
        for k, u in enumerate(self.us or ()):
            self.ge.strain_energy_device(u, out=self.ce)
            L.lpb_sensitivity(self.dc.data_ptr(), self.xphys.data_ptr(), self.ce.data_ptr(), self.e.data_ptr(),
                              self.penal, self.emin, 1.0, int(k > 0), self._part.data_ptr(),
                              self._scal[8 + k:].data_ptr(), *g.args, st)
        if self.shards is not None:
            # this rank's cases summed; one all-reduce gives every rank the totals, and every rank
            # then takes the same design step
            if not self.fs:
                self.dc.zero_()
            local = float(self._scal[8:8 + len(self.fs)].sum().item()) if self.fs else 0.0
            self.c_total = self.shards.reduce(self.dc, local)
        self.filter.apply(self.dcf, self.dc, hs_in=self.filter.hs)

    def oc(self):
        """top3d's bisection on the volume multiplier (loadpath/benchmarks/reference.py:100-110);
        the multipliers are evaluated on the device, 31 per pass over the cells. With device_oc
        (the default) the walk itself runs on the device too (lpb_oc_walk): with graphs the
        passes are one graph launch whose WHILE node repeats volumes + walk while candidates are
        open, so the step reads nothing back; the multiplier and the pass count reach the host
        with the step's scalars. Otherwise the host walks (oc_bisection), reading each pass."""
        L = lib()
        st = stream_handle()
        g = self.grid
        target = self.volfrac * self.ncell
        if not self.device_oc:
            def volumes(cands):
                self._lam.copy_(torch.tensor(cands, dtype=torch.float64))
                L.lpb_oc_volumes(self._vols.data_ptr(), self.x.data_ptr(), self.dcf.data_ptr(),
                                 self.filter.gv.data_ptr(), self.filter.gv.data_ptr(), self._lam.data_ptr(), 31,
                                 self.move, self._part.data_ptr(), *g.args, st)
                return self._vols.cpu().numpy()

            lmid, self.oc_passes = oc_bisection(volumes, target)
            L.lpb_oc_apply(self.xnew.data_ptr(), self.x.data_ptr(), self.dcf.data_ptr(), self.filter.gv.data_ptr(),
                           lmid, self.move, self._part.data_ptr(), self._scal[1:].data_ptr(), *g.args, st)
            self.lmid = lmid
            return
        state = self._oc_state
        L.lpb_oc_walk_init(state.data_ptr(), self._lam.data_ptr(), 1e9, target, OC_TOL, st)

        def body(handle):
            stb = stream_handle()
            L.lpb_oc_volumes(self._vols.data_ptr(), self.x.data_ptr(), self.dcf.data_ptr(), self.filter.gv.data_ptr(),
                             self.filter.gv.data_ptr(), self._lam.data_ptr(), 31, self.move, self._part.data_ptr(),
                             *g.args, stb)
            L.lpb_oc_walk(handle, state.data_ptr(), self._vols.data_ptr(), self._lam.data_ptr(), target, OC_TOL, stb)

        if self.ge.use_graphs:
            self._oc_graph = self.ge._graph(("oc_walk", self.x.data_ptr(), target, self.move), body, loop=True)
            self.ge._replay(self._oc_graph)
        else:
            self._oc_graph = None
            while True:
                body(0)
                if float(state[6].item()) != 0.0:
                    break
        L.lpb_oc_apply_at(self.xnew.data_ptr(), self.x.data_ptr(), self.dcf.data_ptr(), self.filter.gv.data_ptr(),
                          state[4:].data_ptr(), self.move, self._part.data_ptr(), self._scal[1:].data_ptr(), *g.args, st)
        # the multiplier and the pass count, read with the step's scalars
        L.lpb_memcpy_async(self._scal[2:].data_ptr(), state[4:].data_ptr(), 16, st)
        self.lmid = None

    def step(self):
        """One iteration; returns (compliance, change) as top3d reports them."""
        g = self.grid
        self.loop += 1
        t = self.timing
        if t is not None:
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            ev[0].record()
            self._set_moduli()
            ev[1].record()
            self._solve_cases()
            ev[2].record()
            self.sensitivities()
            ev[3].record()
            self.oc()
            ev[4].record()
            t.append(ev)
        else:
            self.solve()
            self.sensitivities()
            self.oc()
        # xphys = H xnew / hs, and the next iteration's moduli
        self.filter.apply(self.xphys, self.xnew, hs_out=self.filter.hs, e_out=self.e, penal=self.penal,
                          emin=self.emin)
        self.x, self.xnew = self.xnew, self.x
        vals = self._scal[:8 + len(self.fs)].cpu().numpy()
        if self.device_oc:
            self.lmid, self.oc_passes = float(vals[2]), int(vals[3])
            if self._oc_graph is not None and self.oc_passes > 1:
                add_launches(self._oc_graph[2] * (self.oc_passes - 1))   # the body ran once per pass
        if self.shards is not None:
            c, change = self.c_total, float(vals[1])
        else:
            c, change = float(vals[8:].sum()) if len(self.fs) > 1 else float(vals[8]), float(vals[1])
        self.history.append((c, change, self.ge.last_iters))
        return c, change

    def step_host(self, x_host, out_host, restart=False):
        """One iteration on a design held in host memory (pinned, so the copies are async):
        the design x (cells, float64) goes in, its physical densities H x / hs and moduli are
        formed on the device, and the updated design comes back in out_host. With restart the
        design is taken as its own physical density and the solve starts from zero (restart()).
        Returns (compliance, change)."""
        g = self.grid
        if self._x_stage is None:
            self._x_stage = torch.empty(g.cells, dtype=torch.float64, device=g.device)
        self._x_stage.copy_(x_host, non_blocking=True)
        if restart:
            g.set_cells(self.xphys, self._x_stage)
            self.restart(self.xphys)
        else:
            g.set_cells(self.x, self._x_stage)
            self.filter.apply(self.xphys, self.x, hs_out=self.filter.hs, e_out=self.e, penal=self.penal,
                              emin=self.emin)
        c, change = self.step()
        out_host.copy_(g.cell_grid(self.x), non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return c, change

    def run(self, maxit=200, on_iter=None):
        change = 1.0
        while change > 0.01 and self.loop < maxit:
            c, change = self.step()
            if on_iter is not None:
                on_iter(self.loop, c, change)
        return self

    def xphys_host(self):
        return self.grid.cells_to_host(self.xphys)
