"""Matrix-free geometric-multigrid PCG for K(E) u = f on a voxel grid, on one B200.

The call surface of loadpath's `mg.GridElasticity` (loadpath/mg.py:411-988):
`GridElasticity(mesh, nu, fixed, ...)`, `.set_moduli(e)`, `.solve_many(fs, x0s)`,
`.live_dofs()`, `.strain_energy(u)`, `.apply(u)`, `.last_iters`, `.strict`, `.levels`,
`.to_grid / .from_grid / .cell_grid`. All arithmetic runs in this package's CUDA kernels
(liblpb200.so); torch only allocates device memory and supplies the stream.

Hierarchy (built on the device at every set_moduli, as the reference builds it):
  level 0   "scaled"   E per cell times the unit-cube Ke (float64 for the outer CG, and a copy
                       in the V-cycle precision)
  level 1   "weights"  the eight child moduli per coarse cell with the eight fixed Galerkin
                       matrices M_k = P_k^T Ke P_k; cells touching held dofs as explicit patches
  level >=2 "explicit" Galerkin 24 x 24 per coarse cell, P^T K P over the eight children
  coarsest  dense D K D + (I - D), Cholesky-factored once per hierarchy and applied as a
            dense inverse (the reference factors the same operator with SuperLU on the host
            and round-trips every V-cycle; here it stays on the device)
Smoother: Chebyshev of `degree` on D^-1 A over [lmax/30, lmax] with lmax from 12 power
iterations x 1.3 (the reference's), or damped Jacobi (smoother="jacobi", omega).
Precision: the V-cycle in `dtype` (float32 = mixed, float64 = the plain FP64 path); the
outer CG, its operator, residual and inner products always in float64.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import fem
from ._lib import LpError, add_launches, launches, lib
from .grid import DevGrid, ptr, stream_handle, torch_dtype

__all__ = ["GridElasticity", "BoxMesh", "LMAX_SAFETY", "STALL", "prolong", "restrict"]


def prolong(c):
    """Trilinear prolongation of a (3, n0, n1, n2) node field to (3, 2n0-1, 2n1-1, 2n2-1)
    (loadpath/mg.py:84-108), on the device."""
    from .mgops import prolong as _prolong

    return _prolong(c)


def restrict(f):
    """Full-weighting restriction, the transpose of prolong (loadpath/mg.py:111-132), on the
    device."""
    from .mgops import restrict as _restrict

    return _restrict(f)

LMAX_SAFETY = 1.3          # loadpath/mg.py:81
STALL = 100                # loadpath/mg.py:930
DENSE_COARSE_MAX = 12_000  # dofs of the coarsest level solved by the dense factor (1.2 GB)
# off-pattern weight (relative to a cell's largest corner-parity entry) above which an explicit
# cell is applied from its node-basis matrix; float32 storage leaves ~1e-7 on pattern cells
MODAL_TOL = 1e-5


class BoxMesh:
    """The HexMesh fields GridElasticity reads, for a full box of unit cells
    (loadpath/fem.py:317-374: elements and nodes in C order, dof = 3 node + component)."""

    def __init__(self, dims, pitch=1.0):
        self.dims = tuple(int(d) for d in dims)
        nx, ny, nz = self.dims
        self.pitch = float(pitch)
        self.elem_ijk = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"),
                                 -1).reshape(-1, 3)
        self.node_ijk = np.stack(np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1),
                                             indexing="ij"), -1).reshape(-1, 3)
        self.n_nodes = len(self.node_ijk)
        self.n_dof = 3 * self.n_nodes

    @property
    def n_elem(self):
        return len(self.elem_ijk)


class FineApplyProbe:
    """CUDA events around every fine-level tiled apply while set (bench.py's roofline).

    The events are recorded as external event nodes, so inside a CUDA graph every replay
    records them again; the solver hands the pairs of a replay back (harvest) once that replay
    is known to be complete."""

    def __init__(self, n=512):
        self.pending = []        # eager launches, read at summary()
        self.capture = None      # pairs recorded while a graph is being captured
        # f32 / f64: the plain applies; f32c1..f32c3: the float32 applies that form a Chebyshev
        # update as they store (modes 1..3 of lpb_apply_fine_cheb_f32)
        self.totals = {f"{k}_{v}": (0.0 if v == "ms" else 0) for k in ("f32", "f64", "f32c1", "f32c2", "f32c3")
                       for v in ("ms", "count")}
        self.pool = []
        self._grow(n)

    def _grow(self, n):
        # torch creates a CUDA event at its first record: record each once here, outside any
        # capture, so the raw handles exist
        for _ in range(n):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            b.record()
            self.pool.append((a, b))

    def take(self):
        if not self.pool:
            if torch.cuda.is_current_stream_capturing():
                raise RuntimeError("fine-apply probe: event pool exhausted during a graph capture")
            self._grow(256)
        return self.pool.pop()

    def harvest(self, pairs, recycle=False):
        for dt, a, b in pairs:
            k = dt if isinstance(dt, str) else ("f32" if dt == torch.float32 else "f64")
            self.totals[k + "_ms"] += a.elapsed_time(b)
            self.totals[k + "_count"] += 1
            if recycle:
                self.pool.append((a, b))

    def summary(self):
        torch.cuda.synchronize()
        self.harvest(self.pending, recycle=True)
        self.pending = []
        return dict(self.totals)


_PROBE = [None]


def set_probe(p):
    _PROBE[0] = p


class DevLevel:
    """One level on the device (loadpath/mg.py:174-199)."""

    def __init__(self, kind, grid: DevGrid, dtype: torch.dtype):
        self.kind = kind
        self.grid = grid
        self.dtype = dtype
        self.e = self.ke = self.kmodal = None
        self.err = None          # device int the tiled fine kernel flags a given-up wait in
        self.w = self.mcat = self.patch_id = self.patch_k = None
        self.npatch = 0
        self.k = None
        self.kp = None           # explicit: packed symmetric (300, cells)
        self.km = None           # explicit, plain hierarchy: corner-parity pattern entries (150, cells)
        self.glist = self.gcount = self.kpc = None   # ...and the cells applied from node-basis entries
        self.ft = None           # explicit: (24, cells) scratch of the cell pass
        self.g1 = None           # weights: 279 corner-parity coefficients (host)
        self.wc = None           # weights: Walsh coefficients (cpz/4, ny, nx, 4, 8)
        self.pbox = None         # weights: node box of the patch cells (host, 6 ints)
        self.mask = None
        self.dinv = None
        self.coef = None         # device: lmax and the Chebyshev coefficients (lpb_cheb_coef)
        self.n_active = 0

    @property
    def lmax(self):
        """The smoother's upper eigenvalue bound (read from the device)."""
        return None if self.coef is None else float(self.coef[0].item())

    @property
    def dims(self):
        return self.grid.cells

    @property
    def node_shape(self):
        return self.grid.node_shape

    def _sfx(self):
        return "f32" if self.dtype == torch.float32 else "f64"

    def apply(self, out, u, mask_in=False, fine_kernel=True):
        """out = m K (m u) + (1 - m) u; the tiled kernel on the fine level when u is known to
        be zero on masked dofs (mask_in False), the general kernel otherwise."""
        L = lib()
        g = self.grid
        st = stream_handle()
        sfx = self._sfx()
        if self.kind == "scaled":
            if fine_kernel and not mask_in:
                probe = _PROBE[0]
                if probe is not None:
                    a, b = probe.take()
                    L.lpb_event_record(a.cuda_event, st)
                getattr(L, f"lpb_apply_fine_{sfx}")(out.data_ptr(), u.data_ptr(), self.e.data_ptr(),
                                                     self.mask.data_ptr(), self.kmodal.ctypes.data,
                                                     self.err.data_ptr(), *g.args, st)
                if probe is not None:
                    L.lpb_event_record(b.cuda_event, st)
                    if probe.capture is not None:
                        probe.capture.append((self.dtype, a, b))
                    else:
                        probe.pending.append((self.dtype, a, b))
            else:
                getattr(L, f"lpb_apply_scaled_{sfx}")(out.data_ptr(), u.data_ptr(), self.e.data_ptr(),
                                                       self.mask.data_ptr(), self.ke.data_ptr(), *g.args,
                                                       int(mask_in), 1, st)
        elif self.kind == "weights":
            if fine_kernel and not mask_in:
                getattr(L, f"lpb_apply_weights_tma_{sfx}")(out.data_ptr(), u.data_ptr(), self.wc.data_ptr(),
                                                            ptr(self.patch_id) if self.npatch else None,
                                                            ptr(self.patch_k) if self.npatch else None,
                                                            self.mask.data_ptr(), self.g1.ctypes.data,
                                                            self.pbox.ctypes.data, self.err.data_ptr(), *g.args, st)
            else:
                getattr(L, f"lpb_apply_weights_{sfx}")(out.data_ptr(), u.data_ptr(), self.w.data_ptr(),
                                                        self.mcat.data_ptr(), ptr(self.patch_id),
                                                        ptr(self.patch_k), self.mask.data_ptr(), *g.args,
                                                        int(mask_in), 1, st)
        else:
            if fine_kernel and not mask_in and self.km is not None:
                L.lpb_apply_explicit_modal_f32(out.data_ptr(), u.data_ptr(), self.km.data_ptr(), self.kpc.data_ptr(),
                                               self.glist.data_ptr(), self.gcount.data_ptr(), self.ft.data_ptr(),
                                               self.mask.data_ptr(), *g.args, st)
            elif fine_kernel and not mask_in:
                getattr(L, f"lpb_apply_explicit_sym_{sfx}")(out.data_ptr(), u.data_ptr(), self.kp.data_ptr(),
                                                             self.ft.data_ptr(), self.mask.data_ptr(), *g.args, st)
            else:
                getattr(L, f"lpb_apply_explicit_{sfx}")(out.data_ptr(), u.data_ptr(), self.k.data_ptr(),
                                                         self.mask.data_ptr(), *g.args, int(mask_in), 1, st)
        return out

    def apply_dot(self, out, u, part, dot):
        """out = m K u on the float64 fine level (u zero on masked dofs) and *dot = u . out, in one
        pass (the PCG's A p and p . A p)."""
        L = lib()
        g = self.grid
        st = stream_handle()
        probe = _PROBE[0]
        if probe is not None:
            a, b = probe.take()
            L.lpb_event_record(a.cuda_event, st)
        L.lpb_apply_fine_dot_f64(out.data_ptr(), u.data_ptr(), self.e.data_ptr(), self.mask.data_ptr(),
                                 self.kmodal.ctypes.data, self.err.data_ptr(), part.data_ptr(), part.numel(),
                                 dot.data_ptr(), *g.args, st)
        if probe is not None:
            L.lpb_event_record(b.cuda_event, st)
            if probe.capture is not None:
                probe.capture.append((self.dtype, a, b))
            else:
                probe.pending.append((self.dtype, a, b))
        return out

    def diagonal(self, d):
        L = lib()
        g = self.grid
        st = stream_handle()
        sfx = self._sfx()
        if self.kind == "scaled":
            raise RuntimeError("the scaled level's diagonal is built from its float64 moduli")
        if self.kind == "weights":
            getattr(L, f"lpb_diag_weights_{sfx}")(d.data_ptr(), self.w.data_ptr(), self.mcat.data_ptr(),
                                                   ptr(self.patch_id), ptr(self.patch_k), *g.args, st)
        else:
            getattr(L, f"lpb_diag_explicit_{sfx}")(d.data_ptr(), self.k.data_ptr(), *g.args, st)
        return d


class GridElasticity:
    """Matrix-free multigrid-preconditioned CG on the device (loadpath/mg.py:411-988).

    mesh: any object with elem_ijk (ne, 3), node_ijk (nn, 3) and pitch (a loadpath
    HexMesh or BoxMesh); nu: Poisson's ratio; fixed: bool per mesh dof. springs/lowrank are
    not supported on this path (the benchmark problems have none). device: a CUDA device, or any
    other name ("cpu", "auto", None) for the default CUDA device."""

    def __init__(self, mesh, nu, fixed, springs=None, rtol=1e-6, maxiter=500, coarse_cells=2000, degree=2,
                 dtype=np.float32, lu_max_dofs=60_000, device=None, lowrank=None, smoother="chebyshev",
                 omega=0.6, element=None):
        if springs is not None or lowrank is not None:
            raise NotImplementedError("springs and low-rank extra terms are not on the B200 path")
        if not torch.cuda.is_available():
            raise RuntimeError("loadpath_b200 needs a CUDA device (it has no CPU fallback)")
        lib()  # fail loudly here if the extension is missing
        self.mesh = mesh
        self.nu = nu
        self.rtol = rtol
        self.maxiter = maxiter
        self.coarse_cells = int(coarse_cells)
        self.degree = int(degree)
        self.dtype = np.dtype(dtype)
        self.tdtype = torch_dtype(self.dtype)
        self.lu_max_dofs = int(lu_max_dofs)
        self.smoother = smoother
        self.omega = float(omega)
        # every solve of this package runs on a CUDA device: a caller's "cpu" (loadpath's build
        # simulation asks for it, loadpath/buildsim.py:612) selects the default one as "auto" does
        dev = torch.device(device) if isinstance(device, (str, torch.device)) and str(device).startswith("cuda") \
            else torch.device("cuda")
        self.device = dev
        cells = np.asarray(mesh.elem_ijk).max(axis=0) + 1
        cells = cells + cells % 2
        self.cells = tuple(int(c) for c in cells)
        self.node_shape = tuple(int(c) + 1 for c in cells)
        self.nn = int(np.prod(self.node_shape))
        self.node_flat = np.ravel_multi_index(tuple(np.asarray(mesh.node_ijk).T), self.node_shape)
        self.elem_ijk = np.asarray(mesh.elem_ijk)
        self.element = element or fem.hex8_element()
        self.ke = fem.hex8_ke(nu, self.element) * mesh.pitch
        fixed = np.asarray(fixed, bool)
        fg = np.zeros((3, self.nn), bool)
        for i in range(3):
            fg[i, self.node_flat] = fixed[i::3]
        self.fixed_grid = fg.reshape((3,) + self.node_shape)
        self.g0 = DevGrid(self.cells, self.device)
        self.fixed_bits = self.g0.bits_to_dev(self.fixed_grid)
        km = np.zeros(45)
        n = lib().lpb_modal_ke(self.ke.ctypes.data, km.ctypes.data)
        if n != 45:
            raise LpError("the element matrix is not in the corner-parity pattern the fine kernel uses")
        # host array: the fine kernel takes the coefficients as launch parameters
        self.kmodal = np.ascontiguousarray(km, np.float64)
        self._err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.ke64 = torch.tensor(self.ke.reshape(-1), dtype=torch.float64, device=self.device)
        self.ke32 = self.ke64.float()
        # level 1: M_k = P_k^T Ke P_k (8 x 576); level 2 from level 1: N_(k,q) = P_k^T M_q P_k
        # (64 x 576, index 8 k + q); formed by the library, so the C-ABI solver handle
        # (lpb_mg_create) shares their bits
        self._mcat = np.zeros((8, 576))
        self._nkq = np.zeros((64, 576))
        lib().lpb_level1_products(np.ascontiguousarray(self.ke).ctypes.data, self._mcat.ctypes.data,
                                  self._nkq.ctypes.data)
        self._nkq_dev = {}
        g1 = np.zeros(279)
        if lib().lpb_modal_g1(np.ascontiguousarray(self.ke).ctypes.data, g1.ctypes.data) != 279:
            raise LpError("the level-1 Galerkin matrices are not in the corner-parity pattern of the kernel")
        self.g1 = g1
        self.levels = []
        self.strict = False
        self.last_iters = 0
        self._lmax_init = {}
        self._coarse = None
        self._plan = None
        self._patch_plan = None
        self._mcat_dev = {}
        self._scal = torch.zeros(64, dtype=torch.float64, device=self.device)
        # device scalars of a build: [0] cells with E > 0, [d] active cells of level d, [31]
        # patch-flag mismatches, [40 + d] largest diagonal of level d; power-iteration dots
        # (32 per level) and Chebyshev coefficients (16 per level)
        self._chk = torch.zeros(64, dtype=torch.float64, device=self.device)
        self._chk_host = torch.zeros(32, dtype=torch.float64, pin_memory=True)
        self._info_host = torch.zeros(2, dtype=torch.int32, pin_memory=True)
        self._pw = torch.zeros(32 * 32, dtype=torch.float64, device=self.device)
        self._coef = torch.zeros(16 * 32, dtype=torch.float64, device=self.device)
        # reduction partials: the vector kernels' blocks, and one per block of the fine float64
        # apply with p . A p (15 x 15 node columns by z segments of at least two chunks)
        g0 = self.g0
        fine_blocks = ((g0.NX + 14) // 15) * ((g0.NY + 14) // 15) * (g0.pz // 4)
        self._part = torch.zeros(max(lib().lpb_reduce_blocks() * 2, 2048, fine_blocks), dtype=torch.float64,
                                 device=self.device)
        self._host = torch.zeros(8, dtype=torch.float64, pin_memory=True)
        # the device-side CG loop: its stopping test's state (iterations, status) and its copy
        self._loop_state = torch.zeros(2, dtype=torch.int64, device=self.device)
        self._loop_out = torch.zeros(2, dtype=torch.int64, pin_memory=True)
        self.device_loop = True  # graphed solves test convergence on the device (no host read per iteration)
        self._work = {}
        self._e_dev = None
        # CUDA graphs for the CG iteration (captured once per solve)
        self.use_graphs = True
        self._gcache = {}
        self._gen = 0            # bumped whenever a work buffer is (re)allocated
        self._cap_stream = torch.cuda.Stream(device=self.device)
        self._side = torch.cuda.Stream(device=self.device, priority=-1)   # coarsest factorisation
        self._ev_fork = torch.cuda.Event()
        self._ev_join = torch.cuda.Event()
        self._pw_stream = torch.cuda.Stream(device=self.device)             # coarse power iterations
        self._ev_pw_fork = torch.cuda.Event()
        self._ev_pw_join = torch.cuda.Event()
        self._part_pw = torch.zeros(lib().lpb_reduce_blocks() * 2, dtype=torch.float64, device=self.device)
        # the fine two levels' power iterations: on the working stream, or (a planned rebuild) on a
        # stream of their own as soon as level 1 is built, beside the coarser levels' Galerkin
        # products; their own reduction scratch either way
        self._pw01_stream = torch.cuda.Stream(device=self.device)
        self._ev_pw01_fork = torch.cuda.Event()
        self._ev_pw01_join = torch.cuda.Event()
        self._part_pw01 = torch.zeros(lib().lpb_reduce_blocks() * 2, dtype=torch.float64, device=self.device)
        self._pw01_early = False
        self._joined = True

    # --- layout conversion (loadpath/mg.py:495-511) -----------------------------------
    def to_grid(self, v, dtype=np.float64):
        out = np.zeros((3, self.nn), dtype)
        for i in range(3):
            out[i, self.node_flat] = v[i::3]
        return out.reshape((3,) + self.node_shape)

    def from_grid(self, g):
        flat = np.asarray(g).reshape(3, -1)
        out = np.empty(3 * len(self.node_flat))
        for i in range(3):
            out[i::3] = flat[i, self.node_flat]
        return out

    def cell_grid(self, e, dtype=np.float64):
        g = np.zeros(self.cells, dtype)
        g[tuple(self.elem_ijk.T)] = e
        return g

    # --- device work buffers -----------------------------------------------------------
    def _flat_buf(self, key, n, dtype):
        t = self._work.get(key)
        if t is None or t.dtype != dtype or t.numel() < n:
            t = torch.zeros(max(n, 1), dtype=dtype, device=self.device)
            self._work[key] = t
            self._gen += 1
        return t

    def _buf(self, key, grid: DevGrid, dtype):
        t = self._work.get(key)
        if t is None or t.dtype != dtype or tuple(t.shape) != (3, grid.pz // 4, grid.NY, grid.NX, 4):
            t = grid.node_field(dtype)
            self._work[key] = t
            self._gen += 1
        return t

    # --- hierarchy (loadpath/mg.py:515-754) --------------------------------------------
    def set_moduli(self, e):
        """Per-element moduli in mesh order (host array): rebuild every level."""
        e = np.asarray(e, np.float64)
        self._e_host = e
        e_dev = self.g0.cells_to_dev(self.cell_grid(e), torch.float64)
        self.set_moduli_device(e_dev)

    def _tbuf(self, key, shape, dtype, fill=0):
        """A persistent device buffer (stable address across rebuilds), filled when created."""
        t = self._work.get(key)
        if t is None or t.dtype != dtype or tuple(t.shape) != tuple(shape):
            t = torch.full(tuple(shape), fill, dtype=dtype, device=self.device)
            self._work[key] = t
            self._gen += 1
        return t

    def set_moduli_device(self, e_dev: torch.Tensor):
        """Moduli already on the device as a float64 cell field of the fine level.

        The host decisions of a build (how many levels, which level-1 cells carry patch
        matrices, the coarsest factor's success) depend on the design only through which cells
        are non-void, so the first build makes them with host reads and records them; a
        rebuild with the same record runs without any host read and checks every decision in
        one copy at the end (active-cell counts, patch flags, factor status), redoing the
        build from scratch when one differs."""
        self._e_dev = e_dev
        plan = self._plan
        if plan is not None and plan["strict"] == self.strict and plan["shape"] == tuple(e_dev.shape):
            if self._build(e_dev, plan):
                return
        self._plan = None
        self._build(e_dev, None)

    def _build(self, e_dev, plan):
        """One hierarchy build (loadpath/mg.py:515-591). plan None: discovery (host reads,
        records a plan). Returns False when a planned build's checks fail."""
        L = lib()
        st = stream_handle()
        g0 = self.g0
        dt = self.tdtype
        chk = self._chk
        part = self._part
        # power iterations launched early by a build before this one are done before anything of
        # this one is written
        torch.cuda.current_stream().wait_event(self._ev_pw01_join)
        self._pw01_early = False
        if plan is None:
            self._gen += 1       # captured graphs may hold launch parameters of the last structure
        l0 = DevLevel("scaled", g0, torch.float64)
        # the moduli in a buffer of this solver's own, so captured graphs can keep its address
        l0.e = self._tbuf("e0_64", e_dev.shape, torch.float64)
        if e_dev.data_ptr() != l0.e.data_ptr():
            L.lpb_memcpy_async(l0.e.data_ptr(), e_dev.data_ptr(), 8 * e_dev.numel(), st)
        e_dev = self._e_dev = l0.e
        l0.ke = self.ke64
        l0.kmodal = self.kmodal
        l0.err = self._err
        d0 = self._buf("diag0", g0, torch.float64)
        L.lpb_diag_scaled_f64(d0.data_ptr(), e_dev.data_ptr(), self.ke64.data_ptr(), *g0.args, st)
        l0.mask = self._tbuf("mask0", g0.mask_field().shape, torch.uint8)
        l0.dinv = self._buf("dinv0_64", g0, torch.float64)
        dinv32 = self._buf("dinv0_32", g0, torch.float32) if dt == torch.float32 else None
        L.lpb_masks(l0.mask.data_ptr(), l0.dinv.data_ptr(), ptr(dinv32), d0.data_ptr(), self.fixed_bits.data_ptr(),
                    None, *g0.args, 1e-300, 1e-300, None, st)
        levels = [l0]
        if dt == torch.float32:
            s = DevLevel("scaled", g0, torch.float32)
            s.e = self._tbuf("e0_32", e_dev.shape, torch.float32)
            L.lpb_cast_f64_f32(s.e.data_ptr(), e_dev.data_ptr(), g0.n_cell_field, st)
            s.ke = self.ke32
            s.kmodal = self.kmodal
            s.err = self._err
            s.mask = l0.mask
            s.dinv = dinv32
            l0s = s
        else:
            l0s = l0
        L.lpb_count_positive_f64(e_dev.data_ptr(), e_dev.numel(), part.data_ptr(), chk[0:].data_ptr(), st)
        counts = [None if plan else int(chk[0].item())]
        fine = l0
        depth = 0
        held = None
        if self.strict:
            held = self._tbuf("held0", l0.mask.shape, torch.uint8)
            L.lpb_held0(held.data_ptr(), l0.mask.data_ptr(), self.fixed_bits.data_ptr(), held.numel(), st)

        def more():
            if plan is not None:
                return depth < plan["depth"]
            return counts[-1] > self.coarse_cells and min(fine.dims) >= 2

        while more():
            depth += 1
            if depth >= 30:
                raise RuntimeError("hierarchy deeper than 30 levels")
            coarse = self._coarsen(fine, depth, plan)
            gc = coarse.grid
            d = self._buf(f"diag{depth}", gc, torch.float64)
            coarse.diagonal(d)
            L.lpb_max_f64(d.data_ptr(), d.numel(), part.data_ptr(), chk[40 + depth:].data_ptr(), st)
            held_c = kept = None
            if self.strict:
                held_c = self._tbuf(f"held{depth}", gc.mask_field().shape, torch.uint8)
                kept = self._buf(f"kept{depth}", gc, torch.float32)
                L.lpb_strict_held_kept(held_c.data_ptr(), kept.data_ptr(), held.data_ptr(), fine.mask.data_ptr(),
                                       *fine.grid.args, *gc.args, st)
                held = held_c
            coarse.mask = self._tbuf(f"mask{depth}", gc.mask_field().shape, torch.uint8)
            coarse.dinv = self._buf(f"dinv{depth}", gc, dt)
            d64 = coarse.dinv if dt == torch.float64 else None
            d32 = coarse.dinv if dt == torch.float32 else None
            # live = d > 1e-12 max(dmax, 1e-300), dmax read on the device
            L.lpb_masks(coarse.mask.data_ptr(), ptr(d64), ptr(d32), d.data_ptr(), ptr(held_c), ptr(kept), *gc.args,
                        1e-12, 1e-12, chk[40 + depth:].data_ptr(), st)
            self._count_active(coarse, chk[depth:])
            counts.append(None if plan else int(chk[depth].item()))
            levels.append(coarse)
            fine = coarse
            if plan is not None and depth == 1:
                self.levels = levels
                self._l0s = l0s
                self._lmax_fine_early(plan["depth"] + 1)
        self.levels = levels
        self._l0s = l0s
        info = self._build_coarse(levels[-1])
        self._all_lmax(len(levels))
        self._join_coarse()
        if plan is None:
            if info is not None:
                st_pivot, st_barrier = (int(v) for v in info.cpu().numpy())
                if st_barrier:
                    raise RuntimeError("coarsest-level factorisation: a grid-barrier wait gave up")
                if st_pivot:
                    return self._singular()
            self._plan = {"strict": self.strict, "shape": tuple(e_dev.shape), "depth": depth,
                          "counts": counts, "patch": self._patch_plan}
            return True
        # one copy back: every count the plan's decisions rest on, the patch-flag mismatches
        # and the coarse factor's status
        hc = self._chk_host
        L.lpb_memcpy_async(hc.data_ptr(), chk.data_ptr(), 8 * 32, st)
        if info is not None:
            L.lpb_memcpy_async(self._info_host.data_ptr(), info.data_ptr(), 8, st)
        torch.cuda.current_stream().synchronize()
        # the same decisions as discovery's: coarsen while the active cells exceed
        # coarse_cells, and the same level-1 patch cells
        n_act = [int(hc[i]) for i in range(depth + 1)]
        if any(c <= self.coarse_cells for c in n_act[:depth]):
            return False
        if n_act[depth] > self.coarse_cells and min(levels[-1].dims) >= 2:
            return False
        if depth >= 1 and int(hc[31]) != 0:
            return False
        if info is not None:
            if int(self._info_host[1]) != 0:
                raise RuntimeError("coarsest-level factorisation: a grid-barrier wait gave up")
            if int(self._info_host[0]) != 0:
                return self._singular()
        return True

    def _singular(self):
        """The coarsest factor failed (loadpath/mg.py:586-591): take the strict hierarchy."""
        if self.strict:
            raise RuntimeError("coarsest-level factor is singular in the strict hierarchy")
        self.strict = True
        self._plan = None
        self._build(self._e_dev, None)
        return True

    def _count_active(self, lv, out):
        """Active cells of a coarse level into a device scalar (loadpath/mg.py:593-599)."""
        L = lib()
        g = lv.grid
        sfx = "f32" if lv.dtype == torch.float32 else "f64"
        if lv.kind == "weights":
            getattr(L, f"lpb_count_active_weights_{sfx}")(lv.w.data_ptr(), ptr(lv.patch_id) if lv.npatch else None,
                                                          *g.args, self._part.data_ptr(), out.data_ptr(),
                                                          stream_handle())
        else:
            getattr(L, f"lpb_count_active_explicit_{sfx}")(lv.k.data_ptr(), *g.args, self._part.data_ptr(),
                                                           out.data_ptr(), stream_handle())

    def _coarsen(self, fine: DevLevel, depth: int, plan) -> DevLevel:
        """Galerkin coarse level (loadpath/mg.py:601-677)."""
        L = lib()
        st = stream_handle()
        dt = self.tdtype
        sfx = "f32" if dt == torch.float32 else "f64"
        nx, ny, nz = fine.dims
        half = (nx // 2, ny // 2, nz // 2)
        cdims = tuple(h + h % 2 if h > 1 else h for h in half)
        gc = DevGrid(cdims, self.device)
        gf = fine.grid
        ncp = gc.nx * gc.ny * gc.cpz
        if depth == 1:
            lv = DevLevel("weights", gc, dt)
            lv.w = self._tbuf("w1", (8, gc.cpz // 4, gc.ny, gc.nx, 4), dt)
            getattr(L, f"lpb_weights_from_e_f64_{sfx}")(lv.w.data_ptr(), fine.e.data_ptr(), *gf.args, *gc.args, st)
            lv.mcat = self._mcat_dev.get(dt)
            if lv.mcat is None:
                lv.mcat = torch.tensor(self._mcat.reshape(-1), dtype=dt, device=self.device)
                self._mcat_dev[dt] = lv.mcat
            flag = self._tbuf("pflag_new" if plan else "pflag", (gc.cpz // 4, gc.ny, gc.nx, 4), torch.uint8)
            L.lpb_patch_flags(flag.data_ptr(), fine.e.data_ptr(), fine.mask.data_ptr(), *gf.args, *gc.args, st)
            if plan is not None:
                pp = plan["patch"]
                L.lpb_count_ne_u8(flag.data_ptr(), self._work["pflag"].data_ptr(), flag.numel(),
                                  self._part.data_ptr(), self._chk[31:].data_ptr(), st)
                pcells, lv.npatch, lv.pbox = pp["cells"], pp["n"], pp["box"]
            else:
                pcells = torch.nonzero(flag.reshape(-1)).reshape(-1).to(torch.int64).contiguous()
                lv.npatch = int(pcells.numel())
                lv.pbox = np.zeros(6, np.int32)
                if lv.npatch:
                    col = pcells // 4          # cell index -> (x, y, z), chunked layout
                    x = col % gc.nx
                    y = (col // gc.nx) % gc.ny
                    z = 4 * (col // (gc.nx * gc.ny)) + pcells % 4
                    lo = torch.stack([x.min(), y.min(), z.min()]).cpu().numpy()
                    hi = torch.stack([x.max(), y.max(), z.max()]).cpu().numpy() + 2   # nodes of the last cell
                    lv.pbox[:3] = lo
                    lv.pbox[3:] = hi - lo
                self._patch_plan = {"cells": pcells, "n": lv.npatch, "box": lv.pbox}
            lv.patch_id = self._tbuf("patch_id", (gc.cpz // 4, gc.ny, gc.nx, 4), torch.int32, -1)
            if plan is None:
                lv.patch_id.fill_(-1)
            if lv.npatch:
                lv.patch_k = self._tbuf("patch_k", (lv.npatch, 576), dt)
                getattr(L, f"lpb_patch_matrices_{sfx}")(lv.patch_k.data_ptr(), lv.w.data_ptr(), lv.patch_id.data_ptr(),
                                                        pcells.data_ptr(), lv.npatch, fine.e.data_ptr(),
                                                        self.ke64.data_ptr(), fine.mask.data_ptr(), *gf.args,
                                                        *gc.args, st)
            else:
                lv.patch_k = None
            lv.patch_cells = pcells
            lv.g1 = self.g1
            # the Walsh coefficients of each cell's child moduli, chunked for the march kernel
            lv.wc = self._tbuf("wc1", (gc.cpz // 4, gc.ny, gc.nx, 4, 8), dt)
            getattr(L, f"lpb_walsh_chunks_{sfx}")(lv.wc.data_ptr(), lv.w.data_ptr(), *gc.args, st)
            lv.err = self._err
            return lv
        lv = DevLevel("explicit", gc, dt)
        lv.k = self._tbuf(f"k{depth}", (ncp, 576), dt)
        if fine.kind == "weights" and not self.strict:
            # the 64 products N_(k,q) = P_k^T M_q P_k: each coarse entry is a 64-term sum
            nkq = self._nkq_dev.get(dt)
            if nkq is None:
                nkq = torch.tensor(self._nkq, dtype=dt, device=self.device)
                self._nkq_dev[dt] = nkq
            getattr(L, f"lpb_galerkin_w2_{sfx}")(lv.k.data_ptr(), fine.w.data_ptr(), nkq.data_ptr(),
                                                 ptr(fine.patch_id) if fine.npatch else None,
                                                 ptr(fine.patch_k) if fine.npatch else None, *gf.args, *gc.args, st)
        elif fine.kind == "weights":
            getattr(L, f"lpb_galerkin_explicit_{sfx}")(lv.k.data_ptr(), 1, fine.w.data_ptr(), fine.mcat.data_ptr(),
                                                       ptr(fine.patch_id), ptr(fine.patch_k), None,
                                                       fine.mask.data_ptr(), int(self.strict), *gf.args, *gc.args, st)
        else:
            getattr(L, f"lpb_galerkin_explicit_{sfx}")(lv.k.data_ptr(), 2, None, None, None, None, fine.k.data_ptr(),
                                                       fine.mask.data_ptr(), int(self.strict), *gf.args, *gc.args, st)
        lv.ft = self._tbuf(f"ft{depth}", (24, ncp), dt)
        lv.km = lv.kp = None
        if dt != torch.float32 or self.strict:
            lv.kp = self._tbuf(f"kp{depth}", (300, ncp), dt)
            getattr(L, f"lpb_pack_sym_{sfx}")(lv.kp.data_ptr(), lv.k.data_ptr(), ncp, st)
        else:
            # the plain hierarchy's cell matrices keep the corner-parity pattern: half the bytes
            lv.km = self._tbuf(f"km{depth}", (150, ncp), dt)
            lv.glist = self._tbuf(f"glist{depth}", (ncp,), torch.int32)
            lv.gcount = self._tbuf(f"gcount{depth}", (1,), torch.int32)
            lv.kpc = self._tbuf(f"kpc{depth}", (ncp, 300), dt)
            L.lpb_pack_modal_f32(lv.km.data_ptr(), lv.glist.data_ptr(), lv.gcount.data_ptr(), lv.kpc.data_ptr(),
                                 lv.k.data_ptr(), ncp, MODAL_TOL, st)
        return lv

    def _build_coarse(self, lv: DevLevel):
        """Direct solve of the coarsest level (loadpath/mg.py:708-754): its operator as a band,
        a tiled band Cholesky and the dense inverse from it, all on the device, once per
        hierarchy; the V-cycle then applies the inverse with one GEMV. Returns the device status
        pair (0 0 when fine; [0]: a non-positive pivot, the operator is singular; [1]: a
        grid-barrier wait of the factorisation gave up), or None when there is no coarse solve."""
        self._coarse = None
        if lv is self.levels[0]:
            return None
        g = lv.grid
        n = 3 * g.NX * g.NY * g.NZ
        if n > DENSE_COARSE_MAX:
            return None
        L = lib()
        st = stream_handle()
        dt = self.tdtype
        sfx = "f32" if dt == torch.float32 else "f64"
        dims = np.zeros(4, np.int64)
        ntiles = int(L.lpb_band_dims(g.nx, g.ny, g.nz, dims.ctypes.data))
        nt = int(dims[1])
        npad = 32 * nt
        t = self._tbuf("band_t", (ntiles * 1024,), torch.float64)
        if lv.kind == "weights":
            getattr(L, f"lpb_coarse_band_{sfx}")(t.data_ptr(), 1, lv.w.data_ptr(), lv.mcat.data_ptr(),
                                                 ptr(lv.patch_id), ptr(lv.patch_k), None, lv.mask.data_ptr(),
                                                 *g.args, st)
        else:
            getattr(L, f"lpb_coarse_band_{sfx}")(t.data_ptr(), 2, None, None, None, None, lv.k.data_ptr(),
                                                 lv.mask.data_ptr(), *g.args, st)
        linv = self._tbuf("band_linv", (nt * 1024,), torch.float64)
        info = self._tbuf("band_info", (2,), torch.int32)
        bar = self._tbuf("band_bar", (2 * max(64, nt),), torch.int32)
        ainv = self._tbuf("band_ainv", (npad, npad), torch.float64)
        sgn = self._tbuf("band_sgn", (npad,), torch.float64)
        self._coarse = {"ainv": ainv, "v": self._tbuf("coarse_v", (npad,), torch.float64), "n": n}
        # The factorisation and the inverse are latency-bound chains on a fraction of the SMs;
        # they run on a high-priority side stream, overlapped with the power iterations the
        # caller issues next on the main stream, which joins before anything reads them.
        main = torch.cuda.current_stream()
        self._ev_fork.record(main)
        self._side.wait_event(self._ev_fork)
        ss = self._side.cuda_stream
        L.lpb_memset_async(info.data_ptr(), 0, 8, ss)
        L.lpb_band_factor(t.data_ptr(), linv.data_ptr(), sgn.data_ptr(), info.data_ptr(), bar.data_ptr(),
                          info[1:].data_ptr(), *g.args, ss)
        L.lpb_band_inverse(ainv.data_ptr(), t.data_ptr(), linv.data_ptr(), sgn.data_ptr(), *g.args, ss)
        self._ev_join.record(self._side)
        self._joined = False
        return info

    def _join_coarse(self):
        """The main stream waits for the side stream's factorisation and inverse."""
        if not self._joined:
            torch.cuda.current_stream().wait_event(self._ev_join)
            self._joined = True

    def _op(self, i):
        return self._l0s if i == 0 else self.levels[i]

    def _lmax_vectors(self, i):
        """The power iteration's buffers of level i; the start vector is drawn once per level
        shape and then warm-started from the last hierarchy's, as the reference does."""
        lv = self._op(i)
        g = lv.grid
        dt = lv.dtype
        v = self._buf(f"pw_v{i}", g, dt)
        av = self._buf(f"pw_av{i}", g, dt)
        keep = self._buf(f"pw_keep{i}", g, dt)
        if self._lmax_init.get(i) != (tuple(keep.shape), dt):
            rng = np.random.default_rng(i)
            host = (rng.random(lv.node_shape) - 0.5).astype(np.float32 if dt == torch.float32 else np.float64)
            g.nodes_to_dev(host, dt, out=keep)
            self._lmax_init[i] = (tuple(keep.shape), dt)
        return v, av, keep

    def _estimate_lmax(self, i, its=12, part=None):
        """Largest eigenvalue of D^-1 A by power iteration, times 1.3, and the Chebyshev
        coefficients from it, all on the device (loadpath/mg.py:771-794). Launches only (the
        buffers come from _lmax_vectors), so a level's iterations can be one graph."""
        L = lib()
        st = stream_handle()
        part = self._part if part is None else part
        lv = self._op(i)
        g = lv.grid
        dt = lv.dtype
        sfx = "f32" if dt == torch.float32 else "f64"
        v, av, keep = self._lmax_vectors(i)
        getattr(L, f"lpb_mask_field_{sfx}")(v.data_ptr(), keep.data_ptr(), lv.mask.data_ptr(), *g.args, 0, st)
        n = g.n_node_field
        pw = self._pw[32 * i:32 * (i + 1)]
        for it in range(its):
            getattr(L, f"lpb_dot_{sfx}")(v.data_ptr(), v.data_ptr(), n, part.data_ptr(),
                                         pw[it:].data_ptr(), st)
            getattr(L, f"lpb_scale_rsqrt_{sfx}")(v.data_ptr(), n, pw[it:].data_ptr(), st)
            lv.apply(av, v)
            getattr(L, f"lpb_dinv_mask_{sfx}")(av.data_ptr(), lv.dinv.data_ptr(), lv.mask.data_ptr(), *g.args, st)
            getattr(L, f"lpb_dot_{sfx}")(v.data_ptr(), av.data_ptr(), n, part.data_ptr(),
                                         pw[16 + it:].data_ptr(), st)
            v, av = av, v
        # the final vector is kept for the next hierarchy (already masked)
        getattr(L, f"lpb_mask_field_{sfx}")(keep.data_ptr(), v.data_ptr(), lv.mask.data_ptr(), *g.args, 0, st)
        L.lpb_cheb_coef(self._coef[16 * i:].data_ptr(), pw.data_ptr(), pw[16:].data_ptr(), its,
                        max(self.degree, 1), LMAX_SAFETY, st)

    def _run_lmax(self, i, nl, part):
        if self.use_graphs:
            self._replay(self._graph(("lmax", i, nl), lambda: self._estimate_lmax(i, part=part)))
        else:
            self._estimate_lmax(i, part=part)

    def _lmax_fine_early(self, nl):
        """A planned rebuild (the level count known): levels 0 and 1's power iterations on their
        own stream as soon as level 1 is built, beside the Galerkin products of the coarser levels
        and the coarsest factorisation; _all_lmax joins them."""
        for i in range(2):
            self._op(i).coef = self._coef[16 * i:16 * (i + 1)]
            self._lmax_vectors(i)
        self._ev_pw01_fork.record()
        with torch.cuda.stream(self._pw01_stream):
            self._pw01_stream.wait_event(self._ev_pw01_fork)
            for i in range(2):
                self._run_lmax(i, nl, self._part_pw01)
            self._ev_pw01_join.record()
        self._pw01_early = True

    def _all_lmax(self, nl):
        """λmax of every level. The levels are independent: the fine two run on the working
        stream (or already run on their own, _lmax_fine_early), the coarse ones (chains of small
        kernels) on a stream of their own beside them; with graphs on, each level's twelve
        iterations are one graph launch."""
        for i in range(nl):
            self._op(i).coef = self._coef[16 * i:16 * (i + 1)]
            self._lmax_vectors(i)

        def run(i, part):
            self._run_lmax(i, nl, part)

        if nl > 2:
            self._ev_pw_fork.record()
        if self._pw01_early:
            torch.cuda.current_stream().wait_event(self._ev_pw01_join)
        else:
            for i in range(min(nl, 2)):
                run(i, self._part_pw01)
        if nl > 2:
            with torch.cuda.stream(self._pw_stream):
                self._pw_stream.wait_event(self._ev_pw_fork)
                for i in range(2, nl):
                    run(i, self._part_pw)
                self._ev_pw_join.record()
            torch.cuda.current_stream().wait_event(self._ev_pw_join)

    # --- V-cycle (loadpath/mg.py:796-864) -----------------------------------------------
    def _smooth(self, i, b, x, from_zero):
        """Chebyshev (or damped Jacobi) smoothing of level i."""
        L = lib()
        st = stream_handle()
        lv = self._op(i)
        g = lv.grid
        dt = lv.dtype
        sfx = "f32" if dt == torch.float32 else "f64"
        n = g.n_node_field
        r = self._buf(f"r{i}", g, dt)
        d = self._buf(f"d{i}", g, dt)
        t = self._buf(f"t{i}", g, dt)
        if self.smoother == "jacobi":
            om = self.omega
            for it in range(self.degree):
                if from_zero and it == 0:
                    getattr(L, f"lpb_jacobi_{sfx}")(x.data_ptr(), b.data_ptr(), b.data_ptr(), lv.dinv.data_ptr(), om,
                                                    1, n, st)
                else:
                    lv.apply(t, x)
                    getattr(L, f"lpb_jacobi_{sfx}")(x.data_ptr(), b.data_ptr(), t.data_ptr(), lv.dinv.data_ptr(), om,
                                                    0, n, st)
            return x
        coef = lv.coef.data_ptr()
        if self.degree == 2 and lv.kind == "scaled" and dt == torch.float32:
            # the fine float32 level forms each update where its tiled apply stores A u
            def fused(mode, u):
                probe = _PROBE[0]
                if probe is not None:
                    ea, eb = probe.take()
                    L.lpb_event_record(ea.cuda_event, st)
                L.lpb_apply_fine_cheb_f32(mode, x.data_ptr(), r.data_ptr(), d.data_ptr(), u.data_ptr(), b.data_ptr(),
                                          lv.dinv.data_ptr(), coef, lv.e.data_ptr(), lv.mask.data_ptr(),
                                          lv.kmodal.ctypes.data, lv.err.data_ptr(), *g.args, st)
                if probe is not None:
                    L.lpb_event_record(eb.cuda_event, st)
                    (probe.capture if probe.capture is not None else probe.pending).append((f"f32c{mode}", ea, eb))
            if from_zero:
                getattr(L, f"lpb_cheb_d_start_{sfx}")(b.data_ptr(), lv.dinv.data_ptr(), coef, d.data_ptr(), n, st)
                fused(1, d)
            else:
                fused(2, x)
                fused(3, d)
            return x
        if self.degree == 2 and lv.kind == "explicit" and lv.km is not None:
            # the explicit levels form each update in the gather of A u (the same expressions)
            def fused(mode, u):
                L.lpb_apply_explicit_modal_cheb_f32(mode, x.data_ptr(), r.data_ptr(), d.data_ptr(), u.data_ptr(),
                                                    b.data_ptr(), lv.dinv.data_ptr(), coef, lv.km.data_ptr(),
                                                    lv.kpc.data_ptr(), lv.glist.data_ptr(), lv.gcount.data_ptr(),
                                                    lv.ft.data_ptr(), lv.mask.data_ptr(), *g.args, st)
            if from_zero:
                getattr(L, f"lpb_cheb_d_start_{sfx}")(b.data_ptr(), lv.dinv.data_ptr(), coef, d.data_ptr(), n, st)
                fused(1, d)
            else:
                fused(2, x)
                fused(3, d)
            return x
        if self.degree == 2:
            # the two Chebyshev steps in two passes (same bits as the step-by-step form)
            if from_zero:
                getattr(L, f"lpb_cheb_d_start_{sfx}")(b.data_ptr(), lv.dinv.data_ptr(), coef, d.data_ptr(), n, st)
                lv.apply(t, d)
                getattr(L, f"lpb_cheb2_zero_{sfx}")(x.data_ptr(), b.data_ptr(), t.data_ptr(), d.data_ptr(),
                                                    lv.dinv.data_ptr(), coef, n, st)
            else:
                lv.apply(t, x)
                getattr(L, f"lpb_residual_scaled_{sfx}")(b.data_ptr(), t.data_ptr(), lv.dinv.data_ptr(), coef,
                                                         r.data_ptr(), d.data_ptr(), n, st)
                lv.apply(t, d)
                getattr(L, f"lpb_cheb2_{sfx}")(x.data_ptr(), d.data_ptr(), r.data_ptr(), t.data_ptr(),
                                               lv.dinv.data_ptr(), coef, n, st)
            return x
        if from_zero:
            getattr(L, f"lpb_cheb_start_{sfx}")(b.data_ptr(), lv.dinv.data_ptr(), coef, x.data_ptr(), r.data_ptr(),
                                                d.data_ptr(), n, st)
        else:
            lv.apply(t, x)
            getattr(L, f"lpb_residual_scaled_{sfx}")(b.data_ptr(), t.data_ptr(), lv.dinv.data_ptr(), coef,
                                                     r.data_ptr(), d.data_ptr(), n, st)
        for it in range(self.degree):
            last = it + 1 == self.degree
            if not last:
                lv.apply(t, d)
            getattr(L, f"lpb_cheb_{sfx}")(x.data_ptr(), d.data_ptr(), r.data_ptr(), (d if last else t).data_ptr(),
                                          lv.dinv.data_ptr(), coef, it, int(last), n, st)
        return x

    def _vcycle(self, i, b, dot=None):
        """x = V(b) on level i; b and the result live in level-i buffers. dot = (r64, out): also
        out = r64 . x (the PCG's r . z)."""
        L = lib()
        st = stream_handle()
        lv = self._op(i)
        g = lv.grid
        dt = lv.dtype
        sfx = "f32" if dt == torch.float32 else "f64"
        x = self._buf(f"x{i}", g, dt)
        if i == len(self.levels) - 1:
            if self._coarse is not None:
                c = self._coarse
                getattr(L, f"lpb_band_solve_{sfx}")(x.data_ptr(), b.data_ptr(), c["ainv"].data_ptr(),
                                                    c["v"].data_ptr(), *g.args, st)
            else:
                self._smooth(i, b, x, True)
                self._smooth(i, b, x, False)
            if dot is not None:
                L.lpb_dot_f64_f32(dot[0].data_ptr(), x.data_ptr(), x.numel(), self._part.data_ptr(),
                                  dot[1].data_ptr(), st)
            return x
        self._smooth(i, b, x, True)
        t = self._buf(f"t{i}", g, dt)
        lv.apply(t, x)
        nxt = self._op(i + 1)
        gc = nxt.grid
        bc = self._buf(f"b{i + 1}", gc, dt)
        getattr(L, f"lpb_restrict_residual_{sfx}")(bc.data_ptr(), b.data_ptr(), t.data_ptr(), lv.mask.data_ptr(),
                                                   nxt.mask.data_ptr(), *g.args, *gc.args, st)
        xc = self._vcycle(i + 1, bc)
        getattr(L, f"lpb_prolong_add_{sfx}")(x.data_ptr(), xc.data_ptr(), nxt.mask.data_ptr(), lv.mask.data_ptr(),
                                             *g.args, *gc.args, st)
        self._smooth(i, b, x, False)
        if dot is not None:
            # its own pass: folded into the last smoothing pass it evicts that pass's inputs from
            # L2 (the float64 r is 103 MB at 256 x 128 x 128) and runs slower than the two
            L.lpb_dot_f64_f32(dot[0].data_ptr(), x.data_ptr(), x.numel(), self._part.data_ptr(), dot[1].data_ptr(), st)
        return x

    def precondition_device(self, r64, z_out):
        """z = V(r) with the cast to and from the V-cycle precision (loadpath/mg.py:862-864)."""
        L = lib()
        st = stream_handle()
        g = self.g0
        n = g.n_node_field
        if self.tdtype == torch.float32:
            b = self._buf("b0", g, torch.float32)
            L.lpb_cast_f64_f32(b.data_ptr(), r64.data_ptr(), n, st)
            x = self._vcycle(0, b)
            L.lpb_cast_f32_f64(z_out.data_ptr(), x.data_ptr(), n, st)
        else:
            b = self._buf("b0", g, torch.float64)
            b.copy_(r64)
            x = self._vcycle(0, b)
            z_out.copy_(x)
        return z_out

    # --- PCG (loadpath/mg.py:872-926) ---------------------------------------------------
    def _dot64(self, a, b, slot):
        lib().lpb_dot_f64(a.data_ptr(), b.data_ptr(), a.numel(), self._part.data_ptr(),
                          self._scal[slot].data_ptr(), stream_handle())

    def _solve_buffers(self):
        """Every buffer a solve's launches name, created before any capture (a capture must
        not allocate) and then reused, so captured graphs stay valid across solves."""
        g = self.g0
        for k in ("cg_x", "cg_r", "cg_p", "cg_ap", "cg_z", "cg_rs"):
            self._buf(k, g, torch.float64)
        if self.tdtype == torch.float32:
            self._buf("cg_r32", g, torch.float32)
        self._buf("b0", g, self.tdtype)
        for i in range(len(self.levels)):
            gi = self._op(i).grid
            for k in ("x", "r", "d", "t"):
                self._buf(f"{k}{i}", gi, self.tdtype)
            if i + 1 < len(self.levels):
                self._buf(f"b{i + 1}", self._op(i + 1).grid, self.tdtype)

    def _graph(self, key, fn, loop=False):
        """fn's launches captured as one CUDA graph, kept until a buffer it names is replaced
        (a new allocation or a new hierarchy structure) or the probe changes. Returns
        (exec, probe event pairs recorded by each replay, kernels per replay). loop: fn(handle)
        records the body of a device-side while loop whose condition handle it is given."""
        L = lib()
        cache = self._gcache
        probe = _PROBE[0]
        sig = (self._gen, id(probe))
        if cache.get("sig") != sig:
            self._free_graphs()
            cache = self._gcache          # the new, empty cache
            cache["sig"] = sig
        if key not in cache:
            pairs = []
            if probe is not None:
                probe.capture = pairs
            gen = self._gen
            c0 = launches()
            # captured on a side stream (the legacy default stream cannot be captured), launched
            # on the working stream
            with torch.cuda.stream(self._cap_stream):
                st0 = stream_handle()
                if loop:
                    handle, outer = ctypes.c_longlong(), ctypes.c_void_p()
                    L.lpb_while_begin(st0, ctypes.byref(handle), ctypes.byref(outer))
                else:
                    L.lpb_capture_begin(st0)
                try:
                    fn(handle.value) if loop else fn()
                finally:
                    exec_ = ctypes.c_void_p()
                    if loop:
                        L.lpb_while_end(st0, outer, ctypes.byref(exec_))
                    else:
                        L.lpb_capture_end(st0, ctypes.byref(exec_))
                    if probe is not None:
                        probe.capture = None
            nk = launches() - c0
            add_launches(-nk)              # recorded, not run
            if self._gen != gen:
                L.lpb_graph_free(exec_)
                raise RuntimeError("a buffer was allocated during a graph capture")
            cache[key] = (exec_, pairs, nk)
        return cache[key]

    def _replay(self, entry):
        """Launch a cached graph on the working stream (its kernels join the launch count)."""
        lib().lpb_graph_launch(entry[0], stream_handle())
        add_launches(entry[2])

    def _pcg_device(self, b, x0):
        """float64 PCG on padded device fields (loadpath/mg.py:872-926). Returns (x, iterations,
        converged). Nothing waits on the host before the first iteration: the warm-start
        choice is made on the device, and |b| reaches the host with the first iteration's
        scalars. With graphs on, the set-up, the CG head (A p, alpha, x, r, |r|^2) and the CG
        tail (V-cycle, beta, p) are each one graph launch.

        When converged is False, x is undefined: the host-tested loop queues an iteration's
        tail (which moves x by alpha p) before it reads that iteration's p.Ap, so on the
        p.Ap <= 0 exit x has taken one step past the iterate the reference returns
        (loadpath/mg.py:903-905). Callers discard it (solve_device raises, the strict fallback
        starts again from the caller's x0)."""
        L = lib()
        g = self.g0
        n = g.n_node_field
        a = self.levels[0]
        sc = self._scal
        self._solve_buffers()
        x = self._buf("cg_x", g, torch.float64)
        r = self._buf("cg_r", g, torch.float64)
        p = self._buf("cg_p", g, torch.float64)
        ap = self._buf("cg_ap", g, torch.float64)
        z = self._buf("cg_z", g, torch.float64)
        rs = self._buf("cg_rs", g, torch.float64)
        r32 = self._buf("cg_r32", g, torch.float32) if self.tdtype == torch.float32 else None
        host = self._host
        nb = 8 * n
        src = self._buf("cg_b", g, torch.float64)
        if b.data_ptr() != src.data_ptr():
            L.lpb_memcpy_async(src.data_ptr(), b.data_ptr(), nb, stream_handle())
        if x0 is not None:
            L.lpb_memcpy_async(x.data_ptr(), x0.data_ptr(), nb, stream_handle())

        def pre(warm):
            st = stream_handle()
            self._dot64(src, src, 0)
            if warm:
                a.apply(ap, x)
                self._dot64(x, ap, 5)
                self._dot64(src, x, 6)
                L.lpb_warm_residual(rs.data_ptr(), src.data_ptr(), ap.data_ptr(), sc.data_ptr(), n, st)
                self._dot64(rs, rs, 7)
                L.lpb_warm_select(x.data_ptr(), r.data_ptr(), src.data_ptr(), rs.data_ptr(), sc.data_ptr(), n, st)
            else:
                L.lpb_memset_async(x.data_ptr(), 0, nb, st)
                L.lpb_memcpy_async(r.data_ptr(), src.data_ptr(), nb, st)
            self.precondition_device(r, z)
            L.lpb_memcpy_async(p.data_ptr(), z.data_ptr(), nb, st)
            self._dot64(r, z, 1)

        def head():
            # ap = A p and pap in one pass; r -= alpha ap (and its float32 copy); |r|^2; scalars
            # out. x += alpha p waits for the tail's pass over p.
            st = stream_handle()
            a.apply_dot(ap, p, self._part, sc[3])
            L.lpb_cg_step_r(r.data_ptr(), ap.data_ptr(), ptr(r32), n, sc[1].data_ptr(), sc[3].data_ptr(),
                            self._part.data_ptr(), sc[4].data_ptr(), st)
            L.lpb_memcpy_async(host.data_ptr(), sc[3:5].data_ptr(), 16, st)
            L.lpb_memcpy_async(host[2:].data_ptr(), sc[0:1].data_ptr(), 8, st)

        def tail():
            # z = V(r) and rz_new (formed by the V-cycle's last pass); x += alpha p;
            # p = z + (rz_new / rz) p; rz = rz_new
            st = stream_handle()
            if r32 is not None:
                xv = self._vcycle(0, r32, dot=(r, sc[2]))
                L.lpb_xpby_x_f32(p.data_ptr(), x.data_ptr(), xv.data_ptr(), n, sc[1].data_ptr(), sc[3].data_ptr(),
                                 sc[2].data_ptr(), st)
            else:
                self.precondition_device(r, z)
                self._dot64(r, z, 2)
                L.lpb_xpby_x_f64(p.data_ptr(), x.data_ptr(), z.data_ptr(), n, sc[1].data_ptr(), sc[3].data_ptr(),
                                 sc[2].data_ptr(), st)
            L.lpb_memcpy_async(sc[1:2].data_ptr(), sc[2:3].data_ptr(), 8, st)

        warm = x0 is not None
        probe = _PROBE[0]
        graphed = self.use_graphs and self.maxiter > 1
        if graphed and self.device_loop and probe is None:
            # the whole iteration loop as one graph launch: head, the stopping test, tail per
            # iteration, the test on the device (the graph's WHILE node); the host reads the
            # outcome once
            st = stream_handle()
            state = self._loop_state
            rtol, maxiter = float(self.rtol), int(self.maxiter)

            def body(handle):
                stb = stream_handle()
                a.apply_dot(ap, p, self._part, sc[3])
                L.lpb_cg_step_r(r.data_ptr(), ap.data_ptr(), ptr(r32), n, sc[1].data_ptr(), sc[3].data_ptr(),
                                self._part.data_ptr(), sc[4].data_ptr(), stb)
                L.lpb_cg_continue(handle, sc.data_ptr(), state.data_ptr(), rtol, maxiter, stb)
                tail()

            g_pre = self._graph(("pre", warm), lambda: pre(warm))
            g_loop = self._graph(("loop", rtol, maxiter), body, loop=True)
            L.lpb_memset_async(state.data_ptr(), 0, 16, st)
            self._replay(g_pre)
            self._replay(g_loop)
            L.lpb_memcpy_async(self._loop_out.data_ptr(), state.data_ptr(), 16, st)
            torch.cuda.current_stream().synchronize()
            it, status = int(self._loop_out[0]), int(self._loop_out[1])
            add_launches(g_loop[2] * (it - 1))          # the body ran `it` times
            if status == 2:
                L.lpb_memset_async(x.data_ptr(), 0, nb, st)
                return x, 0, True
            return x, it, status == 1
        if graphed:
            g_pre = self._graph(("pre", warm), lambda: pre(warm))
            g_head = self._graph("head", head)
            # with the probe set, two instances of the tail take turns: the one replayed at
            # iteration it - 1 is complete (and not replayed again) when iteration it's head is
            g_tails = [self._graph("tail", tail)]
            if probe is not None:
                g_tails.append(self._graph("tail2", tail))
            pre_pairs, head_pairs = g_pre[1], g_head[1]
            self._replay(g_pre)
        else:
            pre(warm)
        ev = torch.cuda.Event()
        last_tail = [None]

        def finish(result):
            if graphed and probe is not None:
                torch.cuda.current_stream().synchronize()
                probe.harvest(last_tail[0][1])     # the last (speculative) tail replay
            return result

        tol = None
        for it in range(1, self.maxiter + 1):
            if graphed:
                self._replay(g_head)
            else:
                head()
            ev.record()
            # the next preconditioner step is queued before the host looks at |r|: the
            # device never waits on the convergence test (a converged solve discards it)
            prev_tail = last_tail[0]
            if graphed:
                last_tail[0] = g_tails[it % len(g_tails)]
                self._replay(last_tail[0])
            else:
                tail()
            ev.synchronize()
            if graphed and probe is not None:
                # this head replay and the previous tail replay are complete, and neither graph
                # instance is queued again before the next harvest
                if it == 1:
                    probe.harvest(pre_pairs)
                else:
                    probe.harvest(prev_tail[1])
                probe.harvest(head_pairs)
            if tol is None:
                bb = float(host[2])
                if bb == 0.0:
                    torch.cuda.current_stream().synchronize()
                    L.lpb_memset_async(x.data_ptr(), 0, nb, stream_handle())
                    return finish((x, 0, True))
                tol = self.rtol * math.sqrt(bb)
            pap, rr = float(host[0]), float(host[1])
            if not pap > 0:
                return finish((x, it, False))
            if math.sqrt(rr) <= tol:
                return finish((x, it, True))
        return finish((x, self.maxiter, False))

    def _solve_device(self, b, x0):
        """One right-hand side with the strict fallback (loadpath/mg.py:951-965)."""
        if self.strict or len(self.levels) < 2:
            return self._pcg_device(b, x0)
        full = self.maxiter
        self.maxiter = min(full, STALL)
        try:
            x, it, ok = self._pcg_device(b, x0)
        finally:
            self.maxiter = full
        if ok:
            return x, it, ok
        self.strict = True
        self.set_moduli_device(self._e_dev)
        x, it2, ok = self._pcg_device(b, x0)
        return x, it + it2, ok

    def solve_device(self, b, x0=None):
        """Solve with padded float64 device fields; b and x0 are masked here. Returns a new
        device field (masked). Raises RuntimeError when CG does not converge."""
        L = lib()
        st = stream_handle()
        g = self.g0
        m = self.levels[0].mask
        bm = self._buf("cg_b", g, torch.float64)
        L.lpb_mask_field_f64(bm.data_ptr(), b.data_ptr(), m.data_ptr(), *g.args, 0, st)
        x0m = None
        if x0 is not None:
            x0m = self._buf("solve_x0", g, torch.float64)
            L.lpb_mask_field_f64(x0m.data_ptr(), x0.data_ptr(), m.data_ptr(), *g.args, 0, st)
        x, it, ok = self._solve_device(bm, x0m)
        self.last_iters = it
        self.check_device()
        if not ok:
            raise RuntimeError(f"linear solve did not converge ({it} iterations); "
                               "the structure may be a mechanism (check supports)")
        out = g.node_field(torch.float64)
        L.lpb_mask_field_f64(out.data_ptr(), x.data_ptr(), m.data_ptr(), *g.args, 0, st)
        return out

    def solve_many(self, fs, x0s=None):
        """Solve for each right-hand side (mesh dof numbering); dofs without stiffness come
        back as zero (loadpath/mg.py:932-949)."""
        x0s = x0s or [None] * len(fs)
        out = []
        iters = 0
        for f, x0 in zip(fs, x0s):
            b = self.g0.nodes_to_dev(self.to_grid(f), torch.float64)
            x0d = self.g0.nodes_to_dev(self.to_grid(x0), torch.float64) if x0 is not None else None
            x = self.solve_device(b, x0d)
            iters = max(iters, self.last_iters)
            out.append(self.from_grid(self.g0.nodes_to_host(x)))
        self.last_iters = iters
        return out

    # --- k right-hand sides as one block ----------------------------------------------------
    # The reference solves its load cases one after another (loadpath/mg.py:932-949). Here k
    # columns advance together: one traversal of the hierarchy per PCG iteration runs every
    # column's smoothing, transfers and operator applies level by level (so a level's
    # coefficients - moduli, level-1 weights, explicit matrices - are read from L2 by the
    # columns after the first), one kernel solves the coarsest level for all columns (its
    # dense inverse read once per eight), and the host reads every column's scalars with one
    # copy per iteration. Each column keeps its own scalars and stopping test and runs the
    # same kernels on the same data as a lone solve, so a column's answer has the same bits.
    def _blk(self, key, k, grid: DevGrid, dtype):
        """k node fields of a level as one (k, field) tensor; [j] is column j's field."""
        return self._tbuf(key, (k, 3, grid.pz // 4, grid.NY, grid.NX, 4), dtype)

    def _tbuf_host(self, key, shape, dtype):
        """A persistent pinned host buffer (for copies a solve makes once)."""
        t = self._work.get(key)
        if t is None or t.dtype != dtype or tuple(t.shape) != tuple(shape):
            t = torch.zeros(tuple(shape), dtype=dtype, pin_memory=True)
            self._work[key] = t
        return t

    def _block_buffers(self, k):
        g = self.g0
        bufs = {key: self._blk(f"bcg_{key}", k, g, torch.float64) for key in ("x", "r", "p", "ap", "rs", "b", "snap")}
        for i in range(len(self.levels)):
            lv = self._op(i)
            self._blk(f"bx{i}", k, lv.grid, self.tdtype)
            self._blk(f"bb{i}", k, lv.grid, self.tdtype)
            for key in ("r", "d", "t"):
                self._buf(f"{key}{i}", lv.grid, self.tdtype)
        if self._coarse is not None:
            self._flat_buf("band_vcols", k * self._coarse["v"].numel(), torch.float64)
        bufs["sc"] = self._tbuf("bcg_sc", (k, 8), torch.float64)
        if getattr(self, "_bhost", None) is None or self._bhost.shape[0] != k:
            self._bhost = torch.zeros((k, 8), dtype=torch.float64, pin_memory=True)
            self._gen += 1               # graphs that copy into the old one are not replayed again
        return bufs

    def _vcycle_cols(self, i, bb, dots=None):
        """The V-cycle of level i for every column of bb (a (k, field) level-i block); returns
        the level's x block. dots: [(r64, out)] per column, out = r64 . x."""
        L = lib()
        st = stream_handle()
        lv = self._op(i)
        g = lv.grid
        dt = lv.dtype
        sfx = "f32" if dt == torch.float32 else "f64"
        k = bb.shape[0]
        xb = self._blk(f"bx{i}", k, g, dt)
        if i == len(self.levels) - 1:
            if self._coarse is not None:
                c = self._coarse
                v = self._flat_buf("band_vcols", k * c["v"].numel(), torch.float64)
                getattr(L, f"lpb_band_solve_cols_{sfx}")(xb.data_ptr(), bb.data_ptr(), xb[0].numel(), k,
                                                         c["ainv"].data_ptr(), v.data_ptr(), *g.args, st)
            else:
                for j in range(k):
                    self._smooth(i, bb[j], xb[j], True)
                    self._smooth(i, bb[j], xb[j], False)
        else:
            t = self._buf(f"t{i}", g, dt)
            nxt = self._op(i + 1)
            gc = nxt.grid
            bc = self._blk(f"bb{i + 1}", k, gc, dt)
            for j in range(k):
                self._smooth(i, bb[j], xb[j], True)
                lv.apply(t, xb[j])
                getattr(L, f"lpb_restrict_residual_{sfx}")(bc[j].data_ptr(), bb[j].data_ptr(), t.data_ptr(),
                                                           lv.mask.data_ptr(), nxt.mask.data_ptr(), *g.args,
                                                           *gc.args, st)
            xc = self._vcycle_cols(i + 1, bc)
            for j in range(k):
                getattr(L, f"lpb_prolong_add_{sfx}")(xb[j].data_ptr(), xc[j].data_ptr(), nxt.mask.data_ptr(),
                                                     lv.mask.data_ptr(), *g.args, *gc.args, st)
                self._smooth(i, bb[j], xb[j], False)
        if dots is not None:
            dot = L.lpb_dot_f64_f32 if dt == torch.float32 else L.lpb_dot_f64
            for j, (r64, out) in enumerate(dots):
                dot(r64.data_ptr(), xb[j].data_ptr(), xb[j].numel(), self._part.data_ptr(), out.data_ptr(), st)
        return xb

    def _pcg_block(self, bs, x0s, outs):
        """float64 PCG on k columns at once (the per-column algorithm of _pcg_device). bs, x0s:
        lists of masked padded fields (x0s entries may be None); outs: the k result fields, each
        written once its column has converged. Returns (iterations, converged) per column."""
        L = lib()
        g = self.g0
        n = g.n_node_field
        k = len(bs)
        a = self.levels[0]
        probe = _PROBE[0]
        _PROBE[0] = None                 # the block path records no fine-apply events
        try:
            B = self._block_buffers(k)
            x, r, p, ap, rs, src, sc = B["x"], B["r"], B["p"], B["ap"], B["rs"], B["b"], B["sc"]
            host = self._bhost
            nb = 8 * n
            f32 = self.tdtype == torch.float32
            bb0 = self._blk("bb0", k, g, self.tdtype)
            for j in range(k):
                L.lpb_memcpy_async(src[j].data_ptr(), bs[j].data_ptr(), nb, stream_handle())
                if x0s[j] is not None:
                    L.lpb_memcpy_async(x[j].data_ptr(), x0s[j].data_ptr(), nb, stream_handle())
            warm = tuple(x0 is not None for x0 in x0s)

            def dot(u, v, out):
                L.lpb_dot_f64(u.data_ptr(), v.data_ptr(), n, self._part.data_ptr(), out.data_ptr(), stream_handle())

            def precondition_all():
                # z = V(r) for every column, z left in the level-0 x block
                st = stream_handle()
                for j in range(k):
                    if f32:
                        L.lpb_cast_f64_f32(bb0[j].data_ptr(), r[j].data_ptr(), n, st)
                    else:
                        L.lpb_memcpy_async(bb0[j].data_ptr(), r[j].data_ptr(), nb, st)
                return self._vcycle_cols(0, bb0)

            def pre():
                st = stream_handle()
                for j in range(k):
                    s = sc[j]
                    dot(src[j], src[j], s[0])
                    if warm[j]:
                        a.apply(ap[j], x[j])
                        dot(x[j], ap[j], s[5])
                        dot(src[j], x[j], s[6])
                        L.lpb_warm_residual(rs[j].data_ptr(), src[j].data_ptr(), ap[j].data_ptr(), s.data_ptr(), n,
                                            st)
                        dot(rs[j], rs[j], s[7])
                        L.lpb_warm_select(x[j].data_ptr(), r[j].data_ptr(), src[j].data_ptr(), rs[j].data_ptr(),
                                          s.data_ptr(), n, st)
                    else:
                        L.lpb_memset_async(x[j].data_ptr(), 0, nb, st)
                        L.lpb_memcpy_async(r[j].data_ptr(), src[j].data_ptr(), nb, st)
                z = precondition_all()
                for j in range(k):
                    if f32:
                        L.lpb_cast_f32_f64(p[j].data_ptr(), z[j].data_ptr(), n, st)
                    else:
                        L.lpb_memcpy_async(p[j].data_ptr(), z[j].data_ptr(), nb, st)
                    dot(r[j], p[j], sc[j][1])

            def head(to_host=True):
                st = stream_handle()
                for j in range(k):
                    s = sc[j]
                    a.apply_dot(ap[j], p[j], self._part, s[3])
                    L.lpb_cg_step_r(r[j].data_ptr(), ap[j].data_ptr(), bb0[j].data_ptr() if f32 else None, n,
                                    s[1].data_ptr(), s[3].data_ptr(), self._part.data_ptr(), s[4].data_ptr(), st)
                if to_host:
                    L.lpb_memcpy_async(host.data_ptr(), sc.data_ptr(), 8 * 8 * k, st)

            def tail():
                st = stream_handle()
                if f32:
                    # cg_step_r left each column's float32 residual in the level-0 b block
                    z = self._vcycle_cols(0, bb0, dots=[(r[j], sc[j][2]) for j in range(k)])
                else:
                    z = precondition_all()
                    for j in range(k):
                        dot(r[j], z[j], sc[j][2])
                for j in range(k):
                    s = sc[j]
                    getattr(L, "lpb_xpby_x_f32" if f32 else "lpb_xpby_x_f64")(
                        p[j].data_ptr(), x[j].data_ptr(), z[j].data_ptr(), n, s[1].data_ptr(), s[3].data_ptr(),
                        s[2].data_ptr(), st)
                    L.lpb_memcpy_async(s[1].data_ptr(), s[2].data_ptr(), 8, st)

            graphed = self.use_graphs and self.maxiter > 1
            if graphed and self.device_loop:
                # the loop on the device (as in _pcg_device): per iteration every column's head,
                # the columns' stopping test, every tail, and the masked copy of each column that
                # converged in this iteration
                st = stream_handle()
                state = self._tbuf("bloop_state", (k + 1, 2), torch.int64)
                rtol, maxiter = float(self.rtol), int(self.maxiter)
                mk = a.mask.data_ptr()

                snap = B["snap"]

                def body(handle):
                    stb = stream_handle()
                    head(to_host=False)
                    L.lpb_cg_continue_cols(handle, sc.data_ptr(), state.data_ptr(), k, rtol, maxiter, stb)
                    tail()
                    for j in range(k):
                        L.lpb_snapshot_converged(snap[j].data_ptr(), x[j].data_ptr(), mk, state.data_ptr(), j, k,
                                                 *g.args, stb)

                g_pre = self._graph(("bpre", k, warm), pre)
                g_loop = self._graph(("bloop", k, rtol, maxiter), body, loop=True)
                L.lpb_memset_async(state.data_ptr(), 0, state.numel() * 8, st)
                self._replay(g_pre)
                self._replay(g_loop)
                hs = self._tbuf_host("bloop_host", (k + 1, 2), torch.int64)
                L.lpb_memcpy_async(hs.data_ptr(), state.data_ptr(), state.numel() * 8, st)
                torch.cuda.current_stream().synchronize()
                sv = hs.numpy().copy()
                it_all = int(sv[k, 0])
                add_launches(g_loop[2] * (it_all - 1))
                iters, ok = [], []
                for j in range(k):
                    done_at, status = int(sv[j, 0]), int(sv[j, 1])
                    if status == 2:
                        L.lpb_memset_async(outs[j].data_ptr(), 0, nb, st)
                        iters.append(0)
                    else:
                        if status == 1:
                            L.lpb_memcpy_async(outs[j].data_ptr(), snap[j].data_ptr(), nb, st)
                        iters.append(done_at if status else self.maxiter)
                    ok.append(status in (1, 2))
                return iters, ok
            if graphed:
                g_pre = self._graph(("bpre", k, warm), pre)
                g_head = self._graph(("bhead", k), head)
                g_tail = self._graph(("btail", k), tail)
                self._replay(g_pre)
            else:
                pre()
            ev = torch.cuda.Event()
            iters = [0] * k
            ok = [False] * k
            done = [False] * k
            tol = [None] * k
            for it in range(1, self.maxiter + 1):
                if graphed:
                    self._replay(g_head)
                else:
                    head()
                ev.record()
                if graphed:
                    self._replay(g_tail)
                else:
                    tail()
                ev.synchronize()
                hv = host.numpy()
                for j in range(k):
                    if done[j]:
                        continue
                    if tol[j] is None:
                        bbj = float(hv[j, 0])
                        if bbj == 0.0:
                            L.lpb_memset_async(outs[j].data_ptr(), 0, nb, stream_handle())
                            done[j], ok[j], iters[j] = True, True, 0
                            continue
                        tol[j] = self.rtol * math.sqrt(bbj)
                    pap, rr = float(hv[j, 3]), float(hv[j, 4])
                    if not pap > 0:
                        done[j], iters[j] = True, it
                    elif math.sqrt(rr) <= tol[j]:
                        # this iteration's tail (already queued) completes x; its masked copy
                        # follows it
                        L.lpb_mask_field_f64(outs[j].data_ptr(), x[j].data_ptr(), a.mask.data_ptr(), *g.args, 0,
                                             stream_handle())
                        done[j], ok[j], iters[j] = True, True, it
                if all(done):
                    break
            for j in range(k):
                if not done[j]:
                    iters[j] = self.maxiter
            return iters, ok
        finally:
            _PROBE[0] = probe

    def solve_block_device(self, bs, x0s=None):
        """Solve for k right-hand sides at once (padded float64 device fields); b and x0 are
        masked here. Returns a list of new device fields (masked); self.last_iters is the list of
        per-column iteration counts. A column not converged within the stall limit switches the
        hierarchy to strict and is solved again with the rest that failed (loadpath/mg.py:951-965).
        Raises RuntimeError when a column does not converge."""
        L = lib()
        st = stream_handle()
        g = self.g0
        m = self.levels[0].mask
        k = len(bs)
        x0s = list(x0s) if x0s is not None else [None] * k
        bm, x0m, outs = [], [], []
        for j in range(k):
            b = g.node_field(torch.float64)
            L.lpb_mask_field_f64(b.data_ptr(), bs[j].data_ptr(), m.data_ptr(), *g.args, 0, st)
            bm.append(b)
            if x0s[j] is not None:
                x0 = g.node_field(torch.float64)
                L.lpb_mask_field_f64(x0.data_ptr(), x0s[j].data_ptr(), m.data_ptr(), *g.args, 0, st)
                x0m.append(x0)
            else:
                x0m.append(None)
            outs.append(g.node_field(torch.float64))
        todo = list(range(k))
        iters = [0] * k
        stall = not (self.strict or len(self.levels) < 2)
        full = self.maxiter
        if stall:
            self.maxiter = min(full, STALL)
        try:
            its, ok = self._pcg_block([bm[j] for j in todo], [x0m[j] for j in todo], [outs[j] for j in todo])
        finally:
            self.maxiter = full
        for j, it_ in zip(todo, its):
            iters[j] += it_
        todo = [j for j, o in zip(todo, ok) if not o]
        if todo and stall:
            self.strict = True
            self.set_moduli_device(self._e_dev)
            its, ok = self._pcg_block([bm[j] for j in todo], [x0m[j] for j in todo], [outs[j] for j in todo])
            for j, it_ in zip(todo, its):
                iters[j] += it_
            todo = [j for j, o in zip(todo, ok) if not o]
        self.last_iters = iters
        self.check_device()
        if todo:
            raise RuntimeError(f"linear solve did not converge ({max(iters[j] for j in todo)} iterations); "
                               "the structure may be a mechanism (check supports)")
        return outs

    # --- other reference methods ----------------------------------------------------------
    def apply(self, u):
        """The float64 operator on a host node-grid field (loadpath/mg.py:868-870)."""
        g = self.g0
        ud = g.nodes_to_dev(u, torch.float64)
        out = g.node_field(torch.float64)
        self.levels[0].apply(out, ud, mask_in=True)
        return g.nodes_to_host(out)

    def live_dofs(self):
        """Bool per mesh dof: carries stiffness (loadpath/mg.py:967-973)."""
        m = self.g0.node_grid(self.levels[0].mask).cpu().numpy()
        a = np.stack([(m >> (3 + c)) & 1 for c in range(3)]).astype(bool).reshape(3, -1)
        out = np.empty(3 * len(self.node_flat), bool)
        for i in range(3):
            out[i::3] = a[i, self.node_flat]
        return out

    def strain_energy_device(self, u_dev, v_dev=None, out=None):
        """Per-cell u_e^T Ke v_e at unit modulus, float64 padded cell field."""
        g = self.g0
        out = out if out is not None else g.cell_field(torch.float64)
        lib().lpb_element_energy_f64(out.data_ptr(), u_dev.data_ptr(), ptr(v_dev), self.ke64.data_ptr(), *g.args,
                                     stream_handle())
        return out

    def strain_energy(self, u):
        """Per element u_e^T Ke u_e at unit modulus, mesh order (loadpath/mg.py:975-988)."""
        g = self.g0
        ud = g.nodes_to_dev(self.to_grid(u), torch.float64)
        se = g.cells_to_host(self.strain_energy_device(ud))
        return se[tuple(self.elem_ijk.T)]

    def _free_graphs(self):
        execs = [v[0] for k, v in self._gcache.items() if k != "sig"]
        if execs:
            torch.cuda.current_stream().synchronize()
            for gexec in execs:
                lib().lpb_graph_free(gexec)
        self._gcache = {}

    def __del__(self):
        try:
            self._free_graphs()
        except Exception:
            pass

    # --- float32-only solve (loadpath/gpu.py:399-481, TorchMG._pcg32 / solve_fp32) -------------
    def apply_rf(self, out, h, l=None):
        """out = m K (h + l) + (1 - m) h on the fine level in float32, each cell's matrix applied to
        its rigid-motion-free deformation formed in pair arithmetic (loadpath/gpu.py:119-149,
        :233-258); h, l, out: float32 device node fields (l None: h alone)."""
        lv = self._l0s
        g = self.g0
        if lv.dtype != torch.float32:
            raise ValueError("apply_rf needs the float32 fine level (dtype=np.float32)")
        ft = self._tbuf("rf_ft", (24, g.n_cell_field), torch.float32)
        lib().lpb_apply_rf_f32(out.data_ptr(), h.data_ptr(), ptr(l), lv.mask.data_ptr(), lv.e.data_ptr(),
                               self.ke32.data_ptr(), ft.data_ptr(), *g.args, stream_handle())
        return out

    def _dot32(self, a, b):
        out = self._tbuf("dot32", (1,), torch.float64)
        lib().lpb_dot_f32(a.data_ptr(), b.data_ptr(), a.numel(), self._part.data_ptr(), out.data_ptr(),
                          stream_handle())
        return float(out.item())

    def _pcg32(self, r, tol, maxiter):
        """Plain float32 PCG on the fine level's rigid-free operator for a correction K d = r to
        tol relative (loadpath/gpu.py:399-427). Returns (d, iterations); r is not changed."""
        L = lib()
        st = stream_handle()
        g = self.g0
        n = g.n_node_field
        f32 = torch.float32
        d = self._buf("rf_d", g, f32)
        d.zero_()
        rnorm = self._dot32(r, r) ** 0.5
        if rnorm == 0:
            return d, 0
        rr = self._buf("rf_r", g, f32)
        rr.copy_(r)
        p = self._buf("rf_p", g, f32)
        ap = self._buf("rf_ap", g, f32)
        z = self._vcycle(0, rr)
        p.copy_(z)
        rz = self._dot32(rr, z)
        for it in range(1, maxiter + 1):
            self.apply_rf(ap, p)
            pap = self._dot32(p, ap)
            if pap <= 0:
                return d, it
            alpha = rz / pap
            L.lpb_axpby_f32(d.data_ptr(), 1.0, d.data_ptr(), alpha, p.data_ptr(), n, st)
            L.lpb_axpby_f32(rr.data_ptr(), 1.0, rr.data_ptr(), -alpha, ap.data_ptr(), n, st)
            if self._dot32(rr, rr) ** 0.5 <= tol * rnorm:
                return d, it
            z = self._vcycle(0, rr)
            rz_new = self._dot32(rr, z)
            L.lpb_axpby_f32(p.data_ptr(), rz_new / rz, p.data_ptr(), 1.0, z.data_ptr(), n, st)
            rz = rz_new
        return d, maxiter

    def solve_fp32_device(self, b, x0=None, inner_rtol=3e-3, inner_max=50, outer_max=40):
        """The float32-only solve (loadpath/gpu.py:429-481): iterative refinement on the pair
        x = hi + lo. Each outer step forms the residual with the rigid-free operator from the pair,
        solves the correction with float32 PCG to inner_rtol and adds it in pair arithmetic;
        converged when the correction's energy |d . r| is under rtol^2 of x . b. b, x0: float64
        device node fields (b masked by the caller). Returns (x float64 device field, V-cycles,
        converged). For devices without fast float64; the mixed solve is the default."""
        L = lib()
        st = stream_handle()
        g = self.g0
        n = g.n_node_field
        f32, f64 = torch.float32, torch.float64
        out = g.node_field(f64)
        if float(torch.count_nonzero(b)) == 0:
            return out, 0, True
        bh, bl = self._buf("rf_bh", g, f32), self._buf("rf_bl", g, f32)
        t64 = self._buf("rf_t64", g, f64)
        L.lpb_cast_f64_f32(bh.data_ptr(), b.data_ptr(), n, st)
        L.lpb_cast_f32_f64(t64.data_ptr(), bh.data_ptr(), n, st)
        L.lpb_axpby_f64(t64.data_ptr(), 1.0, b.data_ptr(), -1.0, t64.data_ptr(), n, st)
        L.lpb_cast_f64_f32(bl.data_ptr(), t64.data_ptr(), n, st)
        xh, xl = self._buf("rf_xh", g, f32), self._buf("rf_xl", g, f32)
        xh.zero_()
        xl.zero_()
        ax, r = self._buf("rf_ax", g, f32), self._buf("rf_res", g, f32)

        def split(x64):   # float64 field -> (hi, lo) float32 pair in xh, xl
            L.lpb_cast_f64_f32(xh.data_ptr(), x64.data_ptr(), n, st)
            L.lpb_cast_f32_f64(t64.data_ptr(), xh.data_ptr(), n, st)
            L.lpb_axpby_f64(t64.data_ptr(), 1.0, x64.data_ptr(), -1.0, t64.data_ptr(), n, st)
            L.lpb_cast_f64_f32(xl.data_ptr(), t64.data_ptr(), n, st)

        if x0 is not None and float(torch.count_nonzero(x0)) > 0:
            # the energy-optimal multiple of x0, or zero if even that is worse
            split(x0)
            self.apply_rf(ax, xh, xl)
            xax = self._dot32(xh, ax) + self._dot32(xl, ax)
            sc = (self._dot32(bh, xh) + self._dot32(bh, xl)) / xax if xax > 0 else 0.0
            keep = False
            if sc > 0:
                L.lpb_axpby_f32(r.data_ptr(), 1.0, bh.data_ptr(), -sc, ax.data_ptr(), n, st)
                keep = self._dot32(r, r) < self._dot32(bh, bh)
            if keep:
                xs = self._buf("rf_xs", g, f64)
                L.lpb_axpby_f64(xs.data_ptr(), sc, x0.data_ptr(), 0.0, x0.data_ptr(), n, st)
                split(xs)
            else:
                xh.zero_()
                xl.zero_()
        tol2 = self.rtol ** 2
        total = 0
        ok = False
        for _ in range(outer_max):
            self.apply_rf(ax, xh, xl)
            L.lpb_pair_residual_f32(r.data_ptr(), bh.data_ptr(), ax.data_ptr(), bl.data_ptr(), n, st)
            d, it = self._pcg32(r, inner_rtol, inner_max)
            total += it
            L.lpb_pair_add_f32(xh.data_ptr(), xl.data_ptr(), d.data_ptr(), n, st)
            de = abs(self._dot32(d, r))
            xe = self._dot32(xh, bh)
            if xe <= 0 or not np.isfinite(de):
                break
            if de <= tol2 * xe:
                ok = True
                break
        L.lpb_cast_f32_f64(out.data_ptr(), xh.data_ptr(), n, st)
        L.lpb_cast_f32_f64(t64.data_ptr(), xl.data_ptr(), n, st)
        L.lpb_axpby_f64(out.data_ptr(), 1.0, out.data_ptr(), 1.0, t64.data_ptr(), n, st)
        self.last_iters = total
        return out, total, ok

    def set_moduli_live(self, e_dev, live, xp_dev, loads=()):
        """set_moduli with the live-cell reduction (loadpath/simp.py:795-806): the moduli of the
        cells `live` (simp.LiveCells) does not keep for the projected densities xp_dev are zeroed;
        if that leaves a load on a dof without stiffness (loads: float64 device node fields), the
        full grid is solved instead. Returns True when the reduced grid was kept."""
        keep = live.keep(xp_dev)
        if keep is None:
            self.set_moduli_device(e_dev)
            return False
        er = self._tbuf("e_live", e_dev.shape, torch.float64)
        live.moduli(e_dev, er)
        self.set_moduli_device(er)
        if getattr(live, "reused", False):
            return True          # a cached reduced system: its loads were found held when it was built
        L = lib()
        st = stream_handle()
        g = self.g0
        cnt = self._tbuf("dead_cnt", (1,), torch.float64)
        for f in loads:
            L.lpb_dead_loads(f.data_ptr(), self.levels[0].mask.data_ptr(), self._part.data_ptr(), cnt.data_ptr(),
                             *g.args, st)
            if float(cnt.item()) > 0:
                if hasattr(live, "record"):
                    live.record(False)
                self.set_moduli_device(e_dev)
                return False
        if hasattr(live, "record"):
            live.record(True)
        return True

    def check_device(self):
        """Raise if a tiled fine-apply launch flagged a shared-memory wait that gave up."""
        if int(self._err.item()) != 0:
            raise RuntimeError("fine-level apply: a TMA load wait gave up (device error flag set)")

    # diagnostics used by the parity tests
    def level_mask(self, i):
        return self._op(i).grid.mask_to_host(self._op(i).mask)

    def level_dinv(self, i):
        lv = self._op(i)
        return lv.grid.nodes_to_host(lv.dinv)
