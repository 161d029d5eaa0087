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
from ._lib import LpError, lib
from .grid import DevGrid, ptr, stream_handle, torch_dtype

__all__ = ["GridElasticity", "BoxMesh", "LMAX_SAFETY", "STALL"]

LMAX_SAFETY = 1.3          # loadpath/mg.py:81
STALL = 100                # loadpath/mg.py:930
DENSE_COARSE_MAX = 12_000  # dofs of the coarsest level solved by the dense factor (1.2 GB)


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
        self.totals = {"f32_ms": 0.0, "f32_count": 0, "f64_ms": 0.0, "f64_count": 0}
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
            k = "f32" if dt == torch.float32 else "f64"
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
        self.ft = None           # explicit: (24, cells) scratch of the cell pass
        self.g1 = None           # weights: 279 corner-parity coefficients (host)
        self.pbox = None         # weights: node box of the patch cells (host, 6 ints)
        self.mask = None
        self.dinv = None
        self.lmax = None
        self.n_active = 0

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
                getattr(L, f"lpb_apply_weights_march_{sfx}")(out.data_ptr(), u.data_ptr(), self.w.data_ptr(),
                                                              ptr(self.patch_id) if self.npatch else None,
                                                              ptr(self.patch_k) if self.npatch else None,
                                                              self.mask.data_ptr(), self.g1.ctypes.data,
                                                              self.pbox.ctypes.data, *g.args, st)
            else:
                getattr(L, f"lpb_apply_weights_{sfx}")(out.data_ptr(), u.data_ptr(), self.w.data_ptr(),
                                                        self.mcat.data_ptr(), ptr(self.patch_id),
                                                        ptr(self.patch_k), self.mask.data_ptr(), *g.args,
                                                        int(mask_in), 1, st)
        else:
            if fine_kernel and not mask_in:
                getattr(L, f"lpb_apply_explicit_sym_{sfx}")(out.data_ptr(), u.data_ptr(), self.kp.data_ptr(),
                                                             self.ft.data_ptr(), self.mask.data_ptr(), *g.args, st)
            else:
                getattr(L, f"lpb_apply_explicit_{sfx}")(out.data_ptr(), u.data_ptr(), self.k.data_ptr(),
                                                         self.mask.data_ptr(), *g.args, int(mask_in), 1, st)
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
    not supported on this path (the benchmark problems have none)."""

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
        self.device = torch.device(device if device not in (None, "b200", "auto") else "cuda")
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
        pk = fem.child_prolongations()
        self._mcat = np.einsum("kai,ab,kbj->kij", pk, self.ke, pk).reshape(8, 576)
        g1 = np.zeros(279)
        if lib().lpb_modal_g1(np.ascontiguousarray(self.ke).ctypes.data, g1.ctypes.data) != 279:
            raise LpError("the level-1 Galerkin matrices are not in the corner-parity pattern of the kernel")
        self.g1 = g1
        self.levels = []
        self.strict = False
        self.last_iters = 0
        self._lmax_vec = {}
        self._coarse = None
        self._scal = torch.zeros(64, dtype=torch.float64, device=self.device)
        self._part = torch.zeros(max(lib().lpb_reduce_blocks(), 1024) * 2, dtype=torch.float64, device=self.device)
        self._host = torch.zeros(8, dtype=torch.float64, pin_memory=True)
        self._work = {}
        self._e_dev = None
        # CUDA graphs for the CG iteration (captured once per solve)
        self.use_graphs = True
        self._graphs = None
        self._cap_stream = torch.cuda.Stream(device=self.device)

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
        return t

    def _buf(self, key, grid: DevGrid, dtype):
        t = self._work.get(key)
        if t is None or t.dtype != dtype or tuple(t.shape) != (3, grid.NX, grid.NY, grid.pz):
            t = grid.node_field(dtype)
            self._work[key] = t
        return t

    # --- hierarchy (loadpath/mg.py:515-754) --------------------------------------------
    def set_moduli(self, e):
        """Per-element moduli in mesh order (host array): rebuild every level."""
        e = np.asarray(e, np.float64)
        self._e_host = e
        e_dev = self.g0.cells_to_dev(self.cell_grid(e), torch.float64)
        self.set_moduli_device(e_dev)

    def set_moduli_device(self, e_dev: torch.Tensor):
        """Moduli already on the device as a padded (nx, ny, pz) float64 cell field."""
        self._e_dev = e_dev
        L = lib()
        st = stream_handle()
        g0 = self.g0
        dt = self.tdtype
        l0 = DevLevel("scaled", g0, torch.float64)
        l0.e = e_dev
        l0.ke = self.ke64
        l0.kmodal = self.kmodal
        l0.err = self._err
        d0 = self._buf("diag0", g0, torch.float64)
        L.lpb_diag_scaled_f64(d0.data_ptr(), e_dev.data_ptr(), self.ke64.data_ptr(), *g0.args, st)
        l0.mask = g0.mask_field()
        l0.dinv = g0.node_field(torch.float64)
        dinv32 = g0.node_field(torch.float32) if dt == torch.float32 else None
        L.lpb_masks(l0.mask.data_ptr(), l0.dinv.data_ptr(), ptr(dinv32), d0.data_ptr(), self.fixed_bits.data_ptr(),
                    None, *g0.args, 1e-300, 1e-300, st)
        self.levels = [l0]
        if dt == torch.float32:
            s = DevLevel("scaled", g0, torch.float32)
            s.e = g0.cell_field(torch.float32)
            L.lpb_cast_f64_f32(s.e.data_ptr(), e_dev.data_ptr(), g0.n_cell_field, st)
            s.ke = self.ke32
            s.kmodal = self.kmodal
            s.err = self._err
            s.mask = l0.mask
            s.dinv = dinv32
            self._l0s = s
        else:
            self._l0s = l0
        fine = l0
        n_active = int((e_dev > 0).sum().item())
        depth = 0
        held = None
        if self.strict:
            held = g0.mask_field()
            L.lpb_held0(held.data_ptr(), l0.mask.data_ptr(), self.fixed_bits.data_ptr(), held.numel(), st)
        while n_active > self.coarse_cells and min(fine.dims) >= 2:
            coarse = self._coarsen(fine, first=(depth == 0))
            depth += 1
            gc = coarse.grid
            d = self._buf(f"diag{depth}", gc, torch.float64)
            coarse.diagonal(d)
            L.lpb_max_f64(d.data_ptr(), d.numel(), self._part.data_ptr(), self._scal[40:].data_ptr(), st)
            dmax = float(self._scal[40].item())
            thr = 1e-12 * max(dmax, 1e-300)
            held_c = kept = None
            if self.strict:
                held_c = gc.mask_field()
                kept = gc.node_field(torch.float32)
                L.lpb_strict_held_kept(held_c.data_ptr(), kept.data_ptr(), held.data_ptr(), fine.mask.data_ptr(),
                                       *fine.grid.args, *gc.args, st)
                held = held_c
            coarse.mask = gc.mask_field()
            coarse.dinv = gc.node_field(dt)
            if dt == torch.float32:
                L.lpb_masks(coarse.mask.data_ptr(), None, coarse.dinv.data_ptr(), d.data_ptr(), ptr(held_c),
                            ptr(kept), *gc.args, thr, thr, st)
            else:
                L.lpb_masks(coarse.mask.data_ptr(), coarse.dinv.data_ptr(), None, d.data_ptr(), ptr(held_c),
                            ptr(kept), *gc.args, thr, thr, st)
            n_active = self._active_cells(coarse)
            self.levels.append(coarse)
            fine = coarse
        ok = self._build_coarse(self.levels[-1])
        if not ok:
            if self.strict:
                raise RuntimeError("coarsest-level factor is singular in the strict hierarchy")
            self.strict = True
            return self.set_moduli_device(e_dev)
        for i in range(len(self.levels)):
            self._op(i).lmax = self._estimate_lmax(i)

    def _active_cells(self, lv):
        """(loadpath/mg.py:593-599)"""
        g = lv.grid
        if lv.kind == "weights":
            act = (lv.w[:, :, :, :g.nz] != 0).any(dim=0)
            if lv.npatch:
                act = act | (lv.patch_id[:, :, :g.nz] >= 0)
            return int(act.sum().item())
        k = lv.k.view(g.nx, g.ny, g.cpz, 576)[:, :, :g.nz]
        return int((k != 0).any(dim=-1).sum().item())

    def _coarsen(self, fine: DevLevel, first: bool) -> DevLevel:
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
        if first:
            lv = DevLevel("weights", gc, dt)
            lv.w = torch.zeros((8, gc.nx, gc.ny, gc.cpz), dtype=dt, device=self.device)
            getattr(L, f"lpb_weights_from_e_f64_{sfx}")(lv.w.data_ptr(), fine.e.data_ptr(), *gf.args, *gc.args, st)
            lv.mcat = torch.tensor(self._mcat.reshape(-1), dtype=dt, device=self.device)
            flag = torch.zeros((gc.nx, gc.ny, gc.cpz), dtype=torch.uint8, device=self.device)
            L.lpb_patch_flags(flag.data_ptr(), fine.e.data_ptr(), fine.mask.data_ptr(), *gf.args, *gc.args, st)
            pcells = torch.nonzero(flag.reshape(-1)).reshape(-1).to(torch.int64).contiguous()
            lv.npatch = int(pcells.numel())
            lv.patch_id = torch.full((gc.nx, gc.ny, gc.cpz), -1, dtype=torch.int32, device=self.device)
            if lv.npatch:
                lv.patch_k = torch.zeros((lv.npatch, 576), dtype=dt, device=self.device)
                getattr(L, f"lpb_patch_matrices_{sfx}")(lv.patch_k.data_ptr(), lv.w.data_ptr(), lv.patch_id.data_ptr(),
                                                        pcells.data_ptr(), lv.npatch, fine.e.data_ptr(),
                                                        self.ke64.data_ptr(), fine.mask.data_ptr(), *gf.args,
                                                        *gc.args, st)
            else:
                lv.patch_k = None
            lv.patch_cells = pcells
            lv.g1 = self.g1
            lv.pbox = np.zeros(6, np.int32)
            if lv.npatch:
                z = pcells % gc.cpz
                yx = pcells // gc.cpz
                y = yx % gc.ny
                x = yx // gc.ny
                lo = torch.stack([x.min(), y.min(), z.min()]).cpu().numpy()
                hi = torch.stack([x.max(), y.max(), z.max()]).cpu().numpy() + 2   # nodes of the last cell
                lv.pbox[:3] = lo
                lv.pbox[3:] = hi - lo
            return lv
        lv = DevLevel("explicit", gc, dt)
        lv.k = torch.zeros((gc.nx * gc.ny * gc.cpz, 576), dtype=dt, device=self.device)
        if fine.kind == "weights":
            getattr(L, f"lpb_galerkin_explicit_{sfx}")(lv.k.data_ptr(), 1, fine.w.data_ptr(), fine.mcat.data_ptr(),
                                                       ptr(fine.patch_id), ptr(fine.patch_k), None,
                                                       fine.mask.data_ptr(), int(self.strict), *gf.args, *gc.args, st)
        else:
            getattr(L, f"lpb_galerkin_explicit_{sfx}")(lv.k.data_ptr(), 2, None, None, None, None, fine.k.data_ptr(),
                                                       fine.mask.data_ptr(), int(self.strict), *gf.args, *gc.args, st)
        ncp = gc.nx * gc.ny * gc.cpz
        lv.kp = torch.empty((300, ncp), dtype=dt, device=self.device)
        getattr(L, f"lpb_pack_sym_{sfx}")(lv.kp.data_ptr(), lv.k.data_ptr(), ncp, st)
        lv.ft = torch.empty((24, ncp), dtype=dt, device=self.device)
        return lv

    def _build_coarse(self, lv: DevLevel) -> bool:
        """Dense factor of the coarsest level (loadpath/mg.py:708-754). False when singular."""
        if lv is self.levels[0]:
            self._coarse = None
            return True
        g = lv.grid
        n = 3 * g.NX * g.NY * g.NZ
        if n > DENSE_COARSE_MAX:
            self._coarse = None
            return True
        L = lib()
        st = stream_handle()
        dt = self.tdtype
        sfx = "f32" if dt == torch.float32 else "f64"
        a = torch.empty((n, n), dtype=torch.float64, device=self.device)
        if lv.kind == "weights":
            getattr(L, f"lpb_coarse_dense_{sfx}")(a.data_ptr(), 1, lv.w.data_ptr(), lv.mcat.data_ptr(),
                                                  ptr(lv.patch_id), ptr(lv.patch_k), None, lv.mask.data_ptr(),
                                                  *g.args, st)
        else:
            getattr(L, f"lpb_coarse_dense_{sfx}")(a.data_ptr(), 2, None, None, None, None, lv.k.data_ptr(),
                                                  lv.mask.data_ptr(), *g.args, st)
        # the dense inverse on the device, once per hierarchy (cuSOLVER potrf + potri); the
        # V-cycle applies it with this package's GEMV kernel
        lw = int(L.lpb_coarse_inverse_work(n))
        work = self._flat_buf("coarse_work", lw, torch.float64)
        info = self._flat_buf("coarse_info", 2, torch.int32)
        L.lpb_coarse_inverse(a.data_ptr(), n, work.data_ptr(), lw, info.data_ptr(), st)
        if bool((info[:2] != 0).any().item()):
            return False
        self._coarse = {"ainv": a, "v": torch.zeros(n, dtype=torch.float64, device=self.device), "n": n}
        return True

    def _op(self, i):
        return self._l0s if i == 0 else self.levels[i]

    def _estimate_lmax(self, i, its=12):
        """Largest eigenvalue of D^-1 A by power iteration, times 1.3 (loadpath/mg.py:771-794)."""
        L = lib()
        st = stream_handle()
        lv = self._op(i)
        g = lv.grid
        dt = lv.dtype
        sfx = "f32" if dt == torch.float32 else "f64"
        v = self._buf(f"pw_v{i}", g, dt)
        av = self._buf(f"pw_av{i}", g, dt)
        prev = self._lmax_vec.get(i)
        if prev is not None and prev.shape == v.shape and prev.dtype == dt:
            src = prev
        else:
            rng = np.random.default_rng(i)
            host = (rng.random(lv.node_shape) - 0.5).astype(np.float32 if dt == torch.float32 else np.float64)
            src = g.nodes_to_dev(host, dt)
        getattr(L, f"lpb_mask_field_{sfx}")(v.data_ptr(), src.data_ptr(), lv.mask.data_ptr(), *g.args, 0, st)
        n = g.n_node_field
        sc = self._scal
        for it in range(its):
            getattr(L, f"lpb_dot_{sfx}")(v.data_ptr(), v.data_ptr(), n, self._part.data_ptr(),
                                         sc[it].data_ptr(), st)
            getattr(L, f"lpb_scale_rsqrt_{sfx}")(v.data_ptr(), n, sc[it].data_ptr(), st)
            lv.apply(av, v)
            getattr(L, f"lpb_dinv_mask_{sfx}")(av.data_ptr(), lv.dinv.data_ptr(), lv.mask.data_ptr(), *g.args, st)
            getattr(L, f"lpb_dot_{sfx}")(v.data_ptr(), av.data_ptr(), n, self._part.data_ptr(),
                                         sc[16 + it].data_ptr(), st)
            v, av = av, v
        vals = sc[:32].cpu().numpy()
        self._lmax_vec[i] = v.clone()
        if np.any(vals[:its] == 0):
            return 2.0
        return LMAX_SAFETY * max(float(vals[16 + its - 1]), 1e-12)

    # --- V-cycle (loadpath/mg.py:796-864) -----------------------------------------------
    def _smooth(self, i, b, x, from_zero):
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
        hi = lv.lmax
        lo = hi / 30.0
        theta = 0.5 * (hi + lo)
        delta = 0.5 * (hi - lo)
        sigma = theta / delta
        rho = 1.0 / sigma
        if from_zero:
            getattr(L, f"lpb_cheb_start_{sfx}")(b.data_ptr(), lv.dinv.data_ptr(), 1.0 / theta, x.data_ptr(),
                                                r.data_ptr(), d.data_ptr(), n, st)
        else:
            lv.apply(t, x)
            getattr(L, f"lpb_residual_scaled_{sfx}")(b.data_ptr(), t.data_ptr(), lv.dinv.data_ptr(), 1.0 / theta,
                                                     r.data_ptr(), d.data_ptr(), n, st)
        for it in range(self.degree):
            last = it + 1 == self.degree
            if not last:
                lv.apply(t, d)
            rho_new = 1.0 / (2.0 * sigma - rho)
            getattr(L, f"lpb_cheb_{sfx}")(x.data_ptr(), d.data_ptr(), r.data_ptr(), (d if last else t).data_ptr(),
                                          lv.dinv.data_ptr(), rho_new * rho, 2.0 * rho_new / delta, int(last), n, st)
            rho = rho_new
        return x

    def _vcycle(self, i, b):
        """x = V(b) on level i; b and the result live in level-i buffers."""
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
                getattr(L, f"lpb_coarse_solve_{sfx}")(x.data_ptr(), b.data_ptr(), c["ainv"].data_ptr(),
                                                      c["v"].data_ptr(), *g.args, st)
                return x
            self._smooth(i, b, x, True)
            return self._smooth(i, b, x, False)
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
        return self._smooth(i, b, x, False)

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

    def _pcg_device(self, b, x0):
        """float64 PCG on padded device fields. Returns (x, iterations, converged)."""
        L = lib()
        st = stream_handle()
        g = self.g0
        n = g.n_node_field
        a = self.levels[0]
        sc = self._scal
        x = self._buf("cg_x", g, torch.float64)
        r = self._buf("cg_r", g, torch.float64)
        p = self._buf("cg_p", g, torch.float64)
        ap = self._buf("cg_ap", g, torch.float64)
        z = self._buf("cg_z", g, torch.float64)
        self._dot64(b, b, 0)
        bnorm = math.sqrt(float(sc[0].item()))
        if bnorm == 0:
            x.zero_()
            return x, 0, True
        r.copy_(b)
        if x0 is not None:
            x.copy_(x0)
            a.apply(ap, x)
            self._dot64(x, ap, 5)
            self._dot64(b, x, 6)
            xax, bx = (float(v) for v in sc[5:7].cpu().numpy())
            s = bx / xax if xax > 0 else 0.0
            if s > 0:
                L.lpb_axpby_f64(z.data_ptr(), 1.0, b.data_ptr(), -s, ap.data_ptr(), n, st)
                self._dot64(z, z, 7)
                if math.sqrt(float(sc[7].item())) < bnorm:
                    L.lpb_axpby_f64(x.data_ptr(), s, x.data_ptr(), 0.0, None, n, st)
                    r.copy_(z)
                else:
                    x.zero_()
            else:
                x.zero_()
        else:
            x.zero_()
        self.precondition_device(r, z)
        p.copy_(z)
        self._dot64(r, z, 1)
        tol = self.rtol * bnorm
        r32 = self._buf("cg_r32", g, torch.float32) if self.tdtype == torch.float32 else None
        host = self._host

        def head():
            # ap = A p; pap; x += alpha p; r -= alpha ap (and its float32 copy); |r|^2; scalars out
            a.apply(ap, p)
            self._dot64(p, ap, 3)
            L.lpb_cg_step(x.data_ptr(), r.data_ptr(), p.data_ptr(), ap.data_ptr(), ptr(r32), n,
                          sc[1].data_ptr(), sc[3].data_ptr(), self._part.data_ptr(), sc[4].data_ptr(),
                          stream_handle())
            L.lpb_memcpy_async(host.data_ptr(), sc[3:5].data_ptr(), 16, stream_handle())

        def tail():
            # z = V(r); rz_new; p = z + (rz_new / rz) p; rz = rz_new
            if r32 is not None:
                xv = self._vcycle(0, r32)
                L.lpb_dot_f64_f32(r.data_ptr(), xv.data_ptr(), n, self._part.data_ptr(), sc[2].data_ptr(),
                                  stream_handle())
                L.lpb_xpby_f32(p.data_ptr(), xv.data_ptr(), n, sc[2].data_ptr(), sc[1].data_ptr(), stream_handle())
            else:
                self.precondition_device(r, z)
                self._dot64(r, z, 2)
                L.lpb_xpby_f64(p.data_ptr(), z.data_ptr(), n, sc[2].data_ptr(), sc[1].data_ptr(), stream_handle())
            L.lpb_memcpy_async(sc[1:2].data_ptr(), sc[2:3].data_ptr(), 8, stream_handle())

        graphs = None
        probe = _PROBE[0]
        gpairs = [[], []]
        if self.use_graphs and self.maxiter > 1:
            # one capture per solve: buffers and smoother coefficients are fixed within it
            self._free_graphs()
            graphs = []
            # captured on a side stream (the legacy default stream cannot be captured), launched
            # on the working stream
            for gi, fn in enumerate((head, tail)):
                if probe is not None:
                    probe.capture = gpairs[gi]
                with torch.cuda.stream(self._cap_stream):
                    st0 = stream_handle()
                    L.lpb_capture_begin(st0)
                    try:
                        fn()
                    finally:
                        exec_ = ctypes.c_void_p()
                        L.lpb_capture_end(st0, ctypes.byref(exec_))
                        if probe is not None:
                            probe.capture = None
                graphs.append(exec_)
            self._graphs = graphs      # freed at the next capture
        ev = torch.cuda.Event()

        def finish(result):
            if graphs is not None and probe is not None:
                torch.cuda.current_stream().synchronize()
                probe.harvest(gpairs[1])          # the last (speculative) tail replay
            return result

        for it in range(1, self.maxiter + 1):
            if graphs is not None:
                L.lpb_graph_launch(graphs[0], stream_handle())
            else:
                head()
            ev.record()
            # the next preconditioner step is queued before the host looks at |r|: the
            # device never waits on the convergence test (a converged solve discards it)
            if graphs is not None:
                L.lpb_graph_launch(graphs[1], stream_handle())
            else:
                tail()
            ev.synchronize()
            if graphs is not None and probe is not None:
                # this head replay is complete and the next is not launched yet; a tail replay
                # may be re-recording its events now, so tails are read once, at the end
                probe.harvest(gpairs[0])
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
        bm = self._buf("solve_b", g, torch.float64)
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
        m = self.levels[0].mask[:, :, :self.g0.NZ].cpu().numpy()
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
        if self._graphs:
            torch.cuda.current_stream().synchronize()
            for gexec in self._graphs:
                lib().lpb_graph_free(gexec)
        self._graphs = None

    def __del__(self):
        try:
            self._free_graphs()
        except Exception:
            pass

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
