"""The reference's `mgops` call surface (loadpath/mgops.py) on host numpy arrays, computed on the
device.

loadpath's solver calls these helpers on numpy node grids (3, X+1, Y+1, Z+1) and cell data of
one dtype; each returns what the reference's returns (an array, a bool, or the in-place update
of `out`). Here every call copies its inputs to the device, runs this package's kernels and copies
the result back: a drop-in with the reference's argument meaning for callers that hold host
arrays (and the functions the parity tests call). The solver itself (`mg.GridElasticity`) keeps
its fields on the device and never goes through this module.

`available()` is the reference's feature gate: True when the CUDA library and a device are
there (and LOADPATH_MGOPS is not "numpy"); there is no host fallback inside this module.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from ._lib import lib
from .grid import DevGrid, stream_handle

__all__ = ["available", "Cells", "apply_masked", "apply_scaled", "apply_weights", "apply_explicit", "cast", "dot",
           "coarse_residual", "add_correction", "prolong", "restrict"]


def available():
    if os.environ.get("LOADPATH_MGOPS", "").lower() == "numpy" or not torch.cuda.is_available():
        return False
    try:
        lib()
    except Exception:  # noqa: BLE001 - a missing library means "not available", as the reference's gate
        return False
    return True


class Cells:
    """The cells of a level that carry stiffness, with the fields the reference's callers read
    (loadpath/mgops.py:220-244):

    - cells: (n, 3) int64, the (x, y, z) of each listed cell, x-major (C order of the grid);
    - n: their count; rows: an int64 grid, a listed cell's position in `cells`, -1 elsewhere;
    - base: (n,) the flat index of each cell's low corner in the node grid (X+1, Y+1, Z+1);
    - off: (24,) the flat offset of element dof 3k + d from `base` in a (3, X+1, Y+1, Z+1) field:
      component d's plane plus corner k's step, bit a of k stepping along axis a;
    - ft(dtype): a (24, n) work array kept per dtype."""

    def __init__(self, active: np.ndarray):
        self.active = np.asarray(active, bool)
        shape = self.active.shape
        listed = np.flatnonzero(self.active)
        self.n = int(listed.size)
        self.cells = np.ascontiguousarray(np.column_stack(np.unravel_index(listed, shape)), np.int64)
        rows = np.full(self.active.size, -1, np.int64)
        rows[listed] = np.arange(self.n, dtype=np.int64)
        self.rows = rows.reshape(shape)
        nodes = np.array(shape, np.int64) + 1
        stride = np.array([nodes[1] * nodes[2], nodes[2], 1], np.int64)
        self.base = np.ascontiguousarray(self.cells @ stride)
        bits = (np.arange(8)[:, None] >> np.arange(3)[None, :]) & 1
        plane = int(np.prod(nodes)) * np.arange(3, dtype=np.int64)
        self.off = np.ascontiguousarray((bits @ stride)[:, None] + plane[None, :]).reshape(24)
        self._work = {}

    def ft(self, dtype):
        dtype = np.dtype(dtype)
        if dtype not in self._work:
            self._work[dtype] = np.empty((24, self.n), dtype)
        return self._work[dtype]


def _sfx(dtype):
    dtype = np.dtype(dtype)
    if dtype == np.float32:
        return "f32", torch.float32
    if dtype == np.float64:
        return "f64", torch.float64
    raise TypeError(f"mgops works on float32 or float64 fields, not {dtype}")


def _grid_of(u):
    if u.ndim != 4 or u.shape[0] != 3:
        raise ValueError(f"a node field is (3, X+1, Y+1, Z+1), got {u.shape}")
    return DevGrid(tuple(int(n) - 1 for n in u.shape[1:]))


def _mask_dev(g, m):
    """a float 0/1 mask (3, nodes...) -> the byte mask (bit c: component c solved)."""
    bits = np.zeros(g.node_shape[1:], np.uint8)
    for c in range(3):
        bits |= (np.asarray(m[c]) != 0).astype(np.uint8) << c
    t = g.mask_field()
    return g.set_nodes(t, torch.from_numpy(bits))


def _cells_to_dev(g, cells, values, dtype):
    """per-listed-cell values (n,) -> a device cell field (zero where no cell is listed)."""
    full = np.zeros(g.cells, dtype)
    full[tuple(cells.cells.T)] = values
    return g.cells_to_dev(full, torch.float32 if dtype == np.float32 else torch.float64)


def _cell_rows_to_dev(g, cells, rows, dtype):
    """(r, n) per-listed-cell rows -> (r, padded cells) device rows in the cell layout."""
    out = torch.zeros((rows.shape[0], g.n_cell_field), dtype=_sfx(dtype)[1], device=g.device)
    for i in range(rows.shape[0]):
        out[i].copy_(_cells_to_dev(g, cells, rows[i], dtype).reshape(-1))
    return out


def _cell_matrices_to_dev(g, cells, k_c, dtype):
    """(24, 24, n) matrices -> (padded cells, 576) device, cell-major in the cell layout."""
    full = np.zeros(tuple(g.cells) + (576,), dtype)
    full[tuple(cells.cells.T)] = np.moveaxis(np.asarray(k_c, dtype).reshape(576, -1), 0, 1)
    pad = np.zeros((g.nx, g.ny, g.cpz, 576), dtype)
    pad[:, :, :g.nz] = full
    t = torch.from_numpy(pad).to(g.device)
    t = t.view(g.nx, g.ny, g.cpz // 4, 4, 576).permute(2, 1, 0, 3, 4).reshape(-1, 576).contiguous()
    return t


def _apply(kind, u, a, b, cells, m, finish, acc=None):
    """the level operator on host arrays; acc: a host field the result is added to (on the
    device) instead of returned alone"""
    sfx, tdt = _sfx(u.dtype)
    g = _grid_of(u)
    L = lib()
    st = stream_handle()
    ud = g.nodes_to_dev(np.asarray(u), tdt)
    md = _mask_dev(g, m) if m is not None else _mask_dev(g, np.ones_like(u))
    out = g.node_field(tdt)
    mask_in = int(m is not None)
    if kind == "scaled":
        ke = torch.as_tensor(np.asarray(a, u.dtype), device=g.device)
        e = _cells_to_dev(g, cells, np.asarray(b, u.dtype), u.dtype)
        getattr(L, f"lpb_apply_scaled_{sfx}")(out.data_ptr(), ud.data_ptr(), e.data_ptr(), md.data_ptr(),
                                               ke.data_ptr(), *g.args, mask_in, int(finish), st)
    elif kind == "weights":
        mk = torch.as_tensor(np.asarray(a, u.dtype).reshape(8, 576), device=g.device)
        w = _cell_rows_to_dev(g, cells, np.asarray(b, u.dtype).reshape(8, -1), u.dtype)
        getattr(L, f"lpb_apply_weights_{sfx}")(out.data_ptr(), ud.data_ptr(), w.data_ptr(), mk.data_ptr(), None,
                                                None, md.data_ptr(), *g.args, mask_in, int(finish), st)
    elif kind == "explicit":
        k = _cell_matrices_to_dev(g, cells, a, u.dtype)
        getattr(L, f"lpb_apply_explicit_{sfx}")(out.data_ptr(), ud.data_ptr(), k.data_ptr(), md.data_ptr(),
                                                 *g.args, mask_in, int(finish), st)
    else:
        raise ValueError(f"unknown level kind {kind!r}")
    if acc is not None:
        accd = g.nodes_to_dev(np.asarray(acc), tdt)
        getattr(L, f"lpb_axpby_{sfx}")(accd.data_ptr(), 1.0, accd.data_ptr(), 1.0, out.data_ptr(), accd.numel(), st)
        out = accd
    return g.nodes_to_host(out)


def apply_masked(kind, u, a, b, cells: Cells, m, out, finish):
    """K (u * m) into `out` (u, m, out: (3, nodes...) of one dtype); with `finish` also
    out = out * m + (1 - m) * u (loadpath/mgops.py:247-264). kind "scaled": a = ke (24, 24),
    b = the listed cells' moduli; "weights": a = the eight (24, 24) matrices, b = (8, n) weights;
    "explicit": a = (24, 24, n) cell matrices."""
    out[...] = _apply(kind, u, a, b, cells, m, finish)
    return out


def apply_scaled(u, ke, e_c, cells: Cells, out):
    """out += sum over the listed cells of e_c[cell] ke u[cell corners] (loadpath/mgops.py:274-279)."""
    out[...] = _apply("scaled", u, ke, e_c, cells, None, False, acc=out)
    return out


def apply_weights(u, mk, w_c, cells: Cells, out):
    """out += sum over cells of (sum_q w_c[q, cell] M_q) u[cell corners] (loadpath/mgops.py:282-287)."""
    out[...] = _apply("weights", u, mk, w_c, cells, None, False, acc=out)
    return out


def apply_explicit(u, k_c, cells: Cells, out):
    """out += sum over cells of K[cell] u[cell corners] (loadpath/mgops.py:290-295)."""
    out[...] = _apply("explicit", u, k_c, None, cells, None, False, acc=out)
    return out


def cast(a, dtype):
    """a.astype(dtype), the conversion on the device (loadpath/mgops.py:564-575)."""
    dtype = np.dtype(dtype)
    a = np.asarray(a)
    if a.dtype == dtype:
        return a.copy()
    if {a.dtype, dtype} != {np.dtype(np.float32), np.dtype(np.float64)}:
        return a.astype(dtype)
    L = lib()
    src = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    out = torch.empty(src.shape, dtype=_sfx(dtype)[1], device="cuda")
    if dtype == np.float32:
        L.lpb_cast_f64_f32(out.data_ptr(), src.data_ptr(), src.numel(), stream_handle())
    else:
        L.lpb_cast_f32_f64(out.data_ptr(), src.data_ptr(), src.numel(), stream_handle())
    return out.cpu().numpy()


def dot(a, b) -> float:
    """The dot product of two same-shape fields, a float64 device reduction
    (loadpath/mgops.py:578-585)."""
    ad = torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()
    bd = torch.from_numpy(np.ascontiguousarray(b, np.float64)).cuda()
    part = torch.zeros(lib().lpb_reduce_blocks() * 2, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib().lpb_dot_f64(ad.data_ptr(), bd.data_ptr(), ad.numel(), part.data_ptr(), out.data_ptr(), stream_handle())
    return float(out.item())


def coarse_residual(b, ax, m, cm, coarse_shape):
    """restrict(((b - ax) * m) zero-padded) * cm onto coarse_shape (loadpath/mgops.py:753-763)."""
    if not (b.dtype == ax.dtype == m.dtype == cm.dtype):
        return None
    sfx, tdt = _sfx(b.dtype)
    gf = _grid_of(b)
    gc = DevGrid(tuple(int(n) - 1 for n in coarse_shape[1:]))
    st = stream_handle()
    bd, axd = gf.nodes_to_dev(np.asarray(b), tdt), gf.nodes_to_dev(np.asarray(ax), tdt)
    md, cmd = _mask_dev(gf, m), _mask_dev(gc, cm)
    rc = gc.node_field(tdt)
    getattr(lib(), f"lpb_restrict_residual_{sfx}")(rc.data_ptr(), bd.data_ptr(), axd.data_ptr(), md.data_ptr(),
                                                   cmd.data_ptr(), *gf.args, *gc.args, st)
    return gc.nodes_to_host(rc)


def add_correction(xc, cm, m, x) -> bool:
    """x += prolong(xc * cm)[:, :x's nodes] * m in place (loadpath/mgops.py:766-773)."""
    if not (xc.dtype == cm.dtype == m.dtype == x.dtype):
        return False
    sfx, tdt = _sfx(x.dtype)
    gf, gc = _grid_of(x), _grid_of(xc)
    st = stream_handle()
    xd, xcd = gf.nodes_to_dev(np.asarray(x), tdt), gc.nodes_to_dev(np.asarray(xc), tdt)
    md, cmd = _mask_dev(gf, m), _mask_dev(gc, cm)
    getattr(lib(), f"lpb_prolong_add_{sfx}")(xd.data_ptr(), xcd.data_ptr(), cmd.data_ptr(), md.data_ptr(), *gf.args,
                                              *gc.args, st)
    x[...] = gf.nodes_to_host(xd)
    return True


def prolong(c):
    """mg.prolong of a (3, nodes...) field (loadpath/mgops.py:776-782): trilinear, the fine grid
    2n - 1 nodes per axis."""
    c = np.asarray(c)
    fine = np.zeros((3,) + tuple(2 * n - 1 for n in c.shape[1:]), c.dtype)
    ones_c, ones_f = np.ones_like(c), np.ones_like(fine)
    add_correction(c, ones_c, ones_f, fine)
    return fine


def restrict(f):
    """mg.restrict of a (3, nodes...) field (loadpath/mgops.py:785-791): full weighting onto
    (n + 1) // 2 nodes per axis. An axis of odd cell count is padded with a zero node plane (the
    kernels take a coarse grid of ceil(cells / 2) cells) and the extra coarse plane dropped."""
    f = np.asarray(f)
    want = (3,) + tuple((n + 1) // 2 for n in f.shape[1:])
    fp = np.zeros((3,) + tuple(n + (1 - n % 2) for n in f.shape[1:]), f.dtype)   # odd node counts
    fp[:, :f.shape[1], :f.shape[2], :f.shape[3]] = f
    shape = (3,) + tuple((n + 1) // 2 for n in fp.shape[1:])
    z = np.zeros_like(fp)
    out = coarse_residual(fp, z, np.ones_like(fp), np.ones(shape, f.dtype), shape)
    return np.ascontiguousarray(out[:, :want[1], :want[2], :want[3]])
