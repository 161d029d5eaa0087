"""CPU restatement (numpy, float64 / float32) of loadpath's voxel SIMP inner loop.

TEST INFRASTRUCTURE ONLY. This module is the oracle the CUDA path is checked
against: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
may import it, and only as the checker. The product package (loadpath_b200)
never imports it and has no CPU fallback.

Pinning: every function below is checked against golden vectors produced by
the reference implementation itself (tests/golden/make_golden.py imports
loadpath read-only and writes tests/golden/*.npz; tests/test_oracle_golden.py
compares). Each function names the reference file:line whose algorithm it
restates (paths are relative to the loadpath project root).

Layouts follow the reference:
- corner k of a cell sits at (k & 1, k >> 1 & 1, k >> 2 & 1)   (loadpath/fem.py:30)
- node fields are (3, nx+1, ny+1, nz+1), component-major, C order (loadpath/mg.py:495-511)
- cell fields are (nx, ny, nz)
- a cell's 24 dofs are ordered 3 * corner + component          (loadpath/fem.py:127-145)
"""
from __future__ import annotations

import numpy as np

CORNERS = np.array([[(k >> 0) & 1, (k >> 1) & 1, (k >> 2) & 1] for k in range(8)])
OFFS = [tuple(int(v) for v in c) for c in CORNERS]
LMAX_SAFETY = 1.3          # loadpath/mg.py:81
STALL = 100                # loadpath/mg.py:930


# --------------------------------------------------------------------------
# element (loadpath/fem.py:113-224)
# --------------------------------------------------------------------------

def elastic_c(nu: float) -> np.ndarray:
    """Isotropic 6x6 elasticity at E = 1, engineering shear (loadpath/fem.py:113-124)."""
    lam = nu / ((1 + nu) * (1 - 2 * nu))
    mu = 1.0 / (2 * (1 + nu))
    c = np.zeros((6, 6))
    c[:3, :3] = lam
    for i in range(3):
        c[i, i] = lam + 2 * mu
        c[3 + i, 3 + i] = mu
    return c


def _strain_rows(b, col, g):
    """Fill the six strain rows for one displacement basis function whose
    gradient is g = (gx, gy, gz); shear order xy, yz, zx (loadpath/fem.py:40)."""
    gx, gy, gz = g
    b[0, col] = gx
    b[1, col + 1] = gy
    b[2, col + 2] = gz
    b[3, col] = gy
    b[3, col + 1] = gx
    b[4, col + 1] = gz
    b[4, col + 2] = gy
    b[5, col] = gz
    b[5, col + 2] = gx


def b_matrix(xi, eta, zeta) -> np.ndarray:
    """6x24 strain-displacement of the unit cube at a natural point (loadpath/fem.py:127-145)."""
    s = 2.0 * CORNERS - 1.0
    b = np.zeros((6, 24))
    for k in range(8):
        gx = 0.25 * s[k, 0] * (1 + eta * s[k, 1]) * (1 + zeta * s[k, 2])
        gy = 0.25 * s[k, 1] * (1 + xi * s[k, 0]) * (1 + zeta * s[k, 2])
        gz = 0.25 * s[k, 2] * (1 + xi * s[k, 0]) * (1 + eta * s[k, 1])
        _strain_rows(b, 3 * k, (gx, gy, gz))
    return b


def b_bubble(xi, eta, zeta) -> np.ndarray:
    """6x9 strain of Wilson's incompatible modes (1 - x_m^2) (loadpath/fem.py:172-188)."""
    x = (xi, eta, zeta)
    b = np.zeros((6, 9))
    for m in range(3):
        g = [0.0, 0.0, 0.0]
        g[m] = -4.0 * x[m]
        _strain_rows(b, 3 * m, g)
    return b


def hex8_ke(nu: float, element: str = "im") -> np.ndarray:
    """Unit-cube stiffness at E = 1 with 2x2x2 Gauss; "im" condenses the nine
    bubble modes, "plain" is the trilinear brick; symmetrised
    (loadpath/fem.py:191-224)."""
    c = elastic_c(nu)
    g = 1.0 / np.sqrt(3.0)
    kuu = np.zeros((24, 24))
    kua = np.zeros((24, 9))
    kaa = np.zeros((9, 9))
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                b = b_matrix(xi, eta, zeta)
                ba = b_bubble(xi, eta, zeta)
                kuu += b.T @ c @ b * 0.125
                kua += b.T @ c @ ba * 0.125
                kaa += ba.T @ c @ ba * 0.125
    if element == "plain":
        k = kuu
    elif element == "im":
        k = kuu - kua @ np.linalg.solve(kaa, kua.T)
    else:
        raise ValueError(element)
    return 0.5 * (k + k.T)


# --------------------------------------------------------------------------
# grid transfers (loadpath/mg.py:57-132)
# --------------------------------------------------------------------------

def child_prolongations() -> np.ndarray:
    """P_k (8, 24, 24): coarse-cell dofs -> dofs of the child at CORNERS[k]
    (loadpath/mg.py:57-75)."""
    out = np.zeros((8, 24, 24))
    for k in range(8):
        for q in range(8):
            pos = (CORNERS[k] + CORNERS[q]) / 2.0
            for r in range(8):
                w = np.prod(np.where(CORNERS[r] == 1, pos, 1.0 - pos))
                if w:
                    for i in range(3):
                        out[k, 3 * q + i, 3 * r + i] = w
    return out


PK = child_prolongations()


def prolong(c: np.ndarray) -> np.ndarray:
    """Trilinear (..., n0, n1, n2) -> (..., 2n0-1, 2n1-1, 2n2-1) (loadpath/mg.py:84-108)."""
    out = c
    for ax in (-3, -2, -1):
        out = np.moveaxis(out, ax, 0)
        n = out.shape[0]
        f = np.empty((2 * n - 1,) + out.shape[1:], out.dtype)
        f[0::2] = out
        f[1::2] = (out[:-1] + out[1:]) * out.dtype.type(0.5)
        out = np.moveaxis(f, 0, ax)
    return np.ascontiguousarray(out)


def restrict(f: np.ndarray) -> np.ndarray:
    """Transpose of prolong (loadpath/mg.py:111-132)."""
    out = f
    for ax in (-3, -2, -1):
        out = np.moveaxis(out, ax, 0)
        n = (out.shape[0] + 1) // 2
        c = out[0::2].copy()
        half = out[1::2] * out.dtype.type(0.5)
        c[:n - 1] += half
        c[1:n] += half
        out = np.moveaxis(c, 0, ax)
    return np.ascontiguousarray(out)


def restrict_masked_residual(b, ax, m, cm, coarse_shape):
    """restrict(((b - ax) * m) zero-padded to twice the coarse cells) * cm
    (loadpath/mgops.py:753-763, with :666-711)."""
    rf = np.zeros((3,) + tuple(2 * n - 1 for n in coarse_shape[1:]), b.dtype)
    sx, sy, sz = b.shape[1:]
    rf[:, :sx, :sy, :sz] = (b - ax) * m
    return restrict(rf) * cm


def prolong_add(xc, cm, m, x):
    """x += prolong(xc * cm)[:, :x's nodes] * m (loadpath/mgops.py:766-773)."""
    sx, sy, sz = x.shape[1:]
    x += prolong(xc * cm)[:, :sx, :sy, :sz] * m
    return x


# --------------------------------------------------------------------------
# levels and operators (loadpath/mg.py:174-387)
# --------------------------------------------------------------------------

def gather_cells(u, dims):
    """(24, nx, ny, nz): the 24 corner dofs of every cell of a node field."""
    nx, ny, nz = dims
    out = np.empty((24, nx, ny, nz), u.dtype)
    for k, (dx, dy, dz) in enumerate(OFFS):
        out[3 * k:3 * k + 3] = u[:, dx:dx + nx, dy:dy + ny, dz:dz + nz]
    return out


def scatter_cells(f, out):
    """out += f (24, cells) at every cell's corners."""
    nx, ny, nz = f.shape[1:]
    for k, (dx, dy, dz) in enumerate(OFFS):
        out[:, dx:dx + nx, dy:dy + ny, dz:dz + nz] += f[3 * k:3 * k + 3]
    return out


def prolong_rows(fine_ijk, coarse_node_shape):
    """Scalar trilinear prolongation rows (len(fine_ijk), coarse nodes) for the given fine nodes
    (loadpath/mg.py:390-408): an odd index lies halfway between two coarse nodes (0.5 each), an
    even one on its coarse node (1)."""
    import scipy.sparse as sp

    n = len(fine_ijk)
    rows, cols, vals = [], [], []
    for corner in range(8):
        w = np.ones(n)
        ci = np.empty((n, 3), np.int64)
        for d in range(3):
            i = fine_ijk[:, d]
            odd = i % 2 == 1
            hi = (corner >> d) & 1
            ci[:, d] = i // 2 + (hi & odd)
            w *= np.where(odd, 0.5, 1.0 if not hi else 0.0)
        ok = w > 0
        rows.append(np.nonzero(ok)[0])
        cols.append(np.ravel_multi_index(tuple(ci[ok].T), coarse_node_shape))
        vals.append(w[ok])
    nc = int(np.prod(coarse_node_shape))
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, nc))


def coarse_extra(fine, cdims, mask_fine):
    """The fine level's extra operator S carried to the coarse level as P^T S P, P the trilinear
    prolongation of the dofs S touches, each row times the fine mask at the first coarsening
    (loadpath/mg.py:679-706). None without an extra operator."""
    import scipy.sparse as sp

    s = fine.extra
    if s is None or s.nnz == 0:
        return None
    nshape_f = fine.node_shape[1:]
    nshape_c = tuple(c + 1 for c in cdims)
    nn_f, nn_c = int(np.prod(nshape_f)), int(np.prod(nshape_c))
    s = s.tocsr()
    mark = np.zeros(s.shape[0], bool)
    mark[s.indices] = True
    mark[np.diff(s.indptr) > 0] = True
    dofs = np.flatnonzero(mark)
    comp, node = np.divmod(dofs, nn_f)
    ijk = np.stack(np.unravel_index(node, nshape_f), axis=1)
    pr = prolong_rows(ijk, nshape_c).tocoo()
    cols = comp[pr.row] * nn_c + pr.col
    vals = pr.data
    if mask_fine is not None:
        vals = vals * np.asarray(mask_fine).reshape(-1)[dofs[pr.row]]
    p = sp.csr_matrix((vals, (dofs[pr.row], cols)), shape=(s.shape[0], 3 * nn_c))
    return (p.T @ s @ p).tocsr()


def springs_to_grid(springs, node_ijk, node_shape):
    """A sparse operator in mesh dof numbering (3 node + component) on the flat (3, nodes) grid
    dofs (component nn + node) of a node grid of shape node_shape (loadpath/mg.py:475-513)."""
    import scipy.sparse as sp

    nn = int(np.prod(node_shape))
    flat = np.ravel_multi_index(tuple(np.asarray(node_ijk).T), node_shape)
    g = np.empty(3 * len(flat), np.int64)
    for i in range(3):
        g[i::3] = i * nn + flat
    c = springs.tocoo()
    return sp.csr_matrix((c.data, (g[c.row], g[c.col])), shape=(3 * nn, 3 * nn))


class Level:
    """One grid level (loadpath/mg.py:174-199).

    kind "scaled": cell matrix e[c] * ke.  kind "weights": sum_k w[k, c] M_k
    plus an explicit patch (patch_ijk, patch_k).  kind "explicit": k (24, 24,
    cells).  The operator is mask * K * mask + (1 - mask)."""

    def __init__(self, kind, dims, dtype):
        self.kind = kind
        self.dims = tuple(int(d) for d in dims)
        self.dtype = np.dtype(dtype)
        self.ke = self.e = self.mcat = self.w = None
        self.patch_ijk = self.patch_k = self.k = None
        self.mask = self.dinv = self.lmax = None
        self.extra = None   # a sparse operator on the flat (3, nodes) dofs, added to K (springs)

    @property
    def node_shape(self):
        return (3,) + tuple(d + 1 for d in self.dims)

    def cell_products(self, cells24):
        """(24, cells) products of every cell's matrix with its gathered dofs
        (loadpath/mg.py:213-230)."""
        flat = cells24.reshape(24, -1)
        if self.kind == "scaled":
            f = (self.ke.astype(flat.dtype) @ flat) * self.e.reshape(1, -1).astype(flat.dtype)
        elif self.kind == "weights":
            g = (self.mcat.astype(flat.dtype) @ flat).reshape(8, 24, -1)
            w = self.w.reshape(8, 1, -1).astype(flat.dtype)
            f = (g * w).sum(axis=0)
        else:
            kk = self.k.reshape(24, 24, -1).astype(flat.dtype)
            f = np.einsum("ijn,jn->in", kk, flat)
        return f.reshape(cells24.shape)

    def patch_index(self):
        """(npatch, 24) flat (3, nodes) indices of patch cells' dofs (loadpath/mg.py:299-309)."""
        nshape = self.node_shape[1:]
        nn = int(np.prod(nshape))
        idx = np.empty((len(self.patch_ijk), 24), np.int64)
        for k, off in enumerate(OFFS):
            node = np.ravel_multi_index(tuple((self.patch_ijk + np.array(off)).T), nshape)
            for i in range(3):
                idx[:, 3 * k + i] = i * nn + node
        return idx

    def apply_k(self, u):
        """Unmasked K u (loadpath/mg.py:251-276)."""
        out = np.zeros(self.node_shape, u.dtype)
        scatter_cells(self.cell_products(gather_cells(u, self.dims)), out)
        if self.patch_ijk is not None and len(self.patch_ijk):
            idx = self.patch_index()
            fe = np.einsum("nij,nj->ni", self.patch_k.astype(u.dtype), u.reshape(-1)[idx])
            np.add.at(out.reshape(-1), idx.ravel(), fe.ravel())
        if self.extra is not None:
            # (loadpath/mg.py:278-296: the extra operator in float64, added in the level's dtype)
            out += (self.extra @ u.reshape(-1).astype(np.float64)).astype(u.dtype).reshape(out.shape)
        return out

    def apply(self, u):
        """mask * K (mask * u) + (1 - mask) * u (loadpath/mg.py:317-346)."""
        m = self.mask.astype(u.dtype)
        out = self.apply_k(u * m)
        return out * m + (1 - m) * u

    def cell_matrices(self):
        """float64 (24, 24, nx, ny, nz) matrices of every cell (loadpath/mg.py:373-387)."""
        if self.kind == "explicit":
            return self.k.astype(np.float64)
        if self.kind == "scaled":
            return self.ke.astype(np.float64)[:, :, None, None, None] * self.e[None, None].astype(np.float64)
        mk = self.mcat.reshape(8, 576).astype(np.float64)
        out = (mk.T @ self.w.reshape(8, -1).astype(np.float64)).reshape((24, 24) + self.dims)
        if self.patch_ijk is not None and len(self.patch_ijk):
            p = self.patch_ijk
            out[:, :, p[:, 0], p[:, 1], p[:, 2]] += np.moveaxis(self.patch_k.astype(np.float64), 0, -1)
        return out

    def diagonal(self):
        """float64 diagonal of the unmasked K (loadpath/mg.py:348-371)."""
        km = self.cell_matrices()
        dc = np.einsum("iixyz->ixyz", km)
        d = np.zeros(self.node_shape)
        d = scatter_cells(dc, d)
        if self.extra is not None:
            d += self.extra.diagonal().reshape(d.shape)   # loadpath/mg.py:369-370
        return d

    def active(self):
        """Cells with a nonzero matrix outside the patch (loadpath/mg.py:205-211)."""
        if self.kind == "scaled":
            return self.e != 0
        if self.kind == "weights":
            return self.w.any(axis=0)
        return np.einsum("iixyz->xyz", self.k) > 0


# --------------------------------------------------------------------------
# hierarchy (loadpath/mg.py:515-754)
# --------------------------------------------------------------------------

class Hierarchy:
    """GridElasticity's level hierarchy and PCG on a full rectangular grid.

    ke: (24, 24) unit-cube stiffness already multiplied by the pitch
    (loadpath/mg.py:446). fixed_grid: bool (3, nodes). Cells are padded to
    even counts by the caller (loadpath/mg.py:438-442)."""

    def __init__(self, ke, cells, fixed_grid, rtol=1e-6, maxiter=500, coarse_cells=2000, degree=2,
                 dtype=np.float32, lu_max_dofs=60_000, springs=None):
        self.springs = None if springs is None else springs.tocsr()   # on the flat (3, nodes) dofs
        self.ke = np.asarray(ke, np.float64)
        self.cells = tuple(int(c) for c in cells)
        self.fixed_grid = np.asarray(fixed_grid, bool)
        self.rtol, self.maxiter = rtol, maxiter
        self.coarse_cells, self.degree = int(coarse_cells), int(degree)
        self.dtype = np.dtype(dtype)
        self.lu_max_dofs = lu_max_dofs
        self.strict = False
        self.levels = []
        self.coarse = None
        self.lmax_vec = {}
        self.last_iters = 0

    def op(self, i):
        return self.l0s if i == 0 else self.levels[i]

    def set_moduli(self, e_grid):
        """Rebuild every level for cell moduli (loadpath/mg.py:515-591)."""
        e_grid = np.asarray(e_grid, np.float64)
        self.e_grid = e_grid
        dt = self.dtype
        l0 = Level("scaled", self.cells, np.float64)
        l0.ke = self.ke
        l0.e = e_grid
        l0.extra = self.springs
        d0 = l0.diagonal()
        alive = d0 > 1e-300
        l0.mask = (alive & ~self.fixed_grid).astype(np.float64)
        l0.dinv = np.where(l0.mask > 0, 1.0 / np.where(alive, d0, 1.0), 1.0)
        self.alive = alive
        self.levels = [l0]
        s = Level("scaled", self.cells, dt)
        s.ke = self.ke.astype(dt)
        s.e = e_grid.astype(dt)
        s.mask = l0.mask.astype(dt)
        s.dinv = l0.dinv.astype(dt)
        s.extra = self.springs
        self.l0s = s
        fine = l0
        n_active = int((e_grid > 0).sum())
        depth = 0
        held = alive & self.fixed_grid
        while n_active > self.coarse_cells and min(fine.dims) >= 2:
            coarse = self.coarsen(fine, first=(depth == 0))
            depth += 1
            d = coarse.diagonal()
            dmax = float(d.max()) if d.size else 0.0
            live = d > 1e-12 * max(dmax, 1e-300)
            if self.strict:
                hc = np.zeros((3,) + coarse.node_shape[1:], bool)
                inj = held[:, ::2, ::2, ::2]
                hc[:, :inj.shape[1], :inj.shape[2], :inj.shape[3]] = inj[:, :hc.shape[1], :hc.shape[2], :hc.shape[3]]
                held = hc
                kept = np.zeros((3,) + coarse.node_shape[1:])
                r = restrict(np.asarray(fine.mask, np.float64))
                kept[:, :r.shape[1], :r.shape[2], :r.shape[3]] = r[:, :kept.shape[1], :kept.shape[2], :kept.shape[3]]
                live &= ~held & (kept >= 1.0)
            coarse.mask = live.astype(dt)
            coarse.dinv = np.where(live, 1.0 / np.where(live, d, 1.0), 1.0).astype(dt)
            n_active = self.active_cells(coarse)
            self.levels.append(coarse)
            fine = coarse
        try:
            self.build_coarse(self.levels[-1])
        except RuntimeError:                     # "Factor is exactly singular"
            if self.strict:
                raise
            self.strict = True
            return self.set_moduli(e_grid)
        for i in range(len(self.levels)):
            self.op(i).lmax = self.estimate_lmax(i)

    @staticmethod
    def active_cells(lv):
        """(loadpath/mg.py:593-599)"""
        if lv.kind == "weights":
            act = lv.w.any(axis=0)
            if lv.patch_ijk is not None and len(lv.patch_ijk):
                act[tuple(lv.patch_ijk.T)] = True
            return int(act.sum())
        return int(np.abs(lv.k).max(axis=(0, 1)).astype(bool).sum())

    def coarsen(self, fine, first):
        """Galerkin coarse level (loadpath/mg.py:601-677)."""
        dt = self.dtype
        nx, ny, nz = fine.dims
        half = (nx // 2, ny // 2, nz // 2)
        cdims = tuple(h + h % 2 if h > 1 else h for h in half)
        hx, hy, hz = half
        if first:
            held = (1 - fine.mask) * self.alive
            held_node = held.any(axis=0)
            touch = np.zeros(fine.dims, bool)
            for (dx, dy, dz) in OFFS:
                touch |= held_node[dx:dx + nx, dy:dy + ny, dz:dz + nz]
            touch &= fine.e > 0
            w = np.zeros((8,) + cdims)
            ptouch = np.zeros(cdims, bool)
            for k, (a, b, c) in enumerate(OFFS):
                w[k, :hx, :hy, :hz] = fine.e[a::2, b::2, c::2]
                ptouch[:hx, :hy, :hz] |= touch[a::2, b::2, c::2]
            lv = Level("weights", cdims, dt)
            mk = np.einsum("kai,ab,kbj->kij", PK, fine.ke, PK)
            lv.mcat = mk.reshape(8 * 24, 24).astype(dt)
            pij = np.argwhere(ptouch)
            pk = np.zeros((len(pij), 24, 24))
            fm = fine.mask
            for k, (a, b, c) in enumerate(OFFS):
                fi = 2 * pij + np.array([a, b, c])
                ec = fine.e[tuple(fi.T)]
                dm = np.empty((len(pij), 24))
                for q, (qx, qy, qz) in enumerate(OFFS):
                    dm[:, 3 * q:3 * q + 3] = fm[:, fi[:, 0] + qx, fi[:, 1] + qy, fi[:, 2] + qz].T
                kc = ec[:, None, None] * fine.ke[None] * dm[:, :, None] * dm[:, None, :]
                pk += PK[k].T[None] @ kc @ PK[k][None]
            w[:, ptouch] = 0.0
            lv.w = w.astype(dt)
            lv.patch_ijk = pij
            lv.patch_k = pk.astype(dt)
            lv.extra = coarse_extra(fine, cdims, fine.mask)
            return lv
        lv = Level("explicit", cdims, dt)
        k = np.zeros((24, 24) + cdims, dt)
        kf = fine.cell_matrices()
        if self.strict:
            fm = fine.mask
            dm = np.empty((24,) + kf.shape[2:])
            for q, (qx, qy, qz) in enumerate(OFFS):
                dm[3 * q:3 * q + 3] = fm[:, qx:qx + nx, qy:qy + ny, qz:qz + nz]
            kf = kf * dm[:, None] * dm[None, :]
        for ch, (ox, oy, oz) in enumerate(OFFS):
            sub = kf[:, :, ox::2, oy::2, oz::2]
            shp = sub.shape[2:]
            t = np.einsum("ai,abn,bj->ijn", PK[ch], sub.reshape(24, 24, -1), PK[ch])
            k[:, :, :shp[0], :shp[1], :shp[2]] += t.reshape((24, 24) + shp).astype(dt)
        lv.k = k
        lv.extra = coarse_extra(fine, cdims, None)
        return lv

    def build_coarse(self, lv):
        """Assemble the coarsest level over the dofs of its active cells, as
        D K D + (I - D), symmetrised, and factor it (loadpath/mg.py:708-754)
        with the reference's own call: SuperLU in symmetric mode without pivoting
        (scipy.sparse.linalg.splu, MMD_AT_PLUS_A, diag_pivot_thresh 0), which raises
        RuntimeError on an exactly singular factor."""
        if lv is self.levels[0]:
            self.coarse = None
            return
        kall = lv.cell_matrices()
        act = np.abs(kall).max(axis=(0, 1)) > 0
        ijk = np.argwhere(act)
        if len(ijk) == 0:
            self.coarse = None
            return
        nshape = lv.node_shape[1:]
        nn = int(np.prod(nshape))
        used = np.zeros(nn, bool)
        for off in OFFS:
            used[np.ravel_multi_index(tuple((ijk + np.array(off)).T), nshape)] = True
        gnode = np.flatnonzero(used)
        gdof = np.concatenate([[i * nn + gnode[j] for i in range(3)] for j in range(len(gnode))]).astype(np.int64)
        loc = np.full(3 * nn, -1, np.int64)
        loc[gdof] = np.arange(len(gdof))
        n = len(gdof)
        kd = np.zeros((n, n))
        for c, (i, j, l) in enumerate(ijk):
            dofs = np.empty(24, np.int64)
            for q, off in enumerate(OFFS):
                node = np.ravel_multi_index((i + off[0], j + off[1], l + off[2]), nshape)
                for comp in range(3):
                    dofs[3 * q + comp] = loc[comp * nn + node]
            kd[np.ix_(dofs, dofs)] += kall[:, :, i, j, l]
        if lv.extra is not None:
            kd += lv.extra[gdof][:, gdof].toarray()   # loadpath/mg.py:734-735
        m = lv.mask.reshape(-1)[gdof].astype(np.float64)
        kd = m[:, None] * kd * m[None, :] + np.diag(1.0 - m)
        kd = 0.5 * (kd + kd.T)
        import scipy.sparse as sp
        from scipy.sparse.linalg import splu

        lu = splu(sp.csc_matrix(kd), permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                  options={"SymmetricMode": True})
        self.coarse = {"gdof": gdof, "lu": lu, "n": n}

    def coarse_solve(self, b):
        """(loadpath/mg.py:756-766)"""
        c = self.coarse
        flat = b.reshape(-1)
        rhs = flat[c["gdof"]].astype(np.float64)
        x = c["lu"].solve(rhs)
        out = np.zeros_like(flat)
        out[c["gdof"]] = x
        return out.reshape(b.shape)

    def initial_vector(self, i):
        """The power iteration's start on level i (loadpath/mg.py:779-786)."""
        lv = self.op(i)
        prev = self.lmax_vec.get(i)
        if prev is not None and prev.shape == lv.node_shape:
            return prev.astype(lv.dinv.dtype) * lv.mask
        rng = np.random.default_rng(i)
        return (rng.random(lv.node_shape) - 0.5).astype(lv.dinv.dtype) * lv.mask

    def estimate_lmax(self, i, its=12):
        """12 power iterations of D^-1 A, times 1.3 (loadpath/mg.py:771-794)."""
        lv = self.op(i)
        v = self.initial_vector(i)
        lam = 1.0
        for _ in range(its):
            nv = float(np.dot(v.reshape(-1).astype(np.float64), v.reshape(-1).astype(np.float64))) ** 0.5
            if nv == 0:
                return 2.0
            v = v / v.dtype.type(nv)
            av = lv.dinv * lv.apply(v) * lv.mask
            lam = float(np.dot(v.reshape(-1).astype(np.float64), av.reshape(-1).astype(np.float64)))
            v = av
        self.lmax_vec[i] = v
        return LMAX_SAFETY * max(lam, 1e-12)

    def smooth(self, lv, b, x):
        """Chebyshev on D^-1 A over [lmax/30, lmax], degree self.degree
        (loadpath/mg.py:796-835, fused-kernel arithmetic of loadpath/mgops.py:312-343)."""
        t = b.dtype.type
        hi = lv.lmax
        lo = hi / 30.0
        theta = 0.5 * (hi + lo)
        delta = 0.5 * (hi - lo)
        sigma = theta / delta
        rho = 1.0 / sigma
        if x is None:
            x = np.zeros_like(b)
            r = b.copy()
            d = (lv.dinv * b) * t(1.0 / theta)
        else:
            r = b - lv.apply(x)
            d = t(1.0 / theta) * lv.dinv * r
        for it in range(self.degree):
            x = x + d
            if it + 1 == self.degree:
                break
            r = r - lv.apply(d)
            rho_new = 1.0 / (2.0 * sigma - rho)
            d = t(rho_new * rho) * d + t(2.0 * rho_new / delta) * lv.dinv * r
            rho = rho_new
        return x

    def vcycle(self, i, b):
        """(loadpath/mg.py:837-860)"""
        lv = self.op(i)
        if i == len(self.levels) - 1:
            if self.coarse is not None:
                return self.coarse_solve(b)
            x = self.smooth(lv, b, None)
            return self.smooth(lv, b, x)
        x = self.smooth(lv, b, None)
        ax = lv.apply(x)
        nxt = self.op(i + 1)
        rc = restrict_masked_residual(b, ax, lv.mask, nxt.mask, nxt.node_shape)
        xc = self.vcycle(i + 1, rc.astype(self.dtype))
        prolong_add(xc, nxt.mask, lv.mask, x)
        return self.smooth(lv, b, x)

    def precondition(self, r):
        return self.vcycle(0, r.astype(self.dtype)).astype(np.float64)

    def pcg(self, b, x0):
        """float64 PCG with the energy-optimal warm start (loadpath/mg.py:872-926)."""
        a = self.levels[0]
        dot = lambda p, q: float(np.dot(p.reshape(-1), q.reshape(-1)))
        bnorm = dot(b, b) ** 0.5
        if bnorm == 0:
            return np.zeros_like(b), 0, True
        x = np.zeros(a.node_shape) if x0 is None else x0.copy()
        r = b.copy()
        if x0 is not None:
            ax = a.apply(x)
            xax = dot(x, ax)
            s = dot(b, x) / xax if xax > 0 else 0.0
            if s > 0:
                rs = b - s * ax
                if dot(rs, rs) ** 0.5 < bnorm:
                    x *= s
                    r = rs
                else:
                    x[:] = 0
            else:
                x[:] = 0
        z = self.precondition(r)
        p = z.copy()
        rz = dot(r, z)
        tol = self.rtol * bnorm
        for it in range(1, self.maxiter + 1):
            ap = a.apply(p)
            pap = dot(p, ap)
            if pap <= 0:
                return x, it, False
            alpha = rz / pap
            x += alpha * p
            r -= alpha * ap
            if dot(r, r) ** 0.5 <= tol:
                return x, it, True
            z = self.precondition(r)
            rz_new = dot(r, z)
            p = z + (rz_new / rz) * p
            rz = rz_new
        return x, self.maxiter, False

    def solve(self, b, x0=None):
        """One right-hand side on the grid (masked), with the strict fallback
        after STALL iterations (loadpath/mg.py:932-965)."""
        m = self.levels[0].mask
        b = b * m
        g0 = x0 * m if x0 is not None else None
        if self.strict or len(self.levels) < 2:
            x, it, ok = self.pcg(b, g0)
        else:
            full = self.maxiter
            self.maxiter = min(full, STALL)
            try:
                x, it, ok = self.pcg(b, g0)
            finally:
                self.maxiter = full
            if not ok:
                self.strict = True
                self.set_moduli(self.e_grid)
                x, it2, ok = self.pcg(b, g0)
                it += it2
        if not ok:
            raise RuntimeError(f"linear solve did not converge ({it} iterations); "
                               "the structure may be a mechanism (check supports)")
        self.last_iters = it
        return x * m

    def strain_energy(self, u_grid):
        """Per-cell u_e^T Ke u_e at unit modulus (loadpath/mg.py:975-988)."""
        g = gather_cells(u_grid, self.cells).reshape(24, -1)
        return np.einsum("in,in->n", g, self.ke @ g).reshape(self.cells)


# --------------------------------------------------------------------------
# SIMP pieces (loadpath/simp.py, loadpath/benchmarks/reference.py)
# --------------------------------------------------------------------------

def filter_taps(radius: float, pitch: float = 1.0):
    """Cone taps w = r - |d| pitch > 0 within floor(r / pitch) cells
    (loadpath/simp.py:1148-1161)."""
    reach = int(np.floor(radius / pitch))
    taps = []
    for dx in range(-reach, reach + 1):
        for dy in range(-reach, reach + 1):
            for dz in range(-reach, reach + 1):
                w = radius - np.sqrt(dx * dx + dy * dy + dz * dz) * pitch
                if w > 0:
                    taps.append(((dx, dy, dz), float(w)))
    return taps


def grid_filter(v: np.ndarray, taps) -> np.ndarray:
    """H v on the cell grid with zeros outside it (loadpath/simp.py:1164-1172).
    H is symmetric, so this is also H^T v."""
    reach = max(max(abs(c) for c in d) for d, _ in taps)
    nx, ny, nz = v.shape
    g = np.zeros((nx + 2 * reach, ny + 2 * reach, nz + 2 * reach))
    g[reach:reach + nx, reach:reach + ny, reach:reach + nz] = v
    out = np.zeros(v.shape)
    for (dx, dy, dz), w in taps:
        out += w * g[reach + dx:reach + dx + nx, reach + dy:reach + dy + ny, reach + dz:reach + dz + nz]
    return out


def filter_row_sums(dims, taps):
    """Row sums of the truncated stencil (top3d's Hs; loadpath/benchmarks/reference.py:48-71)."""
    return grid_filter(np.ones(dims), taps)


def simp_moduli(xphys, penal=3.0, emin=1e-9):
    """E = Emin + x^p (1 - Emin) (loadpath/benchmarks/reference.py:89; loadpath/simp.py:1861)."""
    return emin + xphys ** penal * (1 - emin)


def oc_top3d(x, dc, dv, volfrac, h_apply, hs, move=0.2):
    """top3d's OC bisection on the volume multiplier; volume measured on the
    filtered physical densities (loadpath/benchmarks/reference.py:100-110).
    Returns (xnew, xphys)."""
    n = x.size
    l1, l2 = 0.0, 1e9
    while (l2 - l1) / (l1 + l2) > 1e-3:
        lmid = 0.5 * (l2 + l1)
        xnew = np.maximum(0, np.maximum(x - move, np.minimum(1, np.minimum(x + move, x * np.sqrt(-dc / dv / lmid)))))
        xphys = h_apply(xnew) / hs
        if xphys.sum() > volfrac * n:
            l1 = lmid
        else:
            l2 = lmid
    return xnew, xphys


def project(xt, beta, eta):
    """tanh Heaviside projection (loadpath/simp.py:1443-1446)."""
    den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
    return (np.tanh(beta * eta) + np.tanh(beta * (xt - eta))) / den


def dproject(xt, beta, eta):
    """its derivative in xt (loadpath/simp.py:1448-1450)."""
    den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
    return beta * (1 - np.tanh(beta * (xt - eta)) ** 2) / den


VOLUME_RTOL = 1e-13   # loadpath/simp.py:1234


def mirror_average(v, mirror):
    """loadpath/simp.py:1476-1482 `_symmetrize` on a box whose every cell has a mirror image: per
    axis in order, v = (v + v mirrored across the mid-plane) / 2."""
    for ax in mirror:
        v = 0.5 * (v + np.flip(v, axis=ax))
    return v


def oc_loadpath_step(x, dc, dv, move, beta, eta, h_apply, hs, w, target, pres=None, void=None,
                     lam_last=None, mirror=()):
    """loadpath's optimality-criteria step (loadpath/simp.py:2249-2376, the volume-constrained
    path: no thermal swing constraint, mirror, extrusion or blockage term). The step
    x sqrt(-dc / dv / lm) clipped to [max(0, x - move), min(1, x + move)] (passive cells held),
    measured on the physical volume sum(project(H x / hs) w); the multiplier is bracketed outward
    from lam_last in log space (reach 0.25, x4 per try, range 1e-12..1e12), then found by false
    position with the Illinois halving, to |f| <= 1e-13 target. Returns (x_new, lm, n_eval, held)."""
    lo_x = np.maximum(0.0, x - move)
    hi_x = np.minimum(1.0, x + move)
    ratio = np.sqrt(-dc / dv)
    n_eval = [0]

    def physical(xv):
        xp = project(h_apply(xv) / hs, beta, eta)
        if pres is not None:
            xp[pres] = 1.0
        if void is not None:
            xp[void] = 0.0
        return xp

    def stepped(lm_):
        n_eval[0] += 1
        xn = np.clip(x * ratio / np.sqrt(lm_), lo_x, hi_x)
        if pres is not None:
            xn[pres] = 1.0
        if void is not None:
            xn[void] = 0.0
        if mirror:
            xn = mirror_average(xn, mirror)
        return xn, float(np.sum(physical(xn) * w)) - target

    l1, l2 = 1e-12, 1e12
    s_lo, s_hi = np.log(l1), np.log(l2)
    sm = min(max(np.log(lam_last), s_lo), s_hi) if lam_last else 0.0
    x_new, f = stepped(float(np.exp(sm)))
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
        x_new, f = stepped(lm)
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
            x_new, f = stepped(lm)
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
    return x_new, lm, n_eval[0], f1 is not None and f2 is not None


ALIVE = 1e-3          # loadpath/simp.py:59
REDUCE_BELOW = 0.8    # loadpath/simp.py:61


def connected_keep(alive, support_touch):
    """The cells the solve keeps (loadpath/simp.py:263-289 `_connected`): alive cells in a
    26-connected component (scipy.ndimage.label, as the reference) holding an alive cell that
    touches a support. Grid-order bool arrays."""
    from scipy import ndimage

    lbl, _ = ndimage.label(alive, structure=np.ones((3, 3, 3), bool))
    keep_l = np.unique(lbl[alive & support_touch])
    return alive & np.isin(lbl, keep_l[keep_l > 0])


def cells_touching(node_flags):
    """Cells with any of their eight corners set in node_flags (nx+1, ny+1, nz+1): the cells
    touching a support or a load (loadpath/simp.py:150-151, `support_nodes[mesh.enode].any(axis=1)`)."""
    n = np.asarray(node_flags, bool)
    dims = tuple(d - 1 for d in n.shape)
    out = np.zeros(dims, bool)
    for (i, j, k) in OFFS:
        out |= n[i:i + dims[0], j:j + dims[1], k:k + dims[2]]
    return out


def live_solve(ke, fixed_grid, f_grid, support_touch, anchor):
    """solve(e, xphys) with the SIMP driver's live-cell reduction (loadpath/simp.py:725, 795-826):
    alive = xphys > ALIVE or an anchor cell; when fewer than REDUCE_BELOW of the cells are alive,
    only the cells connected_keep keeps carry their moduli, dofs left without stiffness are
    dropped (and are zero in u), and a load on such a dof sends the solve back to the full grid.
    Direct sparse solves (assembled_solve)."""
    def solve(e, xphys):
        alive = (xphys > ALIVE) | anchor
        if alive.mean() < REDUCE_BELOW:
            keep = connected_keep(alive, support_touch)
            er = np.where(keep, e, 0.0)
            u = assembled_solve(ke, er, fixed_grid, f_grid, drop_dead=True)
            stiff = np.zeros(tuple(d + 1 for d in e.shape), bool)
            for (i, j, k) in OFFS:
                stiff[i:i + e.shape[0], j:j + e.shape[1], k:k + e.shape[2]] |= keep
            if not np.any(np.asarray(f_grid)[:, ~stiff]):
                return u
        return assembled_solve(ke, e, fixed_grid, f_grid)
    return solve


class LiveSystem:
    """The SIMP driver's solves with the live-cell reduction (loadpath/simp.py:114-330 `_Analysis`):
    alive = xphys > ALIVE or an anchor cell; under REDUCE_BELOW alive, only the cells connected_keep
    keeps carry their moduli (dofs without stiffness dropped, zero in u), unless a load is left
    on such a dof. reuse = 0 is the multigrid path's rule (:795-826, the kept cells found every
    solve); reuse = n the direct path's (:288-315 `_subsystem`): a reduced system is kept for up
    to n further solves while every alive cell is inside it. resolve() solves another right-hand
    side on the last solve's system (:828-876). Direct sparse solves (assembled_solve)."""

    def __init__(self, ke, fixed_grid, support_touch, anchor, reuse=0):
        self.ke, self.fixed = ke, np.asarray(fixed_grid, bool)
        self.support_touch, self.anchor, self.reuse = support_touch, anchor, reuse
        self.cache, self.age = None, 0
        self.er, self.drop, self.cells = None, False, None

    def _stiff_nodes(self, cells):
        dims = cells.shape
        stiff = np.zeros(tuple(d + 1 for d in dims), bool)
        for (i, j, k) in OFFS:
            stiff[i:i + dims[0], j:j + dims[1], k:k + dims[2]] |= cells
        return stiff

    def solve(self, e, xphys, f_grid):
        """u for the load f_grid, or the list of u for a list of loads (the reduction decided on all
        of them, as the reference's analysis decides it on every case)."""
        many = isinstance(f_grid, (list, tuple))
        fs = [np.asarray(f, float) for f in (f_grid if many else [f_grid])]
        dead = lambda nodes: any(np.any(f[:, ~nodes]) for f in fs)   # noqa: E731
        alive = (xphys > ALIVE) | self.anchor
        self.er, self.drop, self.cells = e, False, e.size
        if alive.mean() < REDUCE_BELOW and not dead(self._stiff_nodes(alive)):
            keep = None
            if self.reuse and self.cache is not None and self.age < self.reuse and not np.any(alive & ~self.cache):
                self.age += 1
                keep = self.cache
            else:
                keep = connected_keep(alive, self.support_touch)
                if dead(self._stiff_nodes(keep)):
                    self.cache, keep = None, None
                elif self.reuse:
                    self.cache, self.age = keep, 0
            if keep is not None:
                self.er, self.drop, self.cells = np.where(keep, e, 0.0), True, int(keep.sum())
        us = [assembled_solve(self.ke, self.er, self.fixed, f, drop_dead=self.drop) for f in fs]
        return us if many else us[0]

    def resolve(self, rhs):
        return assembled_solve(self.ke, self.er, self.fixed, rhs, drop_dead=self.drop)


# --------------------------------------------------------------------------
# assembled direct solve for tiny grids (loadpath/benchmarks/evaluate.py:111-117)
# --------------------------------------------------------------------------

def assembled_solve(ke, e_grid, fixed_grid, f_grid, drop_dead=False):
    """Direct sparse solve of K(e) u = f on the full node grid, fixed dofs
    removed (the evaluator's scheme). With drop_dead, dofs without stiffness
    (zero diagonal, cells of modulus 0 only) are removed too and come back as
    zero, as the multigrid's masks do (loadpath/mg.py:537-550). Returns the
    node-grid displacement."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    dims = e_grid.shape
    nshape = tuple(d + 1 for d in dims)
    nn = int(np.prod(nshape))
    ijk = np.argwhere(np.ones(dims, bool))
    dofs = np.empty((len(ijk), 24), np.int64)
    for q, off in enumerate(OFFS):
        node = np.ravel_multi_index(tuple((ijk + np.array(off)).T), nshape)
        for c in range(3):
            dofs[:, 3 * q + c] = c * nn + node
    rows = np.repeat(dofs, 24, axis=1).ravel()
    cols = np.tile(dofs, (1, 24)).ravel()
    data = (e_grid[tuple(ijk.T)][:, None, None] * ke[None]).ravel()
    k = sp.csr_matrix((data, (rows, cols)), shape=(3 * nn, 3 * nn))
    keep = ~fixed_grid.reshape(-1)
    if drop_dead:
        keep &= k.diagonal() > 1e-300
    free = np.flatnonzero(keep)
    u = np.zeros(3 * nn)
    u[free] = spla.spsolve(k[free][:, free].tocsc(), f_grid.reshape(-1)[free])
    return u.reshape((3,) + nshape)


def top3d_loop(dims, volfrac, rmin, ke, fixed_grid, f_grid, iters, penal=3.0, emin=1e-9, move=0.2,
               solve=None, x0=None, with_xphys=False, reduce=None):
    """top3d's loop with the density filter (loadpath/benchmarks/reference.py:74-117).
    Returns (x, xphys, compliance history, change history). f_grid may be a list of load cases:
    the objective is then their equally weighted compliance sum, and its sensitivity the sum of
    the cases' (the reference's loop has one load; its sums over cases are those of
    loadpath/simp.py:1901-1904 applied per case). solve(e) returns u, or a list of u per case
    (solve(e, xphys) with with_xphys). x0: the starting design (default volfrac everywhere),
    taken as its own physical density as top3d starts. reduce(ce, c) -> (ce, c): the totals over
    the load cases other processes solved (the cell energies and compliance summed over ranks)."""
    if solve is None:
        if isinstance(f_grid, (list, tuple)):
            solve = lambda e: [assembled_solve(ke, e, fixed_grid, fk) for fk in f_grid]
        else:
            solve = lambda e: assembled_solve(ke, e, fixed_grid, f_grid)
    taps = filter_taps(rmin)
    hs = filter_row_sums(dims, taps)
    hap = lambda v: grid_filter(v, taps)
    x = np.full(dims, volfrac) if x0 is None else np.array(x0, np.float64)
    xphys = x.copy()
    hist_c, hist_ch = [], []
    for _ in range(iters):
        e = simp_moduli(xphys, penal, emin)
        us = solve(e, xphys) if with_xphys else solve(e)
        ce = np.zeros(dims)
        c = 0.0
        for u in (us if isinstance(us, list) else [us]):
            g = gather_cells(u, dims).reshape(24, -1)
            ce_k = np.einsum("in,in->n", g, ke @ g).reshape(dims)
            c += float(np.sum(e * ce_k))
            ce += ce_k
        if reduce is not None:
            ce, c = reduce(ce, c)
        dc = -penal * (1 - emin) * xphys ** (penal - 1) * ce
        dc = hap(dc / hs)
        dv = hap(np.ones(dims) / hs)
        xnew, xphys = oc_top3d(x, dc, dv, volfrac, hap, hs, move)
        hist_c.append(c)
        hist_ch.append(float(np.abs(xnew - x).max()))
        x = xnew
    return x, xphys, hist_c, hist_ch


def optimize_loop(dims, ke, fixed_grid, f_grid, volfrac, radius, iters, pres=None, pad=True, pitch=1.0,
                  eta=0.5, erode=0.15, move=0.2, tol=0.01, beta_max=32.0, beta_every=10, emin=1e-6, penal=3.0,
                  mirror=(), reuse=6, adaptive_move=True, stall_rtol=2e-3, stall_window=6, weights=None):
    """loadpath's own SIMP loop for one load case with its default options (loadpath/simp.py:
    1640-2455): blueprint and eroded projections of xt = H x / hs (`physical`, `eroded`), the SIMP
    law on the eroded design, the solve with the live-cell reduction (LiveSystem with the direct
    path's reuse of a reduced system, the anchor cells being those touching a support or the load
    and the pinned ones), dc = min(H (dc_xe P'_e / hs), 0),
    dv = max(H (w P'_b / hs), 1e-12), the move limit measured from the Lagrangian's slope along
    the last step (t = a / (a - b), the limit times t clipped to [0.5, 1.2], capped at move), the
    step of oc_loadpath_step, and beta doubling after beta_every iterations or a free step of
    change < 2 tol, halving the limit (with adaptive_move off, the fixed limits: move, move / 2 past
    beta 4), and at beta_max the stopping rules; with mirror planes (axes) dc, dv and every trial
    design are averaged across them (:2222-2224, :2300). Ke and the loads' work scale with the pitch. Returns the
    per-iteration records (compliance, beta, change, move, volume, volumeSolves, xphys) and x."""
    pres = np.zeros(dims, bool) if pres is None else np.asarray(pres, bool)
    design = ~pres
    w = design.astype(float)
    taps = filter_taps(radius, pitch)
    hs = np.full(dims, sum(t for _, t in taps)) if pad else filter_row_sums(dims, taps)
    hap = lambda v: grid_filter(v, taps)   # noqa: E731
    fs = [np.asarray(f, float) for f in (f_grid if isinstance(f_grid, (list, tuple)) else [f_grid])]
    weights = [1.0] * len(fs) if weights is None else [float(w_) for w_ in weights]
    held = np.asarray(fixed_grid, bool).any(axis=0)
    loaded = np.zeros(held.shape, bool)
    for f in fs:
        loaded |= (f != 0).any(axis=0)
    system = LiveSystem(ke * pitch, fixed_grid, cells_touching(held), cells_touching(held | loaded) | pres,
                        reuse=reuse)
    x = np.full(dims, volfrac)
    x[pres] = 1.0
    target = volfrac * float(w.sum())
    beta, since_beta, move_k, lam_last, step_prev = 1.0, 0, move, None, None
    recs = []
    for _ in range(iters):
        xt = hap(x) / hs
        xp = project(xt, beta, eta)
        xp[pres] = 1.0
        xe = project(xt, beta, eta + erode)
        xe[pres] = 1.0
        e = emin + xe ** penal * (1 - emin)
        us = system.solve(e, xe, fs)
        comp, dc_xe = 0.0, np.zeros(dims)
        for f, u, wk in zip(fs, us, weights):
            # per case: its weight times f.u, and its sensitivity (loadpath/simp.py:1901-1904)
            g = gather_cells(u, dims).reshape(24, -1)
            ce = np.einsum("in,in->n", g, (ke * pitch) @ g).reshape(dims)
            comp += wk * float(np.sum(f * u))
            dc_xe -= wk * penal * xe ** (penal - 1) * (1 - emin) * ce
        dpe = dproject(xt, beta, eta + erode)
        dpe[pres] = 0.0
        dpb = dproject(xt, beta, eta)
        dpb[pres] = 0.0
        dc = np.minimum(hap(dc_xe * dpe / hs), 0.0)
        dv = np.maximum(hap(w * dpb / hs), 1e-12)
        if mirror:
            dc, dv = mirror_average(dc, mirror), mirror_average(dv, mirror)
        if adaptive_move:
            if step_prev is not None:
                dxp, gp, lam_p = step_prev
                a_s = float(np.sum(gp * dxp))
                b_s = float(np.sum((dc + lam_p * dv) * dxp))
                if a_s < 0:
                    t_s = a_s / (a_s - b_s) if b_s > a_s else np.inf
                    move_k = min(move_k * min(max(t_s, 0.5), 1.2), move)
            mv = move_k
        else:
            mv = move if beta <= 4 else move / 2
        x_new, lm, n_eval, held = oc_loadpath_step(x, dc, dv, mv, beta, eta, hap, hs, w, target, pres=pres,
                                                lam_last=lam_last, mirror=mirror)
        lam_last = lm
        change = float(np.abs(x_new - x)[design].max())
        step_prev = (x_new - x, dc + lm * dv, lm)
        x = x_new
        since_beta += 1
        recs.append(dict(compliance=comp, beta=beta, change=change, move=mv if adaptive_move else np.nan,
                         volume=float(xp[design].mean()), volumeSolves=n_eval, xphys=xp))
        free_step = not adaptive_move or change < 0.999 * mv
        if beta < beta_max and ((change < 2 * tol and free_step) or since_beta >= beta_every):
            beta = min(2 * beta, beta_max)
            since_beta = 0
            step_prev = None
            move_k = move_k / 2
        elif beta >= beta_max and len(recs) >= 3:
            # the stopping rules (loadpath/simp.py:2431-2450); the schedule's rule needs the
            # measured step, the stall rule holds otherwise
            if change < tol and free_step:
                break
            if adaptive_move and held:
                if since_beta >= beta_every:
                    break
            elif since_beta >= stall_window and len(recs) > stall_window:
                old = recs[-1 - stall_window]["compliance"]
                if abs(comp - old) <= stall_rtol * abs(old):
                    break
    return recs, x


VM = np.array([[1.0, -0.5, -0.5, 0, 0, 0], [-0.5, 1.0, -0.5, 0, 0, 0], [-0.5, -0.5, 1.0, 0, 0, 0],
               [0, 0, 0, 3.0, 0, 0], [0, 0, 0, 0, 3.0, 0], [0, 0, 0, 0, 0, 3.0]])   # loadpath/constrained.py:107-114


def hex8_b(xi, eta, zeta, nu, element="im"):
    """Strain-displacement (6x24) of the unit cube at a natural point with the condensed
    bubbles' strain (loadpath/fem.py:227-237)."""
    c = elastic_c(nu)
    g = 1.0 / np.sqrt(3.0)
    kua = np.zeros((24, 9))
    kaa = np.zeros((9, 9))
    for a in (-g, g):
        for b_ in (-g, g):
            for cz in (-g, g):
                b = b_matrix(a, b_, cz)
                ba = b_bubble(a, b_, cz)
                kua += b.T @ c @ ba * 0.125
                kaa += ba.T @ c @ ba * 0.125
    out = b_matrix(xi, eta, zeta)
    if element == "im":
        out = out + b_bubble(xi, eta, zeta) @ (-np.linalg.solve(kaa, kua.T))
    return out


def corner_stress_ops(nu, pitch=1.0, element="im"):
    """The 8 (6x24) stress operators C B at the cube's corners, x outermost
    (loadpath/constrained.py:443-446, STRESS_POINTS = "corners")."""
    c = elastic_c(nu)
    return [c @ hex8_b(a, b, cz, nu, element) / pitch for a in (-1.0, 1.0) for b in (-1.0, 1.0) for cz in (-1.0, 1.0)]


def scatter_cell_vectors(fe, dims):
    """Node field (3, nx+1, ny+1, nz+1) summing per-cell 24-vectors fe (24, nx, ny, nz) onto the
    cells' corners (the transpose of gather_cells)."""
    out = np.zeros((3,) + tuple(d + 1 for d in dims))
    nx, ny, nz = dims
    for k, (dx, dy, dz) in enumerate(OFFS):
        out[:, dx:dx + nx, dy:dy + ny, dz:dz + nz] += fe[3 * k:3 * k + 3]
    return out


def constrained_loop(dims, nu, fixed_grid, f_grid, vf0, radius, iters, stress_limit, deflection_limit, modulus,
                     pres=None, pad=True, pitch=1.0, mirror=(), eta=0.5, erode=0.15, move=0.2, tol=0.01,
                     beta_max=32.0, beta_every=10, stall_window=6, emin=1e-6, penal=3.0, element="im", reuse=6):
    """loadpath's minimum-mass loop under a stress and a deflection limit for one load case
    (loadpath/constrained.py:295-854 with Limits(stress, deflection, modulus) and default options;
    either limit may be None; f_grid one load or a list of load cases, each with its own
    deflection and stress constraint, deflections first):
    per iteration the blueprint and eroded designs, the solve on the live cells (LiveSystem, as
    optimize_loop) and the adjoint solves on the same system, the deflection f.u / (sum_n |f_n| E) against its limit with gradient
    -dE ce / (sum |f| E); the relaxed von Mises xe * vm(C B_k u_e) / limit at the 8 corners of every
    cell that moved and touches no support or load, aggregated by a P-mean (P = 8) over the counted
    corners with the adaptive normalisation kappa (Le et al.), its adjoint solve and gradient;
    the volume objective 10 mean(xp) over the design cells; MMA (move 0.1, halved and its asymptotes
    tightened while the worst constraint grows above 0.02, grown by 1.2 up to the cap inside);
    beta doubling once feasible after beta_every iterations or a small change (or after 3
    beta_every), the cap times 0.6; at beta_max the lightest feasible design is kept and the run
    stops on a feasible small change or a stalled volume. Returns (records, x, converged)."""
    pres = np.zeros(dims, bool) if pres is None else np.asarray(pres, bool)
    design = ~pres
    free = np.flatnonzero(design.reshape(-1))
    taps = filter_taps(radius, pitch)
    hs = np.full(dims, sum(t for _, t in taps)) if pad else filter_row_sums(dims, taps)
    hap = lambda v: grid_filter(v, taps)   # noqa: E731
    ke = hex8_ke(nu, element) * pitch
    fs = [np.asarray(f, float) for f in (f_grid if isinstance(f_grid, (list, tuple)) else [f_grid])]
    held = np.asarray(fixed_grid, bool).any(axis=0)
    loaded = np.zeros(held.shape, bool)
    for f in fs:
        loaded |= (f != 0).any(axis=0)
    system = LiveSystem(ke, fixed_grid, cells_touching(held), cells_touching(held | loaded) | pres, reuse=reuse)
    counted = ~cells_touching(held | loaded)
    nc = max(int(counted.sum()), 1) * 8
    load_size = [float(np.linalg.norm(f.reshape(3, -1), axis=0).sum()) for f in fs]
    defl_cases = [c for c in range(len(fs)) if deflection_limit is not None and load_size[c] > 0]
    stress_cases = list(range(len(fs))) if stress_limit is not None else []
    cbs = corner_stress_ops(nu, pitch, element)
    sym = (lambda v: mirror_average(v, mirror)) if mirror else (lambda v: v)   # noqa: E731
    x = np.full(dims, vf0)
    x[pres] = 1.0
    mma = MMA(len(free), len(defl_cases) + len(stress_cases), 0.0, 1.0, move=min(move, 0.1))
    move_cap = mma.move
    worst_prev, kappa, beta, since_beta = np.inf, [1.0] * len(fs), 1.0, 0
    best, trail, recs, converged = None, [], [], False
    for it in range(1, iters + 1):
        x_now = x
        xt = hap(x) / hs
        xp = project(xt, beta, eta)
        xp[pres] = 1.0
        xe = project(xt, beta, eta + erode)
        xe[pres] = 1.0
        dpb = dproject(xt, beta, eta)
        dpb[pres] = 0.0
        dpe = dproject(xt, beta, eta + erode)
        dpe[pres] = 0.0
        e = emin + xe ** penal * (1 - emin)
        de = penal * xe ** (penal - 1) * (1 - emin)
        us = system.solve(e, xe, fs)
        to_x = lambda g: hap(g * dpe / hs)   # noqa: E731
        ues = [gather_cells(u, dims).reshape(24, -1) for u in us]
        cons, grads, defls, stresses = [], [], [], []
        for c in defl_cases:
            ce = np.einsum("in,in->n", ues[c], ke @ ues[c]).reshape(dims)
            defl = float(np.sum(fs[c] * us[c])) / (load_size[c] * modulus)
            cons.append(defl / deflection_limit - 1.0)
            grads.append(to_x(-de * ce / (load_size[c] * modulus)) / deflection_limit)
            defls.append(defl)
        for c in stress_cases:
            ue = ues[c]
            moved = np.any(ue != 0, axis=0)
            act = (moved & counted.reshape(-1))
            xa = xe.reshape(-1)[act]
            ua = ue[:, act]
            parts = []
            for cbk in cbs:
                sig = cbk @ ua
                sv = VM @ sig
                vm = np.sqrt(np.maximum(np.einsum("in,in->n", sv, sig), 1e-30))
                parts.append((cbk, sv, vm, xa * vm / stress_limit))
            smax = max((float(p[3].max()) for p in parts if p[3].size), default=0.0)
            sc = max(smax, 1e-30)
            pm = sc * (sum(float(np.sum((p[3] / sc) ** 8)) for p in parts) / nc) ** (1.0 / 8)
            kk = smax / max(pm, 1e-30)
            kappa[c] = 0.5 * (kappa[c] + kk) if it > 1 else kk
            g = kappa[c] * pm
            g_xe = np.zeros(ue.shape[1])
            fe = np.zeros((24, ue.shape[1]))
            for cbk, sv, vm, srel in parts:
                dg_ds = kappa[c] * (srel / max(pm, 1e-30)) ** 7 / nc
                g_xe[act] += dg_ds * (vm / stress_limit)
                fe[:, act] += (dg_ds * (xa / (vm * stress_limit)))[None, :] * (cbk.T @ sv)
            rhs = scatter_cell_vectors(fe.reshape((24,) + dims), dims)
            rhs[np.asarray(fixed_grid, bool)] = 0.0
            lam = system.resolve(rhs)
            le = gather_cells(lam, dims).reshape(24, -1)
            g_xe[moved] -= de.reshape(-1)[moved] * np.einsum("in,in->n", le, ke @ ue)[moved]
            cons.append(g - 1.0)
            grads.append(to_x(g_xe.reshape(dims)))
            stresses.append(smax * stress_limit)

        f0 = 10.0 * float(xp[design].mean())
        df0 = sym(hap(10.0 * design / design.sum() * dpb / hs))
        grads = [sym(gr) for gr in grads]
        worst = max(cons)
        if worst > 0.02 and worst > worst_prev:
            mma.move = max(0.02, 0.5 * mma.move)
            mma.tighten(0.5)
        elif worst <= 0.02:
            mma.move = min(move_cap, 1.2 * mma.move)
        worst_prev = worst
        xf = mma.update(x.reshape(-1)[free], f0, df0.reshape(-1)[free], np.array(cons),
                        np.array([gr.reshape(-1)[free] for gr in grads]))
        xnew = x.copy().reshape(-1)
        xnew[free] = xf
        xnew = sym(xnew.reshape(dims))
        change = float(np.abs(xnew - x)[design].max())
        x = xnew
        since_beta += 1
        rec = dict(volume=float(xp[design].mean()), beta=beta, change=change, constraints=list(cons),
                   deflection=defls[0] if defls else np.nan, stress=stresses[0] if stresses else np.nan,
                   deflections=defls, stresses=stresses, xphys=xp)
        recs.append(rec)
        feasible = max(cons) <= 0.02
        if beta < beta_max and ((feasible and (since_beta >= beta_every or change < 2 * tol))
                                or since_beta >= 3 * beta_every):
            beta = min(beta * 2, beta_max)
            since_beta = 0
            move_cap = max(0.02, move_cap * 0.6)
            mma.move = min(mma.move, move_cap)
        elif beta >= beta_max:
            if feasible and (best is None or rec["volume"] < best[1]["volume"]):
                best = (x_now, rec)
            trail.append(best[1]["volume"] if best is not None else np.inf)
            if best is not None and ((feasible and change < tol) or (
                    len(trail) > stall_window and trail[-1] > (1.0 - 5e-3) * trail[-1 - stall_window])):
                converged = True
                break
    if best is not None:
        x = best[0]
    return recs, x, converged

# --------------------------------------------------------------------------
# MMA (loadpath/mma.py:31-214), restated from Svanberg's published method
# --------------------------------------------------------------------------

class MMA:
    """Svanberg's MMA with a primal-dual interior-point subproblem solver, in
    the reference's parameterisation (loadpath/mma.py:31-55)."""

    def __init__(self, n, m, xmin=0.0, xmax=1.0, move=0.2, c=1000.0, asyinit=0.5, asyincr=1.2, asydecr=0.7):
        self.n, self.m = n, m
        self.xmin = np.broadcast_to(np.asarray(xmin, float), (n,)).copy()
        self.xmax = np.broadcast_to(np.asarray(xmax, float), (n,)).copy()
        self.move = move
        self.a0, self.a, self.c, self.d = 1.0, np.zeros(m), np.full(m, float(c)), np.ones(m)
        self.asyinit, self.asyincr, self.asydecr = asyinit, asyincr, asydecr
        self.xold1 = self.xold2 = self.low = self.upp = None
        self.iter = 0

    def tighten(self, factor):
        """Pull the asymptotes toward the last design by factor (loadpath/mma.py:49-55)."""
        if self.xold1 is not None and self.low is not None:
            self.low = self.xold1 - factor * (self.xold1 - self.low)
            self.upp = self.xold1 + factor * (self.upp - self.xold1)

    def update(self, x, f0, df0, f, df):
        """One MMA step (loadpath/mma.py:57-112)."""
        xmin, xmax = self.xmin, self.xmax
        x = np.clip(np.nan_to_num(np.asarray(x, float), nan=0.5), xmin, xmax)
        f = np.nan_to_num(np.asarray(f, float).reshape(self.m), nan=1e6, posinf=1e6, neginf=-1e6)
        df = np.nan_to_num(np.asarray(df, float).reshape(self.m, self.n), nan=0.0, posinf=1e6, neginf=-1e6)
        df0 = np.nan_to_num(np.asarray(df0, float), nan=0.0, posinf=1e6, neginf=-1e6)
        self.iter += 1
        span = xmax - xmin
        if self.iter <= 2 or self.low is None:
            self.low = x - self.asyinit * span
            self.upp = x + self.asyinit * span
        else:
            sgn = (x - self.xold1) * (self.xold1 - self.xold2)
            fac = np.where(sgn > 0, self.asyincr, np.where(sgn < 0, self.asydecr, 1.0))
            self.low = np.clip(x - fac * (self.xold1 - self.low), x - 10 * span, x - 0.01 * span)
            self.upp = np.clip(x + fac * (self.upp - self.xold1), x + 0.01 * span, x + 10 * span)
        low, upp = self.low, self.upp
        alfa = np.maximum(np.maximum(low + 0.1 * (x - low), x - self.move * span), xmin)
        beta = np.minimum(np.minimum(upp - 0.1 * (upp - x), x + self.move * span), xmax)
        xmami = np.maximum(span, 1e-5)
        ux1, xl1 = upp - x, x - low
        ux2, xl2 = ux1 * ux1, xl1 * xl1
        p0, q0 = np.maximum(df0, 0.0), np.maximum(-df0, 0.0)
        pq0 = 0.001 * (p0 + q0) + 1e-5 / xmami
        p0, q0 = (p0 + pq0) * ux2, (q0 + pq0) * xl2
        P, Q = np.maximum(df, 0.0), np.maximum(-df, 0.0)
        PQ = 0.001 * (P + Q) + 1e-5 / xmami
        P, Q = (P + PQ) * ux2, (Q + PQ) * xl2
        b = P @ (1.0 / ux1) + Q @ (1.0 / xl1) - f
        with np.errstate(divide="ignore", invalid="ignore"):
            xnew = self.subsolv(low, upp, alfa, beta, p0, q0, P, Q, b)
        if not np.all(np.isfinite(xnew)):
            xnew = np.where(np.isfinite(xnew), xnew, x)
        xnew = np.clip(xnew, alfa, beta)
        self.xold2 = self.xold1 if self.xold1 is not None else x.copy()
        self.xold1 = x.copy()
        return xnew

    def subsolv(self, low, upp, alfa, beta, p0, q0, P, Q, b, epsimin=1e-7):
        """Primal-dual Newton on the separable subproblem (loadpath/mma.py:114-214)."""
        m = self.m
        a0, a, c, d = self.a0, self.a, self.c, self.d
        x = 0.5 * (alfa + beta)
        y, z, lam = np.ones(m), 1.0, np.ones(m)
        xsi = np.maximum(1.0 / (x - alfa), 1.0)
        eta = np.maximum(1.0 / (beta - x), 1.0)
        mu, zet, s = np.maximum(1.0, 0.5 * c), 1.0, np.ones(m)
        epsi = 1.0

        def resid(x, y, z, lam, xsi, eta, mu, zet, s, epsi):
            ux1, xl1 = upp - x, x - low
            plam, qlam = p0 + P.T @ lam, q0 + Q.T @ lam
            gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
            dpsidx = plam / (ux1 * ux1) - qlam / (xl1 * xl1)
            return np.concatenate([dpsidx - xsi + eta, c + d * y - mu - lam, [a0 - zet - a @ lam],
                                   gvec - a * z - y + s - b, xsi * (x - alfa) - epsi, eta * (beta - x) - epsi,
                                   mu * y - epsi, [zet * z - epsi], lam * s - epsi])

        while epsi > epsimin:
            r = resid(x, y, z, lam, xsi, eta, mu, zet, s, epsi)
            norm = np.linalg.norm(r)
            rmax = np.abs(r).max()
            it = 0
            while rmax > 0.9 * epsi and it < 200:
                it += 1
                ux1, xl1 = upp - x, x - low
                ux2, xl2 = ux1 * ux1, xl1 * xl1
                ux3, xl3 = ux1 * ux2, xl1 * xl2
                plam, qlam = p0 + P.T @ lam, q0 + Q.T @ lam
                gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
                GG = P / ux2 - Q / xl2
                dpsidx = plam / ux2 - qlam / xl2
                delx = dpsidx - epsi / (x - alfa) + epsi / (beta - x)
                dely = c + d * y - lam - epsi / y
                delz = a0 - a @ lam - epsi / z
                dellam = gvec - a * z - y - b + epsi / lam
                diagx = 2.0 * (plam / ux3 + qlam / xl3) + xsi / (x - alfa) + eta / (beta - x)
                diagy = d + mu / y
                diaglamyi = s / lam + 1.0 / diagy
                blam = dellam + dely / diagy - GG @ (delx / diagx)
                aa = np.zeros((m + 1, m + 1))
                aa[:m, :m] = np.diag(diaglamyi) + (GG / diagx) @ GG.T
                aa[:m, m] = a
                aa[m, :m] = a
                aa[m, m] = -zet / z
                sol = np.linalg.solve(aa, np.concatenate([blam, [delz]]))
                dlam, dz = sol[:m], sol[m]
                dx = -delx / diagx - (GG.T @ dlam) / diagx
                dy = -dely / diagy + dlam / diagy
                dxsi = -xsi + epsi / (x - alfa) - xsi * dx / (x - alfa)
                deta = -eta + epsi / (beta - x) + eta * dx / (beta - x)
                dmu = -mu + epsi / y - mu * dy / y
                dzet = -zet + epsi / z - zet * dz / z
                ds = -s + epsi / lam - s * dlam / lam
                xx = np.concatenate([y, [z], lam, xsi, eta, mu, [zet], s])
                dxx = np.concatenate([dy, [dz], dlam, dxsi, deta, dmu, [dzet], ds])
                stmxx = np.max(-1.01 * dxx / xx)
                stmalfa = np.max(-1.01 * dx / (x - alfa))
                stmbeta = np.max(1.01 * dx / (beta - x))
                steg = 1.0 / max(stmalfa, stmbeta, stmxx, 1.0)
                old = (x, y, z, lam, xsi, eta, mu, zet, s)
                for _ in range(50):
                    x, y, z, lam, xsi, eta, mu, zet, s = (o + steg * dd for o, dd in zip(
                        old, (dx, dy, dz, dlam, dxsi, deta, dmu, dzet, ds)))
                    r = resid(x, y, z, lam, xsi, eta, mu, zet, s, epsi)
                    newnorm = np.linalg.norm(r)
                    if newnorm < 2.0 * norm:
                        break
                    steg /= 2.0
                norm = newnorm
                rmax = np.abs(r).max()
            epsi *= 0.1
        self.lam = lam
        return x



def mma_simp_loop(dims, volfrac, rmin, ke, fixed_grid, f_grid, iters, penal=3.0, penal0=1.0, ramp=20,
                  move=0.2, emin=1e-9, solve=None):
    """SIMP with the MMA update (m = 1, volume of the filtered design), the penalty ramped from
    penal0 to penal over `ramp` iterations and the objective scaled by the first compliance: the
    sensitivities of loadpath/simp.py:1901-1904 chained through the filter (loadpath/simp.py:2001),
    one MMA step per iteration (loadpath/mma.py:57-112). Returns (x, xphys, history) with history
    rows (compliance, volume fraction, change)."""
    solve = solve or (lambda e: assembled_solve(ke, e, fixed_grid, f_grid))
    taps = filter_taps(rmin)
    hs = filter_row_sums(dims, taps)
    hap = lambda v: grid_filter(v, taps)
    n = int(np.prod(dims))
    x = np.full(dims, volfrac)
    dg = (hap(np.ones(dims) / hs) / (n * volfrac)).reshape(1, -1)
    opt = MMA(n, 1, 0.0, 1.0, move)
    c0 = None
    hist = []
    for k in range(iters):
        p = penal0 + (penal - penal0) * min(k, ramp) / ramp
        xphys = hap(x) / hs
        e = simp_moduli(xphys, p, emin)
        u = solve(e)
        g = gather_cells(u, dims).reshape(24, -1)
        ce = np.einsum("in,in->n", g, ke @ g).reshape(dims)
        c = float(np.sum(e * ce))
        dc = hap(-p * (1 - emin) * xphys ** (p - 1) * ce / hs)
        c0 = c0 if c0 is not None else (abs(c) if c != 0 else 1.0)
        vol = float(xphys.sum()) / n
        xnew = opt.update(x.reshape(-1), c / c0, dc.reshape(-1) / c0, np.array([vol / volfrac - 1.0]), dg)
        xnew = np.asarray(xnew).reshape(dims)
        hist.append((c, vol, float(np.abs(xnew - x).max())))
        x = xnew
    return x, hap(x) / hs, hist

# --------------------------------------------------------------------------
# problem builders shared by the tests and the CPU baseline
# --------------------------------------------------------------------------

def cantilever_bc(dims, total=-1.0):
    """All dofs of the x = 0 face held; a -z force of `total` spread evenly
    over the nodes of the bottom edge at x = nx (z = 0), as the benchmark
    configs describe (the top3d cantilever, loadpath/benchmarks/problems.py:109-119,
    with the load rescaled to a unit total)."""
    nx, ny, nz = dims
    nshape = (nx + 1, ny + 1, nz + 1)
    fixed = np.zeros((3,) + nshape, bool)
    fixed[:, 0] = True
    f = np.zeros((3,) + nshape)
    f[2, nx, :, 0] = total / (ny + 1)
    return fixed, f


def log_uniform_density(dims, seed, lo=1e-3, radius=2.0):
    """Seeded log-uniform densities in [lo, 1], smoothed by the row-normalised
    cone filter of `radius` (the benchmark configs' synthetic density)."""
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(np.log(lo), 0.0, size=dims))
    taps = filter_taps(radius)
    return grid_filter(x, taps) / filter_row_sums(dims, taps)
