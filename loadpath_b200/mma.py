"""The Method of Moving Asymptotes with its n-sized work on the device (loadpath/mma.py:31-214).

`MMA(n, m, xmin=0.0, xmax=1.0, move=0.2, c=1000.0, asyinit=0.5, asyincr=1.2, asydecr=0.7)` with
`.update(x, f0, df0, f, df) -> xnew` and `.tighten(factor)`, as loadpath's class: the problem

    minimize    f0(x) + a0 z + sum_i (c_i y_i + 0.5 d_i y_i^2)
    subject to  f_i(x) - a_i z - y_i <= 0,   xmin <= x <= xmax,  y_i >= 0, z >= 0

with a0 = 1, a_i = 0, d_i = 1, solved each iteration by Svanberg's primal-dual interior-point
method on the convex separable approximation built from moving asymptotes. The design, the
asymptotes, the approximation's terms and the subsolver's n-sized variables (x, xsi, eta and their
Newton directions) live on the device; each pass over them is one of lp_mma.cu's kernels with its
reductions. The host keeps the m-sized variables (y, z, lam, mu, zet, s), runs the loops (epsi from
1 down to 1e-7, Newton steps, the line search of up to 50 halvings) and solves the (m + 1) x (m + 1)
Newton system, exactly as the reference orders them. m <= 8.

x, df0 and df may be numpy arrays (copied to the device; the result comes back as numpy) or
float64 CUDA tensors (the result is a CUDA tensor).
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import lib
from .grid import stream_handle

__all__ = ["MMA"]

MAXM = 8


def _mround(m):
    return 1 if m <= 1 else 2 if m <= 2 else 4 if m <= 4 else 8


class MMA:
    def __init__(self, n, m, xmin=0.0, xmax=1.0, move=0.2, c=1000.0, asyinit=0.5, asyincr=1.2, asydecr=0.7,
                 device="cuda"):
        if not 1 <= m <= MAXM:
            raise ValueError(f"MMA on the device takes 1 <= m <= {MAXM} constraints, got {m}")
        self.n, self.m = int(n), int(m)
        self.M = _mround(self.m)
        self.device = torch.device(device)
        dev = dict(dtype=torch.float64, device=self.device)
        n = self.n

        def vec(v):
            return torch.as_tensor(np.broadcast_to(np.asarray(v, float), (n,)).copy(), **dev)

        self.xmin, self.xmax = vec(xmin), vec(xmax)
        self.move = float(move)
        self.a0 = 1.0
        self.a = np.zeros(m)
        self.c = np.full(m, float(c))
        self.d = np.ones(m)
        self.asyinit, self.asyincr, self.asydecr = float(asyinit), float(asyincr), float(asydecr)
        self.iter = 0
        self.lam = None
        z = lambda *shape: torch.zeros(shape if shape else (n,), **dev)  # noqa: E731
        self._x, self.low, self.upp, self._xold1, self._xold2 = z(), z(), z(), z(), z()
        self._alfa, self._beta, self._p0, self._q0 = z(), z(), z(), z()
        self._P, self._Q, self._df = z(m, n), z(m, n), z(m, n)
        self._df0, self._xnew = z(), z()
        self._sets = [(z(), z(), z()), (z(), z(), z())]   # (x, xsi, eta) of the subsolver, two sets
        self._dx, self._dxsi, self._deta, self._delx, self._diagx = z(), z(), z(), z(), z()
        self._part = torch.zeros(int(lib().lpb_mma_part_len(m)), **dev)
        self._out = torch.zeros(64, **dev)
        self._have_asy = False
        self._have_old = False

    # -- reference API ------------------------------------------------------------------------
    def tighten(self, factor):
        """Pull the asymptotes toward the last design by `factor` (loadpath/mma.py:48-55)."""
        if self._have_old and self._have_asy:
            self.low.copy_(self._xold1 - factor * (self._xold1 - self.low))
            self.upp.copy_(self._xold1 + factor * (self.upp - self._xold1))

    def update(self, x, f0, df0, f, df):
        """One MMA step (loadpath/mma.py:57-112); returns the new design."""
        L = lib()
        st = stream_handle()
        n, m = self.n, self.m
        host = not isinstance(x, torch.Tensor)
        self._x.copy_(torch.as_tensor(np.asarray(x, float) if host else x).reshape(n))
        self._df0.copy_(torch.as_tensor(np.asarray(df0, float) if not isinstance(df0, torch.Tensor) else df0).reshape(n))
        self._df.copy_(torch.as_tensor(np.asarray(df, float) if not isinstance(df, torch.Tensor) else df).reshape(m, n))
        f = np.nan_to_num(np.asarray(f, float).reshape(m), nan=1e6, posinf=1e6, neginf=-1e6)
        self.iter += 1
        init = self.iter <= 2 or not self._have_asy
        L.lpb_mma_prepare(n, m, self._x.data_ptr(), self.xmin.data_ptr(), self.xmax.data_ptr(), self.low.data_ptr(),
                          self.upp.data_ptr(), None if init else self._xold1.data_ptr(),
                          None if init else self._xold2.data_ptr(), int(init), self.asyinit, self.asyincr,
                          self.asydecr, self.move, self._df0.data_ptr(), self._df.data_ptr(), self._alfa.data_ptr(),
                          self._beta.data_ptr(), self._p0.data_ptr(), self._q0.data_ptr(), self._P.data_ptr(),
                          self._Q.data_ptr(), self._part.data_ptr(), self._out.data_ptr(), st)
        self._have_asy = True
        b = self._out[:m].cpu().numpy() - f
        xs = self._subsolv(b)
        L.lpb_mma_finish(n, xs.data_ptr(), self._x.data_ptr(), self._alfa.data_ptr(), self._beta.data_ptr(),
                         self._xnew.data_ptr(), st)
        self._xold2.copy_(self._xold1 if self._have_old else self._x)
        self._xold1.copy_(self._x)
        self._have_old = True
        return self._xnew.cpu().numpy() if host else self._xnew.clone()

    # -- the subproblem (loadpath/mma.py:114-214) ---------------------------------------------
    def _arrays(self):
        return (self.low.data_ptr(), self.upp.data_ptr(), self._alfa.data_ptr(), self._beta.data_ptr())

    def _residual(self, cur, nxt, d, steg, lam, y, z, mu, zet, s, epsi, b):
        """Norm and largest magnitude of the KKT residual; with d given, the point cur + steg d
        is written to nxt first (the device part), the m-sized part from the host values."""
        L = lib()
        m = self.m
        dx = d[0].data_ptr() if d is not None else None
        dxsi = d[1].data_ptr() if d is not None else None
        deta = d[2].data_ptr() if d is not None else None
        L.lpb_mma_trial(self.n, m, *self._arrays(), self._p0.data_ptr(), self._q0.data_ptr(), self._P.data_ptr(),
                        self._Q.data_ptr(), cur[0].data_ptr(), cur[1].data_ptr(), cur[2].data_ptr(), dx, dxsi, deta,
                        float(steg), np.ascontiguousarray(lam, float).ctypes.data, float(epsi),
                        nxt[0].data_ptr(), nxt[1].data_ptr(), nxt[2].data_ptr(), self._part.data_ptr(),
                        self._out.data_ptr(), stream_handle())
        o = self._out[:2 + self.M].cpu().numpy()
        gvec = o[2:2 + m]
        small = np.concatenate([self.c + self.d * y - mu - lam, [self.a0 - zet - self.a @ lam],
                                gvec - self.a * z - y + s - b, mu * y - epsi, [zet * z - epsi], lam * s - epsi])
        norm = np.sqrt(o[0] + small @ small)
        rmax = max(o[1], np.abs(small).max())
        return norm, rmax

    def _subsolv(self, b, epsimin=1e-7):
        L = lib()
        st = stream_handle()
        n, m, M = self.n, self.m, self.M
        a0, a, c, d = self.a0, self.a, self.c, self.d
        cur, nxt = self._sets
        L.lpb_mma_sub_init(n, self._alfa.data_ptr(), self._beta.data_ptr(), cur[0].data_ptr(), cur[1].data_ptr(),
                           cur[2].data_ptr(), st)
        y = np.ones(m)
        z = 1.0
        lam = np.ones(m)
        mu = np.maximum(1.0, 0.5 * c)
        zet = 1.0
        s = np.ones(m)
        epsi = 1.0
        dvec = (self._dx, self._dxsi, self._deta)
        ntri = M * (M + 1) // 2
        iu = np.triu_indices(M)
        while epsi > epsimin:
            norm, rmax = self._residual(cur, cur, None, 0.0, lam, y, z, mu, zet, s, epsi, b)
            it = 0
            while rmax > 0.9 * epsi and it < 200:
                it += 1
                L.lpb_mma_newton_a(n, m, *self._arrays(), self._p0.data_ptr(), self._q0.data_ptr(),
                                   self._P.data_ptr(), self._Q.data_ptr(), cur[0].data_ptr(), cur[1].data_ptr(),
                                   cur[2].data_ptr(), np.ascontiguousarray(lam, float).ctypes.data, float(epsi),
                                   self._delx.data_ptr(), self._diagx.data_ptr(), self._part.data_ptr(),
                                   self._out.data_ptr(), st)
                o = self._out[:2 * M + ntri].cpu().numpy()
                gvec, bl = o[:m], o[M:M + m]
                tri = np.zeros((M, M))
                tri[iu] = o[2 * M:2 * M + ntri]
                gg = (tri + np.triu(tri, 1).T)[:m, :m]
                dely = c + d * y - lam - epsi / y
                delz = a0 - a @ lam - epsi / z
                dellam = gvec - a * z - y - b + epsi / lam
                diagy = d + mu / y
                diaglamyi = s / lam + 1.0 / diagy
                blam = dellam + dely / diagy - bl
                alam = np.diag(diaglamyi) + gg
                aa = np.zeros((m + 1, m + 1))
                aa[:m, :m] = alam
                aa[:m, m] = a
                aa[m, :m] = a
                aa[m, m] = -zet / z
                sol = np.linalg.solve(aa, np.concatenate([blam, [delz]]))
                dlam, dz = sol[:m], sol[m]
                L.lpb_mma_newton_b(n, m, *self._arrays(), self._P.data_ptr(), self._Q.data_ptr(), cur[0].data_ptr(),
                                   cur[1].data_ptr(), cur[2].data_ptr(), self._delx.data_ptr(), self._diagx.data_ptr(),
                                   np.ascontiguousarray(dlam, float).ctypes.data, float(epsi), self._dx.data_ptr(),
                                   self._dxsi.data_ptr(), self._deta.data_ptr(), self._part.data_ptr(),
                                   self._out.data_ptr(), st)
                mx = self._out[:4].cpu().numpy()
                dy = -dely / diagy + dlam / diagy
                dmu = -mu + epsi / y - mu * dy / y
                dzet = -zet + epsi / z - zet * dz / z
                ds = -s + epsi / lam - s * dlam / lam
                xx = np.concatenate([y, [z], lam, mu, [zet], s])
                dxx = np.concatenate([dy, [dz], dlam, dmu, [dzet], ds])
                stmxx = max(np.max(-1.01 * dxx / xx), mx[0], mx[1])
                steg = 1.0 / max(mx[2], mx[3], stmxx, 1.0)
                old = (y, z, lam, mu, zet, s)
                for _ in range(50):
                    y = old[0] + steg * dy
                    z = old[1] + steg * dz
                    lam = old[2] + steg * dlam
                    mu = old[3] + steg * dmu
                    zet = old[4] + steg * dzet
                    s = old[5] + steg * ds
                    newnorm, newmax = self._residual(cur, nxt, dvec, steg, lam, y, z, mu, zet, s, epsi, b)
                    if newnorm < 2.0 * norm:
                        break
                    steg /= 2.0
                cur, nxt = nxt, cur
                norm, rmax = newnorm, newmax
            epsi *= 0.1
        self._sets = [cur, nxt]
        self.lam = lam
        return cur[0]
