"""Generate the golden fixtures in this folder from the reference implementation.

Run in a container that has the loadpath source tree (read-only is fine):

    LOADPATH_SRC=/path/to/loadpath python tests/golden/make_golden.py [name ...]

(names: element transfers femops filter mma hierarchies top3d config0 oc_step optimize constrained callers
springs; default all but config0,
which runs the reference's top3d port for 20 iterations at 60x20x10 and takes a few minutes).

It imports loadpath's own modules (fem, mg, mgops, femops, simp, mma,
benchmarks.*), runs them on small seeded inputs and stores inputs and outputs
as .npz files here. The tests in tests/test_oracle_golden.py pin the oracle
against these files; the GPU tests then pin the CUDA path against the oracle.
Nothing at test time reads the loadpath tree.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.environ.get("LOADPATH_SRC")
if not SRC:
    raise SystemExit("set LOADPATH_SRC to the loadpath source tree (the folder that holds the loadpath package)")
os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "lp_numba_cache"))
os.environ["LOADPATH_DEVICE"] = "cpu"
sys.path.insert(0, SRC)


def _full_mesh(dims, pitch=1.0):
    from loadpath.fem import HexMesh

    ijk = np.argwhere(np.ones(dims, bool))
    return HexMesh(ijk, pitch, np.zeros(3))


def _cantilever(mesh, dims):
    nx = dims[0]
    fixed = np.zeros(mesh.n_dof, bool)
    root = np.flatnonzero(mesh.node_ijk[:, 0] == 0)
    for i in range(3):
        fixed[3 * root + i] = True
    f = np.zeros(mesh.n_dof)
    tip = np.flatnonzero((mesh.node_ijk[:, 0] == nx) & (mesh.node_ijk[:, 2] == 0))
    f[3 * tip + 2] = -1.0 / len(tip)
    return fixed, f


def make_element():
    from loadpath.fem import hex8_ke

    out = {}
    for el in ("plain", "im"):
        for nu in (0.3, 0.35):
            out[f"ke_{el}_{nu}"] = hex8_ke(nu, el)
    np.savez_compressed(os.path.join(HERE, "element.npz"), **out)


def make_transfers():
    from loadpath.mg import _PK, prolong, restrict

    rng = np.random.default_rng(11)
    c = rng.standard_normal((3, 5, 4, 6))
    f = rng.standard_normal((3, 9, 7, 11))
    c32 = c.astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "transfers.npz"), pk=_PK, c=c, f=f, prolong_c=prolong(c),
                        restrict_f=restrict(f), c32=c32, prolong_c32=prolong(c32))


def make_hierarchy(name, dims, element, seed, coarse_cells, void_frac, pitch=1.0, smooth=True):
    """A GridElasticity hierarchy on a full grid with some removed cells; the
    densities are seeded log-uniform, smoothed by the r = 2 cone filter (as
    the benchmark configs describe) unless `smooth` is False."""
    os.environ["LOADPATH_HEX8"] = element
    from loadpath.mg import GridElasticity
    from loadpath import mgops

    mesh = _full_mesh(dims, pitch)
    fixed, f = _cantilever(mesh, dims)
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(np.log(1e-3), 0.0, mesh.n_elem))
    if smooth:
        x = _smoothed(x.reshape(dims), 2.0).reshape(-1)
    e = 1e-9 + x ** 3 * (1 - 1e-9)
    e[rng.random(mesh.n_elem) < void_frac] = 0.0
    g = GridElasticity(mesh, 0.3, fixed, rtol=1e-10, maxiter=3000, coarse_cells=coarse_cells, device="cpu")
    g.set_moduli(e)
    out = dict(dims=np.array(dims), cells=np.array(g.cells), pitch=pitch, e_mesh=e, f_mesh=f, fixed_mesh=fixed,
               e_grid=g.cell_grid(e), f_grid=g.to_grid(f), fixed_grid=g.fixed_grid, ke=g.ke, strict=g.strict,
               nlevels=len(g.levels), alive=g.alive)
    for i in range(len(g.levels)):
        lv = g._op(i)
        out[f"L{i}_kind"] = lv.kind
        out[f"L{i}_mask"] = lv.mask
        out[f"L{i}_dinv"] = lv.dinv
        out[f"L{i}_lmax"] = lv.lmax
        if lv.kind == "weights":
            out[f"L{i}_w"] = lv.w
            out[f"L{i}_patch_ijk"] = lv.patch_ijk
            out[f"L{i}_patch_k"] = lv.patch_k
            out[f"L{i}_mcat"] = lv.mcat
        elif lv.kind == "explicit":
            out[f"L{i}_k"] = lv.k
        # the operator on seeded inputs, both precisions on the fine level
        u = rng.standard_normal(lv.node_shape).astype(lv.mask.dtype)
        out[f"L{i}_u"] = u
        out[f"L{i}_apply"] = lv.apply(u)
        out[f"L{i}_diag"] = lv.diagonal()
    l0 = g.levels[0]
    u64 = rng.standard_normal(l0.node_shape)
    out["L0_u64"] = u64
    out["L0_apply64"] = l0.apply(u64)
    # transfers between level 0 and 1 in the V-cycle precision
    if len(g.levels) > 1:
        lv, nxt = g._op(0), g._op(1)
        b = rng.standard_normal(lv.node_shape).astype(np.float32)
        ax = rng.standard_normal(lv.node_shape).astype(np.float32)
        xc = rng.standard_normal(nxt.node_shape).astype(np.float32)
        x = rng.standard_normal(lv.node_shape).astype(np.float32)
        out.update(t_b=b, t_ax=ax, t_xc=xc, t_x=x,
                   t_coarse_residual=mgops.coarse_residual(b, ax, lv.mask, nxt.mask, nxt.node_shape))
        x2 = x.copy()
        mgops.add_correction(xc, nxt.mask, lv.mask, x2)
        out["t_add_correction"] = x2
    # one V-cycle on a seeded residual, then the full solve and its energies
    r = (rng.standard_normal(l0.node_shape) * l0.mask)
    out["vc_r"] = r
    out["vc_z"] = g.precondition(r)
    u = g.solve_many([f])[0]
    out["u_mesh"] = u
    out["u_grid"] = g.to_grid(u)
    out["iters"] = g.last_iters
    out["compliance"] = float(f @ u)
    out["strain_energy"] = g.strain_energy(u)
    # warm start from a scaled copy
    g.set_moduli(e * 1.1)
    w = g.solve_many([f], [u])[0]
    out["u_warm_grid"] = g.to_grid(w)
    out["iters_warm"] = g.last_iters
    np.savez_compressed(os.path.join(HERE, f"hier_{name}.npz"), **out)
    print(name, "levels", len(g.levels), "iters", out["iters"], "warm", out["iters_warm"], "strict", g.strict)


def _smoothed(x, radius):
    """Row-normalised cone filter of the reference's top3d port on a full grid."""
    from loadpath.benchmarks.evaluate import Evaluator
    from loadpath.benchmarks.problems import Problem
    from loadpath.benchmarks.reference import _filter

    p = Problem(name="s", title="", source="", dims=x.shape, volfrac=0.3, rmin=radius, fixed=[], loads=[],
                references=[])
    ev = Evaluator(p)
    h, hs = _filter(ev, radius)
    out = np.zeros(x.shape)
    out[ev.cell] = (h @ ev.cells(x)) / hs
    return out


def make_femops():
    os.environ["LOADPATH_HEX8"] = "im"
    from loadpath import femops
    from loadpath.fem import HexMesh, hex8_ke

    rng = np.random.default_rng(5)
    dims = (7, 5, 4)
    mesh = _full_mesh(dims)
    u = rng.standard_normal(mesh.n_dof)
    v = rng.standard_normal(mesh.n_dof)
    ke = hex8_ke(0.3, "im")
    out = femops.element_energy(u, v, mesh.edof, ke)
    uu = femops.element_energy(u, None, mesh.edof, ke)
    assert isinstance(mesh, HexMesh)
    np.savez_compressed(os.path.join(HERE, "femops.npz"), dims=np.array(dims), u=u, v=v, ke=ke, uv=out, uu=uu,
                        edof=mesh.edof)


def make_filter():
    from loadpath.benchmarks.evaluate import Evaluator
    from loadpath.benchmarks.problems import Problem
    from loadpath.benchmarks.reference import _filter
    from loadpath.simp import GridFilter, _dproject, _project

    class _Dom:
        pass

    dims = (9, 7, 5)
    out = {"dims": np.array(dims)}
    rng = np.random.default_rng(7)
    v = rng.random(dims)
    out["v"] = v
    for r in (1.5, 2.0, 3.0):
        d = _Dom()
        d.mesh = _full_mesh(dims)
        d.dims = dims
        d.pitch = 1.0
        h = GridFilter(d, r)
        out[f"grid_{r}"] = h @ v[tuple(d.mesh.elem_ijk.T)]
        out[f"ntaps_{r}"] = len(h.taps)
        p = Problem(name="f", title="", source="", dims=dims, volfrac=0.3, rmin=r, fixed=[], loads=[], references=[])
        ev = Evaluator(p)
        hh, hs = _filter(ev, r)
        out[f"top3d_{r}"] = hh @ ev.cells(v)
        out[f"top3d_hs_{r}"] = hs
        out[f"top3d_cellorder_{r}"] = np.stack(ev.cell, axis=1)
    xt = rng.random(50)
    out["proj_x"] = xt
    for beta in (1.0, 8.0):
        out[f"proj_{beta}"] = _project(xt, beta, 0.5)
        out[f"dproj_{beta}"] = _dproject(xt, beta, 0.5)
    np.savez_compressed(os.path.join(HERE, "filter.npz"), **out)


def make_top3d():
    import loadpath.benchmarks.reference as ref
    from loadpath.benchmarks.problems import cantilever_3d, get

    os.environ["LOADPATH_HEX8"] = "plain"
    p = cantilever_3d(12, 4, 6, 0.3, 1.5)
    hist = []
    ref.TOP3D_MAXIT = 8
    rec = ref.optimize_reference(p, "top3d", on_iter=lambda loop, c, ch: hist.append((c, ch)))
    ref.TOP3D_MAXIT = 200
    stored = ref.load_reference(get("cantilever-3d"), "top3d")
    np.savez_compressed(os.path.join(HERE, "top3d.npz"), dims=np.array(p.dims), volfrac=p.volfrac, rmin=p.rmin,
                        xphys=rec["x"], hist=np.array(hist), stored_x=stored["x"].astype(np.float32),
                        stored_iters=stored["iterations"], stored_c=stored["compliance_reported"],
                        stored_dims=np.array(get("cantilever-3d").dims))


def make_mma():
    from loadpath.mma import MMA

    rng = np.random.default_rng(9)
    n, m = 40, 2
    mma = MMA(n, m, move=0.2)
    x = rng.random(n) * 0.8 + 0.1
    steps = []
    for it in range(4):
        df0 = rng.standard_normal(n)
        f = rng.standard_normal(m) * 0.1
        df = rng.standard_normal((m, n))
        xn = mma.update(x, 1.0, df0, f, df)
        steps.append((x.copy(), df0, f, df, xn))
        x = xn
    out = {}
    for i, (a, b, c, d, e) in enumerate(steps):
        out.update({f"x{i}": a, f"df0{i}": b, f"f{i}": c, f"df{i}": d, f"xn{i}": e})
    np.savez_compressed(os.path.join(HERE, "mma.npz"), n=n, m=m, steps=len(steps), **out)


def make_config0():
    """The 60x20x10 cantilever (top3d's default problem at that size, "im" element) with a unit total
    load: 20 iterations of the reference's top3d port (SuperLU direct solves), its compliance and
    change history and the final physical densities."""
    import dataclasses

    os.environ["LOADPATH_HEX8"] = "im"
    import loadpath.benchmarks.reference as ref
    from loadpath.benchmarks.problems import cantilever_3d

    p = cantilever_3d(60, 20, 10, 0.3, 1.5)
    nodes, comp, val = p.loads[0]
    p = dataclasses.replace(p, loads=[(nodes, comp, val / (p.dims[1] + 1))])
    hist = []
    ref.TOP3D_MAXIT = 20
    rec = ref.optimize_reference(p, "top3d", on_iter=lambda loop, c, ch: hist.append((c, ch)))
    ref.TOP3D_MAXIT = 200
    np.savez_compressed(os.path.join(HERE, "config0.npz"), dims=np.array(p.dims), volfrac=p.volfrac, rmin=p.rmin,
                        xphys=rec["x"], hist=np.array(hist), load_per_node=val / (p.dims[1] + 1))


def make_oc_step():
    """loadpath's design step as a whole (loadpath/simp.py:2249-2376: the optimality-criteria step
    whose volume multiplier is bracketed outward from the last step's in log space, then found by
    false position with the Illinois halving), captured from the reference's own optimize on the
    12x4x6 cantilever of its benchmarks (domain_for: load and support cells pinned, padded filter,
    default options) for its first three iterations. numpy inside loadpath.simp is replaced by a
    pass-through whose clip, called by the step's trial function, records the trial's inputs (the
    design x, ratio = sqrt(-dc / dv), the move limits, beta, the volume target, the last step's
    multiplier) and outputs from the calling frames; the accepted step is the last trial of an
    iteration."""
    os.environ["LOADPATH_HEX8"] = "im"
    import loadpath.simp as S
    from loadpath.benchmarks.problems import cantilever_3d
    from loadpath.benchmarks.run import NU, design_volfrac, domain_for

    p = cantilever_3d(12, 4, 6, 0.3, 1.5)
    dom, _ = domain_for(p)
    opts = S.SimpOptions(volume_fraction=design_volfrac(p, dom), filter_radius=p.rmin, max_iterations=3)
    real_np = S.np
    trials = []

    class _Numpy:
        def __getattr__(self, k):
            return getattr(real_np, k)

        def clip(self, a, lo, hi, *args, **kw):
            out = real_np.clip(a, lo, hi, *args, **kw)
            f1 = sys._getframe(1)
            if f1.f_code.co_name == "stepped":
                l1, l2 = f1.f_locals, f1.f_back.f_locals
                trials.append(dict(it=int(l2["it"]), x=l1["x"].copy(), ratio=l1["ratio"].copy(), move=float(l2["move"]),
                                   beta=float(l1["beta"]), target=float(l1["target"]),
                                   lam_last=float(l2["lam_last"]) if l2["lam_last"] is not None else float("nan"),
                                   lm=float(l1["lm_"]), xn=out.copy(), pres=l1["pres"].copy(),
                                   wdesign=l1["wdesign"].copy(), void=l1["void"]))
            return out

    S.np = _Numpy()
    try:
        S.optimize(dom, NU, opts)
    finally:
        S.np = real_np
    its = sorted({t["it"] for t in trials})
    out = dict(dims=np.array(dom.dims), pitch=float(dom.mesh.pitch), radius=float(opts.filter_radius),
               pad=bool(S._pad(opts)), eta=float(opts.eta), elem_ijk=dom.mesh.elem_ijk, iterations=np.array(its))
    for k, it in enumerate(its):
        mine = [t for t in trials if t["it"] == it]
        first, last = mine[0], mine[-1]
        assert first["void"] is None
        xn = last["xn"].copy()
        xn[first["pres"]] = 1.0
        out.update({f"x{k}": first["x"], f"ratio{k}": first["ratio"], f"move{k}": first["move"],
                    f"beta{k}": first["beta"], f"target{k}": first["target"], f"lam_last{k}": first["lam_last"],
                    f"pres{k}": first["pres"], f"w{k}": first["wdesign"], f"x_new{k}": xn, f"lm{k}": last["lm"],
                    f"n_eval{k}": len(mine)})
    np.savez_compressed(os.path.join(HERE, "oc_step.npz"), **out)


def make_optimize():
    """loadpath's own SIMP loop as a whole (loadpath/simp.py:1640-2455, simp.optimize with its
    default options: blueprint and eroded projections, the measured step length, beta
    continuation, the volume multiplier solved to rounding) on two top3d cantilevers and a bridge
    mirrored in x and y, and with the fixed move schedule (adaptive_move off, beta up to 8, run
    to its stall rule) on the small cantilever, of its benchmarks (domain_for: load and support cells pinned, padded
    filter), with the solves
    tightened to rtol 1e-10 so that a solver of another kind can be compared iteration by
    iteration. Stored per case: the domain on the node / cell grid (supports, load, pinned cells),
    the options, and per iteration the record the loop reports and the blueprint density it
    started from; and the last design."""
    os.environ["LOADPATH_HEX8"] = "im"
    import loadpath.simp as S
    from loadpath.benchmarks.problems import bridge_3d, cantilever_3d
    from loadpath.benchmarks.run import NU, design_volfrac, domain_for

    out = {}
    cases = {"small": (cantilever_3d, (12, 4, 6), 0.3, 1.5, 30, {}),
             "medium": (cantilever_3d, (20, 6, 10), 0.3, 2.0, 24, {}),
             "bridge": (bridge_3d, (16, 4, 6), 0.15, 1.5, 24, {}),
             "fixedmove": (cantilever_3d, (12, 4, 6), 0.3, 1.5, 48, {"adaptive_move": False, "beta_max": 8.0}),
             "twocase": (cantilever_3d, (12, 4, 6), 0.3, 1.5, 24, {})}
    for name, (problem, dims, vf, rmin, iters, extra) in cases.items():
        p = problem(*dims, vf, rmin)
        dom, _ = domain_for(p)
        mesh = dom.mesh
        assert mesh.n_elem == int(np.prod(dims)) and len(dom.loads) == 1 and dom.springs is None
        f_second = None
        if name == "twocase":
            # a second case on the same nodes, an axial pull, weighed at half the first
            f_second = np.zeros_like(dom.loads[0])
            on = np.flatnonzero(dom.loads[0].reshape(-1, 3).any(axis=1))
            f_second[3 * on] = 0.8
            dom.loads = [dom.loads[0], f_second]
            dom.case_weights = [1.0, 0.5]
            dom.spreads = [None, None]
            dom.case_names = ["down", "pull"]
        axes = {"x": 0, "y": 1, "z": 2}
        for ax, m in dom.mirror.items():
            assert np.all(m >= 0)
            mirrored = mesh.elem_ijk.copy()
            mirrored[:, axes[ax]] = dims[axes[ax]] - 1 - mirrored[:, axes[ax]]
            assert np.array_equal(mesh.elem_ijk[m], mirrored)
        opts = S.SimpOptions(volume_fraction=design_volfrac(p, dom), filter_radius=p.rmin, max_iterations=iters,
                             solve_rtol=1e-10, **extra)
        recs, xps = [], []
        res = S.optimize(dom, NU, opts, on_iter=lambda r, xp: (recs.append(r), xps.append(np.array(xp))))
        nxyz = np.array(dims) + 1
        fixed = np.zeros((3, *nxyz), bool)
        f = np.zeros((3, *nxyz))
        nijk = tuple(mesh.node_ijk.T)
        f2 = np.zeros((3, *nxyz))
        for c in range(3):
            fixed[c][nijk] = dom.fixed[c::3]
            f[c][nijk] = dom.loads[0][c::3]
            if f_second is not None:
                f2[c][nijk] = f_second[c::3]
        if f_second is not None:
            out[f"{name}_f2"] = f2
        cells = tuple(mesh.elem_ijk.T)

        def grid(v):
            g = np.zeros(dims, np.asarray(v).dtype)
            g[cells] = v
            return g

        keys = ("compliance", "relative", "volume", "beta", "change", "move", "volumeSolves", "solvedCells")
        out.update({f"{name}_dims": np.array(dims), f"{name}_pitch": float(mesh.pitch), f"{name}_nu": float(NU),
                    f"{name}_fixed": fixed, f"{name}_f": f, f"{name}_pres": grid(dom.preserve),
                    f"{name}_volfrac": float(opts.volume_fraction), f"{name}_radius": float(opts.filter_radius),
                    f"{name}_pad": bool(S._pad(opts)), f"{name}_emin": float(S.E_MIN),
                    f"{name}_penal": float(S.PENALTY), f"{name}_iterations": len(recs),
                    f"{name}_mirror": np.array([axes[a] for a in dom.mirror], np.int64),
                    f"{name}_adaptive_move": bool(opts.adaptive_move), f"{name}_beta_max": float(opts.beta_max),
                    f"{name}_converged": bool(res.converged), f"{name}_weights": np.array(dom.case_weights, float),
                    f"{name}_xphys": np.stack([grid(v) for v in xps]), f"{name}_x_last": grid(res.x)})
        for k in keys:
            out[f"{name}_{k}"] = np.array([float(r.get(k, np.nan)) for r in recs])
        out[f"{name}_stepFit"] = np.array([float(r.get("stepFit", np.nan)) for r in recs])
    np.savez_compressed(os.path.join(HERE, "optimize.npz"), **out)


def make_constrained():
    """loadpath's minimum-mass loop under stress and deflection limits (loadpath/constrained.py:
    295-854, optimize_constrained: relaxed von Mises at the cells' corners aggregated by a P-mean
    with the adaptive normalisation, one adjoint solve per case, MMA on the free cells, its own
    beta continuation) on top3d cantilevers (domain_for), from a uniform 0.5, solves at rtol
    1e-10: both limits on the 12x4x6 one for 40 iterations (constrained.npz), a deflection limit
    alone and a stress limit alone on a 16x4x8 one for 30 (constrained_deflection.npz,
    constrained_stress.npz), both limits with beta_max 4 run to the loop's own stop
    (constrained_converge.npz: the lightest feasible design delivered), and both limits on two
    load cases, the second an axial pull on the loaded nodes (constrained_twocase.npz: four
    constraints). Stored: the domain, the limits, and per iteration the
    record (volume, beta, change, constraints, deflection and stress readings, solved cells) and
    the blueprint; and the last design."""
    os.environ["LOADPATH_HEX8"] = "im"
    import loadpath.simp as S
    from loadpath.benchmarks.problems import cantilever_3d
    from loadpath.benchmarks.run import NU, domain_for
    from loadpath.constrained import Limits, optimize_constrained

    for tag, dims, iters, lim, extra in (("", (12, 4, 6), 40, Limits(12.0, 0.6, 1000.0), {}),
                                         ("_deflection", (16, 4, 8), 30, Limits(None, 0.5, 1000.0), {}),
                                         ("_stress", (16, 4, 8), 30, Limits(9.0, None, 1000.0), {}),
                                         ("_converge", (12, 4, 6), 100, Limits(12.0, 0.6, 1000.0),
                                          {"beta_max": 4.0}),
                                         ("_twocase", (12, 4, 6), 30, Limits(12.0, 0.6, 1000.0), {})):
        _constrained_case(S, cantilever_3d, NU, domain_for, optimize_constrained, tag, dims, iters, lim, extra)


def _constrained_case(S, cantilever_3d, NU, domain_for, optimize_constrained, tag, dims, iters, lim, extra):
    p = cantilever_3d(*dims, 0.3, 1.5)
    dom, _ = domain_for(p)
    mesh = dom.mesh
    assert mesh.n_elem == int(np.prod(dims)) and len(dom.loads) == 1
    f_second = None
    if tag == "_twocase":
        # a second case on the same nodes, an axial pull (its own deflection and stress limits)
        f_second = np.zeros_like(dom.loads[0])
        on = np.flatnonzero(dom.loads[0].reshape(-1, 3).any(axis=1))
        f_second[3 * on] = 0.8
        dom.loads = [dom.loads[0], f_second]
        dom.case_weights = [1.0, 0.5]
        dom.spreads = [None, None]
        dom.case_names = ["down", "pull"]
    opts = S.SimpOptions(volume_fraction=0.5, filter_radius=p.rmin, max_iterations=iters, solve_rtol=1e-10, **extra)
    recs, xps = [], []
    res = optimize_constrained(dom, NU, opts, lim, on_iter=lambda r, xp: (recs.append(r), xps.append(np.array(xp))))
    nxyz = np.array(dims) + 1
    fixed = np.zeros((3, *nxyz), bool)
    f = np.zeros((3, *nxyz))
    nijk = tuple(mesh.node_ijk.T)
    for c in range(3):
        fixed[c][nijk] = dom.fixed[c::3]
        f[c][nijk] = dom.loads[0][c::3]
    cells = tuple(mesh.elem_ijk.T)

    def grid(v):
        g = np.zeros(dims, np.asarray(v).dtype)
        g[cells] = v
        return g

    axes = {"x": 0, "y": 1, "z": 2}
    name = dom.case_names[0]
    out = dict(dims=np.array(dims), pitch=float(mesh.pitch), nu=float(NU), fixed=fixed, f=f, pres=grid(dom.preserve),
               volfrac=float(opts.volume_fraction), radius=float(opts.filter_radius), pad=bool(S._pad(opts)),
               mirror=np.array([axes[a] for a in dom.mirror], np.int64),
               stress_limit=np.nan if lim.stress is None else lim.stress,
               deflection_limit=np.nan if lim.deflection is None else lim.deflection, modulus=lim.modulus,
               iterations=len(recs), converged=bool(res.converged), xphys=np.stack([grid(v) for v in xps]),
               x_last=grid(res.x), constraints=np.array([r["constraints"] for r in recs]),
               deflection=np.array([r.get(f"deflection.{name}", np.nan) for r in recs]),
               stress=np.array([r.get(f"stress.{name}", np.nan) for r in recs]),
               contact=grid((dom.support_nodes | dom.load_nodes)[mesh.enode].any(axis=1)),
               beta_max=float(opts.beta_max), max_iterations=int(iters),
               delivered_iteration=int(res.delivered["iteration"]) if res.delivered else -1)
    if f_second is not None:
        f2 = np.zeros((3, *nxyz))
        for c in range(3):
            f2[c][nijk] = f_second[c::3]
        out["f2"] = f2
        out["deflection_cases"] = np.array([[r.get(f"deflection.{n}", np.nan) for n in dom.case_names] for r in recs])
        out["stress_cases"] = np.array([[r.get(f"stress.{n}", np.nan) for n in dom.case_names] for r in recs])
    for k in ("volume", "beta", "change", "solvedCells"):
        out[k] = np.array([float(r[k]) for r in recs])
    np.savez_compressed(os.path.join(HERE, f"constrained{tag}.npz"), **out)


def make_callers():
    """Two other users of GridElasticity, on a mesh that is not a full box (an L-shaped part:
    a 12x6x8 box at pitch 0.5 without its upper +x quarter), held at its base:
    - verification's re-solve on a delivered grid (loadpath/verify.py:1689-1704): one
      set_moduli with per-cell moduli, two right-hand sides through solve_many;
    - the build simulation's layer-by-layer solves (loadpath/buildsim.py:609-640): one solver,
      set_moduli(e * active) as each layer of cells is added (the cells not yet built at modulus
      0), one load per layer on the built nodes.
    Solves at rtol 1e-10; the reference's own GridElasticity (device "cpu")."""
    os.environ["LOADPATH_HEX8"] = "im"
    from loadpath.fem import HexMesh
    from loadpath.mg import GridElasticity

    rng = np.random.default_rng(12)
    full = np.ones((12, 6, 8), bool)
    full[6:, :, 4:] = False
    mesh = HexMesh(np.argwhere(full), 0.5, np.zeros(3))
    fixed = np.zeros(mesh.n_dof, bool)
    base = np.flatnonzero(mesh.node_ijk[:, 2] == 0)
    for i in range(3):
        fixed[3 * base + i] = True
    e = 1700.0 * (0.5 + rng.random(mesh.n_elem))
    top = mesh.node_ijk[:, 2] == mesh.node_ijk[:, 2].max()
    f1 = np.zeros(mesh.n_dof)
    f1[3 * np.flatnonzero(top) + 2] = -1.0
    f2 = np.zeros(mesh.n_dof)
    f2[3 * np.flatnonzero(mesh.node_ijk[:, 0] == mesh.node_ijk[:, 0].max()) + 1] = 0.5
    ge = GridElasticity(mesh, 0.3, fixed, rtol=1e-10, maxiter=3000, device="cpu")
    ge.set_moduli(e)
    us = ge.solve_many([f1, f2])
    out = dict(elem_ijk=mesh.elem_ijk, node_ijk=mesh.node_ijk, pitch=float(mesh.pitch), fixed=fixed, e=e, f1=f1,
               f2=f2, verify_u1=us[0], verify_u2=us[1], verify_iters=np.array(ge.last_iters))
    ge2 = GridElasticity(mesh, 0.3, fixed, rtol=1e-10, maxiter=3000, device="cpu")
    layers = int(mesh.elem_ijk[:, 2].max()) + 1
    for li in range(layers):
        active = mesh.elem_ijk[:, 2] <= li
        node_on = np.zeros(mesh.n_nodes, bool)
        node_on[mesh.enode[active].ravel()] = True
        f = np.where(np.repeat(node_on, 3), rng.standard_normal(mesh.n_dof), 0.0)
        f[fixed] = 0.0
        ge2.set_moduli(e * active)
        du = ge2.solve_many([f])[0]
        out[f"layer{li}_f"] = f
        out[f"layer{li}_u"] = du
        out[f"layer{li}_iters"] = np.array(ge2.last_iters)
    out["layers"] = layers
    np.savez_compressed(os.path.join(HERE, "callers.npz"), **out)


def make_springs():
    """GridElasticity with a springs term (loadpath/mg.py:415-470, :274-296, :348-371, :679-706,
    :734-735): the sparse operator added on the fine level, coarsened as P^T S P level by level
    and added to the coarsest assembly. A 12x8x8 box at pitch 1 held by springs alone (diagonal
    springs on every base node, as the build simulation's layer springs hold a part) plus a
    spring coupling two top nodes (an off-diagonal term, as a cut cell's operator has); smoothed
    seeded moduli, a top load; rtol 1e-10, coarse_cells 40 so that the hierarchy has three
    levels. Stored: the mesh, the springs (mesh dof numbering, COO), the solve and its count,
    and every level's lmax."""
    os.environ["LOADPATH_HEX8"] = "im"
    import scipy.sparse as sp
    from loadpath.mg import GridElasticity

    dims = (12, 8, 8)
    mesh = _full_mesh(dims)
    rng = np.random.default_rng(31)
    x = _smoothed(np.exp(rng.uniform(np.log(1e-2), 0.0, dims)), 2.0).reshape(-1)
    e = 1e-9 + x ** 3 * (1 - 1e-9)
    base = np.flatnonzero(mesh.node_ijk[:, 2] == 0)
    rows, cols, vals = [], [], []
    for c in range(3):
        rows += list(3 * base + c)
        cols += list(3 * base + c)
        vals += [0.05] * len(base)
    top = np.flatnonzero(mesh.node_ijk[:, 2] == dims[2])
    a, b = int(top[0]), int(top[-1])
    for c in range(3):
        for (i, j, v) in ((a, a, 0.2), (b, b, 0.2), (a, b, -0.2), (b, a, -0.2)):
            rows.append(3 * i + c)
            cols.append(3 * j + c)
            vals.append(v)
    s = sp.csr_matrix((vals, (rows, cols)), shape=(mesh.n_dof, mesh.n_dof))
    fixed = np.zeros(mesh.n_dof, bool)
    f = np.zeros(mesh.n_dof)
    f[3 * top + 2] = -1.0 / len(top)
    f[3 * top + 0] = 0.3 / len(top)
    ge = GridElasticity(mesh, 0.3, fixed, springs=s, rtol=1e-10, maxiter=3000, coarse_cells=40, device="cpu")
    ge.set_moduli(e)
    u = ge.solve_many([f])[0]
    coo = s.tocoo()
    np.savez_compressed(os.path.join(HERE, "springs.npz"), dims=np.array(dims), e_mesh=e, f_mesh=f,
                        fixed_mesh=fixed, s_row=coo.row, s_col=coo.col, s_val=coo.data, u_mesh=u,
                        iters=np.array(ge.last_iters), nlevels=len(ge.levels),
                        lmax=np.array([ge._op(i).lmax for i in range(len(ge.levels))]), strict=ge.strict,
                        u_grid=ge.to_grid(u), f_grid=ge.to_grid(f), e_grid=ge.cell_grid(e))
    print("springs: levels", len(ge.levels), "iters", ge.last_iters, "strict", ge.strict)


def main(names=None):
    gens = {"element": make_element, "transfers": make_transfers, "femops": make_femops, "filter": make_filter,
            "mma": make_mma,
            "hierarchies": lambda: (make_hierarchy("even_im", (12, 6, 6), "im", 1, 50, 0.02),
                                    make_hierarchy("odd_plain", (11, 5, 7), "plain", 2, 30, 0.0),
                                    make_hierarchy("deep_im", (16, 8, 8), "im", 3, 20, 0.0),
                                    make_hierarchy("rough_strict", (8, 4, 4), "im", 4, 20, 0.05, smooth=False)),
            "top3d": make_top3d, "config0": make_config0, "oc_step": make_oc_step,
            "optimize": make_optimize, "constrained": make_constrained, "callers": make_callers,
            "springs": make_springs}
    for name in names or [k for k in gens if k != "config0"]:
        gens[name]()


if __name__ == "__main__":
    main(sys.argv[1:])
