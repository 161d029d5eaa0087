"""The oracle (oracle/ref_numpy.py) against golden vectors made by the
reference implementation itself (tests/golden/make_golden.py). CPU only."""
import os

import numpy as np
import pytest

from oracle import ref_numpy as R

GOLD = os.path.join(os.path.dirname(__file__), "golden")
COARSE_CELLS = {"even_im": 50, "odd_plain": 30, "deep_im": 20, "rough_strict": 20}


def _load(name):
    return np.load(os.path.join(GOLD, name), allow_pickle=False)


def test_element_matrices():
    g = _load("element.npz")
    for el in ("plain", "im"):
        for nu in (0.3, 0.35):
            np.testing.assert_allclose(R.hex8_ke(nu, el), g[f"ke_{el}_{nu}"], rtol=0, atol=1e-14)


def test_transfers():
    g = _load("transfers.npz")
    np.testing.assert_array_equal(R.PK, g["pk"])
    np.testing.assert_allclose(R.prolong(g["c"]), g["prolong_c"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(R.restrict(g["f"]), g["restrict_f"], rtol=0, atol=1e-14)
    # float32: the reference's compiled path sums the corners before scaling, the
    # numpy path axis by axis; the two agree to rounding
    np.testing.assert_allclose(R.prolong(g["c32"]), g["prolong_c32"], rtol=1e-6, atol=1e-6)
    # adjoint pair, as the reference's own test pins (tests/test_mg.py:56-63)
    c, f = g["c"], g["f"]
    assert abs(np.vdot(R.prolong(c), f) - np.vdot(c, R.restrict(f))) < 1e-10


def _hierarchy(name):
    g = _load(f"hier_{name}.npz")
    h = R.Hierarchy(g["ke"], tuple(g["cells"]), g["fixed_grid"], rtol=1e-10, maxiter=3000,
                    coarse_cells=COARSE_CELLS[name])
    h.set_moduli(g["e_grid"])
    return g, h


@pytest.mark.parametrize("name", sorted(COARSE_CELLS))
def test_hierarchy_levels(name):
    g, h = _hierarchy(name)
    assert len(h.levels) == int(g["nlevels"])
    assert h.strict == bool(g["strict"])
    np.testing.assert_array_equal(h.alive, g["alive"])
    for i in range(len(h.levels)):
        lv = h.op(i)
        assert lv.kind == str(g[f"L{i}_kind"])
        np.testing.assert_array_equal(lv.mask, g[f"L{i}_mask"])
        np.testing.assert_allclose(lv.dinv, g[f"L{i}_dinv"], rtol=2e-6)
        np.testing.assert_allclose(lv.lmax, float(g[f"L{i}_lmax"]), rtol=1e-4)
        if lv.kind == "weights":
            np.testing.assert_array_equal(lv.w, g[f"L{i}_w"])
            np.testing.assert_array_equal(lv.patch_ijk, g[f"L{i}_patch_ijk"])
            np.testing.assert_allclose(lv.patch_k, g[f"L{i}_patch_k"], rtol=1e-6, atol=1e-7)
            np.testing.assert_allclose(lv.mcat, g[f"L{i}_mcat"], rtol=1e-6, atol=1e-7)
        elif lv.kind == "explicit":
            ref = g[f"L{i}_k"]
            np.testing.assert_allclose(lv.k, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
        np.testing.assert_allclose(lv.diagonal(), g[f"L{i}_diag"], rtol=1e-6, atol=1e-12)
        u = g[f"L{i}_u"]
        want = g[f"L{i}_apply"]
        tol = 1e-5 if u.dtype == np.float32 else 1e-12
        np.testing.assert_allclose(lv.apply(u), want, rtol=tol, atol=tol * np.abs(want).max())
    want = g["L0_apply64"]
    np.testing.assert_allclose(h.levels[0].apply(g["L0_u64"]), want, rtol=1e-12, atol=1e-13 * np.abs(want).max())


@pytest.mark.parametrize("name", sorted(COARSE_CELLS))
def test_transfers_and_vcycle(name):
    g, h = _hierarchy(name)
    if "t_b" in g:
        lv, nxt = h.op(0), h.op(1)
        rc = R.restrict_masked_residual(g["t_b"], g["t_ax"], lv.mask, nxt.mask, nxt.node_shape)
        np.testing.assert_allclose(rc, g["t_coarse_residual"], rtol=1e-6, atol=1e-6)
        x = g["t_x"].copy()
        R.prolong_add(g["t_xc"], nxt.mask, lv.mask, x)
        np.testing.assert_allclose(x, g["t_add_correction"], rtol=1e-6, atol=1e-6)
    z = h.precondition(g["vc_r"])
    want = g["vc_z"]
    np.testing.assert_allclose(z, want, rtol=1e-4, atol=1e-4 * np.abs(want).max())


@pytest.mark.parametrize("name", sorted(COARSE_CELLS))
def test_solve_matches_reference(name):
    g, h = _hierarchy(name)
    u = h.solve(g["f_grid"])
    ref = g["u_grid"]
    assert np.linalg.norm(u - ref) <= 1e-8 * np.linalg.norm(ref)
    assert abs(h.last_iters - int(g["iters"])) <= max(2, int(0.05 * int(g["iters"])))
    c = float(np.vdot(g["f_grid"], u))
    assert abs(c - float(g["compliance"])) <= 1e-9 * abs(float(g["compliance"]))
    se = h.strain_energy(ref)
    nx, ny, nz = g["dims"]
    np.testing.assert_allclose(se[:nx, :ny, :nz].reshape(-1), g["strain_energy"], rtol=1e-10,
                               atol=1e-12 * np.abs(g["strain_energy"]).max())
    h.set_moduli(g["e_grid"] * 1.1)
    w = h.solve(g["f_grid"], u)
    assert np.linalg.norm(w - g["u_warm_grid"]) <= 1e-8 * np.linalg.norm(g["u_warm_grid"])


def test_element_energy():
    g = _load("femops.npz")
    dims = tuple(g["dims"])
    u, v, edof, ke = g["u"], g["v"], g["edof"], g["ke"]
    ue, ve = u[edof], v[edof]
    np.testing.assert_allclose(np.einsum("ij,jk,ik->i", ue, ke, ve), g["uv"], rtol=1e-13)
    # the grid form used by the CUDA path: node-grid field, cells in C order
    nshape = tuple(d + 1 for d in dims)
    ug = u.reshape(-1, 3).T.reshape((3,) + nshape)
    cells = R.gather_cells(ug, dims).reshape(24, -1)
    np.testing.assert_allclose(np.einsum("in,in->n", cells, ke @ cells), g["uu"], rtol=1e-12)


def test_filters():
    g = _load("filter.npz")
    dims = tuple(g["dims"])
    v = g["v"]
    for r in (1.5, 2.0, 3.0):
        taps = R.filter_taps(r)
        assert len(taps) == int(g[f"ntaps_{r}"])
        np.testing.assert_allclose(R.grid_filter(v, taps).reshape(-1), g[f"grid_{r}"], rtol=1e-13)
        order = tuple(g[f"top3d_cellorder_{r}"].T)
        np.testing.assert_allclose(R.grid_filter(v, taps)[order], g[f"top3d_{r}"], rtol=1e-13)
        np.testing.assert_allclose(R.filter_row_sums(dims, taps)[order], g[f"top3d_hs_{r}"], rtol=1e-13)


def test_top3d_history():
    g = _load("top3d.npz")
    dims = tuple(int(d) for d in g["dims"])
    ke = R.hex8_ke(0.3, "plain")
    nx, ny, nz = dims
    fixed = np.zeros((3, nx + 1, ny + 1, nz + 1), bool)
    fixed[:, 0] = True
    f = np.zeros(fixed.shape)
    f[2, nx, :, 0] = -1.0           # the stock problem: -1 on each bottom-edge node
    hist = g["hist"]
    x, xphys, hc, hch = R.top3d_loop(dims, float(g["volfrac"]), float(g["rmin"]), ke, fixed, f, len(hist))
    np.testing.assert_allclose(hc, hist[:, 0], rtol=1e-9)
    np.testing.assert_allclose(hch, hist[:, 1], rtol=1e-7, atol=1e-12)
    np.testing.assert_allclose(xphys, g["xphys"], rtol=1e-9, atol=1e-12)


@pytest.mark.slow
def test_top3d_stored_cantilever_compliance():
    """The stored top3d design of the 60x4x20 cantilever (the reference's own
    golden file): its penalised compliance, evaluated by the oracle's direct
    solve, is the compliance top3d reported on its last iteration up to the
    float32 storage of the design."""
    g = _load("top3d.npz")
    dims = tuple(int(d) for d in g["stored_dims"])
    nx, ny, nz = dims
    ke = R.hex8_ke(0.3, "plain")
    fixed = np.zeros((3, nx + 1, ny + 1, nz + 1), bool)
    fixed[:, 0] = True
    f = np.zeros(fixed.shape)
    f[2, nx, :, 0] = -1.0
    x = g["stored_x"].astype(np.float64)
    u = R.assembled_solve(ke, R.simp_moduli(x), fixed, f)
    c = float(np.vdot(f, u))
    assert abs(c - float(g["stored_c"])) < 2e-4 * float(g["stored_c"]), (c, float(g["stored_c"]))
    assert int(g["stored_iters"]) == 133


def test_mma_steps():
    g = _load("mma.npz")
    n, m = int(g["n"]), int(g["m"])
    mma = R.MMA(n, m, move=0.2)
    for i in range(int(g["steps"])):
        xn = mma.update(g[f"x{i}"], 1.0, g[f"df0{i}"], g[f"f{i}"], g[f"df{i}"])
        np.testing.assert_allclose(xn, g[f"xn{i}"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", sorted(COARSE_CELLS))
def test_c_port_apply_matches_golden(name):
    """The oracle's C port of the reference's two-pass CPU apply (the CPU baseline) gives the
    reference's level-0 operator."""
    from oracle import cport

    g, h = _hierarchy(name)
    l0 = h.levels[0]
    op = cport.MaskedApply(l0.ke, l0.e, l0.mask, np.float64)
    want = g["L0_apply64"]
    np.testing.assert_allclose(op(g["L0_u64"]), want, rtol=1e-12, atol=1e-13 * np.abs(want).max())
    op32 = cport.MaskedApply(l0.ke, l0.e, l0.mask, np.float32)
    want = g["L0_apply"]
    np.testing.assert_allclose(op32(g["L0_u"]), want, rtol=2e-5, atol=2e-5 * np.abs(want).max())


@pytest.mark.parametrize("name", sorted(COARSE_CELLS))
def test_c_port_weights_apply_matches_golden(name):
    """The oracle's C port of the reference's level-1 (weights) operator, patch cells included
    (the reference arm's level-1 applies), gives the reference's level-1 operator in float32."""
    from oracle import cport

    g, h = _hierarchy(name)
    if len(h.levels) < 2 or h.levels[1].kind != "weights":
        pytest.skip("no weights level in this hierarchy")
    op = cport.WeightsApply(h.levels[1])
    want = g["L1_apply"]
    np.testing.assert_allclose(op(g["L1_u"]), want, rtol=2e-5, atol=2e-5 * np.abs(want).max())


@pytest.mark.parametrize("name", sorted(COARSE_CELLS))
def test_c_port_transfers_match_golden(name):
    """The oracle's C port of the reference's V-cycle transfers (the reference arm's restriction
    of the residual and prolongation of the correction) against the reference's float32 outputs."""
    from oracle import cport

    g, h = _hierarchy(name)
    if "t_b" not in g:
        pytest.skip("a single-level hierarchy")
    lv, nxt = h.op(0), h.op(1)
    rc = cport.coarse_residual(g["t_b"], g["t_ax"], lv.mask, nxt.mask)
    np.testing.assert_allclose(rc, g["t_coarse_residual"], rtol=1e-6, atol=1e-6)
    x = np.ascontiguousarray(g["t_x"], np.float32).copy()
    cport.add_correction(g["t_xc"], nxt.mask, lv.mask, x)
    np.testing.assert_allclose(x, g["t_add_correction"], rtol=1e-6, atol=1e-6)


def test_projection_matches_reference():
    g = _load("filter.npz")
    for beta in (1.0, 8.0):
        np.testing.assert_allclose(R.project(g["proj_x"], beta, 0.5), g[f"proj_{beta}"], rtol=1e-15, atol=0)
        np.testing.assert_allclose(R.dproject(g["proj_x"], beta, 0.5), g[f"dproj_{beta}"], rtol=1e-15, atol=0)


@pytest.mark.parametrize("beta,lam_last", [(1.0, None), (8.0, None), (4.0, 3e-3)])
def test_oracle_oc_loadpath_step_lands_on_the_volume(beta, lam_last):
    """The restated step (the reference's closure inside simp.optimize is not callable alone)
    lands the projected volume on target to the reference's tolerance, moves no cell past its
    move limit and keeps the passive cells."""
    rng = np.random.default_rng(5)
    dims = (14, 9, 7)
    taps = R.filter_taps(2.0)
    hs = R.filter_row_sums(dims, taps)
    x = 0.2 + 0.6 * rng.random(dims)
    dc = -np.exp(rng.uniform(-3, 1, dims))
    dv = R.grid_filter(np.ones(dims) * R.dproject(R.grid_filter(x, taps) / hs, beta, 0.5) / hs, taps)
    pres = np.zeros(dims, bool)
    pres[0, :, :2] = True
    void = np.zeros(dims, bool)
    void[-1, :, -2:] = True
    w = np.ones(dims)
    target = 0.45 * x.size
    xn, lm, n_eval, held = R.oc_loadpath_step(x, dc, dv, 0.2, beta, 0.5, lambda v: R.grid_filter(v, taps), hs, w,
                                              target, pres, void, lam_last)
    assert held and n_eval < 40
    vol = np.sum(np.where(pres, 1.0, np.where(void, 0.0, R.project(R.grid_filter(xn, taps) / hs, beta, 0.5))))
    assert abs(vol - target) <= 1e-12 * target
    free = ~pres & ~void
    assert np.all(np.abs(xn - x)[free] <= 0.2 + 1e-15)
    assert np.all(xn[pres] == 1.0) and np.all(xn[void] == 0.0)


def _oc_golden():
    g = np.load(os.path.join(GOLD, "oc_step.npz"))
    dims = tuple(int(d) for d in g["dims"])
    ijk = g["elem_ijk"]

    def grid(v):
        out = np.zeros(dims, v.dtype)
        out[tuple(ijk.T)] = v
        return out
    return g, dims, grid


def test_oracle_oc_loadpath_step_matches_reference_run():
    """The oracle's restatement of loadpath's design step against the step the reference's own
    optimize took in its first three iterations on the 12x4x6 cantilever (tests/golden/oc_step.npz):
    the accepted design, the multiplier and the number of trial steps."""
    g, dims, grid = _oc_golden()
    taps = R.filter_taps(float(g["radius"]), float(g["pitch"]))
    hs = np.full(dims, sum(w for _, w in taps)) if bool(g["pad"]) else R.filter_row_sums(dims, taps)
    for k in range(len(g["iterations"])):
        ratio = grid(g[f"ratio{k}"])
        lam_last = float(g[f"lam_last{k}"])
        xn, lm, n_eval, held = R.oc_loadpath_step(
            grid(g[f"x{k}"]), -ratio ** 2, np.ones(dims), float(g[f"move{k}"]), float(g[f"beta{k}"]), float(g["eta"]),
            lambda v: R.grid_filter(v, taps), hs, grid(g[f"w{k}"]), float(g[f"target{k}"]), grid(g[f"pres{k}"]), None,
            None if np.isnan(lam_last) else lam_last)
        assert n_eval == int(g[f"n_eval{k}"])
        np.testing.assert_allclose(lm, float(g[f"lm{k}"]), rtol=1e-12)
        np.testing.assert_allclose(xn, grid(g[f"x_new{k}"]), rtol=0, atol=1e-13)


@pytest.mark.parametrize("case", ["small", "medium", "bridge", "fixedmove", "twocase"])
def test_oracle_optimize_loop_matches_reference_run(case):
    """The oracle's restatement of loadpath's SIMP loop (optimize_loop) against the reference's
    own simp.optimize (tests/golden/optimize.npz): every iteration's projection sharpness, move
    limit, multiplier trial count, compliance, change, volume and blueprint, and the last design.
    The medium case's last iterations solve on the live cells only; the cantilevers are mirrored in
    y, the bridge in x and y."""
    g = _load("optimize.npz")
    k = lambda s: g[f"{case}_{s}"]   # noqa: E731
    dims = tuple(int(d) for d in k("dims"))
    loads = [k("f"), k("f2")] if f"{case}_f2" in g.files else k("f")
    recs, x = R.optimize_loop(dims, R.hex8_ke(float(k("nu")), "im"), k("fixed"), loads, float(k("volfrac")),
                              float(k("radius")), int(k("iterations")), pres=k("pres"), pad=bool(k("pad")),
                              pitch=float(k("pitch")), emin=float(k("emin")), penal=float(k("penal")),
                              mirror=tuple(int(a) for a in k("mirror")), adaptive_move=bool(k("adaptive_move")),
                              beta_max=float(k("beta_max")), weights=k("weights"))
    col = lambda key: np.array([r[key] for r in recs], float)   # noqa: E731
    np.testing.assert_array_equal(col("beta"), k("beta"))
    np.testing.assert_array_equal(col("volumeSolves"), k("volumeSolves"))
    # the bridge (volume fraction 0.01, held at its four bottom corners' edges) is badly conditioned:
    # two direct factorisations of it agree on the energy to a few parts in 10^9
    np.testing.assert_allclose(col("compliance"), k("compliance"), rtol=1e-10 if case != "bridge" else 2e-8)
    np.testing.assert_allclose(col("move"), k("move"), rtol=1e-12, equal_nan=True)
    assert len(recs) == int(k("iterations"))
    np.testing.assert_allclose(col("change"), k("change"), rtol=0, atol=1e-10 if case != "bridge" else 1e-9)
    np.testing.assert_allclose(col("volume"), k("volume"), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(np.stack([r["xphys"] for r in recs]), k("xphys"), rtol=0, atol=1e-9)
    np.testing.assert_allclose(x, k("x_last"), rtol=0, atol=1e-9)
    if case == "medium":
        assert k("solvedCells")[-1] < np.prod(dims)


@pytest.mark.parametrize("tag", ["", "_deflection", "_stress", "_converge", "_twocase"])
def test_oracle_constrained_loop_matches_reference_run(tag):
    """The oracle's restatement of loadpath's minimum-mass loop under stress and deflection limits
    (constrained_loop) against the reference's own optimize_constrained on the 12x4x6 cantilever
    (tests/golden/constrained.npz, 40 iterations, beta 1 to 8, the last ones on a reduced system
    the direct path reuses; a deflection limit or a stress limit alone on a 16x4x8 cantilever,
    30 iterations; both limits with beta_max 4, run to the loop's own stop; and both limits on two
    load cases, four constraints): every iteration's
    constraints, readings, volume, change and blueprint, and the delivered design (the last one,
    or the lightest feasible one at beta_max); and the cells whose stress is not counted."""
    g = _load(f"constrained{tag}.npz")
    dims = tuple(int(d) for d in g["dims"])
    lim = lambda key: None if np.isnan(float(g[key])) else float(g[key])   # noqa: E731
    held = g["fixed"].any(axis=0)
    loaded = (g["f"] != 0).any(axis=0)
    np.testing.assert_array_equal(R.cells_touching(held | loaded), g["contact"])
    loads = [g["f"], g["f2"]] if "f2" in g.files else g["f"]
    recs, x, conv = R.constrained_loop(dims, float(g["nu"]), g["fixed"], loads, float(g["volfrac"]),
                                       float(g["radius"]), int(g["max_iterations"]), lim("stress_limit"),
                                       lim("deflection_limit"), float(g["modulus"]), pres=g["pres"],
                                       pad=bool(g["pad"]), pitch=float(g["pitch"]),
                                       mirror=tuple(int(a) for a in g["mirror"]), beta_max=float(g["beta_max"]))
    assert conv == bool(g["converged"]) and len(recs) == int(g["iterations"])
    col = lambda key: np.array([r[key] for r in recs], float)   # noqa: E731
    np.testing.assert_array_equal(col("beta"), g["beta"])
    np.testing.assert_allclose(np.array([r["constraints"] for r in recs]), g["constraints"], rtol=0, atol=1e-10)
    for key in ("deflection", "stress", "volume"):
        np.testing.assert_allclose(col(key), g[key], rtol=1e-10, equal_nan=True)
    np.testing.assert_allclose(col("change"), g["change"], rtol=0, atol=1e-10)
    if "f2" in g.files:
        np.testing.assert_allclose([r["deflections"] for r in recs], g["deflection_cases"], rtol=1e-10)
        np.testing.assert_allclose([r["stresses"] for r in recs], g["stress_cases"], rtol=1e-10)
    np.testing.assert_allclose(np.stack([r["xphys"] for r in recs]), g["xphys"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(x, g["x_last"], rtol=0, atol=1e-10)
    if tag == "":
        assert g["solvedCells"].min() < np.prod(dims)


def test_oracle_springs_solve_matches_reference():
    """The oracle's hierarchy with a springs term (the operator added on the fine level, carried
    to every coarse level as P^T S P and into the coarsest assembly; loadpath/mg.py:274-296,
    :348-371, :679-706, :734-735) against the reference's own GridElasticity with springs
    (tests/golden/springs.npz): a box held by springs alone at its base plus one spring coupling
    two top nodes. Every level's lmax, the solution and the CG count."""
    import scipy.sparse as sp

    g = _load("springs.npz")
    dims = tuple(int(d) for d in g["dims"])
    nshape = tuple(d + 1 for d in dims)
    node_ijk = np.stack(np.meshgrid(*[np.arange(n) for n in nshape], indexing="ij"), -1).reshape(-1, 3)
    ndof = 3 * len(node_ijk)
    s = sp.csr_matrix((g["s_val"], (g["s_row"], g["s_col"])), shape=(ndof, ndof))
    fixed = np.zeros((3,) + nshape, bool)
    h = R.Hierarchy(R.hex8_ke(0.3, "im"), dims, fixed, rtol=1e-10, maxiter=3000, coarse_cells=40,
                    springs=R.springs_to_grid(s, node_ijk, nshape))
    h.set_moduli(g["e_grid"])
    assert len(h.levels) == int(g["nlevels"]) and h.strict == bool(g["strict"])
    np.testing.assert_allclose([h.op(i).lmax for i in range(len(h.levels))], g["lmax"], rtol=1e-4)
    u = h.solve(g["f_grid"])
    np.testing.assert_allclose(u, g["u_grid"], rtol=0, atol=1e-8 * np.abs(g["u_grid"]).max())
    assert abs(h.last_iters - int(g["iters"])) <= 2, (h.last_iters, int(g["iters"]))
    # springs on every level: a coarse operator without them is singular (nothing else holds the box)
    assert all(h.op(i).extra is not None for i in range(len(h.levels)))
