"""CUDA path against the reference's golden vectors and the oracle (GPU).

Tolerances: float64 operator results to 1e-12 relative (different summation order only);
float32 V-cycle quantities to 1e-5; solutions of the float64 PCG to 1e-8 relative at
rtol 1e-10 (both sides converge to the same float64 answer)."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = {"even_im": ("im", 50), "odd_plain": ("plain", 30), "deep_im": ("im", 20), "rough_strict": ("im", 20)}


def _load(name):
    return np.load(os.path.join(GOLD, f"hier_{name}.npz"), allow_pickle=False)


def _ge(name, rtol=1e-10, dtype=np.float32, **kw):
    from loadpath_b200.mg import BoxMesh, GridElasticity

    g = _load(name)
    element, cc = CASES[name]
    mesh = BoxMesh(tuple(int(d) for d in g["dims"]), float(g["pitch"]))
    ge = GridElasticity(mesh, 0.3, g["fixed_mesh"], rtol=rtol, maxiter=3000, coarse_cells=cc, dtype=dtype,
                        element=element, **kw)
    ge.set_moduli(g["e_mesh"])
    return g, ge


@pytest.mark.parametrize("name", sorted(CASES))
def test_hierarchy_matches_reference(name):
    g, ge = _ge(name)
    assert len(ge.levels) == int(g["nlevels"])
    assert ge.strict == bool(g["strict"])
    for i in range(len(ge.levels)):
        np.testing.assert_array_equal(ge.level_mask(i), g[f"L{i}_mask"], err_msg=f"mask L{i}")
        np.testing.assert_allclose(ge.level_dinv(i), g[f"L{i}_dinv"], rtol=2e-6, err_msg=f"dinv L{i}")
        np.testing.assert_allclose(ge._op(i).lmax, float(g[f"L{i}_lmax"]), rtol=1e-4, err_msg=f"lmax L{i}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_level_operators_match_reference(name):
    from loadpath_b200.grid import stream_handle  # noqa: F401

    g, ge = _ge(name)
    for i in range(len(ge.levels)):
        lv = ge._op(i)
        gr = lv.grid
        u = g[f"L{i}_u"]
        want = g[f"L{i}_apply"]
        dt = torch.float32 if u.dtype == np.float32 else torch.float64
        ud = gr.nodes_to_dev(u, dt)
        out = gr.node_field(dt)
        lv.apply(out, ud, mask_in=True)          # general kernel: arbitrary u
        got = gr.nodes_to_host(out)
        tol = 2e-5 if dt == torch.float32 else 1e-12
        np.testing.assert_allclose(got, want, rtol=tol, atol=tol * np.abs(want).max(), err_msg=f"L{i}")
        # the tiled / zero-on-masked path: same numbers on a masked input
        m = ge.level_mask(i).astype(u.dtype)
        um = gr.nodes_to_dev(u * m, dt)
        lv.apply(out, um, mask_in=False)
        ref2 = gr.nodes_to_host(out)
        lv.apply(out, um, mask_in=True, fine_kernel=False)
        np.testing.assert_allclose(ref2, gr.nodes_to_host(out), rtol=tol, atol=tol * np.abs(ref2).max())
    # float64 fine operator
    l0 = ge.levels[0]
    u64 = g["L0_u64"]
    out = l0.grid.node_field(torch.float64)
    l0.apply(out, l0.grid.nodes_to_dev(u64, torch.float64), mask_in=True)
    want = g["L0_apply64"]
    np.testing.assert_allclose(l0.grid.nodes_to_host(out), want, rtol=1e-12, atol=1e-13 * np.abs(want).max())


@pytest.mark.parametrize("name", sorted(CASES))
def test_vcycle_and_solve_match_reference(name):
    g, ge = _ge(name)
    gr = ge.g0
    r = gr.nodes_to_dev(g["vc_r"], torch.float64)
    z = gr.node_field(torch.float64)
    ge.precondition_device(r, z)
    want = g["vc_z"]
    np.testing.assert_allclose(gr.nodes_to_host(z), want, rtol=1e-4, atol=1e-4 * np.abs(want).max())
    u = ge.solve_many([g["f_mesh"]])[0]
    ref = g["u_mesh"]
    assert np.linalg.norm(u - ref) <= 1e-8 * np.linalg.norm(ref)
    assert abs(ge.last_iters - int(g["iters"])) <= max(2, int(0.05 * int(g["iters"])))
    c = float(g["f_mesh"] @ u)
    assert abs(c - float(g["compliance"])) <= 1e-9 * abs(float(g["compliance"]))
    se = ge.strain_energy(ref)
    np.testing.assert_allclose(se, g["strain_energy"], rtol=1e-10, atol=1e-12 * np.abs(g["strain_energy"]).max())
    ge.set_moduli(g["e_mesh"] * 1.1)
    w = ge.solve_many([g["f_mesh"]], [u])[0]
    w_ref = ge.from_grid(g["u_warm_grid"])
    assert np.linalg.norm(w - w_ref) <= 1e-8 * np.linalg.norm(w_ref)


def test_fine_kernel_matches_general_kernel_medium():
    """The tiled fine-level kernel against the general node-centric kernel on a grid that
    spans several blocks in x and y and odd z padding, float32 and float64."""
    from loadpath_b200.mg import BoxMesh, GridElasticity

    dims = (40, 34, 21)
    mesh = BoxMesh(dims)
    rng = np.random.default_rng(3)
    fixed = np.zeros(mesh.n_dof, bool)
    fixed[3 * np.flatnonzero(mesh.node_ijk[:, 0] == 0)[:, None] + np.arange(3)] = True
    e = 1e-9 + rng.random(mesh.n_elem) ** 3
    e[rng.random(mesh.n_elem) < 0.05] = 0.0
    ge = GridElasticity(mesh, 0.3, fixed, coarse_cells=10 ** 9)
    ge.set_moduli(e)
    for lv in (ge.levels[0], ge._l0s):
        gr = lv.grid
        m = ge.level_mask(0)
        u = (rng.standard_normal(gr.node_shape) * m).astype(np.float64 if lv.dtype == torch.float64 else np.float32)
        ud = gr.nodes_to_dev(u, lv.dtype)
        a = gr.node_field(lv.dtype)
        b = gr.node_field(lv.dtype)
        lv.apply(a, ud, mask_in=False, fine_kernel=True)
        lv.apply(b, ud, mask_in=False, fine_kernel=False)
        tol = 1e-12 if lv.dtype == torch.float64 else 2e-5
        ga, gb = gr.nodes_to_host(a), gr.nodes_to_host(b)
        np.testing.assert_allclose(ga, gb, rtol=tol, atol=tol * np.abs(gb).max())
        # padding stays zero
        zpad = a.permute(0, 3, 2, 1, 4).reshape(3, gr.NX, gr.NY, gr.pz)[..., gr.NZ:]
        assert zpad.numel() == 0 or float(zpad.abs().max()) == 0.0


def test_solve_matches_oracle_mixed_and_fp64():
    """A 24x12x12 cantilever with smoothed log-uniform density (the benchmark's synthetic
    field): the device solve in both precisions against the oracle's float64 solve."""
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    dims = (24, 12, 12)
    x = R.log_uniform_density(dims, 7)
    e = R.simp_moduli(x)
    fixed, f = R.cantilever_bc(dims)
    ke = R.hex8_ke(0.3, "im")
    h = R.Hierarchy(ke, dims, fixed, rtol=1e-10, maxiter=2000, coarse_cells=100)
    h.set_moduli(e)
    u_ref = h.solve(f)
    c_ref = float(np.vdot(f, u_ref))
    mesh = BoxMesh(dims)
    for dt in (np.float32, np.float64):
        ge = GridElasticity(mesh, 0.3, ge_fixed(mesh, fixed), rtol=1e-10, maxiter=2000, coarse_cells=100, dtype=dt,
                            element="im")
        ge.set_moduli(e.reshape(-1))
        u = ge.solve_many([ge.from_grid(f)])[0]
        ug = ge.to_grid(u)
        assert np.linalg.norm(ug - u_ref) <= 1e-8 * np.linalg.norm(u_ref)
        assert abs(float(np.vdot(f, ug)) - c_ref) <= 1e-9 * c_ref
        assert abs(ge.last_iters - h.last_iters) <= 2


def ge_fixed(mesh, fixed_grid):
    """bool per mesh dof from a (3, nodes...) grid."""
    flat = fixed_grid.reshape(3, -1)
    out = np.empty(mesh.n_dof, bool)
    for i in range(3):
        out[i::3] = flat[i]
    return out


@pytest.mark.parametrize("name", ["deep_im", "odd_plain"])
def test_band_direct_solve_matches_dense(name):
    """The coarsest level's band Cholesky + inverse against numpy on the dense operator the same
    level assembles (lpb_coarse_dense_*), float64 to 1e-10 relative."""
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import ptr, stream_handle

    g, ge = _ge(name)
    lv = ge.levels[-1]
    gr = lv.grid
    L = lib()
    n = 3 * gr.NX * gr.NY * gr.NZ
    a = torch.empty((n, n), dtype=torch.float64, device="cuda")
    sfx = "f32"
    if lv.kind == "weights":
        L.lpb_coarse_dense_f32(a.data_ptr(), 1, lv.w.data_ptr(), lv.mcat.data_ptr(), ptr(lv.patch_id),
                               ptr(lv.patch_k), None, lv.mask.data_ptr(), *gr.args, stream_handle())
    else:
        L.lpb_coarse_dense_f32(a.data_ptr(), 2, None, None, None, None, lv.k.data_ptr(), lv.mask.data_ptr(),
                               *gr.args, stream_handle())
    dense = a.cpu().numpy()
    rng = np.random.default_rng(3)
    for _ in range(2):
        b = rng.standard_normal(gr.node_shape).astype(np.float32)
        bd = gr.nodes_to_dev(b, torch.float32)
        xd = gr.node_field(torch.float32)
        c = ge._coarse
        getattr(L, f"lpb_band_solve_{sfx}")(xd.data_ptr(), bd.data_ptr(), c["ainv"].data_ptr(), c["v"].data_ptr(),
                                           *gr.args, stream_handle())
        got = gr.nodes_to_host(xd).astype(np.float64).reshape(-1)
        want = np.linalg.solve(dense, b.astype(np.float64).reshape(-1))
        np.testing.assert_allclose(got, want, rtol=2e-6, atol=2e-6 * np.abs(want).max())
    # the inverse itself, in float64
    c = ge._coarse
    ainv = c["ainv"].cpu().numpy()
    dims = np.zeros(4, np.int64)
    L.lpb_band_dims(gr.nx, gr.ny, gr.nz, dims.ctypes.data)
    # band numbering -> the dense (component-major) numbering
    ext = np.array([gr.NX, gr.NY, gr.NZ])
    perm = np.argsort(-ext, kind="stable")
    idx = np.arange(n)
    node_b, comp = idx // 3, idx % 3
    p2 = node_b % ext[perm[2]]
    q = node_b // ext[perm[2]]
    p1, p0 = q % ext[perm[1]], q // ext[perm[1]]
    coords = np.zeros((3, n), np.int64)
    coords[perm[0]], coords[perm[1]], coords[perm[2]] = p0, p1, p2
    dense_idx = comp * (gr.NX * gr.NY * gr.NZ) + (coords[0] * gr.NY + coords[1]) * gr.NZ + coords[2]
    inv_dense = np.linalg.inv(dense)
    got_inv = ainv[:n, :n]
    want_inv = inv_dense[np.ix_(dense_idx, dense_idx)]
    np.testing.assert_allclose(got_inv, want_inv, rtol=1e-9, atol=1e-10 * np.abs(want_inv).max())


@pytest.mark.parametrize("cells", [(6, 10, 6), (16, 8, 12), (10, 6, 14)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_grid_transfers_match_oracle(cells, dtype):
    """Masked residual restriction and masked prolongation against the oracle, on grids whose
    coarse level is padded up to even cells (6 -> 4, 10 -> 6, 14 -> 8): float32 to 2e-6,
    float64 to 1e-12 relative (the same sums in another order)."""
    from oracle import ref_numpy as R
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import DevGrid, stream_handle

    L = lib()
    st = stream_handle()
    sfx = "f32" if dtype == np.float32 else "f64"
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    half = tuple(c // 2 for c in cells)
    cdims = tuple(h + h % 2 if h > 1 else h for h in half)
    gf, gc = DevGrid(cells), DevGrid(cdims)
    rng = np.random.default_rng(11)
    b = rng.standard_normal(gf.node_shape).astype(dtype)
    ax = rng.standard_normal(gf.node_shape).astype(dtype)
    mbits = rng.integers(0, 8, gf.node_shape[1:]).astype(np.uint8)
    cbits = rng.integers(0, 8, gc.node_shape[1:]).astype(np.uint8)
    m = np.stack([(mbits >> i) & 1 for i in range(3)]).astype(dtype)
    cm = np.stack([(cbits >> i) & 1 for i in range(3)]).astype(dtype)

    def mask_dev(g, bits):
        return g.set_nodes(g.mask_field(), torch.from_numpy(bits))

    md, cmd = mask_dev(gf, mbits), mask_dev(gc, cbits)
    rc = gc.node_field(tdt)
    bd, axd = gf.nodes_to_dev(b, tdt), gf.nodes_to_dev(ax, tdt)   # held: the launch is asynchronous
    getattr(L, f"lpb_restrict_residual_{sfx}")(rc.data_ptr(), bd.data_ptr(), axd.data_ptr(), md.data_ptr(),
                                               cmd.data_ptr(), *gf.args, *gc.args, st)
    want = R.restrict_masked_residual(b.astype(np.float64), ax.astype(np.float64), m, cm, gc.node_shape)
    tol = 2e-6 if dtype == np.float32 else 1e-12
    got = gc.nodes_to_host(rc)
    np.testing.assert_allclose(got, want, rtol=tol, atol=tol * np.abs(want).max())
    assert np.all(gc.nodes_to_host(rc) * (1 - cm) == 0)

    xc = rng.standard_normal(gc.node_shape).astype(dtype)
    x = rng.standard_normal(gf.node_shape).astype(dtype)
    xd, xcd = gf.nodes_to_dev(x, tdt), gc.nodes_to_dev(xc, tdt)
    getattr(L, f"lpb_prolong_add_{sfx}")(xd.data_ptr(), xcd.data_ptr(), cmd.data_ptr(), md.data_ptr(), *gf.args,
                                         *gc.args, st)
    want = R.prolong_add(xc.astype(np.float64), cm, m, x.astype(np.float64).copy())
    np.testing.assert_allclose(gf.nodes_to_host(xd), want, rtol=tol, atol=tol * np.abs(want).max())


def test_coarse_factor_takes_roundoff_negative_pivots():
    """A thin bar in 1e-9 void: the float32 Galerkin levels leave the coarsest operator indefinite
    by rounding. The reference's SuperLU (symmetric mode, no pivoting) factors it and so does the
    band's signed Cholesky: no strict fallback, and the solve agrees with the oracle's."""
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    dims = (24, 8, 8)
    fixed = np.zeros((3,) + tuple(d + 1 for d in dims), bool)
    fixed[:, 0] = True
    xp = np.full(dims, 1e-6)
    xp[:, 2:6, 2:6] = 1.0
    xp[10:14, 0, 0] = 1.0
    e = 1e-9 + xp ** 3
    f = np.zeros(fixed.shape)
    f[2, -1, 4, 4] = -1.0
    ke = R.hex8_ke(0.3, "im")
    h = R.Hierarchy(ke, dims, fixed, rtol=1e-10, maxiter=3000, coarse_cells=200)
    h.set_moduli(e)
    assert not h.strict                   # the build factors the coarsest level as it is
    mesh = BoxMesh(dims)
    ge = GridElasticity(mesh, 0.3, ge_fixed(mesh, fixed), rtol=1e-10, maxiter=3000, coarse_cells=200, element="im")
    ge.set_moduli(e.reshape(-1))
    assert not ge.strict
    u_ref = h.solve(f)                    # (a stalled solve may still take the strict hierarchy)
    u = ge.to_grid(ge.solve_many([ge.from_grid(f)])[0])
    assert ge.strict == h.strict
    # at a 1e9 stiffness contrast the void nodes' displacements are ill-determined at any
    # residual tolerance; the compliance is not
    c, c_ref = float(np.vdot(f, u)), float(np.vdot(f, u_ref))
    assert abs(c - c_ref) <= 1e-9 * abs(c_ref)
    assert np.linalg.norm(u - u_ref) <= 1e-5 * np.linalg.norm(u_ref)


def test_explicit_levels_modal_form_matches_node_basis():
    """The explicit levels' corner-parity storage (150 pattern entries per cell, listed cells from
    the node-basis form) gives the general kernel's operator; the supports' patch cells make some
    cells listed, so both paths run."""
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    dims = (32, 16, 16)
    x = R.log_uniform_density(dims, 5)
    e = R.simp_moduli(x)
    fixed, f = R.cantilever_bc(dims)
    mesh = BoxMesh(dims)
    ge = GridElasticity(mesh, 0.3, ge_fixed(mesh, fixed), coarse_cells=20, element="im")
    ge.set_moduli(e.reshape(-1))
    explicit = [lv for lv in ge.levels[1:] if lv.kind == "explicit" and lv.km is not None]
    assert explicit
    listed = 0
    rng = np.random.default_rng(2)
    for lv in explicit:
        gr = lv.grid
        listed += int(lv.gcount.item())
        m = gr.mask_to_host(lv.mask)
        u = (rng.standard_normal(gr.node_shape) * m).astype(np.float32)
        ud = gr.nodes_to_dev(u, torch.float32)
        a, b = gr.node_field(torch.float32), gr.node_field(torch.float32)
        lv.apply(a, ud)
        lv.apply(b, ud, fine_kernel=False)
        ga, gb = gr.nodes_to_host(a), gr.nodes_to_host(b)
        np.testing.assert_allclose(ga, gb, rtol=2e-5, atol=2e-5 * np.abs(gb).max())
    assert listed > 0


def test_smoothing_forms_match_two_launch_form():
    """The applies that form a Chebyshev update where they store A u (the fine float32 stencil
    kernel and the explicit levels' gather, modes 1-3) give the bits of the plain apply followed
    by the vector kernel of the same step (lpb_cheb2_zero / lpb_residual_scaled / lpb_cheb2)."""
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import stream_handle
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    dims = (32, 16, 16)
    x = R.log_uniform_density(dims, 6)
    e = R.simp_moduli(x)
    fixed, _ = R.cantilever_bc(dims)
    mesh = BoxMesh(dims)
    ge = GridElasticity(mesh, 0.3, ge_fixed(mesh, fixed), coarse_cells=20, element="im")
    ge.set_moduli(e.reshape(-1))
    L, st = lib(), stream_handle()
    coef = torch.tensor([0.0, 0.7, 0.3, 0.2] + [0.0] * 12, dtype=torch.float64, device="cuda")
    levels = [ge._l0s] + [lv for lv in ge.levels[1:] if lv.kind == "explicit" and lv.km is not None]
    assert levels[0].kind == "scaled" and levels[0].dtype == torch.float32 and len(levels) > 1
    rng = np.random.default_rng(7)
    for lv in levels:
        gr = lv.grid
        n = gr.n_node_field
        m = gr.mask_to_host(lv.mask)

        def fld():
            return gr.nodes_to_dev((rng.standard_normal(gr.node_shape) * m).astype(np.float32), torch.float32)

        b0, d0, x0, r0 = fld(), fld(), fld(), fld()

        def fused(mode, xx, rr, dd, u):
            if lv.kind == "scaled":
                rc = L.lpb_apply_fine_cheb_f32(mode, xx.data_ptr(), rr.data_ptr(), dd.data_ptr(), u.data_ptr(),
                                               b0.data_ptr(), lv.dinv.data_ptr(), coef.data_ptr(), lv.e.data_ptr(),
                                               lv.mask.data_ptr(), lv.kmodal.ctypes.data, lv.err.data_ptr(),
                                               *gr.args, st)
            else:
                rc = L.lpb_apply_explicit_modal_cheb_f32(mode, xx.data_ptr(), rr.data_ptr(), dd.data_ptr(),
                                                         u.data_ptr(), b0.data_ptr(), lv.dinv.data_ptr(),
                                                         coef.data_ptr(), lv.km.data_ptr(), lv.kpc.data_ptr(),
                                                         lv.glist.data_ptr(), lv.gcount.data_ptr(), lv.ft.data_ptr(),
                                                         lv.mask.data_ptr(), *gr.args, st)
            assert rc == 0

        t = gr.node_field(torch.float32)
        # mode 1: x = d + (c1 d + c2 dinv (b - A d))
        xa = x0.clone()
        fused(1, xa, r0.clone(), d0, d0)
        xb = x0.clone()
        lv.apply(t, d0)
        L.lpb_cheb2_zero_f32(xb.data_ptr(), b0.data_ptr(), t.data_ptr(), d0.data_ptr(), lv.dinv.data_ptr(),
                             coef.data_ptr(), n, st)
        assert torch.equal(xa, xb)
        # mode 2: r = b - A x, d = s dinv r
        ra, da = r0.clone(), d0.clone()
        fused(2, x0, ra, da, x0)
        rb, db = r0.clone(), d0.clone()
        lv.apply(t, x0)
        L.lpb_residual_scaled_f32(b0.data_ptr(), t.data_ptr(), lv.dinv.data_ptr(), coef.data_ptr(), rb.data_ptr(),
                                  db.data_ptr(), n, st)
        assert torch.equal(ra, rb) and torch.equal(da, db)
        # mode 3: x = (x + d) + (c1 d + c2 dinv (r - A d))
        xa = x0.clone()
        fused(3, xa, r0, d0, d0)
        xb = x0.clone()
        lv.apply(t, d0)
        L.lpb_cheb2_f32(xb.data_ptr(), d0.data_ptr(), r0.data_ptr(), t.data_ptr(), lv.dinv.data_ptr(),
                        coef.data_ptr(), n, st)
        assert torch.equal(xa, xb)
        assert float(xa.abs().max()) > 0
    ge.check_device()
