"""The reference-facing host-array mirrors: mgops (loadpath/mgops.py), femops.element_energy
(loadpath/femops.py:236-242) and the device seam gpu.resolve_device / TorchMG (loadpath/gpu.py),
against the oracle and the reference's own golden vectors (GPU)."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _level(kind, dims, dtype, rng):
    """An oracle level with about a fifth of its cells inactive, and the mgops arguments."""
    from loadpath_b200.mgops import Cells
    from oracle import ref_numpy as R

    active = rng.random(dims) > 0.2
    cells = Cells(active)
    lv = R.Level(kind, dims, dtype)
    ke = R.hex8_ke(0.3, "im")
    if kind == "scaled":
        e = rng.random(dims) * active
        lv.ke, lv.e = ke.astype(dtype), e.astype(dtype)
        return lv, cells, lv.ke, e[active].astype(dtype)
    if kind == "weights":
        mk = np.stack([ke * (1.0 + 0.1 * q) for q in range(8)]).astype(dtype)
        w = rng.random((8,) + dims) * active
        lv.mcat, lv.w = mk.reshape(8 * 24, 24), w.astype(dtype)
        return lv, cells, mk, w[:, active].astype(dtype)
    k = np.zeros((24, 24) + dims)
    for idx in np.argwhere(active):
        s = rng.random() + 0.5
        k[(slice(None), slice(None)) + tuple(idx)] = s * ke + 0.01 * np.diag(rng.random(24))
    lv.k = k.astype(dtype)
    return lv, cells, k[:, :, active].astype(dtype), None


@pytest.mark.parametrize("kind", ["scaled", "weights", "explicit"])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 2e-5)])
def test_apply_masked_and_accumulating_applies(kind, dtype, tol):
    from loadpath_b200 import mgops

    rng = np.random.default_rng(7)
    dims = (6, 4, 5)
    lv, cells, a, b = _level(kind, dims, dtype, rng)
    u = rng.standard_normal(lv.node_shape).astype(dtype)
    m = (rng.random(lv.node_shape) > 0.1).astype(dtype)
    lv.mask = m
    scale = np.abs(lv.apply_k(u)).max()
    out = np.empty_like(u)
    mgops.apply_masked(kind, u, a, b, cells, m, out, True)
    np.testing.assert_allclose(out, lv.apply(u), rtol=0, atol=tol * scale)
    mgops.apply_masked(kind, u, a, b, cells, m, out, False)
    np.testing.assert_allclose(out, lv.apply_k(u * m), rtol=0, atol=tol * scale)
    acc = rng.standard_normal(lv.node_shape).astype(dtype)
    want = acc + lv.apply_k(u)
    fn = {"scaled": mgops.apply_scaled, "weights": mgops.apply_weights}.get(kind)
    if fn is not None:
        fn(u, a, b, cells, acc)
    else:
        mgops.apply_explicit(u, a, cells, acc)
    np.testing.assert_allclose(acc, want, rtol=0, atol=tol * scale)


def test_transfers_cast_dot():
    from loadpath_b200 import mgops
    from oracle import ref_numpy as R

    rng = np.random.default_rng(3)
    f = rng.standard_normal((3, 7, 5, 9))
    np.testing.assert_allclose(mgops.restrict(f), R.restrict(f), rtol=1e-13, atol=1e-13)
    c = rng.standard_normal((3, 4, 3, 5))
    np.testing.assert_allclose(mgops.prolong(c), R.prolong(c), rtol=1e-13, atol=1e-13)
    from loadpath_b200 import mg

    np.testing.assert_array_equal(mg.prolong(c), mgops.prolong(c))
    np.testing.assert_array_equal(mg.restrict(f), mgops.restrict(f))
    fine = (3, 8, 6, 10)                              # 7 x 5 x 9 cells: a padded coarse level
    coarse = (3, 5, 4, 6)
    b, ax = rng.standard_normal(fine), rng.standard_normal(fine)
    m = (rng.random(fine) > 0.2).astype(float)
    cm = (rng.random(coarse) > 0.2).astype(float)
    np.testing.assert_allclose(mgops.coarse_residual(b, ax, m, cm, coarse),
                               R.restrict_masked_residual(b, ax, m, cm, coarse), rtol=1e-13, atol=1e-13)
    x = rng.standard_normal(fine)
    xc = rng.standard_normal(coarse)
    want = R.prolong_add(xc, cm, m, x.copy())
    assert mgops.add_correction(xc, cm, m, x)
    np.testing.assert_allclose(x, want, rtol=1e-13, atol=1e-13)
    a64 = rng.standard_normal((3, 5, 5, 5))
    assert mgops.cast(a64, np.float32).dtype == np.float32
    np.testing.assert_array_equal(mgops.cast(a64, np.float32), a64.astype(np.float32))
    assert mgops.dot(a64, a64) == pytest.approx(float(np.vdot(a64, a64)), rel=1e-13)
    assert mgops.available()


def test_element_energy_matches_reference_golden():
    from loadpath_b200.femops import element_energy

    g = np.load(os.path.join(GOLD, "femops.npz"))
    np.testing.assert_allclose(element_energy(g["u"], g["v"], g["edof"], g["ke"]), g["uv"], rtol=1e-12,
                               atol=1e-12 * np.abs(g["uv"]).max())
    np.testing.assert_allclose(element_energy(g["u"], None, g["edof"], g["ke"]), g["uu"], rtol=1e-12,
                               atol=1e-12 * np.abs(g["uu"]).max())
    with pytest.raises(IndexError):
        bad = g["edof"].copy()
        bad[0, 0] = len(g["u"])
        element_energy(g["u"], None, bad, g["ke"])


def test_device_seam_solves_like_the_solver():
    from loadpath_b200.gpu import TorchMG, resolve_device
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    assert resolve_device("cpu") is None and resolve_device("b200").type == "cuda"
    dims = (16, 8, 8)
    fixed, f = R.cantilever_bc(dims)
    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, rtol=1e-10, coarse_cells=100, element="im")
    ge.set_moduli(R.simp_moduli(R.log_uniform_density(dims, 4)).reshape(-1))
    dev = TorchMG(ge, resolve_device("b200"))
    dev.load()
    x, it, ok = dev.solve(f, None)
    want = ge.g0.nodes_to_host(ge.solve_device(ge.g0.nodes_to_dev(f, torch.float64)))
    assert ok and it == ge.last_iters
    np.testing.assert_array_equal(x, want)
