"""The float32-only solve mode (loadpath/gpu.py:119-149, :233-258, :399-481) on the device (GPU)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _solver(dims, seed, rtol=1e-6):
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    x = R.log_uniform_density(dims, seed)
    e = R.simp_moduli(x)
    fixed, f = R.cantilever_bc(dims)
    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, rtol=rtol, maxiter=2000, coarse_cells=100, element="im")
    ge.set_moduli(e.reshape(-1))
    return ge, e, fixed, f


def test_rigid_free_apply_on_a_displaced_field():
    """u = a large rigid translation and rotation plus a small deformation: the pair operator keeps
    the deformation's digits, a plain float32 apply loses them to the rigid part."""
    dims = (16, 8, 8)
    ge, e, fixed, f = _solver(dims, 3)
    g = ge.g0
    rng = np.random.default_rng(0)
    X, Y, Z = np.meshgrid(*[np.arange(n + 1, dtype=float) for n in dims], indexing="ij")
    rigid = np.stack([1e3 + 0.02 * Y, 5e2 - 0.02 * X + 0.01 * Z, -3e2 - 0.01 * Y])
    u = rigid + 1e-3 * rng.standard_normal(rigid.shape)
    m = ge.level_mask(0)
    u = u * m
    want = ge.apply(u)                                  # float64
    h = u.astype(np.float32)
    l = (u - h.astype(np.float64)).astype(np.float32)
    hd, ld = g.nodes_to_dev(h, torch.float32), g.nodes_to_dev(l, torch.float32)
    out = g.node_field(torch.float32)
    ge.apply_rf(out, hd, ld)
    got = g.nodes_to_host(out).astype(np.float64)
    plain = g.node_field(torch.float32)
    ge._l0s.apply(plain, hd, mask_in=True, fine_kernel=False)
    got_plain = g.nodes_to_host(plain).astype(np.float64)
    # compare away from the support: its zeroed layer breaks the rigid motion next to it
    far = np.zeros_like(m)
    far[:, 2:] = m[:, 2:]
    scale = np.abs(want * far).max()
    err_rf = np.abs((got - want) * far).max() / scale
    err_plain = np.abs((got_plain - want) * far).max() / scale
    assert err_rf < 1e-4
    assert err_plain > 10 * err_rf


def test_fp32_solve_matches_oracle():
    from oracle import ref_numpy as R

    dims = (24, 12, 12)
    ge, e, fixed, f = _solver(dims, 7, rtol=1e-6)
    ke = R.hex8_ke(0.3, "im")
    h = R.Hierarchy(ke, dims, fixed, rtol=1e-10, maxiter=2000, coarse_cells=100)
    h.set_moduli(e)
    u_ref = h.solve(f)
    g = ge.g0
    b = g.nodes_to_dev(f * ge.level_mask(0), torch.float64)
    x, vcycles, ok = ge.solve_fp32_device(b)
    assert ok and 0 < vcycles < 400
    u = g.nodes_to_host(x)
    assert np.linalg.norm(u - u_ref) <= 1e-5 * np.linalg.norm(u_ref)
    # a warm start from the answer converges at once
    x2, v2, ok2 = ge.solve_fp32_device(b, x)
    assert ok2 and v2 <= vcycles
