"""The compliant-mechanism adjoint sensitivity (loadpath/mechanism.py:156-165) and a load case's
compliance (loadpath/directions.py:167-180) on the device (GPU)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_adjoint_sensitivity_matches_formula_and_reciprocity():
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from loadpath_b200.simp import adjoint_sensitivity, case_compliance
    from oracle import ref_numpy as R

    dims = (20, 8, 8)
    nx, ny, nz = dims
    rng = np.random.default_rng(4)
    xp = 0.3 + 0.7 * rng.random(dims)
    e = R.simp_moduli(xp)
    mesh = BoxMesh(dims)
    fixed = np.zeros((3, nx + 1, ny + 1, nz + 1), bool)
    fixed[:, 0] = True
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, rtol=1e-10, maxiter=2000, coarse_cells=100, element="im")
    ge.set_moduli(e.reshape(-1))
    g = ge.g0
    f = np.zeros((3, nx + 1, ny + 1, nz + 1))
    f[0, nx, 4, 4] = 1.0                  # the input push
    l = np.zeros_like(f)
    l[2, nx, 4, nz] = 1.0                 # the output displacement u_z at the top of the free end
    fd, ld = g.nodes_to_dev(f, torch.float64), g.nodes_to_dev(l, torch.float64)
    u = ge.solve_device(fd)
    lam = ge.solve_device(ld)
    # reciprocity (K symmetric): l . u = lam . f
    lu, lf = case_compliance(ld, u), case_compliance(fd, lam)
    assert abs(lu - lf) <= 1e-8 * abs(lu)
    xt = 0.2 + 0.6 * rng.random(dims)
    beta = 4.0
    dproj = R.dproject(xt, beta, 0.5)
    out = g.cell_field(torch.float64)
    adjoint_sensitivity(ge, [(u, lam)], g.cells_to_dev(xp, torch.float64), g.cells_to_dev(dproj, torch.float64),
                        out, modulus=2.5)
    ug, lg = g.nodes_to_host(u), g.nodes_to_host(lam)
    want = -np.einsum("ixyz,ij,jxyz->xyz", R.gather_cells(lg, dims), ge.ke, R.gather_cells(ug, dims))
    want = want * 2.5 * 3.0 * (1 - 1e-9) * xp ** 2 * dproj
    got = g.cells_to_host(out)
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * np.abs(want).max())
