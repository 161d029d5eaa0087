"""Compliance and point displacement as torch.autograd.Functions (loadpath_b200.autograd): the
backward against the reference's sensitivity formulas (loadpath/simp.py:1901-1904, :2001;
loadpath/mechanism.py:13-22, 156-164) computed by the oracle, and against central finite
differences along seeded random design directions (GPU)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

EMIN = 1e-9


def _raw_design(dims, seed, lo=1e-3):
    """The benchmark's log-uniform draws before their r = 2 smoothing: the design x whose filtered
    field H x / hs is the benchmark density."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), 0.0, size=dims))


def _problem(dims, dtype, rtol):
    from loadpath_b200.autograd import SimpProblem
    from oracle import ref_numpy as R

    fixed, f = R.cantilever_bc(dims)
    p = SimpProblem(dims, fixed, rmin=2.0, dtype=dtype, rtol=rtol, coarse_cells=200)
    return p, p.node_load(f), fixed, f


def _oracle_state(dims, x, fixed, f, l=None):
    from oracle import ref_numpy as R

    taps = R.filter_taps(2.0)
    hs = R.filter_row_sums(dims, taps)
    xp = R.grid_filter(x, taps) / hs
    e = R.simp_moduli(xp, 3.0, EMIN)
    ke = R.hex8_ke(0.3, "im")
    h = R.Hierarchy(ke, dims, fixed, rtol=1e-13, maxiter=3000, coarse_cells=200)
    h.set_moduli(e)
    u = h.solve(f)
    lam = h.solve(l) if l is not None else None
    return taps, hs, xp, ke, u, lam


def _pair_energy(ke, a, b, dims):
    from oracle import ref_numpy as R

    ga = R.gather_cells(a, dims).reshape(24, -1)
    gb = R.gather_cells(b, dims).reshape(24, -1)
    return np.einsum("in,in->n", ga, ke @ gb).reshape(dims)


@pytest.mark.parametrize("dtype,rtol,tol", [(np.float64, 1e-13, 1e-10), (np.float32, 1e-8, 1e-6)])
def test_compliance_gradient_matches_reference_formula(dtype, rtol, tol):
    from oracle import ref_numpy as R

    from loadpath_b200.autograd import compliance

    dims = (24, 12, 12)
    x = _raw_design(dims, 11)
    p, fd_, fixed, f = _problem(dims, dtype, rtol)
    xt = torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True)
    c = compliance(xt, p, [fd_])
    c.backward()
    taps, hs, xp, ke, u, _ = _oracle_state(dims, x, fixed, f)
    c_ref = float((f * u).sum())
    ce = _pair_energy(ke, u, u, dims)
    dc = -3.0 * (1 - EMIN) * xp ** 2 * ce                         # loadpath/simp.py:1901-1904
    g_ref = R.grid_filter(dc / hs, taps)                           # loadpath/simp.py:2001
    assert abs(float(c.detach()) - c_ref) <= tol * abs(c_ref)
    g = xt.grad.cpu().numpy()
    assert np.linalg.norm(g - g_ref) <= tol * np.linalg.norm(g_ref)


@pytest.mark.parametrize("dtype,rtol,tol", [(np.float64, 1e-13, 1e-10), (np.float32, 1e-8, 1e-6)])
def test_point_displacement_gradient_matches_adjoint_formula(dtype, rtol, tol):
    from oracle import ref_numpy as R

    from loadpath_b200.autograd import point_displacement

    dims = (24, 12, 12)
    node = (24, 6, 0)
    x = _raw_design(dims, 12)
    p, fd_, fixed, f = _problem(dims, dtype, rtol)
    xt = torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True)
    j = point_displacement(xt, p, fd_, node, 2)
    j.backward()
    l = np.zeros_like(f)
    l[(2,) + node] = 1.0
    taps, hs, xp, ke, u, lam = _oracle_state(dims, x, fixed, f, l)
    j_ref = float(u[(2,) + node])
    dj = -3.0 * (1 - EMIN) * xp ** 2 * _pair_energy(ke, lam, u, dims)   # loadpath/mechanism.py:156-164
    g_ref = R.grid_filter(dj / hs, taps)
    assert abs(float(j.detach()) - j_ref) <= tol * abs(j_ref)
    g = xt.grad.cpu().numpy()
    assert np.linalg.norm(g - g_ref) <= tol * np.linalg.norm(g_ref)


def _fd_check(objective, x, ndir, seed, h=1e-6):
    """(directional derivatives from the gradient, central differences) along ndir unit
    directions drawn N(0, 1) from default_rng(seed)."""
    xt = torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True)
    objective(xt).backward()
    g = xt.grad.double()
    rng = np.random.default_rng(seed)
    an, fd = [], []
    with torch.no_grad():
        for _ in range(ndir):
            d = rng.standard_normal(x.shape)
            d /= np.linalg.norm(d)
            dt = torch.tensor(d, dtype=torch.float64, device="cuda")
            jp = float(objective(xt + h * dt))
            jm = float(objective(xt - h * dt))
            fd.append((jp - jm) / (2 * h))
            an.append(float((g * dt).sum()))
    return np.array(an), np.array(fd), float(torch.linalg.vector_norm(g))


@pytest.mark.parametrize("dtype,ndir", [(np.float64, 64), (np.float32, 16)])
def test_point_displacement_central_differences_128x64x64(dtype, ndir):
    """The differentiation check at 128 x 64 x 64 (1.6M dof): the z displacement of node
    (128, 32, 0), 64 seeded directions (default_rng(202)) in float64, step 1e-6."""
    from loadpath_b200.autograd import PointDisplacement

    dims = (128, 64, 64)
    x = _raw_design(dims, 2)
    p, fd_, _, _ = _problem(dims, dtype, 1e-13)
    l = p.unit_load((128, 32, 0), 2)

    an, fd, gn = _fd_check(lambda xt: PointDisplacement.apply(xt, p, fd_, l), x, ndir, 202)
    err = np.abs(an - fd)
    print(f"point displacement {np.dtype(dtype).name}: |g| {gn:.3e}, |g.d| median {np.median(np.abs(an)):.3e}, "
          f"err max {err.max():.3e}, rel max {np.max(err / np.abs(an)):.3e}, solves {p.solves}, "
          f"iterations {p.iterations}")
    # measured on a B200: errors below 5e-7 against |g| ~ 2e3 and |g . d| ~ 2
    assert np.all(err <= 2e-5 * np.abs(an) + 1e-9 * gn)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_compliance_central_differences_128x64x64(dtype):
    from loadpath_b200.autograd import Compliance

    dims = (128, 64, 64)
    x = _raw_design(dims, 2)
    p, fd_, _, _ = _problem(dims, dtype, 1e-13)
    an, fd, gn = _fd_check(lambda xt: Compliance.apply(xt, p, [fd_]), x, 16, 203)
    err = np.abs(an - fd)
    print(f"compliance {np.dtype(dtype).name}: |g| {gn:.3e}, |g.d| median {np.median(np.abs(an)):.3e}, "
          f"err max {err.max():.3e}, rel max {np.max(err / np.abs(an)):.3e}, solves {p.solves}, "
          f"iterations {p.iterations}")
    # measured on a B200: errors below 5e-7 against |g| ~ 2e3 and |g . d| ~ 2
    assert np.all(err <= 2e-5 * np.abs(an) + 1e-9 * gn)


def test_checkpointed_cases_give_the_saved_gradient():
    """Load cases past the saved-field budget are solved again in the backward; the gradient is
    the one the saved fields give."""
    from oracle import ref_numpy as R

    from loadpath_b200.autograd import SimpProblem, compliance

    dims = (16, 8, 8)
    fixed, f = R.cantilever_bc(dims)
    x = _raw_design(dims, 13)
    rng = np.random.default_rng(4)
    loads = []
    for _ in range(3):
        fk = np.zeros_like(f)
        fk[:, dims[0], rng.integers(0, dims[1] + 1), rng.integers(0, dims[2] + 1)] = rng.standard_normal(3)
        loads.append(fk)
    grads = []
    for budget in (1 << 40, 0):
        p = SimpProblem(dims, fixed, dtype=np.float64, rtol=1e-13, coarse_cells=100, save_bytes=budget)
        xt = torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True)
        c = compliance(xt, p, [p.node_load(fk) for fk in loads])
        # another design in between: the backward puts its own design back
        compliance(xt.detach() * 0.5, p, [p.node_load(loads[0])])
        c.backward()
        grads.append((float(c.detach()), xt.grad.cpu().numpy(), p.solves))
    (c0, g0, s0), (c1, g1, s1) = grads
    assert c0 == pytest.approx(c1, rel=1e-12)
    assert s1 == s0 + 3
    assert np.linalg.norm(g1 - g0) <= 1e-10 * np.linalg.norm(g0)
