"""loadpath's own design update on the device (simp.ProjectedDesign) against the reference's
projection values and the oracle's restatement of its optimality-criteria step (GPU)."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _design(dims, rng):
    from loadpath_b200.grid import DevGrid
    from loadpath_b200.simp import DeviceFilter, ProjectedDesign

    g = DevGrid(dims)
    flt = DeviceFilter(g, 2.0)
    pres = np.zeros(dims, bool)
    pres[0, :, :2] = True
    void = np.zeros(dims, bool)
    void[-1, :, -2:] = True
    flags = g.set_cells(g.cell_field(torch.uint8),
                        torch.from_numpy(pres.astype(np.uint8) | (void.astype(np.uint8) << 1)))
    w = 0.5 + rng.random(dims)
    return g, ProjectedDesign(flt, w=g.cells_to_dev(w, torch.float64), flags=flags), pres, void, w


def test_projection_matches_reference_values():
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import DevGrid, stream_handle

    gold = np.load(os.path.join(GOLD, "filter.npz"))
    g = DevGrid((5, 5, 2))
    xt = g.cells_to_dev(gold["proj_x"].reshape(5, 5, 2), torch.float64)
    for beta in (1.0, 8.0):
        xp, dxp = g.cell_field(torch.float64), g.cell_field(torch.float64)
        lib().lpb_project(xp.data_ptr(), dxp.data_ptr(), xt.data_ptr(), beta, 0.5, None, None, None, None, *g.args,
                          stream_handle())
        np.testing.assert_allclose(g.cells_to_host(xp).reshape(-1), gold[f"proj_{beta}"], rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(g.cells_to_host(dxp).reshape(-1), gold[f"dproj_{beta}"], rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("dims,beta,lam_last", [((14, 9, 7), 1.0, None), ((14, 9, 7), 8.0, 2e-2),
                                                ((48, 24, 20), 4.0, None)])
def test_oc_step_matches_oracle(dims, beta, lam_last):
    from oracle import ref_numpy as R

    rng = np.random.default_rng(sum(dims))
    g, pd, pres, void, w = _design(dims, rng)
    taps = R.filter_taps(2.0)
    hs = R.filter_row_sums(dims, taps)
    x = 0.2 + 0.6 * rng.random(dims)
    dc = -np.exp(rng.uniform(-3, 1, dims))
    dv = R.grid_filter(w * R.dproject(R.grid_filter(x, taps) / hs, beta, 0.5) / hs, taps)
    target = 0.45 * float(w.sum())
    want = R.oc_loadpath_step(x, dc, dv, 0.2, beta, 0.5, lambda v: R.grid_filter(v, taps), hs, w, target, pres,
                              void, lam_last)
    pd.lam_last = lam_last
    xd, dcd, dvd = (g.cells_to_dev(a, torch.float64) for a in (x, dc, dv))
    xn, lm, held = pd.oc_step(xd, dcd, dvd, 0.2, beta, 0.5, target)
    assert held == want[3]
    assert pd.n_eval == want[2]
    np.testing.assert_allclose(lm, want[1], rtol=1e-10)
    np.testing.assert_allclose(g.cells_to_host(xn), want[0], rtol=1e-10, atol=1e-12)
    vol = pd.physical(xn, beta, 0.5)
    assert abs(vol - target) <= 1e-12 * target


def test_chain_rule_matches_oracle():
    from oracle import ref_numpy as R

    dims = (20, 12, 9)
    rng = np.random.default_rng(3)
    g, pd, pres, void, w = _design(dims, rng)
    taps = R.filter_taps(2.0)
    hs = R.filter_row_sums(dims, taps)
    x = rng.random(dims)
    grad = -rng.random(dims)
    beta = 6.0
    dxp = g.cell_field(torch.float64)
    pd.physical(g.cells_to_dev(x, torch.float64), beta, 0.5, dxp=dxp)
    want_d = R.dproject(R.grid_filter(x, taps) / hs, beta, 0.5)
    want_d[pres | void] = 0.0
    np.testing.assert_allclose(g.cells_to_host(dxp), want_d, rtol=1e-12, atol=1e-14)
    out = g.cell_field(torch.float64)
    pd.chain(out, g.cells_to_dev(grad, torch.float64), dxp, clip=True)
    want = np.minimum(R.grid_filter(grad * want_d / hs, taps), 0.0)
    np.testing.assert_allclose(g.cells_to_host(out), want, rtol=1e-12, atol=1e-14 * np.abs(want).max())


def test_oc_step_matches_reference_run():
    """The device step against the step the reference's own optimize took in its first three
    iterations on the 12x4x6 cantilever (tests/golden/oc_step.npz, captured from loadpath.simp's
    trial function): the accepted design, the multiplier and the number of trial steps."""
    from loadpath_b200.grid import DevGrid
    from loadpath_b200.simp import DeviceFilter, ProjectedDesign

    gold = np.load(os.path.join(GOLD, "oc_step.npz"))
    dims = tuple(int(d) for d in gold["dims"])
    ijk = gold["elem_ijk"]

    def grid(v):
        out = np.zeros(dims, v.dtype)
        out[tuple(ijk.T)] = v
        return out

    g = DevGrid(dims)
    flt = DeviceFilter(g, float(gold["radius"]), float(gold["pitch"]), pad=bool(gold["pad"]))
    for k in range(len(gold["iterations"])):
        pres = grid(gold[f"pres{k}"])
        flags = g.set_cells(g.cell_field(torch.uint8), torch.from_numpy(pres.astype(np.uint8)))
        pd = ProjectedDesign(flt, w=g.cells_to_dev(grid(gold[f"w{k}"]), torch.float64), flags=flags)
        lam_last = float(gold[f"lam_last{k}"])
        pd.lam_last = None if np.isnan(lam_last) else lam_last
        ratio = grid(gold[f"ratio{k}"])
        xd = g.cells_to_dev(grid(gold[f"x{k}"]), torch.float64)
        dcd = g.cells_to_dev(-ratio ** 2, torch.float64)
        dvd = g.cells_to_dev(np.ones(dims), torch.float64)
        xn, lm, held = pd.oc_step(xd, dcd, dvd, float(gold[f"move{k}"]), float(gold[f"beta{k}"]), float(gold["eta"]),
                                  float(gold[f"target{k}"]))
        assert held
        assert pd.n_eval == int(gold[f"n_eval{k}"])
        np.testing.assert_allclose(lm, float(gold[f"lm{k}"]), rtol=1e-10)
        np.testing.assert_allclose(g.cells_to_host(xn), grid(gold[f"x_new{k}"]), rtol=0, atol=1e-11)
