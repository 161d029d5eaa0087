"""The cone filter on the device (lpb_filter through simp.DeviceFilter) against the oracle's
grid_filter (GPU), in its three forms: H v, H (v / hs) and (H v) / hs with the SIMP law
(loadpath/simp.py:1143-1228, loadpath/benchmarks/reference.py:48-71, :89).

Radii 1.5 and 2.0 reach one cell, 2.5 and 3.0 two (the shared-memory tile's halo), 3.5 three
(the taps gathered from global memory cell by cell). The shapes leave partial tiles in x and y
(tiles of 32 x 8 columns) and z extents that are not a multiple of the 4-cell z chunk."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SHAPES = [(37, 11, 9), (8, 5, 6), (64, 16, 12)]


@pytest.mark.parametrize("radius", [1.5, 2.0, 2.5, 3.0, 3.5])
@pytest.mark.parametrize("dims", SHAPES)
def test_device_filter_matches_oracle(dims, radius):
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import DevGrid, stream_handle
    from loadpath_b200.simp import DeviceFilter
    from oracle import ref_numpy as R

    rng = np.random.default_rng(int(10 * radius) + sum(dims))
    g = DevGrid(dims)
    flt = DeviceFilter(g, radius)
    taps = R.filter_taps(radius)
    assert flt.ntaps == len(taps)
    hs = R.filter_row_sums(dims, taps)
    np.testing.assert_allclose(g.cells_to_host(flt.hs), hs, rtol=1e-14)
    v = np.exp(rng.uniform(-3, 0, dims))
    vd = g.cells_to_dev(v, torch.float64)
    out = g.cell_field(torch.float64)
    # H v
    flt.apply(out, vd)
    np.testing.assert_allclose(g.cells_to_host(out), R.grid_filter(v, taps), rtol=1e-13)
    # H (v / hs): the sensitivity filter
    dc = -v
    flt.apply(out, g.cells_to_dev(dc, torch.float64), hs_in=flt.hs)
    np.testing.assert_allclose(g.cells_to_host(out), R.grid_filter(dc / hs, taps), rtol=1e-13)
    # (H v) / hs and the SIMP law: the density filter
    e = g.cell_field(torch.float64)
    flt.apply(out, vd, hs_out=flt.hs, e_out=e, penal=3.0, emin=1e-9)
    xphys = R.grid_filter(v, taps) / hs
    np.testing.assert_allclose(g.cells_to_host(out), xphys, rtol=1e-13)
    np.testing.assert_allclose(g.cells_to_host(e), R.simp_moduli(xphys), rtol=1e-12)
    # the z padding of the cell field (z from nz to the pitch) is left as it was
    out2 = torch.full_like(out, 7.0)
    flt.apply(out2, vd)
    full = out2.permute(2, 1, 0, 3).reshape(g.nx, g.ny, g.cpz).cpu().numpy()
    assert g.cpz > g.nz and np.all(full[..., g.nz:] == 7.0)
    np.testing.assert_allclose(full[..., :g.nz], R.grid_filter(v, taps), rtol=1e-13)


@pytest.mark.parametrize("dims", [(24, 8, 8), (20, 6, 7), (33, 9, 10)])
def test_oc_volumes_ignore_padding(dims):
    """lpb_oc_volumes sums over the grid's cells only: garbage in the z padding of x, dc, dv and
    gv leaves the 31 volumes unchanged, and they match the oracle's clipped steps."""
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import DevGrid, stream_handle

    rng = np.random.default_rng(sum(dims))
    g = DevGrid(dims)
    x = rng.uniform(0.0, 1.0, dims)
    dc = -np.exp(rng.uniform(-4, 1, dims))
    dv = rng.uniform(0.5, 1.5, dims)
    gv = rng.uniform(0.1, 1.0, dims)
    lam = np.logspace(-2, 2, 31)
    move = 0.2
    vols = {}
    for garbage in (0.0, np.nan, 1e300):
        fields = []
        for a in (x, dc, dv, gv):
            t = g.cell_field(torch.float64)
            t.fill_(garbage)
            full = t.permute(2, 1, 0, 3).reshape(g.nx, g.ny, g.cpz)
            full[..., :g.nz] = torch.from_numpy(a).to(t.device)
            t.copy_(full.reshape(g.nx, g.ny, g.cpz // 4, 4).permute(2, 1, 0, 3))
            fields.append(t)
        lamd = torch.from_numpy(lam).cuda()
        part = torch.zeros(31 * 592, dtype=torch.float64, device="cuda")
        out = torch.zeros(31, dtype=torch.float64, device="cuda")
        rc = lib().lpb_oc_volumes(out.data_ptr(), *(f.data_ptr() for f in fields), lamd.data_ptr(), 31, move,
                                  part.data_ptr(), *g.args, stream_handle())
        assert rc == 0
        vols[garbage] = out.cpu().numpy()
    assert np.array_equal(vols[0.0], vols[np.nan]) and np.array_equal(vols[0.0], vols[1e300])
    want = [float((np.maximum(np.maximum(0.0, x - move), np.minimum(np.minimum(1.0, x + move),
                                                                     x * np.sqrt(-dc / dv / l))) * gv).sum())
            for l in lam]
    np.testing.assert_allclose(vols[0.0], want, rtol=1e-13)
