"""The device SIMP loop against the reference's top3d port (GPU).

The reference solves each iteration with a direct sparse factorization; the device loop with
MG-PCG to rtol 1e-10, so compliances agree to ~1e-9 and the OC bisection takes the same branches.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_top3d_history_matches_reference():
    from loadpath_b200.simp import Top3dLoop

    g = np.load(os.path.join(GOLD, "top3d.npz"))
    dims = tuple(int(d) for d in g["dims"])
    nx, ny, nz = dims
    fixed = np.zeros((3, nx + 1, ny + 1, nz + 1), bool)
    fixed[:, 0] = True
    f = np.zeros(fixed.shape)
    f[2, nx, :, 0] = -1.0
    hist = g["hist"]
    loop = Top3dLoop(dims, float(g["volfrac"]), float(g["rmin"]), fixed, f, rtol=1e-10, element="plain",
                     coarse_cells=20)
    got = [loop.step() for _ in range(len(hist))]
    np.testing.assert_allclose([c for c, _ in got], hist[:, 0], rtol=1e-7)
    np.testing.assert_allclose([ch for _, ch in got], hist[:, 1], rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(loop.xphys_host(), g["xphys"], rtol=1e-6, atol=1e-8)


def test_filter_matches_reference():
    from loadpath_b200.simp import density_filter

    g = np.load(os.path.join(GOLD, "filter.npz"))
    dims = tuple(int(d) for d in g["dims"])
    v = g["v"]
    for r in (1.5, 2.0, 3.0):
        h, hs = density_filter(dims, r, pad=False)
        np.testing.assert_allclose(h @ v.reshape(-1), g[f"grid_{r}"], rtol=1e-13)
        order = tuple(g[f"top3d_cellorder_{r}"].T)
        np.testing.assert_allclose(hs.reshape(dims)[order], g[f"top3d_hs_{r}"], rtol=1e-13)
        np.testing.assert_allclose((h.T @ v.reshape(-1)).reshape(dims)[order], g[f"top3d_{r}"], rtol=1e-13)


def test_smoke_entry():
    import __graft_entry__ as ge

    ge.smoke()


@pytest.mark.parametrize("graphs", [True, False])
def test_device_bisection_walk_equals_host_walk(graphs):
    """The OC bisection walked on the device (lpb_oc_walk, in a graph WHILE loop or looped from
    the host) takes the host walk's (oc_bisection) candidates, passes and multiplier, so the
    designs agree bit for bit."""
    from loadpath_b200.simp import Top3dLoop

    dims = (24, 8, 8)
    nx, ny, nz = dims
    fixed = np.zeros((3, nx + 1, ny + 1, nz + 1), bool)
    fixed[:, 0] = True
    f = np.zeros(fixed.shape)
    f[2, nx, :, 0] = -1.0
    loops = [Top3dLoop(dims, 0.3, 1.5, fixed, f, rtol=1e-10, coarse_cells=40) for _ in range(2)]
    loops[1].device_oc = False
    loops[0].ge.use_graphs = graphs
    for it in range(6):
        (c0, ch0), (c1, ch1) = loops[0].step(), loops[1].step()
        assert (c0, ch0) == (c1, ch1), it
        assert loops[0].lmid == loops[1].lmid and loops[0].oc_passes == loops[1].oc_passes, it
        assert torch.equal(loops[0].x, loops[1].x), it
