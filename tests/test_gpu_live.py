"""The live-cell reduction on the device (simp.LiveCells, GridElasticity.set_moduli_live) against
the oracle's restatement of loadpath's labelling (scipy.ndimage.label, 26-connected) (GPU)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _run(dims, xp, support, anchor):
    from loadpath_b200.grid import DevGrid
    from loadpath_b200.simp import LiveCells

    g = DevGrid(dims)
    live = LiveCells(g, support, anchor)
    keep = live.keep(g.cells_to_dev(xp, torch.float64))
    return live, (None if keep is None else g.cells_to_host(keep) == 2)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_keep_matches_labelling(seed):
    from oracle import ref_numpy as R

    dims = (40, 24, 20)
    rng = np.random.default_rng(seed)
    xp = np.where(rng.random(dims) < 0.12, 0.5, 1e-4)   # near the 26-neighbour percolation threshold
    support = np.zeros(dims, bool)
    support[0] = True
    anchor = support.copy()
    anchor[-1, 10:14, :2] = True
    alive = (xp > R.ALIVE) | anchor
    live, got = _run(dims, xp, support, anchor)
    assert abs(live.alive_share - alive.mean()) < 1e-12
    np.testing.assert_array_equal(got, R.connected_keep(alive, support))
    assert 0 < got.sum() < alive.sum()


def test_keep_long_serpentine_path():
    """One winding path a cell thick through many tiles (many passes), a detached island, and
    corner-only (26-) connections."""
    from oracle import ref_numpy as R

    dims = (48, 40, 6)
    xp = np.full(dims, 1e-5)
    for j in range(0, 40, 4):          # rows joined at alternating ends
        xp[:, j, 2] = 1.0
        if j + 4 < 40:
            end = 47 if (j // 4) % 2 == 0 else 0
            xp[end, j:j + 4, 2] = 1.0
    xp[20:24, 38, 4] = 1.0             # island
    xp[46, 37, 3] = 1.0                # joined to the path's last row by a corner only
    support = np.zeros(dims, bool)
    support[0, 0, 2] = True
    alive = xp > R.ALIVE
    live, got = _run(dims, xp, support, np.zeros(dims, bool))
    want = R.connected_keep(alive, support)
    np.testing.assert_array_equal(got, want)
    assert not got[20, 38, 4] and got[46, 37, 3] and live.passes > 4


def test_dense_design_keeps_everything():
    dims = (16, 8, 8)
    xp = np.full(dims, 0.9)
    live, got = _run(dims, xp, np.zeros(dims, bool), np.zeros(dims, bool))
    assert got is None and live.alive_share == 1.0


def test_set_moduli_live_solves_and_falls_back_on_dead_loads():
    from loadpath_b200.grid import DevGrid
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from loadpath_b200.simp import LiveCells

    dims = (24, 8, 8)
    mesh = BoxMesh(dims)
    fixed = np.zeros((3,) + tuple(d + 1 for d in dims), bool)
    fixed[:, 0] = True
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    g = DevGrid(dims)
    ge = GridElasticity(mesh, 0.3, fx, coarse_cells=200)
    xp = np.full(dims, 1e-6)
    xp[:, 2:6, 2:6] = 1.0              # a bar from the support to the free end
    xp[10:14, 0, 0] = 1.0              # an island
    support = np.zeros(dims, bool)
    support[0] = True
    anchor = support.copy()
    # the moduli are the caller's: void at 1e-3 keeps the full grid's float32 coarse levels
    # positive definite for the fallback build (at 1e-9 their rounding makes the coarsest operator
    # indefinite for this thin bar, and the band Cholesky rejects it)
    e = 1e-3 + xp ** 3
    ed = g.cells_to_dev(e, torch.float64)
    live = LiveCells(g, support, anchor)
    f = np.zeros((3,) + tuple(d + 1 for d in dims))
    f[2, -1, 4, 4] = -1.0              # on the bar
    fd = g.nodes_to_dev(f, torch.float64)
    assert ge.set_moduli_live(ed, live, g.cells_to_dev(xp, torch.float64), [fd])
    kept = g.cells_to_host(live.state) == 2
    assert kept[:, 2:6, 2:6].all() and not kept[10:14, 0, 0].any()
    u = ge.solve_device(fd)
    assert np.isfinite(g.nodes_to_host(u)).all() and ge.last_iters < 200
    f2 = f.copy()
    f2[2, 12, 0, 0] = -1.0             # a load on the island's nodes: the full grid is solved
    assert not ge.set_moduli_live(ed, live, g.cells_to_dev(xp, torch.float64), [g.nodes_to_dev(f2, torch.float64)])
