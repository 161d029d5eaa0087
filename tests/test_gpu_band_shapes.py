"""The coarsest level's band factorisation and dense inverse at band widths that take the
kernels' different paths (GPU), against numpy's inverse of the dense operator the same level
assembles (lpb_coarse_dense_f32):

- D = 2 tile diagonals: no helper rows (the critical block does every row);
- D = 3: helpers form one tile per row;
- D = 6: the helpers' partial sums of the last tiles, inverse with the shared-memory ring;
- D = 13: more of a row's tiles than the helpers' ring holds (their operands staged again) and
  the inverse kernel for wide bands.

Seeded log-uniform moduli smoothed by the r = 2 filter, cantilever supports."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

# fine cells, coarse_cells (the hierarchy stops at the coarsest level below), band tile diagonals
SHAPES = [((16, 4, 4), 100, 2), ((16, 8, 8), 200, 3), ((24, 12, 12), 500, 6), ((40, 20, 20), 2000, 13)]


def _band_to_dense_index(gr):
    ext = np.array([gr.NX, gr.NY, gr.NZ])
    n = 3 * gr.NX * gr.NY * gr.NZ
    perm = np.argsort(-ext, kind="stable")
    idx = np.arange(n)
    node_b, comp = idx // 3, idx % 3
    p2 = node_b % ext[perm[2]]
    q = node_b // ext[perm[2]]
    p1, p0 = q % ext[perm[1]], q // ext[perm[1]]
    coords = np.zeros((3, n), np.int64)
    coords[perm[0]], coords[perm[1]], coords[perm[2]] = p0, p1, p2
    return comp * (gr.NX * gr.NY * gr.NZ) + (coords[0] * gr.NY + coords[1]) * gr.NZ + coords[2]


@pytest.mark.parametrize("dims,cc,dtiles", SHAPES)
def test_band_inverse_matches_dense_at_band_widths(dims, cc, dtiles):
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import ptr, stream_handle
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    x = R.log_uniform_density(dims, 21)
    fixed, _ = R.cantilever_bc(dims)
    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, rtol=1e-10, maxiter=3000, coarse_cells=cc, element="im")
    ge.set_moduli(R.simp_moduli(x).reshape(-1))
    assert not ge.strict
    lv = ge.levels[-1]
    gr = lv.grid
    L = lib()
    bdims = np.zeros(4, np.int64)
    L.lpb_band_dims(gr.nx, gr.ny, gr.nz, bdims.ctypes.data)
    assert int(bdims[2]) == dtiles, (gr.cells, bdims)
    assert [int(v) for v in ge._work["band_info"].cpu().numpy()] == [0, 0]
    n = 3 * gr.NX * gr.NY * gr.NZ
    a = torch.empty((n, n), dtype=torch.float64, device="cuda")
    if lv.kind == "weights":
        L.lpb_coarse_dense_f32(a.data_ptr(), 1, lv.w.data_ptr(), lv.mcat.data_ptr(), ptr(lv.patch_id),
                               ptr(lv.patch_k), None, lv.mask.data_ptr(), *gr.args, stream_handle())
    else:
        L.lpb_coarse_dense_f32(a.data_ptr(), 2, None, None, None, None, lv.k.data_ptr(), lv.mask.data_ptr(),
                               *gr.args, stream_handle())
    dense = a.cpu().numpy()
    del a
    didx = _band_to_dense_index(gr)
    got = ge._coarse["ainv"][:n, :n].cpu().numpy()
    want = np.linalg.inv(dense)[np.ix_(didx, didx)]
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-10 * np.abs(want).max())
    # and a solve through the level's band solve
    rng = np.random.default_rng(4)
    b = rng.standard_normal(gr.node_shape).astype(np.float32)
    bd = gr.nodes_to_dev(b, torch.float32)
    xd = gr.node_field(torch.float32)
    c = ge._coarse
    L.lpb_band_solve_f32(xd.data_ptr(), bd.data_ptr(), c["ainv"].data_ptr(), c["v"].data_ptr(), *gr.args,
                         stream_handle())
    got_x = gr.nodes_to_host(xd).astype(np.float64).reshape(-1)
    want_x = np.linalg.solve(dense, b.astype(np.float64).reshape(-1))
    np.testing.assert_allclose(got_x, want_x, rtol=2e-6, atol=2e-6 * np.abs(want_x).max())
