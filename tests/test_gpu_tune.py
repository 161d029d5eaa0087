"""The launch-geometry autotuner (loadpath_b200.tune) on a built hierarchy (GPU)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_autotune_sets_the_fastest_candidate_and_keeps_the_operator():
    from loadpath_b200 import tune
    from loadpath_b200._lib import lib
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    dims = (64, 32, 32)
    x = R.log_uniform_density(dims, 9)
    fixed, f = R.cantilever_bc(dims)
    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, rtol=1e-8, coarse_cells=200, element="im")
    ge.set_moduli(R.simp_moduli(x).reshape(-1))
    g = ge.g0
    b = g.nodes_to_dev(f, torch.float64)
    u_before = g.nodes_to_host(ge.solve_device(b))
    it_before = ge.last_iters
    res = tune.autotune(ge)
    assert {"fine_f64", "fine_f32", "level1_f32"} <= set(res)
    for name, r in res.items():
        grid = g if name.startswith("fine") else ge.levels[1].grid
        assert r["best"] == min(r["us"], key=r["us"].get)
        assert lib().lpb_tune_get(tune.KNOBS[name], grid.nx, grid.ny, grid.nz) == r["best"]
    u_after = g.nodes_to_host(ge.solve_device(b))
    # the same operator: the solve agrees to its tolerance and takes the same iterations
    assert abs(ge.last_iters - it_before) <= 1
    assert np.linalg.norm(u_after - u_before) <= 1e-7 * np.linalg.norm(u_before)
    # a second tuning of the same grid reuses the timings
    assert tune.autotune(ge)["fine_f32"] is res["fine_f32"]
    for name in res:
        grid = g if name.startswith("fine") else ge.levels[1].grid
        lib().lpb_tune_set(tune.KNOBS[name], grid.nx, grid.ny, grid.nz, 0)
