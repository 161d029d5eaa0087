"""SIMP with the MMA update and a penalty ramp (optimize.MMALoop), its sensitivities from the
autograd path, against the oracle's loop with direct sparse solves (GPU)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,rtol_c,atol_x", [(np.float64, 1e-8, 1e-7), (np.float32, 1e-8, 1e-7)])
def test_mma_loop_matches_oracle(dtype, rtol_c, atol_x):
    from loadpath_b200.optimize import MMALoop
    from oracle import ref_numpy as R

    dims = (16, 8, 8)
    fixed, f = R.cantilever_bc(dims)
    iters = 8
    x_ref, xp_ref, hist = R.mma_simp_loop(dims, 0.25, 1.5, R.hex8_ke(0.3, "im"), fixed, f, iters, ramp=4)
    loop = MMALoop(dims, 0.25, 1.5, fixed, f, ramp=4, rtol=1e-12, dtype=dtype, coarse_cells=20, maxiter=2000)
    loop.run(iters)
    got = np.array([h[:3] for h in loop.history])
    want = np.array(hist)
    np.testing.assert_allclose(got[:, 0], want[:, 0], rtol=rtol_c)
    np.testing.assert_allclose(got[:, 1], want[:, 1], rtol=1e-10)
    np.testing.assert_allclose(loop.x.cpu().numpy(), x_ref, rtol=0, atol=atol_x)
    assert [h[3] for h in loop.history] == [1.0 + 2.0 * min(k, 4) / 4 for k in range(iters)]
