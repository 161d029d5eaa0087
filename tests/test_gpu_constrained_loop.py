"""loadpath's minimum-mass loop under stress and deflection limits on the device
(optimize.ConstrainedLoop) against the reference's own optimize_constrained
(tests/golden/constrained.npz: the 12x4x6 cantilever mirrored in y, Limits(12 MPa, 0.6 mm,
1000 MPa), 40 iterations from a uniform 0.5 with the solves at rtol 1e-10; and a 16x4x8
cantilever under a deflection limit or a stress limit alone, 30 iterations), iteration by
iteration: the projection sharpness, the two constraints and their readings, the volume, the
design change and the blueprint each iteration started from, and the last design (GPU).

The reference solves this small grid directly; the device loop runs MG-PCG to rtol 1e-10 and its
adjoint solves alike, in both V-cycle precisions. The cells touching the supports and the load are
left out of the stress as the reference leaves them out."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("tag", ["", "_deflection", "_stress"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_constrained_loop_matches_reference_run(dtype, tag):
    from loadpath_b200.optimize import ConstrainedLoop, Limits, SimpOptions

    g = np.load(os.path.join(GOLD, f"constrained{tag}.npz"))
    lim_of = lambda key: None if np.isnan(float(g[key])) else float(g[key])   # noqa: E731
    n_it = int(g["iterations"])
    opts = SimpOptions(volume_fraction=float(g["volfrac"]), filter_radius=float(g["radius"]), max_iterations=n_it,
                       solve_rtol=1e-10, pad_filter=bool(g["pad"]))
    lim = Limits(lim_of("stress_limit"), lim_of("deflection_limit"), float(g["modulus"]))
    loop = ConstrainedLoop(tuple(int(d) for d in g["dims"]), g["fixed"], [g["f"]], float(g["nu"]), opts, lim,
                           preserve=g["pres"], pitch=float(g["pitch"]), mirror=tuple(int(a) for a in g["mirror"]),
                           dtype=dtype, coarse_cells=100)
    np.testing.assert_array_equal(loop.grid.cells_to_host(loop.counted).astype(bool), ~g["contact"])
    xps = []
    for _ in range(n_it):
        loop.step()
        xps.append(loop.grid.cells_to_host(loop.xp))
    h = loop.history
    assert len(h) == n_it and loop.converged == bool(g["converged"])
    cons = np.array([r["constraints"] for r in h])
    col = lambda key: np.array([float(r[key]) for r in h])   # noqa: E731
    defl = np.array([r["deflection"][0] if r["deflection"] else np.nan for r in h])
    stress = np.array([r["stress"][0] if r["stress"] else np.nan for r in h])
    print(f"{tag or 'both'} {np.dtype(dtype).name}: constraints {np.abs(cons - g['constraints']).max():.2e}, "
          f"deflection {np.nanmax(np.abs(defl / g['deflection'] - 1)) if lim.deflection else 0:.2e}, "
          f"stress {np.nanmax(np.abs(stress / g['stress'] - 1)) if lim.stress else 0:.2e}, "
          f"blueprint {max(np.abs(xps[i] - g['xphys'][i]).max() for i in range(n_it)):.2e}, "
          f"CG {[r['cgIterations'] for r in h]}")
    np.testing.assert_array_equal(col("beta"), g["beta"])
    np.testing.assert_allclose(cons, g["constraints"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(defl, g["deflection"], rtol=1e-8, equal_nan=True)
    np.testing.assert_allclose(stress, g["stress"], rtol=1e-8, equal_nan=True)
    np.testing.assert_allclose(col("volume"), g["volume"], rtol=1e-8)
    np.testing.assert_allclose(col("change"), g["change"], rtol=0, atol=1e-8)
    for i in range(n_it):
        np.testing.assert_allclose(xps[i], g["xphys"][i], rtol=0, atol=1e-8, err_msg=f"iteration {i + 1}")
    np.testing.assert_allclose(loop.x_host(), g["x_last"], rtol=0, atol=1e-8)
    if tag == "":
        assert any(r["reduced"] for r in h)
