"""loadpath's own SIMP loop on the device (optimize.OptimizeLoop) against the loop of the
reference itself (tests/golden/optimize.npz: simp.optimize on two top3d cantilevers mirrored in y
and a bridge mirrored in x and y, default options with the solves at rtol 1e-10), iteration by
iteration: the projection sharpness, the
measured move limit, the number of volume-multiplier trials, the compliance, the design change
and the blueprint density each iteration starts from (GPU).

The reference solves these small systems directly; the device loop runs MG-PCG to rtol 1e-10 with
a float32 or float64 V-cycle, so the two differ by the solves' residuals, carried through 24 to 30
iterations of a loop whose steps depend smoothly on them."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("case", ["small", "medium", "bridge"])
def test_optimize_loop_matches_reference_run(case, dtype):
    from loadpath_b200.optimize import OptimizeLoop, SimpOptions

    g = np.load(os.path.join(GOLD, "optimize.npz"))
    k = lambda s: g[f"{case}_{s}"]   # noqa: E731
    n_it = int(k("iterations"))
    opts = SimpOptions(volume_fraction=float(k("volfrac")), filter_radius=float(k("radius")), max_iterations=n_it,
                       solve_rtol=1e-10, pad_filter=bool(k("pad")))
    loop = OptimizeLoop(tuple(int(d) for d in k("dims")), k("fixed"), [k("f")], float(k("nu")), opts,
                        preserve=k("pres"), pitch=float(k("pitch")), mirror=tuple(int(a) for a in k("mirror")),
                        dtype=dtype, coarse_cells=100)
    xps = []
    for _ in range(n_it):
        loop.step()
        xps.append(loop.grid.cells_to_host(loop.xp))   # the blueprint the iteration started from
    h = loop.history
    assert len(h) == n_it and not loop.converged
    got = {key: np.array([float(r[key]) for r in h]) for key in ("compliance", "beta", "change", "move", "volume",
                                                                  "volumeSolves")}
    np.testing.assert_array_equal(got["beta"], k("beta"))
    err_c = np.abs(got["compliance"] / k("compliance") - 1)
    print(f"{case} {np.dtype(dtype).name}: compliance rel err max {err_c.max():.2e}, change "
          f"{np.abs(got['change'] - k('change')).max():.2e}, move {np.abs(got['move'] - k('move')).max():.2e}, "
          f"volume solves {int(np.abs(got['volumeSolves'] - k('volumeSolves')).sum())} off, "
          f"CG {[r['cgIterations'] for r in h]}")
    # the bridge (volume fraction 0.01, held at its four bottom corners' edges) is badly conditioned:
    # the reference's own direct solve and the oracle's agree on its energy to a few parts in 10^9
    assert err_c.max() <= (1e-9 if case != "bridge" else 2e-8)
    np.testing.assert_allclose(got["move"], k("move"), rtol=1e-9)
    np.testing.assert_allclose(got["change"], k("change"), rtol=0, atol=1e-9)
    np.testing.assert_allclose(got["volume"], k("volume"), rtol=1e-9)
    np.testing.assert_array_equal(got["volumeSolves"], k("volumeSolves"))
    for i in range(n_it):
        np.testing.assert_allclose(xps[i], k("xphys")[i], rtol=0, atol=1e-9, err_msg=f"iteration {i + 1}")
    np.testing.assert_allclose(loop.x_host(), k("x_last"), rtol=0, atol=1e-9)
