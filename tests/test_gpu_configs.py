"""The device path at the benchmark configurations' own sizes, against the reference (GPU).

- The 60x20x10 cantilever ("im" element, unit total load, volume fraction 0.3, r = 1.5): 20
  iterations of the device top3d loop against the reference's top3d port with direct sparse
  solves (tests/golden/config0.npz, written by tests/golden/make_golden.py config0), on the plain
  FP64 GPU path (rtol 1e-12: compliance to 1e-10), in mixed precision (rtol 1e-10: 1e-6) and with
  the damped-Jacobi smoother (omega 0.6, 2 + 2) over a 3-level hierarchy.
- The 256x128x128 design of the operator/solve benchmark (seeded log-uniform density smoothed by
  the r = 2 filter): one 5-level mixed-precision MG-PCG solve to rtol 1e-6 against the reference's
  own solve of the same design (loadpath/mg.py GridElasticity on the CPU: C = 257.0077140996013 in
  17 CG iterations), and the plain FP64 GPU path at rtol 1e-10 (the FP64 GPU oracle) against it.
- The evolving SIMP loop with the reference driver's live-cell reduction
  (loadpath/simp.py:795-826) for 45 iterations on a small grid, against the oracle's loop with
  the same reduction and direct solves.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

# the reference's solve of the 256x128x128 benchmark design (float32 V-cycle, rtol 1e-6, from zero)
C_REF_256 = 257.0077140996013
CG_REF_256 = 17


def _cantilever(dims, per_node):
    nx, ny, nz = dims
    fixed = np.zeros((3, nx + 1, ny + 1, nz + 1), bool)
    fixed[:, 0] = True
    f = np.zeros(fixed.shape)
    f[2, nx, :, 0] = per_node
    return fixed, f


@pytest.mark.parametrize("dtype,rtol,smoother,tol", [(np.float64, 1e-12, "chebyshev", 1e-10),
                                                     (np.float32, 1e-10, "chebyshev", 1e-6),
                                                     (np.float64, 1e-12, "jacobi", 1e-10)])
def test_config0_history_matches_reference(dtype, rtol, smoother, tol):
    from loadpath_b200.simp import Top3dLoop

    g = np.load(os.path.join(GOLD, "config0.npz"))
    dims = tuple(int(d) for d in g["dims"])
    fixed, f = _cantilever(dims, float(g["load_per_node"]))
    hist = g["hist"]
    loop = Top3dLoop(dims, float(g["volfrac"]), float(g["rmin"]), fixed, f, rtol=rtol, dtype=dtype, element="im",
                     coarse_cells=1000, smoother=smoother)
    got = np.array([loop.step() for _ in range(len(hist))])
    assert len(loop.ge.levels) == 3
    err_c = np.abs(got[:, 0] - hist[:, 0]) / np.abs(hist[:, 0])
    print(f"config 0 ({np.dtype(dtype).name}, {smoother}): C1 {got[0, 0]!r} C20 {got[-1, 0]!r}, "
          f"largest relative compliance difference {err_c.max():.2e}")
    assert err_c.max() <= tol
    np.testing.assert_allclose(got[:, 1], hist[:, 1], rtol=max(tol, 1e-9) * 10, atol=1e-9)
    np.testing.assert_allclose(loop.xphys_host(), g["xphys"], rtol=0, atol=max(tol, 1e-9) * 10)


def _bench_design(dims):
    """The benchmark's density (log-uniform in [1e-3, 1], seed 1, smoothed by the r = 2 cone filter
    normalised by its row sums) and its moduli, as device cell fields."""
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import DevGrid, stream_handle
    from loadpath_b200.simp import DeviceFilter

    g = DevGrid(dims)
    rng = np.random.default_rng(1)
    xr = g.cells_to_dev(np.exp(rng.uniform(np.log(1e-3), 0.0, dims)), torch.float64)
    flt = DeviceFilter(g, 2.0)
    x = flt.apply(g.cell_field(torch.float64), xr, hs_out=flt.hs)
    e = g.cell_field(torch.float64)
    lib().lpb_simp_law(e.data_ptr(), x.data_ptr(), 3.0, 1e-9, *g.args, stream_handle())
    return g, x, e


def test_config1_solve_matches_reference():
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from loadpath_b200.simp import case_compliance

    dims = (256, 128, 128)
    g, _, e = _bench_design(dims)
    fixed, f = _cantilever(dims, -1.0 / (dims[1] + 1))
    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    b = g.nodes_to_dev(f, torch.float64)
    out = {}
    for name, dtype, rtol in (("mixed", np.float32, 1e-6), ("fp64", np.float64, 1e-10)):
        ge = GridElasticity(mesh, 0.3, fx, rtol=rtol, element="im", dtype=dtype)
        ge.set_moduli_device(e)
        u = ge.solve_device(b)
        out[name] = (case_compliance(b, u), ge.last_iters, len(ge.levels))
        del ge, u
        torch.cuda.empty_cache()
    c32, it32, nl = out["mixed"]
    c64, _, _ = out["fp64"]
    print(f"config 1: mixed C {c32!r} in {it32} CG iterations ({nl} levels); FP64 oracle C {c64!r}; "
          f"reference C {C_REF_256!r} in {CG_REF_256}")
    assert nl == 5
    assert abs(it32 - CG_REF_256) <= 2
    assert abs(c32 - C_REF_256) / C_REF_256 <= 1e-6
    assert abs(c64 - C_REF_256) / C_REF_256 <= 1e-6
    assert abs(c32 - c64) / c64 <= 1e-6


def test_live_cell_loop_45_iterations_matches_oracle():
    """45 iterations of the loop from the benchmark's kind of start (log-uniform density), solved on
    the live cells once fewer than 80 % are alive (REDUCE_BELOW), against the oracle's loop making
    the same reduction (alive = density above 1e-3 or an anchor cell, kept = 26-connected to a
    support) with direct solves on the kept dofs."""
    from loadpath_b200.simp import Top3dLoop
    from oracle import ref_numpy as R

    dims = (24, 12, 12)
    iters = 45
    fixed, f = _cantilever(dims, -1.0 / (dims[1] + 1))
    x0 = R.log_uniform_density(dims, 7)
    ke = R.hex8_ke(0.3, "im")
    loop = Top3dLoop(dims, 0.3, 2.0, fixed, f, rtol=1e-10, dtype=np.float32, element="im", x0=x0, coarse_cells=200,
                     live_cells=True)
    got = np.array([loop.step()[0] for _ in range(iters)])
    reduced = loop.reduced
    held = fixed.any(axis=0)
    loaded = (f != 0).any(axis=0)
    support = R.cells_touching(held)
    anchor = R.cells_touching(held | loaded)
    _, _, hist_c, _ = R.top3d_loop(dims, 0.3, 2.0, ke, fixed, f, iters, x0=x0,
                                   solve=R.live_solve(ke, fixed, f, support, anchor), with_xphys=True)
    err = np.abs(got - np.array(hist_c)) / np.abs(np.array(hist_c))
    print(f"live-cell loop: {iters} iterations, CG counts {[h[2] for h in loop.history]}, reduced at the end "
          f"{reduced}, slow solves {loop.slow_solves}, largest relative compliance difference {err.max():.2e}")
    assert reduced
    assert err.max() <= 1e-6
