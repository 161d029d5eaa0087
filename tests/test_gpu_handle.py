"""The solver handle of the C ABI (lpb_mg_create / lpb_mg_set_moduli / lpb_mg_solve /
lpb_mg_destroy) driven through plain ctypes, the way a host in another language binds the
library, against loadpath_b200.mg.GridElasticity (GPU).

Given the same element matrix the two take the same kernels in the same order, so the solutions
must agree bit for bit, with the same CG counts: the float32 V-cycle (mixed) and the float64
hierarchy, from zero and from a warm start, and a design whose coarsest factor or CG stall sends
both to the strict hierarchy (the reference's golden `rough_strict` case). A handle built from the
library's own element matrix (lpb_hex8_ke) agrees with the Python class to the solver tolerance.
torch only allocates the device memory a C host would allocate with cudaMalloc."""
import ctypes
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "loadpath_b200", "liblpb200.so")


def _cdll():
    L = ctypes.CDLL(LIB)
    vp, i, d, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
    L.lpb_mg_create.restype = vp
    L.lpb_mg_create.argtypes = [i, i, i, vp, vp, i, d, i, ll, vp]
    L.lpb_mg_set_moduli.argtypes = [vp, vp, vp]
    L.lpb_mg_solve.argtypes = [vp, vp, vp, vp, vp, vp]
    L.lpb_mg_levels.argtypes = [vp]
    L.lpb_mg_strict.argtypes = [vp]
    L.lpb_mg_destroy.argtypes = [vp]
    L.lpb_mg_destroy.restype = None
    L.lpb_layout_dims.argtypes = [i, i, i, vp]
    L.lpb_layout_nodes_f64.argtypes = [vp, vp, i, i, i]
    L.lpb_layout_cells_f64.argtypes = [vp, vp, i, i, i]
    L.lpb_hex8_ke.argtypes = [d, i, vp]
    return L


def _problem(dims, seed, void_frac=0.0):
    """Cantilever (x = 0 face held, unit -z load on the bottom edge at x = nx), seeded log-uniform
    densities smoothed by the r = 2 filter, some cells removed."""
    from oracle import ref_numpy as R

    x = R.log_uniform_density(dims, seed)
    e = R.simp_moduli(x)
    if void_frac:
        e[np.random.default_rng(seed + 100).random(dims) < void_frac] = 0.0
    fixed, f = R.cantilever_bc(dims)
    return e, fixed, f


class Handle:
    def __init__(self, L, dims, fixed_grid, ke, single, rtol, coarse_cells, maxiter=500):
        self.L, self.dims = L, dims
        bits = (fixed_grid[0].astype(np.uint8) | (fixed_grid[1].astype(np.uint8) << 1)
                | (fixed_grid[2].astype(np.uint8) << 2))
        bits = np.ascontiguousarray(bits)
        ke = np.ascontiguousarray(ke, np.float64)
        st = ctypes.c_int(0)
        self.h = L.lpb_mg_create(*dims, bits.ctypes.data, ke.ctypes.data, int(single), rtol, maxiter, coarse_cells,
                                 ctypes.byref(st))
        assert self.h and st.value == 0, st.value
        sizes = np.zeros(5, np.int64)
        L.lpb_layout_dims(*dims, sizes.ctypes.data)
        self.nnode, self.ncell = int(sizes[2]), int(sizes[3])

    def nodes(self, grid_order):
        out = np.zeros(self.nnode)
        self.L.lpb_layout_nodes_f64(np.ascontiguousarray(grid_order, np.float64).ctypes.data, out.ctypes.data,
                                    *self.dims)
        return torch.from_numpy(out).cuda()

    def set_moduli(self, e_grid):
        out = np.zeros(self.ncell)
        self.L.lpb_layout_cells_f64(np.ascontiguousarray(e_grid, np.float64).ctypes.data, out.ctypes.data, *self.dims)
        self.e = torch.from_numpy(out).cuda()
        rc = self.L.lpb_mg_set_moduli(self.h, self.e.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert rc == 0, rc

    def solve(self, b, x0=None):
        x = torch.empty_like(b)
        it = ctypes.c_int(0)
        rc = self.L.lpb_mg_solve(self.h, b.data_ptr(), x0.data_ptr() if x0 is not None else None, x.data_ptr(),
                                 ctypes.byref(it), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return x, it.value, rc

    def close(self):
        self.L.lpb_mg_destroy(self.h)


def _python(dims, fixed_grid, e_grid, single, rtol, coarse_cells, element="im", maxiter=500):
    from loadpath_b200.mg import BoxMesh, GridElasticity

    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed_grid[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, rtol=rtol, maxiter=maxiter, coarse_cells=coarse_cells,
                        dtype=np.float32 if single else np.float64, element=element)
    ge.set_moduli_device(ge.g0.cells_to_dev(e_grid, torch.float64))
    return ge


@pytest.mark.parametrize("single", [1, 0])
def test_handle_solve_equals_python_class(single):
    from loadpath_b200.fem import hex8_ke

    dims, rtol, cc = (32, 16, 16), 1e-8, 200
    e, fixed, f = _problem(dims, 11, 0.02)
    L = _cdll()
    h = Handle(L, dims, fixed, hex8_ke(0.3, "im"), single, rtol, cc)
    try:
        h.set_moduli(e)
        ge = _python(dims, fixed, e, single, rtol, cc)
        assert L.lpb_mg_levels(h.h) == len(ge.levels) >= 3
        assert bool(L.lpb_mg_strict(h.h)) == ge.strict
        b = h.nodes(f)
        x, it, rc = h.solve(b)
        assert rc == 0
        want = ge.solve_device(ge.g0.nodes_to_dev(f, torch.float64))
        assert it == ge.last_iters
        assert torch.equal(x, want.reshape(-1)), float((x - want.reshape(-1)).abs().max())
        # a warm start: the solution of a scaled load, both sides from the same x0
        x0 = (0.5 * x).contiguous()
        x2, it2, rc2 = h.solve(b, x0)
        want2 = ge.solve_device(ge.g0.nodes_to_dev(f, torch.float64), x0.reshape(want.shape))
        assert rc2 == 0 and it2 == ge.last_iters
        assert torch.equal(x2, want2.reshape(-1))
    finally:
        h.close()


def test_handle_strict_fallback_equals_python_class():
    """The reference's rough design (no smoothing, 5 % of the cells removed): the plain hierarchy
    stalls in the solve and both sides go on in the strict hierarchy, with the same answer."""
    from loadpath_b200.fem import hex8_ke

    g = np.load(os.path.join(GOLD, "hier_rough_strict.npz"), allow_pickle=False)
    dims = tuple(int(d) for d in g["dims"])
    e, fixed, f = g["e_grid"], g["fixed_grid"], g["f_grid"]
    L = _cdll()
    h = Handle(L, dims, fixed, hex8_ke(0.3, "im"), 1, 1e-10, 20, maxiter=3000)
    try:
        h.set_moduli(e)
        ge = _python(dims, fixed, e, 1, 1e-10, 20, maxiter=3000)
        b = h.nodes(f)
        x, it, rc = h.solve(b)
        want = ge.solve_device(ge.g0.nodes_to_dev(f, torch.float64))
        assert rc == 0
        assert bool(L.lpb_mg_strict(h.h)) == ge.strict is True
        assert it == ge.last_iters
        assert torch.equal(x, want.reshape(-1))
    finally:
        h.close()


def test_handle_with_library_element_matches_to_tolerance():
    """A host without numpy: the element matrix from lpb_hex8_ke; the answer agrees with the Python
    class (numpy's element matrix) to the solver tolerance."""
    dims, rtol, cc = (16, 8, 8), 1e-10, 60
    e, fixed, f = _problem(dims, 5)
    L = _cdll()
    ke = np.zeros((24, 24))
    assert L.lpb_hex8_ke(0.3, 1, ke.ctypes.data) == 0
    h = Handle(L, dims, fixed, ke, 1, rtol, cc)
    try:
        h.set_moduli(e)
        x, it, rc = h.solve(h.nodes(f))
        ge = _python(dims, fixed, e, 1, rtol, cc)
        want = ge.solve_device(ge.g0.nodes_to_dev(f, torch.float64)).reshape(-1)
        assert rc == 0
        assert float((x - want).norm() / want.norm()) < 1e-8
    finally:
        h.close()
