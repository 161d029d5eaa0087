"""The other users of GridElasticity, driven through this package's GridElasticity as they drive
the reference's (GPU), against the reference's own solves (tests/golden/callers.npz), on a mesh
that is not a full box (an L-shaped part at pitch 0.5, held at its base):

- verification's re-solve of a delivered grid (loadpath/verify.py:1689-1704): one set_moduli,
  two right-hand sides through solve_many, the mesh and Poisson's ratio read back for the stress
  recovery and a stress mask set on the solver;
- the build simulation's layer-by-layer solves (loadpath/buildsim.py:609-640): one solver made
  with device "cpu", set_moduli(e * active) as each layer of cells is added (the cells not yet
  built at modulus 0), one load per layer.

Solutions to 1e-8 of their largest entry at rtol 1e-10, CG counts within 2 of the reference's."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


class _Mesh:
    """The fields of loadpath's HexMesh that GridElasticity reads."""

    def __init__(self, g):
        self.elem_ijk, self.node_ijk, self.pitch = g["elem_ijk"], g["node_ijk"], float(g["pitch"])
        self.n_elem, self.n_nodes = len(self.elem_ijk), len(self.node_ijk)
        self.n_dof = 3 * self.n_nodes


def _close(got, want):
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-8 * np.abs(want).max())


def test_verification_resolve_matches_reference():
    from loadpath_b200.mg import GridElasticity

    g = np.load(os.path.join(GOLD, "callers.npz"))
    mesh = _Mesh(g)
    ge = GridElasticity(mesh, 0.3, g["fixed"], rtol=1e-10, maxiter=3000, element="im")
    ge.set_moduli(g["e"])
    ge.stress_mask = None
    u1, u2 = ge.solve_many([g["f1"], g["f2"]])
    assert ge.mesh is mesh and ge.nu == 0.3
    _close(u1, g["verify_u1"])
    _close(u2, g["verify_u2"])
    its = ge.last_iters if not isinstance(ge.last_iters, (list, tuple)) else max(ge.last_iters)
    assert abs(int(its) - int(g["verify_iters"])) <= 2, (ge.last_iters, int(g["verify_iters"]))


def test_build_simulation_layers_match_reference():
    from loadpath_b200.mg import GridElasticity

    g = np.load(os.path.join(GOLD, "callers.npz"))
    mesh = _Mesh(g)
    ge = GridElasticity(mesh, 0.3, g["fixed"], rtol=1e-10, maxiter=3000, device="cpu", element="im")
    assert ge.device.type == "cuda"
    for li in range(int(g["layers"])):
        active = mesh.elem_ijk[:, 2] <= li
        ge.set_moduli(g["e"] * active)
        du = ge.solve_many([g[f"layer{li}_f"]])[0]
        _close(du, g[f"layer{li}_u"])
        its = ge.last_iters if not isinstance(ge.last_iters, (list, tuple)) else max(ge.last_iters)
        assert abs(int(its) - int(g[f"layer{li}_iters"])) <= 2, (li, ge.last_iters, int(g[f"layer{li}_iters"]))
