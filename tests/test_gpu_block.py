"""k load cases solved as one block (GridElasticity.solve_block_device): every column's answer
and iteration count equal a lone solve's, bit for bit, in the mixed and the float64 hierarchy;
warm starts, a zero right-hand side and more than eight columns (GPU)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _solver(dims, dtype, seed=5):
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from oracle import ref_numpy as R

    x = R.log_uniform_density(dims, seed)
    fixed, _ = R.cantilever_bc(dims)
    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, rtol=1e-8, maxiter=500, coarse_cells=200, dtype=dtype, element="im")
    ge.set_moduli(R.simp_moduli(x).reshape(-1))
    return ge


def _point_loads(dims, k, seed):
    """k unit point forces at seeded nodes of the x = nx face, directions uniform on the sphere."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        f = np.zeros((3,) + tuple(d + 1 for d in dims))
        j, kk = rng.integers(0, dims[1] + 1), rng.integers(0, dims[2] + 1)
        d = rng.standard_normal(3)
        f[:, dims[0], j, kk] = d / np.linalg.norm(d)
        out.append(f)
    return out


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("k", [3, 9])
def test_block_equals_lone_solves(dtype, k):
    dims = (32, 16, 16)
    ge = _solver(dims, dtype)
    g = ge.g0
    loads = _point_loads(dims, k, 3)
    bs = [g.nodes_to_dev(f, torch.float64) for f in loads]
    lone, lone_its = [], []
    for b in bs:
        lone.append(g.nodes_to_host(ge.solve_device(b)))
        lone_its.append(ge.last_iters)
    xs = ge.solve_block_device(bs)
    assert ge.last_iters == lone_its
    for x, want in zip(xs, lone):
        np.testing.assert_array_equal(g.nodes_to_host(x), want)


def test_block_warm_starts_and_zero_column():
    dims = (32, 16, 16)
    ge = _solver(dims, np.float32)
    g = ge.g0
    loads = _point_loads(dims, 3, 4)
    loads[1] = np.zeros_like(loads[1])
    bs = [g.nodes_to_dev(f, torch.float64) for f in loads]
    first = ge.solve_block_device(bs)
    assert ge.last_iters[1] == 0 and not g.nodes_to_host(first[1]).any()
    # warm starts from a nearby answer: a lone warm solve gives the same bits
    x0s = [None if j == 1 else x * 0.9 for j, x in enumerate(first)]
    xs = ge.solve_block_device(bs, x0s)
    its = list(ge.last_iters)
    for j in (0, 2):
        want = ge.solve_device(bs[j], x0s[j])
        assert ge.last_iters == its[j]
        np.testing.assert_array_equal(g.nodes_to_host(xs[j]), g.nodes_to_host(want))


def test_load_case_simp_loop_matches_oracle():
    """The batched load-case SIMP loop (Top3dLoop with a list of loads, solved as one block) against
    the oracle's top3d loop on the compliance sum, with its direct sparse solves."""
    from loadpath_b200.simp import Top3dLoop
    from oracle import ref_numpy as R

    dims = (16, 8, 8)
    fixed, _ = R.cantilever_bc(dims)
    loads = _point_loads(dims, 4, 7)
    iters = 6
    _, xp_ref, hc, hch = R.top3d_loop(dims, 0.2, 2.0, R.hex8_ke(0.3, "plain"), fixed, loads, iters)
    loop = Top3dLoop(dims, 0.2, 2.0, fixed, loads, rtol=1e-10, element="plain", coarse_cells=20)
    got = [loop.step() for _ in range(iters)]
    np.testing.assert_allclose([c for c, _ in got], hc, rtol=1e-7)
    np.testing.assert_allclose([ch for _, ch in got], hch, rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(loop.xphys_host(), xp_ref, rtol=1e-6, atol=1e-8)
    assert len(loop.history[-1][2]) == 4


def test_sharded_loop_single_rank_equals_block_loop():
    """Top3dLoop with a LoadCaseShards over one rank (no process group: it owns every case) takes the
    sharded path (compliance summed on the host, the reduction a no-op) and equals the plain
    load-case loop."""
    from loadpath_b200.simp import LoadCaseShards, Top3dLoop
    from oracle import ref_numpy as R

    dims = (16, 8, 8)
    fixed, _ = R.cantilever_bc(dims)
    loads = _point_loads(dims, 3, 9)
    a = Top3dLoop(dims, 0.2, 2.0, fixed, loads, rtol=1e-10, element="plain", coarse_cells=20, autotune=False)
    b = Top3dLoop(dims, 0.2, 2.0, fixed, loads, rtol=1e-10, element="plain", coarse_cells=20, autotune=False,
                  shards=LoadCaseShards(len(loads)))
    ga = [a.step() for _ in range(3)]
    gb = [b.step() for _ in range(3)]
    np.testing.assert_allclose([c for c, _ in gb], [c for c, _ in ga], rtol=1e-14)
    assert [ch for _, ch in gb] == [ch for _, ch in ga]
    np.testing.assert_array_equal(b.xphys_host(), a.xphys_host())
