"""The N > 1 path's host logic on CPU ranks (gloo, world size 2): load cases split over ranks and
summed with one all-reduce, and the bench's max-over-ranks timing rule."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case_field(case, shape):
    return np.random.default_rng(100 + case).standard_normal(shape)


def _worker(rank, world, port, n_cases, shape, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from loadpath_b200.simp import LoadCaseShards

        sh = LoadCaseShards(n_cases)
        dc = torch.zeros(shape, dtype=torch.float64)
        comp = 0.0
        for c in sh.mine():
            dc += torch.from_numpy(_case_field(c, shape))
            comp += float(c + 1)
        total = sh.reduce(dc, comp)
        # the bench's timing rule: each rank's time, the job's time is the largest
        t = torch.tensor([1.0 + rank], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out[rank] = (sh.mine(), dc.numpy().copy(), total, float(t.item()))
    finally:
        dist.destroy_process_group()


def test_load_cases_over_two_ranks():
    world, n_cases, shape = 2, 5, (4, 3, 2)
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, n_cases, shape, out), nprocs=world, join=True)
        res = dict(out)
    want_dc = sum(_case_field(c, shape) for c in range(n_cases))
    want_c = float(sum(c + 1 for c in range(n_cases)))
    assert sorted(res[0][0] + res[1][0]) == list(range(n_cases))
    assert not set(res[0][0]) & set(res[1][0])
    for r in range(world):
        np.testing.assert_allclose(res[r][1], want_dc, rtol=1e-14)
        assert res[r][2] == want_c
        assert res[r][3] == 2.0


def _point_loads(dims, k=3, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        j, kk = int(rng.integers(0, dims[1] + 1)), int(rng.integers(0, dims[2] + 1))
        d = rng.standard_normal(3)
        f = np.zeros((3,) + tuple(n + 1 for n in dims))
        f[:, dims[0], j, kk] = d / np.linalg.norm(d)
        out.append(f)
    return out


def _loop_worker(rank, world, port, dims, iters, out):
    """The sharded SIMP loop's host logic (what Top3dLoop(shards=...) does on the device): each
    rank solves its own cases, one all-reduce sums the cell energies and the compliance, every
    rank takes the design step on the totals."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from loadpath_b200.simp import LoadCaseShards
        from oracle import ref_numpy as R

        loads = _point_loads(dims)
        sh = LoadCaseShards(len(loads))
        fixed = np.zeros(loads[0].shape, bool)
        fixed[:, 0] = True

        def reduce(ce, c):
            t = torch.from_numpy(np.ascontiguousarray(ce))
            total = sh.reduce(t, c)
            return t.numpy(), total

        x, xphys, hc, hch = R.top3d_loop(dims, 0.3, 1.5, R.hex8_ke(0.3, "im"), fixed, [loads[i] for i in sh.mine()],
                                         iters, reduce=reduce)
        out[rank] = (sh.mine(), x.copy(), list(hc), list(hch))
    finally:
        dist.destroy_process_group()


def test_sharded_load_case_loop_over_two_ranks():
    """Three load cases over two ranks for three SIMP iterations: the case split is a partition,
    both ranks hold the same design (bit for bit) and it equals the one-process loop over all
    cases, as do the reduced compliances."""
    from oracle import ref_numpy as R

    world, dims, iters = 2, (8, 4, 4), 3
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_loop_worker, args=(world, port, dims, iters, out), nprocs=world, join=True)
        res = dict(out)
    loads = _point_loads(dims)
    fixed = np.zeros(loads[0].shape, bool)
    fixed[:, 0] = True
    x, _, hc, hch = R.top3d_loop(dims, 0.3, 1.5, R.hex8_ke(0.3, "im"), fixed, loads, iters)
    assert sorted(res[0][0] + res[1][0]) == list(range(len(loads)))
    np.testing.assert_array_equal(res[0][1], res[1][1])
    assert res[0][2] == res[1][2]
    np.testing.assert_allclose(res[0][1], x, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(res[0][2], hc, rtol=1e-10)
    np.testing.assert_allclose(res[0][3], hch, rtol=1e-8, atol=1e-12)
