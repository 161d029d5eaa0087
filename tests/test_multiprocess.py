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
