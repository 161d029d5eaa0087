"""The device MMA (loadpath_b200.mma) against the reference's own steps and the oracle (GPU).

The reference's golden steps (n = 40, m = 2, four updates) pin it directly; larger problems are
checked against the oracle's restatement of loadpath/mma.py. Sums are reduced in a different order
on the device, so designs agree to rounding (1e-9 relative here), not bit for bit.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_mma_matches_reference_steps():
    from loadpath_b200.mma import MMA

    g = np.load(os.path.join(GOLD, "mma.npz"))
    n, m = int(g["n"]), int(g["m"])
    mma = MMA(n, m, move=0.2)
    for i in range(int(g["steps"])):
        xn = mma.update(g[f"x{i}"], 1.0, g[f"df0{i}"], g[f"f{i}"], g[f"df{i}"])
        np.testing.assert_allclose(xn, g[f"xn{i}"], rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize("n,m", [(50_000, 1), (20_000, 3)])
def test_mma_matches_oracle_large(n, m):
    """Several updates of a design with random gradients, bounds of both kinds and a few
    non-finite gradient entries (read as the reference reads them)."""
    from loadpath_b200.mma import MMA
    from oracle import ref_numpy as R

    rng = np.random.default_rng(n + m)
    xmin = np.where(rng.random(n) < 0.5, 0.0, 0.05)
    xmax = np.where(rng.random(n) < 0.5, 1.0, 0.9)
    dev = MMA(n, m, xmin=xmin, xmax=xmax, move=0.2)
    ref = R.MMA(n, m, xmin=xmin, xmax=xmax, move=0.2)
    x = xmin + (xmax - xmin) * rng.random(n)
    for it in range(4):
        df0 = -np.abs(rng.standard_normal(n)) * (1 + rng.random(n))
        df0[rng.integers(0, n, 3)] = np.nan
        f = rng.standard_normal(m) * 0.2
        df = rng.standard_normal((m, n)) / n
        want = ref.update(x, 1.0, df0, f, df)
        got = dev.update(x, 1.0, df0, f, df)
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-10)
        x = want


def test_mma_device_tensors():
    """CUDA float64 tensors in, a CUDA tensor out; same steps as the numpy form."""
    from loadpath_b200.mma import MMA

    g = np.load(os.path.join(GOLD, "mma.npz"))
    n, m = int(g["n"]), int(g["m"])
    mma = MMA(n, m, move=0.2)
    for i in range(int(g["steps"])):
        t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
        xn = mma.update(t(g[f"x{i}"]), 1.0, t(g[f"df0{i}"]), g[f"f{i}"], t(g[f"df{i}"]))
        assert xn.is_cuda
        np.testing.assert_allclose(xn.cpu().numpy(), g[f"xn{i}"], rtol=1e-9, atol=1e-11)
