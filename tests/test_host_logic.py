"""Host-side logic that needs no GPU: the batched OC bisection walk."""
import numpy as np
import pytest

from loadpath_b200.simp import oc_bisection


def _volume_fn(seed, n=4000, move=0.2):
    """V(lam) = sum_c clamp(x sqrt(-dc / dv) / sqrt(lam), max(0, x - move), min(1, x + move)) gv,
    the OC step's filtered volume, on random cells."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, n)
    x[rng.random(n) < 0.1] = 0.0
    dc = -10.0 ** rng.uniform(-9, 3, n)
    dv = rng.uniform(0.5, 1.5, n)
    gv = rng.uniform(0.5, 1.5, n)
    ts = x * np.sqrt(-dc / dv)
    lo, hi = np.maximum(0.0, x - move), np.minimum(1.0, x + move)

    def vol(lam):
        return float(np.sum(np.clip(ts / np.sqrt(lam), lo, hi) * gv))

    return vol, float(np.sum(gv))


def _plain(vol, target, l1=0.0, l2=1e9):
    lmid, n = None, 0
    while (l2 - l1) / (l1 + l2) > 1e-3:
        lmid = 0.5 * (l2 + l1)
        n += 1
        if vol(lmid) > target:
            l1 = lmid
        else:
            l2 = lmid
    return lmid, n


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("frac", [0.05, 0.3, 0.6])
def test_oc_bisection_follows_the_plain_walk(seed, frac):
    vol, total = _volume_fn(seed)
    target = frac * total
    want, steps = _plain(vol, target)
    got, passes = oc_bisection(lambda cands: [vol(c) for c in cands], target)
    assert got == want
    # one ladder pass and at most ceil(remaining levels / 5) tree passes
    assert passes <= 1 + (steps + 4) // 5
    assert passes <= 5


def test_oc_bisection_plateaus_and_ties():
    """A step-function V (whole ranges of multipliers give the same volume, one exactly equal to
    the target) still gives the plain walk's midpoint."""
    def vol(lam):
        return float(np.floor(np.log2(1e9 / lam)))

    for target in (0.0, 3.0, 17.0, 40.0, 100.0):
        want, _ = _plain(vol, target)
        got, _ = oc_bisection(lambda cands: [vol(c) for c in cands], target)
        assert got == want


def test_graph_cache_keeps_graphs_across_calls(monkeypatch):
    """GridElasticity._graph captures a key once per buffer generation: a second call with the
    same key and generation reuses the first capture (no GPU: capture and free are stubbed)."""
    import loadpath_b200.mg as mg

    class FakeLib:
        def __init__(self):
            self.captured = 0
            self.freed = 0

        def lpb_capture_begin(self, st):
            self.captured += 1

        def lpb_capture_end(self, st, out):
            out._obj.value = 1000 + self.captured

        def lpb_graph_free(self, g):
            self.freed += 1

    fake = FakeLib()
    monkeypatch.setattr(mg, "lib", lambda: fake)
    monkeypatch.setattr(mg, "stream_handle", lambda: 0)

    class Stream:
        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

    monkeypatch.setattr(mg.torch.cuda, "stream", lambda s: Stream())
    monkeypatch.setattr(mg.torch.cuda, "current_stream", lambda: type("S", (), {"synchronize": lambda self: None})())
    ge = object.__new__(mg.GridElasticity)
    ge._gcache, ge._gen, ge._cap_stream = {}, 0, None
    a = ge._graph("head", lambda: None)
    b = ge._graph("head", lambda: None)
    assert fake.captured == 1 and a is b
    ge._gen += 1                               # a buffer was replaced: the graphs go
    ge._graph("head", lambda: None)
    assert fake.captured == 2 and fake.freed == 1


def test_cells_touching_matches_oracle():
    """The loop's anchor/support cells (any corner node flagged) against the oracle's restatement
    of loadpath/simp.py:150-151 on random node flags."""
    from loadpath_b200.simp import _cells_touching
    from oracle import ref_numpy as R

    rng = np.random.default_rng(4)
    flags = rng.random((7, 5, 9)) < 0.05
    np.testing.assert_array_equal(_cells_touching(flags), R.cells_touching(flags))


def test_oracle_live_solve_reduces_and_falls_back():
    """The oracle's live-cell solve (loadpath/simp.py:795-826): on a design with a floating island
    the island's dofs come back zero and the answer equals a solve on the kept cells alone; with
    the load placed on the island it goes back to the full grid."""
    from oracle import ref_numpy as R

    dims = (8, 3, 3)
    fixed = np.zeros((3, 9, 4, 4), bool)
    fixed[:, 0] = True
    f = np.zeros(fixed.shape)
    f[2, 3, :, 0] = -0.25
    x = np.full(dims, 1e-4)
    x[:4] = 1.0                 # a bar from the support to the load
    x[6] = 1.0                  # an island, not touching the bar (5 of 8 slabs alive: below 0.8)
    ke = R.hex8_ke(0.3, "im")
    e = R.simp_moduli(x)
    held = fixed.any(axis=0)
    support = R.cells_touching(held)
    anchor = R.cells_touching(held | (f != 0).any(axis=0))
    u = R.live_solve(ke, fixed, f, support, anchor)(e, x)
    assert np.all(u[:, 6:] == 0.0) and np.any(u[:, 1:4] != 0.0)
    keep = R.connected_keep((x > R.ALIVE) | anchor, support)
    assert keep[:4].all() and not keep[4:].any()
    np.testing.assert_allclose(u, R.assembled_solve(ke, np.where(keep, e, 0.0), fixed, f, drop_dead=True),
                               rtol=1e-12, atol=1e-14)
    f2 = np.zeros(fixed.shape)
    f2[2, 8, 1, 3] = -1.0       # a load on the island: the full grid solves it
    anchor2 = R.cells_touching(held | (f2 != 0).any(axis=0))
    u2 = R.live_solve(ke, fixed, f2, support, anchor2)(e, x)
    np.testing.assert_allclose(u2, R.assembled_solve(ke, e, fixed, f2), rtol=1e-12)


def test_mgops_cells_fields():
    """mgops.Cells carries the fields the reference's callers read (loadpath/mgops.py:220-244),
    checked here element by element: the dof at base + off[3k + d] of a (3, X+1, Y+1, Z+1) field
    is component d of the cell's corner k."""
    from loadpath_b200.mgops import Cells

    rng = np.random.default_rng(3)
    shape = (4, 3, 5)
    active = rng.random(shape) > 0.3
    c = Cells(active)
    want = [(x, y, z) for x in range(4) for y in range(3) for z in range(5) if active[x, y, z]]
    assert c.n == len(want) and c.cells.tolist() == [list(w) for w in want]
    for i, (x, y, z) in enumerate(want):
        assert c.rows[x, y, z] == i
    assert (c.rows[~active] == -1).all()
    field = np.arange(3 * 5 * 4 * 6).reshape(3, 5, 4, 6)
    flat = field.reshape(-1)
    for i, (x, y, z) in enumerate(want):
        assert flat[c.base[i]] == field[0, x, y, z]
        for k in range(8):
            for d in range(3):
                assert flat[c.base[i] + c.off[3 * k + d]] == field[d, x + (k & 1), y + (k >> 1 & 1), z + (k >> 2 & 1)]
    assert c.ft(np.float32).shape == (24, c.n) and c.ft(np.float32) is c.ft("float32")
    assert c.base.dtype == c.off.dtype == c.cells.dtype == np.int64


def _loop_state(**kw):
    from loadpath_b200.optimize import OptimizeLoop, SimpOptions

    lp = object.__new__(OptimizeLoop)
    lp.opts = SimpOptions(volume_fraction=0.3, filter_radius=1.5, **kw.pop("opts", {}))
    lp.measured, lp.scheduled = True, True
    lp.beta, lp.since_beta, lp.step_prev, lp.move_k = 1.0, 0, 0.5, 0.2
    lp.it, lp.history, lp.converged = 1, [], False
    for key, v in kw.items():
        setattr(lp, key, v)
    return lp


def test_optimize_loop_beta_continuation_and_stops():
    """OptimizeLoop's continuation and stopping rules (loadpath/simp.py:2418-2450): beta doubles
    after beta_every iterations or a free step under 2 tol, dropping the measured step and halving
    the limit; at beta_max a free step under tol stops, the schedule stops a held volume after its
    hold, and otherwise the compliance's stall over stall_window iterations stops."""
    from loadpath_b200.optimize import beta_hold

    assert beta_hold(_loop_state().opts, 1.0) == 10
    sched = _loop_state(opts={"beta_schedule": (20, 15)}).opts
    assert (beta_hold(sched, 1.0), beta_hold(sched, 2.0), beta_hold(sched, 4.0)) == (20, 15, 10)
    # nine iterations at beta 1, a large change: no doubling
    lp = _loop_state(since_beta=9)
    lp._continue(change=0.1, move=0.2, comp=1.0, held=True)
    assert lp.beta == 1.0 and lp.step_prev == 0.5
    # the tenth: doubling
    lp = _loop_state(since_beta=10)
    lp._continue(change=0.1, move=0.2, comp=1.0, held=True)
    assert (lp.beta, lp.since_beta, lp.step_prev, lp.move_k) == (2.0, 0, None, 0.1)
    # a small change doubles early only as a free step (not held at the move limit)
    lp = _loop_state(since_beta=3)
    lp._continue(change=0.015, move=0.015, comp=1.0, held=True)
    assert lp.beta == 1.0
    lp._continue(change=0.015, move=0.2, comp=1.0, held=True)
    assert lp.beta == 2.0
    # at beta_max: a free step under tol stops
    lp = _loop_state(beta=32.0, it=5, since_beta=2)
    lp._continue(change=0.005, move=0.2, comp=1.0, held=True)
    assert lp.converged
    # scheduled with the volume held: stops after the hold, not before
    lp = _loop_state(beta=32.0, it=5, since_beta=9)
    lp._continue(change=0.05, move=0.2, comp=1.0, held=True)
    assert not lp.converged
    lp.since_beta = 10
    lp._continue(change=0.05, move=0.2, comp=1.0, held=True)
    assert lp.converged
    # the volume off target (held False): the stall rule over stall_window = 6 compares with the
    # compliance seven records back
    hist = [{"compliance": c} for c in (10.0, 9.0, 8.5, 8.31, 8.305, 8.30, 8.30, 8.30)]
    lp = _loop_state(beta=32.0, it=8, since_beta=6, history=hist)
    lp._continue(change=0.05, move=0.2, comp=8.30, held=False)
    assert not lp.converged           # against 9.0
    hist += [{"compliance": 8.30}, {"compliance": 8.30}]
    lp._continue(change=0.05, move=0.2, comp=8.30, held=False)
    assert lp.converged               # against 8.31: within 2e-3


def _constrained_state(**kw):
    from types import SimpleNamespace

    from loadpath_b200.optimize import ConstrainedLoop, SimpOptions

    lp = object.__new__(ConstrainedLoop)
    lp.opts = SimpOptions(volume_fraction=0.5, filter_radius=1.5, **kw.pop("opts", {}))
    lp.mma = SimpleNamespace(move=0.1)
    lp.move_cap = 0.1
    lp.beta, lp.since_beta = 1.0, 0
    lp.best, lp.trail, lp.converged = None, [], False
    for key, v in kw.items():
        setattr(lp, key, v)
    return lp


def test_constrained_loop_continuation_and_stops():
    """ConstrainedLoop's rules (loadpath/constrained.py:789-829): beta doubles only once the design
    is feasible (worst constraint <= 0.02) after beta_every iterations or a small change, or after
    three holds whatever; each doubling shrinks the move cap by 0.6 (floor 0.02) and the move to it;
    at beta_max the lightest feasible design is kept, and the run stops on a feasible change under
    tol or when the kept volume gained under STALL_GAIN over stall_window iterations."""
    rec = lambda v, c, ch: {"volume": v, "constraints": c, "change": ch}   # noqa: E731
    # infeasible after the usual hold: no doubling
    lp = _constrained_state(since_beta=10)
    lp._continue(rec(0.4, [0.05, -0.1], 0.05), "x")
    assert lp.beta == 1.0
    # feasible after the hold: doubling, the cap 0.06
    lp = _constrained_state(since_beta=10)
    lp._continue(rec(0.4, [0.01, -0.1], 0.05), "x")
    assert (lp.beta, lp.since_beta) == (2.0, 0) and abs(lp.move_cap - 0.06) < 1e-15 and lp.mma.move == lp.move_cap
    # feasible with a small change before the hold: doubling
    lp = _constrained_state(since_beta=2)
    lp._continue(rec(0.4, [0.0], 0.015), "x")
    assert lp.beta == 2.0
    # three holds, infeasible: doubling all the same
    lp = _constrained_state(since_beta=30)
    lp._continue(rec(0.4, [0.3], 0.05), "x")
    assert lp.beta == 2.0
    # the cap's floor
    lp = _constrained_state(since_beta=10, move_cap=0.03)
    lp._continue(rec(0.4, [0.0], 0.05), "x")
    assert lp.move_cap == 0.02
    # at beta_max: the lightest feasible design is kept; an infeasible one is not
    lp = _constrained_state(beta=32.0)
    lp._continue(rec(0.40, [0.01], 0.05), "x1")
    lp._continue(rec(0.38, [0.10], 0.05), "x2")
    lp._continue(rec(0.39, [0.00], 0.05), "x3")
    assert lp.best[0] == "x3" and lp.trail == [0.40, 0.40, 0.39] and not lp.converged
    # a feasible small change stops
    lp._continue(rec(0.389, [0.0], 0.005), "x4")
    assert lp.converged and lp.best[0] == "x4"
    # the stall over stall_window = 6 kept volumes
    lp = _constrained_state(beta=32.0)
    for k in range(7):
        lp._continue(rec(0.40 - 1e-4 * k, [0.0], 0.05), f"x{k}")
        assert not lp.converged or k == 6
    assert lp.converged   # 0.3994 against 0.40 six records back: under STALL_GAIN
