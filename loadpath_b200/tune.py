"""Launch-geometry autotuner for the stencil applies.

The level-1 apply marches along z in segments of chunks (four node planes); a segment recomputes
one halo cell, so short segments fill the GPU's resident blocks at the cost of more halo work, long
ones the other way round. The fine-level applies run persistent blocks that share the (tile,
chunk) units out evenly; their knob is the number of blocks per SM (0: all that fit). The
launchers pick a geometry by a cost model; `autotune(ge)` instead times the applies of a built
hierarchy at a set of candidates (CUDA events on the working stream, after a warm-up launch) and
records the fastest in the library's tuning table (`lpb_tune_set`), per grid and precision. Only
launch geometry is tuned: the smoothing schedule (Chebyshev degree 2, as the reference's V-cycle)
is part of the algorithm the CG iteration counts are checked against, and stays fixed.

Results are kept for the process (a second hierarchy of the same grid reuses them) and can be
saved to / loaded from a JSON file.
"""
from __future__ import annotations

import json
import os

import torch

from ._lib import lib
from .grid import stream_handle

__all__ = ["KNOBS", "autotune", "candidates", "save", "load", "tuned"]

KNOBS = {"fine_f32": 1, "fine_f64": 2, "level1_f32": 3, "level1_f64": 4}
_RESULTS = {}        # (knob name, nx, ny, nz) -> {"best": value, "us": {value: time}}


def candidates(nchunks, lo):
    """Segment lengths to time: a geometric spread up to the whole column (and 0, the cost
    model's own choice)."""
    c = {0, nchunks}
    v = lo
    while v < nchunks:
        c.add(v)
        v = v + 1 if v < 4 else int(v * 1.5)
    return sorted(x for x in c if x == 0 or lo <= x <= nchunks)


def _time(fn, reps):
    fn()                                               # warm-up (and the tensor-map set-up)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) * 1e3 / reps


FINE_CANDIDATES = (0, 1, 2)   # persistent fine-apply blocks per SM (0: all that fit)


def _tune_one(name, grid, fn, lo, reps):
    L = lib()
    knob = KNOBS[name]
    key = (name, grid.nx, grid.ny, grid.nz)
    if key in _RESULTS:
        L.lpb_tune_set(knob, grid.nx, grid.ny, grid.nz, _RESULTS[key]["best"])
        return _RESULTS[key]
    times = {}
    cands = FINE_CANDIDATES if name.startswith("fine") else candidates(grid.pz // 4, lo)
    for z in cands:
        L.lpb_tune_set(knob, grid.nx, grid.ny, grid.nz, z)
        times[z] = _time(fn, reps)
    best = min(times, key=times.get)
    L.lpb_tune_set(knob, grid.nx, grid.ny, grid.nz, best)
    _RESULTS[key] = {"best": best, "us": times}
    return _RESULTS[key]


def autotune(ge, reps=5):
    """Tune the fine applies (both precisions the hierarchy uses) and the level-1 apply of a
    GridElasticity whose hierarchy is built (after set_moduli). Returns {knob: result}."""
    if not ge.levels:
        raise RuntimeError("autotune needs a built hierarchy (call set_moduli first)")
    out = {}
    L = lib()
    st = stream_handle()
    g = ge.g0
    l0 = ge.levels[0]
    # inputs: random fields with the held dofs zeroed (the applies' precondition)
    raw = g.node_field(torch.float64).normal_()
    u64, o64 = g.node_field(torch.float64), g.node_field(torch.float64)
    L.lpb_mask_field_f64(u64.data_ptr(), raw.data_ptr(), l0.mask.data_ptr(), *g.args, 0, st)
    out["fine_f64"] = _tune_one("fine_f64", g, lambda: l0.apply(o64, u64), 2, reps)
    if ge._l0s is not l0:
        s = ge._l0s
        u32, o32 = u64.float(), g.node_field(torch.float32)
        out["fine_f32"] = _tune_one("fine_f32", g, lambda: s.apply(o32, u32), 2, reps)
    if len(ge.levels) > 1 and ge.levels[1].kind == "weights" and getattr(ge.levels[1], "wc", None) is not None:
        l1 = ge.levels[1]
        g1 = l1.grid
        dt = l1.dtype
        sfx = "f32" if dt == torch.float32 else "f64"
        raw1 = g1.node_field(dt).normal_()
        u1, o1 = g1.node_field(dt), g1.node_field(dt)
        getattr(L, f"lpb_mask_field_{sfx}")(u1.data_ptr(), raw1.data_ptr(), l1.mask.data_ptr(), *g1.args, 0, st)
        out[f"level1_{sfx}"] = _tune_one(f"level1_{sfx}", g1, lambda: l1.apply(o1, u1), 1, reps)
    torch.cuda.synchronize()
    ge._gen += 1          # graphs captured before hold the old launch geometry: capture again
    return out


def tuned():
    """Every result of this process: {"knob nx ny nz": {"best": value, "us": {value: time}}}."""
    return {" ".join(map(str, k)): v for k, v in _RESULTS.items()}


def save(path):
    with open(path, "w") as fh:
        json.dump(tuned(), fh, indent=1)


def load(path):
    """Results saved by save(); they take effect for grids tuned again in this process (which
    then reuses them without timing)."""
    if not os.path.exists(path):
        return 0
    with open(path) as fh:
        d = json.load(fh)
    for k, v in d.items():
        name, nx, ny, nz = k.split()
        _RESULTS[(name, int(nx), int(ny), int(nz))] = {"best": int(v["best"]),
                                                         "us": {int(z): t for z, t in v["us"].items()}}
    return len(d)
