#!/usr/bin/env python
"""SIMP iterations per second at 256x128x128 hex8 (12.8M DOF) on B200, mixed precision,
with the plain FP64 GPU path and the K*u apply's HBM roofline beside it.

One step = one SIMP iteration of the plain top3d loop on the device, from the same seeded
design every step: SIMP law, Galerkin multigrid hierarchy build, MG-PCG solve to rtol 1e-6 from
zero, element energies, compliance and sensitivities, density-filter chain rule, OC bisection,
filtered densities and moduli of the new design. Each step does identical work whatever --steps
is (the solve takes the reference's 17 CG iterations on this design).
Workload (synthetic, seeded): cantilever with the x = 0 face held and a unit -z load spread over
the bottom edge at x = nx; density log-uniform in [1e-3, 1] (seed 1) smoothed by the r = 2 cone
filter (row-normalised); E0 = 1, Emin = 1e-9, nu = 0.3, p = 3, volume fraction 0.3, filter
r = 2, move 0.2, incompatible-mode hex8, 5-level hierarchy (coarse_cells 2000).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--evolve runs the loop instead (each step's design is the last step's output, warm-started
solves) and reports its CG counts; the designs of that loop sharpen into 1e9 stiffness contrasts
that the multigrid takes hundreds of CG iterations on (the reference's SIMP driver leaves the
multigrid past 60 CG iterations for a factorisation or AMG-CG, loadpath/simp.py:85, 735).

Multi-GPU: one process per GPU (torchrun); each rank runs its own replica of the workload
(the loop does not shard: replicas only), the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
DIMS = (256, 128, 128)
CASE_DIMS = (192, 96, 96)
FULL_DIMS = (384, 192, 192)
VOLFRAC, RMIN, RTOL, PENAL, EMIN, MOVE = 0.3, 2.0, 1e-6, 3.0, 1e-9, 0.2
METRIC = "SIMP iter/s & K*u GB/s at 12.7M DOF: mixed-prec vs FP64 GPU, <=1e-6 rel err"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--dims", default=",".join(str(d) for d in DIMS))
    p.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 GPU comparison")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--evolve", action="store_true",
                   help="step the evolving SIMP loop (each step from the last step's design, warm-started "
                        "solves) instead of the fixed-work iteration from the seeded design")
    p.add_argument("--micro", choices=["apply", "band", "cases", "full", "torchref", "optimize"], default=None,
                   help="apply: only the K*u microbenchmarks (fine level in both precisions, then the "
                        "level-1 weights operator; applies on seeded N(0,1) vectors); band: only the "
                        "coarsest level's band assembly, factorisation and inverse; cases: the batched "
                        "load-case SIMP iteration (8 point loads at 192x96x96 unless --dims is given), "
                        "the cases solved as one block and one after another; full: the full-scale MMA "
                        "SIMP run (384x192x192 unless --dims is given, --iters iterations) in mixed "
                        "precision and on the plain FP64 GPU path, final compliance and design compared; torchref: "
                        "the reference's own torch-CUDA multigrid (loadpath.gpu.TorchMG under "
                        "mg.GridElasticity(device='cuda'), from the copy installed in baseline/_ref) on the bench's "
                        "design: hierarchy build and one solve to rtol 1e-6, wall-clock, beside this package's; "
                        "optimize: loadpath's own SIMP loop (optimize.OptimizeLoop) and its stress-constrained "
                        "loop (optimize.ConstrainedLoop) on the bench's cantilever, --iters iterations each")
    p.add_argument("--iters", type=int, default=100, help="SIMP iterations of --micro full")
    p.add_argument("--reps", type=int, default=100)
    p.add_argument("--eager", action="store_true",
                   help="launch every kernel eagerly (no CUDA graphs, convergence tested on the host): the same "
                        "kernels in the same order, for profilers that do not follow graph launches")
    p.add_argument("--kernels", type=int, default=0, metavar="N",
                   help="device time per kernel over N SIMP iterations (after the warm-up), from the CUDA "
                        "activity trace (torch.profiler); a table, not the JSON line")
    a = p.parse_args()
    a.warmup = max(a.warmup, 3)
    if a.micro == "cases" and a.dims == ",".join(str(d) for d in DIMS):
        a.dims = CASE_DIMS
    if a.micro == "full" and a.dims == ",".join(str(d) for d in DIMS):
        a.dims = FULL_DIMS
    a.dims = tuple(int(v) for v in a.dims.split(",")) if isinstance(a.dims, str) else a.dims
    return a


def workload_config(dims, world, evolve=False):
    """The `config` both arms print: the bench workload and its sizes."""
    dof = 3 * math.prod(d + 1 for d in dims)
    if evolve:
        what = (f"evolving plain SIMP loop (warm-started solves), cantilever {'x'.join(map(str, dims))} hex8 "
                f"({dof} DOF), MG-PCG rtol {RTOL}, V-cycle float32, CG float64")
    else:
        what = (f"plain SIMP iteration from the seeded config-1 design (log-uniform density, seed 1, r=2 smoothed), "
                f"cantilever {'x'.join(map(str, dims))} hex8 ({dof} DOF): hierarchy build, MG-PCG from zero to rtol "
                f"{RTOL} (V-cycle float32, CG float64), sensitivities, filter chain rule, OC; same design every step")
    return {"workload": what, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (fields of 51-103 MB)"}


def cantilever(dims):
    nx, ny, nz = dims
    fixed = np.zeros((3, nx + 1, ny + 1, nz + 1), bool)
    fixed[:, 0] = True
    f = np.zeros((3, nx + 1, ny + 1, nz + 1))
    f[2, nx, :, 0] = -1.0 / (ny + 1)
    return fixed, f


def apply_bytes(dims, itemsize):
    """Algorithmic bytes of one fine K*u apply: read u, write K u (3 N values each), read E."""
    nx, ny, nz = dims
    n = (nx + 1) * (ny + 1) * (nz + 1)
    return 2 * 3 * n * itemsize + nx * ny * nz * itemsize


# the float32 fine apply's Chebyshev-update forms (lpb_apply_fine_cheb_f32), as extra node fields
# moved beyond the plain apply's u in / A u out: 1 reads b and dinv (u is d); 2 reads b and dinv
# and writes r and d; 3 reads x, r and dinv and writes x (u is d)
CHEB_FORMS = {"f32c1": 2, "f32c2": 3, "f32c3": 3}


def form_bytes(dims, form):
    """Algorithmic bytes of one float32 fine apply in the given form ("f32" plain, or a
    CHEB_FORMS key)."""
    nx, ny, nz = dims
    field = 3 * (nx + 1) * (ny + 1) * (nz + 1) * 4
    return apply_bytes(dims, 4) + CHEB_FORMS.get(form, 0) * field


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- clocks during the timed region ----------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [v.strip() for v in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- CPU baseline: the oracle's C port of the reference's two-pass CPU operator ---------------
def level1_apply(e, m, ke):
    """The C port's level-1 (weights) operator of the reference's hierarchy for cell moduli e and
    the fine mask m (x = 0 face held): the first Galerkin coarsening of the oracle (the children's
    moduli as weights, the cells touching held nodes as explicit patch matrices), its mask from
    its diagonal (loadpath/mg.py:601-677, :560-591), formed without the dense per-cell matrices."""
    from oracle import cport
    from oracle import ref_numpy as R

    dims = e.shape
    l0 = R.Level("scaled", dims, np.float64)
    l0.ke, l0.e, l0.mask = ke, e, m
    h = R.Hierarchy(ke, dims, m == 0, dtype=np.float32)
    h.alive = np.ones(m.shape, bool)
    l1 = h.coarsen(l0, first=True)
    dm = np.einsum("kii->ki", np.asarray(l1.mcat, np.float64).reshape(8, 24, 24))
    d = R.scatter_cells((dm.T @ l1.w.reshape(8, -1).astype(np.float64)).reshape((24,) + l1.dims),
                        np.zeros(l1.node_shape))
    if l1.patch_ijk is not None and len(l1.patch_ijk):
        np.add.at(d.reshape(-1), l1.patch_index().ravel(),
                  np.einsum("nii->ni", np.asarray(l1.patch_k, np.float64)).ravel())
    l1.mask = (d > 1e-12 * d.max()).astype(np.float32)
    return cport.WeightsApply(l1), l1.node_shape, l1.mask


def transfer_step(m, cm, rng):
    """One V-cycle's transfers between the fine level and level 1 in the C port: the restriction
    of the residual and the prolongation of the correction, on seeded fields."""
    from oracle import cport

    m32 = np.ascontiguousarray(m, np.float32)
    b, ax, x = (rng.standard_normal(m.shape).astype(np.float32) for _ in range(3))
    xc = rng.standard_normal(cm.shape).astype(np.float32)
    rc = np.empty(cm.shape, np.float32)

    def run():
        cport.coarse_residual(b, ax, m32, cm, rc)
        cport.add_correction(xc, cm, m32, x)
    return run


def cpu_apply_times(dims, reps64=3, reps32=3):
    """Seconds per fine-level apply (float64, float32) and per level-1 apply (float32) of the C
    port on all host cores."""
    from oracle import cport
    from oracle import ref_numpy as R

    nx, ny, nz = dims
    rng = np.random.default_rng(101)
    e = R.simp_moduli(np.exp(rng.uniform(np.log(1e-3), 0.0, dims)))
    m = np.ones((3, nx + 1, ny + 1, nz + 1))
    m[:, 0] = 0.0
    ke = R.hex8_ke(0.3, "im")
    u = rng.standard_normal(m.shape) * m
    out = {}
    for dt, reps in ((np.float64, reps64), (np.float32, reps32)):
        op = cport.MaskedApply(ke, e, m, dt)
        uu = u.astype(dt)
        o = np.empty_like(uu)
        op(uu, o)
        t0 = time.perf_counter()
        for _ in range(reps):
            op(uu, o)
        out[np.dtype(dt).name] = (time.perf_counter() - t0) / reps
    op1, shape1, cm = level1_apply(e, m, ke)
    u1 = rng.standard_normal(shape1).astype(np.float32)
    o1 = np.empty_like(u1)
    op1(u1, o1)
    t0 = time.perf_counter()
    for _ in range(reps32):
        op1(u1, o1)
    out["level1"] = (time.perf_counter() - t0) / reps32
    tr = transfer_step(m, cm, rng)
    tr()
    t0 = time.perf_counter()
    for _ in range(reps32):
        tr()
    out["transfers"] = (time.perf_counter() - t0) / reps32
    return out, cport.threads()


# CG iterations of the reference's own solve (loadpath/mg.py GridElasticity, float32 V-cycle,
# rtol 1e-6, from zero) on the bench's design at 256x128x128: C = 257.0077140996013 in 17
CG_REFERENCE_256 = 17
C_REFERENCE_256 = 257.0077140996013


def fine_applies(cg_iters):
    """Fine-level applies of SIMP iterations whose solves start from zero, averaged over
    iterations with these CG counts (loadpath/mg.py:872-926): float64 = one per CG iteration;
    float32 = four per V-cycle (one V-cycle before the loop and one after every iteration but
    the last) + 12 power iterations."""
    n = max(len(cg_iters), 1)
    n64 = sum(c for c in cg_iters) / n
    n32 = sum(12 + 4 * c for c in cg_iters) / n
    return int(round(n64)), int(round(n32))


def cpu_iteration_estimate(dims, n64, n32):
    t, cores = cpu_apply_times(dims)
    nv = (n32 - 12) // 4   # V-cycles (four float32 fine applies each besides the 12 power iterations)
    sec = n64 * t["float64"] + n32 * (t["float32"] + t["level1"]) + nv * t["transfers"]
    return {"value": 1.0 / sec, "unit": "SIMP iter/s", "cores": cores, "kind": "port",
            "sample": (f"C port of the reference's two-pass CPU operator (loadpath/mgops.py), of its level-1 "
                       f"operator and of its fine-level transfers on {cores} threads, 3 runs each: "
                       f"{t['float64'] * 1e3:.1f} ms per float64 and {t['float32'] * 1e3:.1f} ms per float32 "
                       f"fine-level apply, {t['level1'] * 1e3:.1f} ms per level-1 apply, "
                       f"{t['transfers'] * 1e3:.1f} ms per V-cycle's transfers at {dims[0]}x{dims[1]}x{dims[2]}, "
                       f"scaled to the {n64} float64 + {n32} float32 fine and {n32} level-1 applies and {nv} V-cycles "
                       "one SIMP iteration makes; deeper levels, vector passes, setup, filter and OC not counted "
                       "(a lower bound on the CPU iteration time)")}


def run_reference(args):
    """The reference arm: every fine-level and level-1 apply one SIMP iteration of the workload
    makes (its solve's float64 CG applies, float32 V-cycle and power-iteration applies on the fine
    level and as many on level 1) and its V-cycles' fine-level transfers, executed by the oracle's
    C port of the reference's CPU operators on all host cores, per step. Deeper levels, vector
    passes, setup, filter and OC are not run (a lower bound on the reference's CPU time)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import cport
    from oracle import ref_numpy as R

    dims = tuple(args.dims)
    n64, n32 = fine_applies((CG_REFERENCE_256,))
    nx, ny, nz = dims
    rng = np.random.default_rng(101)
    e = R.simp_moduli(R.log_uniform_density(dims, 1))
    m = np.ones((3, nx + 1, ny + 1, nz + 1))
    m[:, 0] = 0.0
    ke = R.hex8_ke(0.3, "im")
    u = rng.standard_normal(m.shape) * m
    ops = {}
    for dt in (np.float64, np.float32):
        op = cport.MaskedApply(ke, e, m, dt)
        uu = u.astype(dt)
        ops[dt] = (op, uu, np.empty_like(uu))
    op1, shape1, cm = level1_apply(e, m, ke)
    u1 = rng.standard_normal(shape1).astype(np.float32)
    o1 = np.empty_like(u1)
    tr = transfer_step(m, cm, rng)
    nv = (n32 - 12) // 4

    def step():
        for dt, n in ((np.float64, n64), (np.float32, n32)):
            op, uu, o = ops[dt]
            for _ in range(n):
                op(uu, o)
        for _ in range(n32):
            op1(u1, o1)
        for _ in range(nv):
            tr()

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    sec = (time.perf_counter() - t0) / args.steps
    v = 1.0 / sec
    cores = cport.threads()
    cb = {"value": v, "unit": "SIMP iter/s", "cores": cores, "kind": "port",
          "sample": (f"per step, the {n64} float64 + {n32} float32 fine-level applies, {n32} level-1 applies and "
                     f"the fine-level transfers of {nv} V-cycles one SIMP iteration of the workload makes "
                     f"({CG_REFERENCE_256} CG iterations, the reference's own count on this design), executed by the "
                     f"C port of the reference's CPU operators and transfers (loadpath/mgops.py, loadpath/mg.py) on "
                     f"{cores} threads at {nx}x{ny}x{nz}; deeper levels, vector passes, setup, filter and OC not run "
                     "(a lower bound on the CPU iteration time)")}
    line = {"metric": METRIC, "value": v, "unit": "SIMP iter/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": workload_config(dims, args.gpus, args.evolve),
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "SIMP iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- the B200 arm ---------------------------------------------------------------------------
def run_b200(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from loadpath_b200 import _lib, mg
    from loadpath_b200.grid import DevGrid
    from loadpath_b200.simp import DeviceFilter, Top3dLoop

    dims = args.dims
    fixed, f = cantilever(dims)
    # synthetic density: seeded log-uniform in [1e-3, 1], smoothed by the r = 2 cone filter
    g = DevGrid(dims)
    rng = np.random.default_rng(1)
    xr = g.cells_to_dev(np.exp(rng.uniform(np.log(1e-3), 0.0, dims)), torch.float64)
    flt = DeviceFilter(g, 2.0)
    x0 = flt.apply(g.cell_field(torch.float64), xr, hs_out=flt.hs)
    x0_host = g.cells_to_host(x0)
    del flt, xr

    def new_loop(dtype):
        return Top3dLoop(dims, VOLFRAC, RMIN, fixed, f, rtol=RTOL, dtype=dtype, x0=x0_host, penal=PENAL, emin=EMIN,
                         move=MOVE, element="im")

    def barrier():
        if world > 1:
            dist.barrier()

    def one_step(lp):
        # the fixed-work step starts every iteration from the seeded design (device copies and
        # the SIMP law, inside the timed region); --evolve steps the loop on
        if not args.evolve:
            lp.restart()
        return lp.step()

    # ---- device-resident timing -----------------------------------------------------------
    loop = new_loop(np.float32)
    if args.eager:
        loop.ge.use_graphs = False
        loop.ge.device_loop = False
    for _ in range(args.warmup):
        one_step(loop)
    barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.start()
    calls0 = _lib.launches()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    loop.timing = []
    torch.cuda.nvtx.range_push("timed")        # the region a profiler can be limited to
    t0.record()
    iters = []
    for _ in range(args.steps):
        one_step(loop)
        iters.append(loop.ge.last_iters)
    t1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    timing, loop.timing = loop.timing, None
    barrier()
    clocks = clk.stop()
    launches = _lib.launches() - calls0
    ms = t0.elapsed_time(t1)
    if world > 1:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * args.steps / (ms / 1e3)
    # the fine kernel's launch times: CUDA events around every fine-level apply over a second
    # pass of as many SIMP iterations, right after the timed one (events cannot sit inside the
    # device-side CG loop's graph, so this pass tests convergence on the host)
    probe = mg.FineApplyProbe()
    mg.set_probe(probe)
    for _ in range(args.steps):
        one_step(loop)
    mg.set_probe(None)
    fine = probe.summary()
    peak, peak_kind = peaks()
    roofline = None
    forms = [f for f in ("f32",) + tuple(CHEB_FORMS) if fine[f + "_count"]]
    if forms:
        # every float32 fine launch (the plain apply and its Chebyshev-update forms): their
        # algorithmic bytes over their event time
        count = sum(fine[f + "_count"] for f in forms)
        sec = sum(fine[f + "_ms"] for f in forms) / 1e3
        nbytes = sum(form_bytes(dims, f) * fine[f + "_count"] for f in forms)
        avg = sec / count
        achieved = nbytes / sec / 1e9
        traffic = None
        prof = os.path.join(ROOT, "profiles", "fine_apply_f32_traffic.json")
        if os.path.exists(prof):
            with open(prof) as fh:
                pd = json.load(fh)
            per = pd.get("forms", {})
            if tuple(pd.get("dims", ())) == tuple(dims) and all(f in per for f in forms):
                traffic = sum(per[f] * fine[f + "_count"] for f in forms) / count
        by_form = {f: {"launches": fine[f + "_count"], "avg_us": fine[f + "_ms"] / fine[f + "_count"] * 1e3,
                       "algorithmic_bytes": form_bytes(dims, f),
                       "GBps": form_bytes(dims, f) / (fine[f + "_ms"] / fine[f + "_count"] / 1e3) / 1e9}
                   for f in forms}
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "kernel": "k_apply_fine<float> (plain A u and the Chebyshev-update "
                                              "forms f32c1..3)",
                    "algorithmic_bytes": nbytes / count, "avg_launch_us": avg * 1e6, "launches_timed": count,
                    "forms": by_form,
                    "timed_over": f"{args.steps} SIMP iterations after the timed region, CUDA events around "
                                  "each fine-level float32 apply on its stream",
                    "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs, burst copy)" if peak_kind == "measured"
                                    else "fallback (6.65 TB/s, a copy measured on B200)")}
    phases = np.array([[a.elapsed_time(b) for a, b in zip(ev[:-1], ev[1:])] for ev in timing])
    extra = {"cg_iterations": iters, "compliance": loop.history[args.warmup + args.steps - 1][0],
             "phase_ms_per_step": dict(zip(("hierarchy", "solve", "sensitivities", "oc"),
                                           np.round(phases.mean(axis=0), 3).tolist())),
             "fine_apply_f64_us": (fine["f64_ms"] / fine["f64_count"] * 1e3) if fine["f64_count"] else None,
             "fine_applies_per_step": dict(zip(("f64", "f32"), fine_applies(iters)))}
    del loop
    torch.cuda.empty_cache()

    # ---- accuracy and the plain FP64 GPU path ---------------------------------------------
    fp64 = None
    if not args.no_fp64:
        ref = new_loop(np.float64)
        mix = new_loop(np.float32)
        # the first design, solved three ways: mixed and plain FP64 at rtol 1e-6, and a tight
        # FP64 solve (rtol 1e-10) as the GPU oracle
        def first(lp, rtol):
            lp.ge.rtol = rtol
            lp.u = None
            lp.solve()
            lp.sensitivities()
            return float(lp._scal[8].item()), lp.u.clone(), lp.dcf.clone()

        c32, u32, dc32 = first(mix, RTOL)
        c64, _, _ = first(ref, RTOL)
        c_or, u_or, dc_or = first(ref, 1e-10)
        du = float((u32 - u_or).norm() / u_or.norm())
        dsens = float((dc32 - dc_or).norm() / dc_or.norm())
        del u32, dc32, u_or, dc_or
        ref.ge.rtol = RTOL
        for _ in range(args.warmup - 1):
            one_step(ref)
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record()
        it64 = []
        for _ in range(args.steps):
            one_step(ref)
            it64.append(ref.ge.last_iters)
        a1.record()
        torch.cuda.synchronize()
        v64 = args.steps / (a0.elapsed_time(a1) / 1e3)
        fp64 = {"value": v64, "unit": "SIMP iter/s", "mixed_over_fp64": value / world / v64, "cg_iterations": it64,
                "rel_err_vs_fp64_oracle": {"compliance": abs(c32 - c_or) / abs(c_or),
                                           "compliance_fp64_path": abs(c64 - c_or) / abs(c_or),
                                           "displacement": du, "sensitivity": dsens},
                "fp64_oracle_compliance": c_or, "mixed_compliance": c32}
        if tuple(dims) == DIMS:
            # the reference's own solve of this design (loadpath/mg.py GridElasticity on the CPU,
            # rtol 1e-6, 17 CG iterations)
            fp64["rel_diff_vs_reference_cpu_solve"] = {"mixed": abs(c32 - C_REFERENCE_256) / C_REFERENCE_256,
                                                       "fp64_oracle": abs(c_or - C_REFERENCE_256) / C_REFERENCE_256}
        del ref, mix
        torch.cuda.empty_cache()

    # ---- end to end through the host-facing step ----------------------------------------------
    e2e = None
    if not args.no_e2e:
        loop = new_loop(np.float32)
        x_host = torch.from_numpy(np.ascontiguousarray(x0_host)).pin_memory()
        out_host = torch.empty_like(x_host).pin_memory()
        # the same warm-up as the device-timed loop, so both time the same SIMP iterations; with
        # --evolve each step's output design is the next step's input (the pinned buffers swap
        # roles), else every step takes the seeded design in again
        for _ in range(args.warmup):
            loop.step_host(x_host, out_host, restart=not args.evolve)
            if args.evolve:
                x_host, out_host = out_host, x_host
        barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e2e_iters = []
        for _ in range(args.steps):
            c, _ = loop.step_host(x_host, out_host, restart=not args.evolve)
            e2e_iters.append(loop.ge.last_iters)
            if args.evolve:
                x_host, out_host = out_host, x_host
        torch.cuda.synchronize()
        w = time.perf_counter() - w0
        if world > 1:
            tt = torch.tensor([w], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            w = float(tt.item())
        nb = int(np.prod(dims)) * 8
        e2e = {"value": world * args.steps / w, "unit": "SIMP iter/s", "h2d_bytes_per_step": nb,
               "d2h_bytes_per_step": nb + 16, "cg_iterations": e2e_iters,
               "api": ("Top3dLoop.step_host: the design in from pinned host memory (restart: taken as its own "
                       "physical density), the updated design, compliance and change out"
                       if not args.evolve else
                       "Top3dLoop.step_host: design in from pinned host memory, updated design and compliance out")}
        del loop

    # ---- CPU baseline (rank 0, N = 1 only) -----------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        n64, n32 = fine_applies(iters)
        cpu = cpu_iteration_estimate(dims, n64, n32)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": "SIMP iter/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded log-uniform density smoothed by the r=2 filter; cantilever loads)",
            "config": workload_config(dims, world, args.evolve),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "fp64_gpu_path": fp64, "detail": extra}
    print(json.dumps(line))
    return 0


def time_cheb_forms(lv, u, m, dims, reps):
    """The three Chebyshev-update forms of the float32 fine apply on seeded fields (held dofs
    zero, as in the V-cycle), each warmed once and timed over reps launches."""
    import torch

    from loadpath_b200._lib import lib
    from loadpath_b200.grid import stream_handle

    L, st, gr = lib(), stream_handle(), lv.grid
    gen = torch.Generator(device="cuda").manual_seed(103)

    def fld():
        return (torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float32) * m).contiguous()

    x, r, b, dinv, d = fld(), fld(), fld(), fld().abs(), u.clone()
    coef = torch.tensor([0.0, 0.5, 0.3, 0.2] + [0.0] * 12, dtype=torch.float64, device="cuda")
    srcs = {1: d, 2: x, 3: d}
    res = {}
    for mode in (1, 2, 3):
        def call():
            L.lpb_apply_fine_cheb_f32(mode, x.data_ptr(), r.data_ptr(), d.data_ptr(), srcs[mode].data_ptr(),
                                      b.data_ptr(), dinv.data_ptr(), coef.data_ptr(), lv.e.data_ptr(),
                                      lv.mask.data_ptr(), lv.kmodal.ctypes.data, lv.err.data_ptr(), *gr.args, st)
        call()
        torch.cuda.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            call()
        e.record()
        torch.cuda.synchronize()
        us = a.elapsed_time(e) / reps * 1e3
        gbs = form_bytes(dims, f"f32c{mode}") / (us * 1e-6) / 1e9
        res[f"mode{mode}"] = {"us_per_apply": us, "GBps": gbs, "frac_of_peak": gbs / peaks()[0]}
    return res


def run_micro_apply(args):
    """args.reps fine-level applies (float32 and float64) on seeded N(0,1) vectors at the bench's
    density, timed with CUDA events; one JSON line."""
    import torch

    from loadpath_b200.grid import DevGrid
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from loadpath_b200.simp import DeviceFilter

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dims = args.dims
    g = DevGrid(dims)
    rng = np.random.default_rng(1)
    flt = DeviceFilter(g, 2.0)
    xr = g.cells_to_dev(np.exp(rng.uniform(np.log(1e-3), 0.0, dims)), torch.float64)
    x = flt.apply(g.cell_field(torch.float64), xr, hs_out=flt.hs)
    e = g.cell_field(torch.float64)
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import stream_handle

    lib().lpb_simp_law(e.data_ptr(), x.data_ptr(), PENAL, EMIN, *g.args, stream_handle())
    fixed, _ = cantilever(dims)
    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, coarse_cells=10 ** 12, element="im")
    ge.set_moduli_device(e)
    out = {}
    for lv in (ge._l0s, ge.levels[0]):
        gr = lv.grid
        m = torch.stack([((lv.mask >> c) & 1) for c in range(3)]).to(lv.dtype)
        u = torch.randn((3, gr.pz // 4, gr.NY, gr.NX, 4), generator=torch.Generator(device="cuda").manual_seed(101),
                        device="cuda", dtype=torch.float64).to(lv.dtype) * m
        o = gr.node_field(lv.dtype)
        for _ in range(3):
            lv.apply(o, u)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.reps):
            lv.apply(o, u)
        b.record()
        torch.cuda.synchronize()
        us = a.elapsed_time(b) / args.reps * 1e3
        isz = 4 if lv.dtype == torch.float32 else 8
        gbs = apply_bytes(dims, isz) / (us * 1e-6) / 1e9
        out["f32" if isz == 4 else "f64"] = {"us_per_apply": us, "GBps": gbs, "frac_of_peak": gbs / peaks()[0]}
        if isz == 4:
            out["f32_cheb_forms"] = time_cheb_forms(lv, u, m, dims, args.reps)
    ge.check_device()
    # the level-1 (weights) operator of the solver's own hierarchy, float32
    ge1 = GridElasticity(mesh, 0.3, fx, element="im")
    ge1.set_moduli_device(e)
    lv = ge1._op(1)
    if lv.kind == "weights":
        gr = lv.grid
        m = torch.stack([((lv.mask >> c) & 1) for c in range(3)]).to(lv.dtype)
        u = torch.randn((3, gr.pz // 4, gr.NY, gr.NX, 4), generator=torch.Generator(device="cuda").manual_seed(102),
                        device="cuda", dtype=torch.float64).to(lv.dtype) * m
        o = gr.node_field(lv.dtype)
        for _ in range(3):
            lv.apply(o, u)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.reps):
            lv.apply(o, u)
        b.record()
        torch.cuda.synchronize()
        us = a.elapsed_time(b) / args.reps * 1e3
        isz = 4 if lv.dtype == torch.float32 else 8
        nb = (2 * 3 * gr.NX * gr.NY * gr.NZ + 8 * gr.nx * gr.ny * gr.nz) * isz
        out["level1"] = {"dims": list(gr.cells), "us_per_apply": us, "GBps": nb / (us * 1e-6) / 1e9,
                         "patch_cells": int(lv.npatch)}
        ge1.check_device()
    print(json.dumps({"micro": "fine K*u apply", "dims": list(dims), "reps": args.reps, **out}))
    return 0


def run_micro_band(args):
    """args.reps rebuilds of the coarsest level's direct solve alone, on the main stream: the band
    assembly, the tiled Cholesky (k_band_factor) and the dense inverse (k_band_inverse), each timed
    with CUDA events; one JSON line."""
    import torch

    from loadpath_b200._lib import lib
    from loadpath_b200.grid import DevGrid, stream_handle
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from loadpath_b200.simp import DeviceFilter

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dims = args.dims
    g = DevGrid(dims)
    rng = np.random.default_rng(1)
    flt = DeviceFilter(g, 2.0)
    xr = g.cells_to_dev(np.exp(rng.uniform(np.log(1e-3), 0.0, dims)), torch.float64)
    x = flt.apply(g.cell_field(torch.float64), xr, hs_out=flt.hs)
    e = g.cell_field(torch.float64)
    L = lib()
    st = stream_handle()
    L.lpb_simp_law(e.data_ptr(), x.data_ptr(), PENAL, EMIN, *g.args, st)
    fixed, _ = cantilever(dims)
    mesh = BoxMesh(dims)
    fx = np.empty(mesh.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed[i].reshape(-1)
    ge = GridElasticity(mesh, 0.3, fx, element="im")
    ge.set_moduli_device(e)
    torch.cuda.synchronize()
    lv = ge.levels[-1]
    gr = lv.grid
    w = ge._work
    t, linv, sgn, info, bar, ainv = (w[k] for k in ("band_t", "band_linv", "band_sgn", "band_info", "band_bar",
                                                    "band_ainv"))
    sfx = "f32" if lv.dtype == torch.float32 else "f64"

    def ptr_or_none(a):
        return None if a is None else a.data_ptr()

    times = {"assemble": [], "factor": [], "inverse": []}
    for r in range(args.reps + 3):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        if lv.kind == "weights":
            getattr(L, f"lpb_coarse_band_{sfx}")(t.data_ptr(), 1, lv.w.data_ptr(), lv.mcat.data_ptr(),
                                                 ptr_or_none(lv.patch_id), ptr_or_none(lv.patch_k), None,
                                                 lv.mask.data_ptr(), *gr.args, st)
        else:
            getattr(L, f"lpb_coarse_band_{sfx}")(t.data_ptr(), 2, None, None, None, None, lv.k.data_ptr(),
                                                 lv.mask.data_ptr(), *gr.args, st)
        L.lpb_memset_async(info.data_ptr(), 0, 8, st)
        ev[1].record()
        L.lpb_band_factor(t.data_ptr(), linv.data_ptr(), sgn.data_ptr(), info.data_ptr(), bar.data_ptr(),
                          info[1:].data_ptr(),
                          *gr.args, st)
        ev[2].record()
        L.lpb_band_inverse(ainv.data_ptr(), t.data_ptr(), linv.data_ptr(), sgn.data_ptr(), *gr.args, st)
        ev[3].record()
        torch.cuda.synchronize()
        if r >= 3:
            for k, (a, b) in zip(times, zip(ev[:-1], ev[1:])):
                times[k].append(a.elapsed_time(b) * 1e3)
    status = [int(v) for v in info.cpu().numpy()]
    out = {k: float(np.median(v)) for k, v in times.items()}
    print(json.dumps({"micro": "coarsest direct solve rebuild", "dims": list(dims),
                      "coarsest_nodes": [gr.NX, gr.NY, gr.NZ], "reps": args.reps, "us": out, "status": status}))
    return 0


def case_loads(dims, k=8, seed=3):
    """k unit point forces at nodes (nx, j, kk) of the free face, j and kk from
    default_rng(seed).integers, each direction a normalised standard_normal(3)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        j, kk = int(rng.integers(0, dims[1] + 1)), int(rng.integers(0, dims[2] + 1))
        d = rng.standard_normal(3)
        f = np.zeros((3,) + tuple(n + 1 for n in dims))
        f[:, dims[0], j, kk] = d / np.linalg.norm(d)
        out.append(f)
    return out


def run_micro_cases(args):
    """The batched load-case SIMP iteration: 8 cases, x = 0 face held, uniform start at volume
    fraction 0.2, filter r = 2, mixed precision; SIMP iterations per second with the cases solved
    as one block of right-hand sides and one after another, CUDA-event timed."""
    import torch

    from loadpath_b200.simp import Top3dLoop

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dims = args.dims
    fixed, _ = cantilever(dims)
    loads = case_loads(dims)
    out = {}
    # the launch geometry is tuned once, before either run builds a hierarchy, so both runs make
    # the same launches from their first build on
    tuner = Top3dLoop(dims, 0.2, 2.0, fixed, loads, rtol=RTOL, dtype=np.float32, penal=PENAL, emin=EMIN,
                      move=MOVE, element="im")
    tuner._set_moduli()
    del tuner
    for block in (True, False):
        loop = Top3dLoop(dims, 0.2, 2.0, fixed, loads, rtol=RTOL, dtype=np.float32, penal=PENAL, emin=EMIN,
                         move=MOVE, element="im", block_cases=block)
        for _ in range(args.warmup):
            loop.step()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(args.steps):
            loop.step()
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / args.steps
        out["block" if block else "one_by_one"] = {
            "simp_iter_per_s": 1e3 / ms, "ms_per_step": ms,
            "cg_iterations": [list(map(int, h[2])) for h in loop.history[-args.steps:]],
            "compliance": [h[0] for h in loop.history[-args.steps:]]}
        del loop
        torch.cuda.empty_cache()
    same = out["block"]["compliance"] == out["one_by_one"]["compliance"]
    print(json.dumps({"micro": "load cases", "dims": list(dims), "cases": len(loads), "steps": args.steps,
                      "warmup": args.warmup, "dtype": "f32+f64", "data": "synthetic (seeded point loads)",
                      "block_over_one_by_one": out["block"]["simp_iter_per_s"] / out["one_by_one"]["simp_iter_per_s"],
                      "same_compliance_bits": same, **out}))
    return 0


def run_micro_full(args):
    """The full-scale SIMP run: cantilever, uniform start at volume fraction 0.25, filter r = 3,
    penalty ramped 1 -> 3 over 20 iterations, MMA, sensitivities from the autograd path; the same
    run in mixed precision (rtol 1e-6) and on the plain FP64 GPU path, CUDA-event timed, with the
    final compliance and filtered design compared."""
    import torch

    from loadpath_b200.optimize import MMALoop

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dims = args.dims
    fixed, f = cantilever(dims)
    out, designs = {}, {}
    for name, dtype in (("mixed", np.float32), ("fp64", np.float64)):
        loop = MMALoop(dims, 0.25, 3.0, fixed, f, penal=3.0, penal0=1.0, ramp=20, rtol=RTOL, dtype=dtype)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0.record()
        loop.run(args.iters)
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / args.iters
        h = loop.history
        out[name] = {"simp_iter_per_s": 1e3 / ms, "ms_per_iteration": ms, "final_compliance": h[-1][0],
                     "final_volume_fraction": h[-1][1], "final_change": h[-1][2],
                     "cg_iterations_total": int(sum(r[4] for r in h)), "levels": len(loop.problem.ge.levels),
                     "compliance_every_10": [h[i][0] for i in range(0, len(h), 10)]}
        designs[name] = loop.problem.xphys.clone()
        del loop
        torch.cuda.empty_cache()
    a, b = designs["mixed"], designs["fp64"]
    print(json.dumps({"micro": "full-scale MMA SIMP", "dims": list(dims), "iterations": args.iters,
                      "dtype": "f32+f64", "data": "synthetic (uniform start, cantilever)",
                      "mixed_over_fp64": out["mixed"]["simp_iter_per_s"] / out["fp64"]["simp_iter_per_s"],
                      "rel_err_vs_fp64_path": {
                          "compliance": abs(out["mixed"]["final_compliance"] - out["fp64"]["final_compliance"])
                          / abs(out["fp64"]["final_compliance"]),
                          "design_max_abs": float((a - b).abs().max()),
                          "design_l2": float((a - b).norm() / b.norm())}, **out}))
    return 0


def run_micro_optimize(args):
    """loadpath's own SIMP loop (default options: blueprint and eroded projections, live cells,
    measured step, Illinois volume step, beta continuation) and its minimum-mass loop under a
    stress and a deflection limit, on the bench's cantilever at the bench's size, mixed precision,
    solves to rtol 1e-6; CUDA-event timed over --iters iterations after one untimed."""
    import torch

    from loadpath_b200.optimize import ConstrainedLoop, Limits, OptimizeLoop, SimpOptions

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dims = args.dims
    fixed, f = cantilever(dims)
    out = {}
    opts = SimpOptions(volume_fraction=0.3, filter_radius=2.0, max_iterations=args.iters + 1, solve_rtol=RTOL)
    copts = SimpOptions(volume_fraction=0.5, filter_radius=2.0, max_iterations=args.iters + 1, solve_rtol=RTOL)
    for name, make in (("optimize", lambda: OptimizeLoop(dims, fixed, [f], 0.3, opts)),
                       ("constrained", lambda: ConstrainedLoop(dims, fixed, [f], 0.3, copts,
                                                               Limits(0.02, 0.5, 1000.0)))):
        loop = make()
        loop.step()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0.record()
        for _ in range(args.iters):
            loop.step()
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / args.iters
        h = loop.history
        out[name] = {"simp_iter_per_s": 1e3 / ms, "ms_per_iteration": ms,
                     "cg_iterations": [r["cgIterations"] for r in h],
                     "last": {k: v for k, v in h[-1].items() if k in ("compliance", "volume", "beta", "change",
                                                                       "constraints", "volumeSolves", "move")}}
        del loop
        torch.cuda.empty_cache()
    print(json.dumps({"micro": "loadpath SIMP loops", "dims": list(dims), "iterations": args.iters,
                      "dtype": "f32+f64", "data": "synthetic (uniform start, cantilever)", **out}))
    return 0


def run_micro_torchref(args):
    """The reference's own GPU path on the bench's design: loadpath.mg.GridElasticity with
    device='cuda' (its hierarchy built on the host by numba, then loaded into torch tensors; the
    solve is gpu.TorchMG.solve_mixed: float64 CG and operator on the device, float32 V-cycle, the
    coarsest level on the host), timed by wall clock (the path synchronises with the host every CG
    iteration), beside this package's hierarchy build + solve of the same design, CUDA-event timed.
    Needs the reference installed in baseline/_ref (pip install --target baseline/_ref); prints an
    `unavailable` line without it."""
    import torch

    ref_dir = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref_dir, "loadpath")):
        print(json.dumps({"micro": "reference torch-CUDA solve", "unavailable": "baseline/_ref holds no loadpath"}))
        return 0
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "lp_numba_cache"))
    sys.path.insert(0, ref_dir)
    from loadpath.fem import HexMesh
    from loadpath.mg import GridElasticity as RefGE

    from loadpath_b200.grid import DevGrid
    from loadpath_b200.mg import BoxMesh, GridElasticity
    from loadpath_b200.simp import case_compliance
    from oracle import ref_numpy as R

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dims = tuple(args.dims)
    x = R.log_uniform_density(dims, 1)
    e = R.simp_moduli(x)
    fixed_g, f_g = R.cantilever_bc(dims)
    mesh = HexMesh(np.argwhere(np.ones(dims, bool)), 1.0, np.zeros(3))
    fixed = fixed_g.transpose(1, 2, 3, 0).reshape(-1)
    f = f_g.transpose(1, 2, 3, 0).reshape(-1)
    out = {"micro": "reference torch-CUDA solve", "dims": list(dims), "rtol": RTOL}
    ref = RefGE(mesh, 0.3, fixed, rtol=RTOL, device="cuda")
    runs = []
    for _ in range(2):       # the first run includes numba compilation
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ref.set_moduli(e.reshape(-1))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        u = ref.solve_many([f])[0]
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        runs.append({"set_moduli_s": t1 - t0, "solve_s": t2 - t1, "cg_iterations": int(ref.last_iters),
                     "compliance": float(f @ u)})
    out["reference"] = dict(runs[-1], first_run=runs[0], levels=len(ref.levels),
                            host_threads=int(os.cpu_count() or 1))
    del ref, u
    torch.cuda.empty_cache()
    # this package on the same design
    bm = BoxMesh(dims)
    fx = np.empty(bm.n_dof, bool)
    for i in range(3):
        fx[i::3] = fixed_g[i].reshape(-1)
    ge = GridElasticity(bm, 0.3, fx, rtol=RTOL, element="im")
    dg = DevGrid(dims)
    ed = dg.cells_to_dev(e, torch.float64)
    b = dg.nodes_to_dev(f_g, torch.float64)
    res = []
    for _ in range(4):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        ge.set_moduli_device(ed)
        ev[1].record()
        ud = ge.solve_device(b)
        ev[2].record()
        torch.cuda.synchronize()
        res.append({"set_moduli_s": ev[0].elapsed_time(ev[1]) / 1e3, "solve_s": ev[1].elapsed_time(ev[2]) / 1e3,
                    "cg_iterations": int(ge.last_iters), "compliance": case_compliance(b, ud)})
    out["b200"] = res[-1]
    out["speedup"] = {"solve": out["reference"]["solve_s"] / res[-1]["solve_s"],
                      "build_and_solve": (out["reference"]["set_moduli_s"] + out["reference"]["solve_s"])
                      / (res[-1]["set_moduli_s"] + res[-1]["solve_s"])}
    print(json.dumps(out))
    return 0


def run_kernels(args):
    """Per-kernel device time of args.kernels SIMP iterations after args.warmup, from the CUDA
    activity records (CUPTI through torch.profiler: kernels are not serialised)."""
    import collections
    import re

    import torch
    from torch.profiler import ProfilerActivity, profile

    from loadpath_b200.grid import DevGrid
    from loadpath_b200.simp import DeviceFilter, Top3dLoop

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dims = args.dims
    fixed, f = cantilever(dims)
    g = DevGrid(dims)
    rng = np.random.default_rng(1)
    xr = g.cells_to_dev(np.exp(rng.uniform(np.log(1e-3), 0.0, dims)), torch.float64)
    flt = DeviceFilter(g, 2.0)
    x0 = g.cells_to_host(flt.apply(g.cell_field(torch.float64), xr, hs_out=flt.hs))
    loop = Top3dLoop(dims, VOLFRAC, RMIN, fixed, f, rtol=RTOL, dtype=np.float32, x0=x0, penal=PENAL, emin=EMIN,
                     move=MOVE, element="im")
    # the activity trace does not list kernels run inside a graph's conditional (WHILE) node,
    # so the table is taken with the host-tested CG loop: the same kernels in the same order
    loop.ge.device_loop = False
    def one_step():
        if not args.evolve:
            loop.restart()
        loop.step()

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(args.kernels):
            one_step()
        torch.cuda.synchronize()
    agg = collections.defaultdict(lambda: [0, 0.0])
    for ev in prof.events():
        if ev.device_type != torch.autograd.DeviceType.CUDA:
            continue
        name = re.sub(r"\(.*", "", ev.name.replace("(anonymous namespace)::", "").replace("<unnamed>::", ""))
        agg[name][0] += 1
        agg[name][1] += getattr(ev, "device_time_total", 0.0) or ev.cuda_time_total
    k = args.kernels
    tot = sum(v[1] for v in agg.values())
    print(f"{k} SIMP iterations after {args.warmup} warm-up at {dims[0]}x{dims[1]}x{dims[2]}: "
          f"CG iterations {[h[2] for h in loop.history[-k:]]} (all: {[h[2] for h in loop.history]}), "
          f"device time {tot / 1e3 / k:.3f} ms per iteration")
    print(f"{'ms/iter':>9} {'share':>7} {'launches/iter':>13} {'us/launch':>10}  kernel")
    for name, (c, t) in sorted(agg.items(), key=lambda kv: -kv[1][1]):
        if t / tot < 0.002:
            continue
        print(f"{t / 1e3 / k:9.3f} {100 * t / tot:6.2f}% {c / k:13.1f} {t / c:10.1f}  {name[:90]}")
    return 0


def main():
    args = parse()
    sys.path.insert(0, ROOT)
    if args.micro == "apply":
        return run_micro_apply(args)
    if args.micro == "band":
        return run_micro_band(args)
    if args.micro == "cases":
        return run_micro_cases(args)
    if args.micro == "full":
        return run_micro_full(args)
    if args.micro == "torchref":
        return run_micro_torchref(args)
    if args.micro == "optimize":
        return run_micro_optimize(args)
    if args.kernels:
        return run_kernels(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
