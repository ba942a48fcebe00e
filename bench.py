"""Benchmark: time to 1e-10 relative residual of the steady 3D heat-conduction
solve on the jittered Kuhn-tet mesh (64^3-node lattice, 1,500,282 cells,
Gaussian-random-field conductivity with contrast 1e3), mixed precision
(FP32 V-cycle under FP64 iterative refinement, FP64 coarsest direct solve)
against the plain FP64 GPU AMG, on the same GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference]

One step = one complete solve through the public API: init(), conductivity
and source from host arrays, advance() until the outer L1 residual ratio is
below 1e-10 (matrix assembly, AMG setup and every outer linearization
included), temperature read back to the host.

Printed: one JSON line (rank 0). `value` is the device time (CUDA events) of
advance() with the fields already resident; `e2e` the host wall clock of the
whole step through the API including host<->device copies. Under torchrun
each rank solves its own replica (the single-mesh solve does not shard:
replicas only, weak scaling) and times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to 1e-10 rel. residual: mixed+learned vs plain FP64 AMG, same B200"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}



def plan_name(p):
    """A level's smoother launch plan: "tpr/block" on SELL-32 levels, "ellW"
    (and "x2" with two rows per thread) on ELL-32 levels."""
    if p[0] < 0:
        return "ell%d" % -p[0] + ("x%d" % -p[1] if p[1] < -1 else "")
    return "%d/%d" % p

def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ---------------------------------------------------------------------------
# distributed plumbing (torchrun), kept optional for N=1


# dram__bytes_read.sum + dram__bytes_write.sum over the algorithmic bytes of
# the finest-level FP32 GS colour launches in an ncu capture of the workload
# (24.69 MB for a 502k-row colour of 24.10 MB algorithmic)
NCU_TRAFFIC_RATIO = {"config1": 24.69 / 24.10}


def Dist():
    from fvm_b200.replicas import Ranks

    return Ranks()


# ---------------------------------------------------------------------------


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# workload


def make_workload(name: str):
    """(mesh, fields, description, generator of other draws by seed)."""
    from fvm_b200 import meshgen

    if name == "config1":
        gen = lambda seed: meshgen.config1(m=64, seed=seed)  # noqa: E731
        desc = "steady 3D heat conduction, Kuhn tets of a jittered 64^3-node lattice"
        seed = 1
    elif name == "config1-small":
        gen = lambda seed: meshgen.config1(m=24, seed=seed)  # noqa: E731
        desc = "steady 3D heat conduction, Kuhn tets of a jittered 24^3-node lattice"
        seed = 1
    elif name == "config0":
        gen = lambda seed: meshgen.config0(n=256, seed=seed)  # noqa: E731
        desc = "steady 2D heat conduction, jittered 256^2 quads"
        seed = 0
    elif name == "config3":
        gen = lambda seed: meshgen.config3(n=100, seed=seed)  # noqa: E731
        desc = ("steady 3D heat conduction, 100^3 hexes, two-phase: k = 1e4 in random spheres "
                "(r 0.02-0.08, 30% volume), 1 outside")
        seed = 3
    elif name == "config4":
        gen = lambda seed: meshgen.config4(n=200, seed=seed)  # noqa: E731
        desc = ("implicit transient 3D heat conduction, 200^3 hexes, k ~ lognormal(0,1), rho c ~ U[0.5,2]: "
                "one backward-Euler step (dt = 1e-3) from T0 = 300 with x=1 held at 400")
        seed = 4
    else:
        raise SystemExit("unknown workload " + name)
    mesh, f = gen(seed)
    return mesh, f, desc, gen, seed


def train_learned(gen, inner_rel, seeds=(101, 102), n_outer=4, per_solve=3, steps=600, lr=1e-3):
    """Learned correction trained on the GPU (the library's own forward /
    backward kernels and Adam) on residuals harvested from plain-solver runs
    of other draws of the workload (other mesh jitter and conductivity
    seeds), with the residual objective |r + A d|^2 / |r|^2. Not timed: it
    is the offline training stage. The solve uses the network only when the
    residual reduction it reaches on its pairs pays for its cost."""
    from fvm_b200.learned import LearnedCorrection

    t0 = time.perf_counter()
    lc = LearnedCorrection(seed=0)
    lc.setObjective(LearnedCorrection.RESIDUAL)
    for seed in seeds:
        mesh, f = gen(seed)
        s = Solve(mesh, f, "plain", inner_rel)
        cells = s.m.getCells()
        s.tm.init()
        s.tf.conductivity[cells] = s.k
        s.tf.source[cells] = s.s
        if s.rc is not None:
            s.tf.specificHeat[cells] = s.rc
        lc.harvest(s.tm, nOuter=n_outer, perSolve=per_solve, relativeTolerance=1e-8, maxCycles=100)
        del s
    before = lc.evaluate()
    t1 = time.perf_counter()
    losses = lc.train(steps=steps, lr=lr, seed=0)  # returns after the device has finished
    train_s = time.perf_counter() - t1
    after = lc.evaluate()
    factor = lc.residualFactor()
    info = {"objective": "residual |r + A d|^2 / |r|^2", "pairs": lc.numPairs(), "instances": len(seeds),
            "train_steps": steps, "loss_before": before, "loss_after": after,
            "residual_factor": factor, "useful_factor": 0.5,
            "used_in_solve": bool(factor <= 0.5),
            "loss_first50": float(np.mean(losses[:50])), "loss_last50": float(np.mean(losses[-50:])),
            "dense_layers": "tcgen05 tf32" if lc.tensorCores else "fp32 cuda cores",
            "train_seconds": train_s, "ms_per_train_step": 1e3 * train_s / max(steps, 1),
            "seconds": time.perf_counter() - t0}
    return lc, info


def size_matched_copy_gbs(nbytes: float, reps: int = 7, launches: int = 1) -> float:
    """Bandwidth of plain device-to-device copies that move the same bytes
    as a kernel (nbytes/2 read + nbytes/2 written), CUDA events, L2 flushed
    before each repetition: what streaming reaches at this transfer size,
    launch and ramp included, beside the large-transfer peak. With
    launches > 1 the bytes are split into that many copies in a row, as a
    multicolour pass splits its rows into one launch per colour."""
    import torch

    n = max(1, int(nbytes // (16 * launches)))
    src = torch.ones(n * launches, dtype=torch.float64, device="cuda")
    dst = torch.empty_like(src)
    flush = torch.empty(64 << 20, dtype=torch.float64, device="cuda")
    # the copies are elementwise kernels (dst = src * 1) replayed as one
    # CUDA graph, so no host launch gap sits between them (as the solver's
    # own launches replay); a captured memcpy would run on a copy engine
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for q in range(launches):  # warm-up outside the capture
            torch.mul(src[q * n:(q + 1) * n], 1.0, out=dst[q * n:(q + 1) * n])
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for q in range(launches):
            torch.mul(src[q * n:(q + 1) * n], 1.0, out=dst[q * n:(q + 1) * n])
    times = []
    for r in range(reps + 2):
        flush.fill_(float(r))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        graph.replay()
        e1.record()
        e1.synchronize()
        if r >= 2:
            times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    del graph, src, dst, flush
    return 16.0 * n * launches / (ms * 1e-3) / 1e9


HOST_SETUP = False  # --host-setup: the mixed path on the reference's host aggregation
USE_GRAPHS = True   # --no-graphs: kernels launched one by one (for ncu launch lists)


# The mixed solver's outer loop per workload: (Anderson depth, inner CG
# relative tolerance). On the non-orthogonal tet meshes the outer
# (deferred-correction) iteration contracts by about 0.4 per step and mixing
# two earlier iterates cuts config 1 from 26 to 19 outer and from 114 to 87
# CG iterations; on the orthogonal hex meshes it converges in 8-10 steps and
# mixing does not pay, so those keep the reference's plain loop.
MIXED_OUTER = {"config1": (2, 0.05), "config1-small": (2, 0.05)}


def solver_for(variant: str, inner_rel: float, accel: int = 0):
    """plain: the reference's default solver on the GPU -- standalone FP64
    AMG, V(1,1), multicolour Gauss-Seidel, coarsest level <= 100 rows
    smoothed. plain-cg: CG preconditioned by that AMG (FP64). mixed /
    learned: CG preconditioned by the FP32 V-cycle (FP64 refinement by the
    CG, FP64 dense inverse on the coarsest level <= 4096 rows, damped Jacobi
    below the finest level, V(0,2): no pre-smoothing, two post-sweeps, as
    the reference's AMG default V(0,1) with one more sweep)."""
    from fvm_b200 import fvmbaseExt

    amg = fvmbaseExt.AMG()
    amg.nPreSweeps = 1
    amg.nPostSweeps = 1
    amg.coarsestSize = 100
    amg.relativeTolerance = inner_rel
    amg.nMaxIterations = 200
    amg.useGraphs = USE_GRAPHS
    if variant in ("mixed", "learned", "mixed-plain-outer"):
        amg.setupOnDevice = not HOST_SETUP
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 4096
        amg.coarseJacobiRows = 1 << 30
        amg.jacobiWeight = 2.0 / 3.0
        amg.nPreSweeps = 0
        amg.nPostSweeps = 2
        if not HOST_SETUP:
            # GPU-built levels: pairs of pairs (aggregates of about 4 rows)
            # of neighbours at least half as strong as a row's strongest,
            # one damped-Jacobi sweep on each level below the finest
            amg.matchPasses = 2
            amg.matchBeta = 0.5
            amg.coarsePostSweeps = 1
    if variant in ("mixed", "learned", "mixed-plain-outer"):
        amg.outerAcceleration = accel
    if variant in ("plain-cg", "mixed", "learned", "mixed-plain-outer"):
        cg = fvmbaseExt.CG()
        cg.preconditioner = amg
        cg.relativeTolerance = inner_rel
        cg.nMaxIterations = 200
        return cg
    return amg


class Solve:
    """One model reused across steps; each step is a full solve from T0."""

    def __init__(self, mesh, fields, variant, inner_rel, outer_rel=1e-10, max_outer=500, accel=0):
        from fvm_b200 import fvmbaseExt, models

        self.mesh_d = mesh
        self.fields = fields
        self.m = fvmbaseExt.Mesh.from_dict(mesh)
        self.tf = models.ThermalFields("therm")
        self.tm = models.ThermalModelA(models.GeomFields("geom"), self.tf, [self.m])
        for gid, (kind, val) in fields["bc"].items():
            bc = self.tm.getBCMap()[gid]
            bc.bcType = "SpecifiedTemperature" if kind == "T" else "SpecifiedHeatFlux"
            bc.setVar("specifiedTemperature" if kind == "T" else "specifiedHeatFlux", val)
        o = self.tm.getOptions()
        o.linearSolver = solver_for(variant, inner_rel, accel)
        o.relativeTolerance = outer_rel
        self.rc = None
        if "rc" in fields:  # transient: one backward-Euler step from T0 per bench step
            o.transient = True
            o["timeStep"] = 1e-3
            o["initialTemperature"] = 300.0
            self.rc = np.ascontiguousarray(fields["rc"])
        self.max_outer = max_outer
        self.k = np.ascontiguousarray(fields["k"])
        self.s = np.ascontiguousarray(fields["s"])

    def step(self):
        """Returns (device seconds of advance, host wall seconds of the whole
        step, report, temperature, h2d bytes, d2h bytes)."""
        cells = self.m.getCells()
        t0 = time.perf_counter()
        self.tm.init()
        self.tf.conductivity[cells] = self.k
        self.tf.source[cells] = self.s
        if self.rc is not None:
            self.tf.specificHeat[cells] = self.rc
        rep = self.tm.advance(self.max_outer)
        T = self.tf.temperature[cells]
        t1 = time.perf_counter()
        n_all = cells.getCount()
        h2d = 8 * (3 if self.rc is None else 4) * n_all  # T (initial), k, source (, rho c)
        d2h = 8 * n_all
        return rep.seconds, t1 - t0, rep, T, h2d, d2h


# ---------------------------------------------------------------------------


REF_CACHE = os.path.join(ROOT, ".ref_cache")


def _host_cpu():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_solve(workload, seed, mesh, fields, inner_rel, use_cache=True):
    """One complete solve by the reference itself (oracle/_ref: its own
    ThermalModel<double> + AMG sources, -O3, one thread -- the reference is
    single-threaded) on the same mesh and fields: init, fields, advance()
    until the outer L1 ratio is below 1e-10, with the reference's default
    solver (AMG, 1 pre + 1 post Gauss-Seidel sweep, lexicographic order,
    inner relTol `inner_rel`). Returns the measured wall time of advance(),
    the reference's own outer-iteration count and the converged field.

    The result is cached (.ref_cache/, not part of the source tree) keyed by
    workload, seed and cell count, so that the product arm of the same run
    states its fields' error against this solve without solving again."""
    from oracle import ref
    from fvm_b200.meshgen import extend_to_ghosts

    n = mesh["nCells"]
    path = os.path.join(REF_CACHE, "%s_seed%d_n%d_rel%g.npz" % (workload, seed, n, inner_rel))
    if use_cache and os.path.exists(path):
        z = np.load(path, allow_pickle=False)
        return {"T": z["T"], "seconds": float(z["seconds"]), "outer": int(z["outer"]), "ratio": float(z["ratio"]),
                "cpu": str(z["cpu"]), "cached": True}
    if not ref.available():
        return None
    r = ref.RefThermal(mesh)
    extra = {"transient": True, "dt": 1e-3} if "rc" in fields else {}
    r.set_options(n_pre=1, n_post=1, max_iter=200, lin_rel=inner_rel, rel=1e-10, **extra)
    for gid, (kind, val) in fields["bc"].items():
        r.set_bc(gid, 0 if kind == "T" else 1, [val] if kind == "T" else [None, val])
    r.init()
    r.set_field(1, extend_to_ghosts(mesh, fields["k"]))
    r.set_field(2, extend_to_ghosts(mesh, fields["s"]))
    if "rc" in fields:
        r.set_field(3, extend_to_ghosts(mesh, fields["rc"]))
    norms, sec = r.advance(500)
    T = r.get_field(0)[:n].copy()
    out = {"T": T, "seconds": sec, "outer": int(len(norms)), "ratio": float(norms[-1] / norms[0]),
           "cpu": _host_cpu(), "cached": False}
    del r
    try:
        os.makedirs(REF_CACHE, exist_ok=True)
        np.savez(path, T=T, seconds=sec, outer=out["outer"], ratio=out["ratio"], cpu=out["cpu"])
    except OSError:
        pass
    return out


def reference_baseline(res, n_cells):
    """cpu_baseline entry of a measured reference solve."""
    return {"value": res["seconds"], "unit": "s", "cores": 1, "kind": "reference",
            "sample": ("one complete solve of the same %d-cell workload by the compiled reference "
                       "(ThermalModel<double> + AMG V(1,1), lexicographic Gauss-Seidel, one thread, host %s): "
                       "%d outer iterations to outer L1 ratio %.2e, wall time of advance() measured%s"
                       % (n_cells, res["cpu"], res["outer"], res["ratio"],
                          " by the reference arm of this run" if res.get("cached") else ""))}


def bench_batch(args, dist, peaks, peak_kind):
    """config 2: a batch of independent jittered quad meshes (sides
    U{32..256}) solved as one system, every mesh to outer relative residual
    1e-10 on its own norm. With N ranks each solves its share of the batch
    (greedy bin-packing by cells, no data-path exchange): strong scaling of
    a fixed batch, timed as the max over ranks."""
    from fvm_b200 import batch, meshgen
    from fvm_b200.replicas import shard_meshes

    ms_all = meshgen.config2(n_meshes=args.batch_meshes)
    n_cells_total = int(sum(m["nCells"] for m, _ in ms_all))
    ms = [ms_all[i] for i in shard_meshes([m["nCells"] for m, _ in ms_all], dist.world, dist.rank)]
    meshes = [m for m, _ in ms]
    ks = [f["k"] for _, f in ms]
    ss = [f["s"] for _, f in ms]
    n_cells = n_cells_total
    bcs = ms[0][1]["bc"]
    results = {}
    for variant in ("plain", "mixed"):
        bt = batch.BatchedThermal(meshes, bcs, solver_for(variant, args.inner_rel))
        for _ in range(args.warmup):
            bt.solve(ks, ss)
        dist.barrier()
        sampler = ClockSampler(dist.local)
        sampler.__enter__()
        dev_t, wall_t, rep = [], [], None
        for _ in range(args.steps):
            t0 = time.perf_counter()
            Ts, rep = bt.solve(ks, ss)
            wall_t.append(time.perf_counter() - t0)
            dev_t.append(rep.seconds)
        sampler.__exit__()
        dist.barrier()
        first, last, at = bt.status()
        n_all = bt.mesh.getCells().getCount()
        prof = bt.model.profile(args.profile_reps)
        plans = bt.model.getLaunchPlans()
        results[variant] = {"profile": prof, "plans": plans,
                            "dev": dist.max(statistics.median(dev_t)), "wall": dist.max(statistics.median(wall_t)),
                            "outer": rep.iterations, "cycles": rep.linearIterations, "setup": rep.setupSeconds,
                            "all_converged": bool(np.all(at >= 0)), "max_ratio": float(np.max(last / first)),
                            "T": np.concatenate(Ts), "launches": rep.launches, "clocks": sampler.summary(),
                            "h2d": 8 * 3 * n_all, "d2h": 8 * n_all}
        del bt
    plain, mixed = results["plain"], results["mixed"]
    peak = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    pm, pp = mixed["profile"], plain["profile"]

    def gbs(b, ms):
        return b / (ms * 1e-3) / 1e9

    roofline = {"bound": "hbm", "achieved": gbs(pm["gs_pass_bytes"], pm["gs_pass_ms"]), "peak": peak,
                "unit": "GB/s", "frac": gbs(pm["gs_pass_bytes"], pm["gs_pass_ms"]) / peak, "traffic": None,
                "kernel": "k_gs_color_ell<float> (one pass over all colours of the batch's finest level)",
                "peak_kind": peak_kind,
                "fp64_gs_pass": {"achieved": gbs(pp["gs_pass_bytes"], pp["gs_pass_ms"]),
                                 "frac": gbs(pp["gs_pass_bytes"], pp["gs_pass_ms"]) / peak},
                "fp64_residual": {"achieved": gbs(pp["residual_bytes"], pp["residual_ms"]),
                                  "frac": gbs(pp["residual_bytes"], pp["residual_ms"]) / peak}}
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_batch(ms, args.inner_rel)
    if dist.rank == 0:
        rel = float(np.linalg.norm(mixed["T"] - plain["T"]) / np.linalg.norm(plain["T"]))
        line = {
            "metric": METRIC, "value": mixed["dev"], "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mixed["dev"] * 1e3, "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32 V-cycle / f64 refinement", "data": "synthetic",
            "config": {"workload": "%d independent jittered quad meshes, sides U{32..256}, one batched solve"
                                   % len(ms_all), "cells": n_cells, "meshes": len(ms_all),
                       "parallelism": ("meshes sharded over %d ranks by cells, no exchange" % dist.world
                                       if dist.world > 1 else "single GPU"), "outer_rel": 1e-10,
                       "inner_rel": args.inner_rel, "convergence": "every mesh on its own L1 norm",
                       "l2": "working set > 126 MB L2"},
            "plain_fp64_s": plain["dev"], "speedup_vs_plain_fp64": plain["dev"] / mixed["dev"],
            "mixed_vs_plain_rel_l2": rel, "cells_per_s": n_cells / mixed["dev"] * args.gpus,
            "counts": {k: {"outer": v["outer"], "cycles": v["cycles"], "setup_s": v["setup"],
                           "all_meshes_converged": v["all_converged"], "max_mesh_ratio": v["max_ratio"]}
                       for k, v in results.items()},
            "gpu_launches": int(mixed["launches"]) * args.steps,
            "launch_plans": {v: [plan_name(p) for p in r["plans"]]
                             for v, r in results.items()},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": mixed["wall"], "unit": "s", "h2d_bytes_per_step": mixed["h2d"],
                    "d2h_bytes_per_step": mixed["d2h"]},
            "clocks": mixed["clocks"],
        }
        print(json.dumps(line))


def bench_transient(args, dist, peaks, peak_kind):
    """config 4 as stated: 200^3 hexes (8M cells), 50 backward-Euler steps
    (dt = 1e-3, updateTime between steps), every step solved to outer
    relative residual 1e-10. Arms, each a full 50-step run from T0 = 300:
    plain FP64 AMG (the reference's default solver on the GPU), mixed
    (CG + FP32 V-cycle), and mixed + learned, whose network is retrained on
    pairs harvested from the first 5 plain steps (an untimed stage). The
    AMG hierarchy is built on the first step and kept (the matrix does not
    change between steps). Times are device times of advance() per step."""
    from fvm_b200.learned import LearnedCorrection

    mesh, fields, desc, gen, seed = make_workload("config4")
    n_cells = mesh["nCells"]
    n_steps = args.time_steps

    def run(variant, lc=None, harvest=None):
        s = Solve(mesh, fields, variant, args.inner_rel)
        if lc is not None:
            s.tm.setLearnedCorrection(lc)
        cells = s.m.getCells()
        s.tm.init()
        s.tf.conductivity[cells] = s.k
        s.tf.source[cells] = s.s
        s.tf.specificHeat[cells] = s.rc
        per, outer, cycles, kept, tried = [], [], [], 0, 0
        t0 = time.perf_counter()
        for step in range(n_steps if harvest is None else harvest[1]):
            if harvest is not None:
                harvest[0].harvest(s.tm, nOuter=200, perSolve=3, relativeTolerance=1e-8, maxCycles=100)
            else:
                rep = s.tm.advance(200)
                rep = s.tm.lastReport()
                if not rep.converged:
                    raise RuntimeError("%s: step %d did not converge" % (variant, step))
                per.append(rep.seconds)
                outer.append(rep.iterations)
                cycles.append(rep.linearIterations)
                kept += rep.learnedAccepted
                tried += rep.learnedSteps
            s.tm.updateTime()
        wall = time.perf_counter() - t0
        T = s.tf.temperature[cells][:n_cells].copy()
        del s
        return {"per_step_s": per, "total_s": float(sum(per)), "outer": outer, "cycles": cycles,
                "learned_tried": tried, "learned_kept": kept, "wall_s": wall, "T": T}

    dist.barrier()
    sampler = ClockSampler(dist.local)
    sampler.__enter__()
    plain = run("plain")
    mixed = run("mixed")
    lc = LearnedCorrection(seed=0)
    t_train = time.perf_counter()
    run("plain", harvest=(lc, 5))
    pairs = lc.numPairs()
    losses = lc.train(steps=args.train_steps, lr=1e-3, seed=0)
    train_s = time.perf_counter() - t_train
    learned = run("learned", lc=lc)
    sampler.__exit__()
    dist.barrier()
    if dist.rank != 0:
        return
    rel = {k: float(np.linalg.norm(v["T"] - plain["T"]) / np.linalg.norm(plain["T"]))
           for k, v in (("mixed", mixed), ("mixed_learned", learned))}

    def summary(r):
        return {"total_s": r["total_s"], "first_step_s": r["per_step_s"][0],
                "mean_later_step_s": float(np.mean(r["per_step_s"][1:])) if len(r["per_step_s"]) > 1 else None,
                "step_ms": [round(1e3 * t, 2) for t in r["per_step_s"]],
                "outer_per_step": r["outer"], "cycles_per_step": r["cycles"],
                "learned_tried": r["learned_tried"], "learned_kept": r["learned_kept"]}

    cpu = None
    if dist.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_transient(mesh, fields, args.inner_rel, args.ref_time_steps)
    head = learned
    line = {
        "metric": METRIC, "value": head["total_s"], "unit": "s", "n_gpus": args.gpus, "steps": 1, "warmup": 0,
        "ms_per_step": head["total_s"] * 1e3 / max(n_steps, 1), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 V-cycle / f64 refinement", "data": "synthetic",
        "config": {"workload": desc.replace("one backward-Euler step (dt = 1e-3) from T0 = 300",
                                            "%d backward-Euler steps (dt = 1e-3) from T0 = 300" % n_steps),
                   "cells": n_cells, "time_steps": n_steps, "outer_rel": 1e-10, "inner_rel": args.inner_rel,
                   "value": "device time of all %d steps of the mixed + learned run" % n_steps},
        "plain_fp64_s": plain["total_s"], "mixed_without_learned_s": mixed["total_s"],
        "speedup_vs_plain_fp64": plain["total_s"] / head["total_s"],
        "field_rel_l2_vs_plain_after_last_step": rel,
        "arms": {"plain": summary(plain), "mixed": summary(mixed), "mixed_learned": summary(learned)},
        "learned_training": {"pairs": pairs, "from": "first 5 plain steps", "train_steps": args.train_steps,
                             "loss_first50": float(np.mean(losses[:50])), "loss_last50": float(np.mean(losses[-50:])),
                             "seconds": train_s},
        "cpu_baseline": cpu,
        "clocks": sampler.summary(),
    }
    print(json.dumps(line))


def bench_learned_protocol(args, dist, peaks, peak_kind):
    """Config 3's learned-correction protocol: 100^3 hexes, two-phase
    conductivity (k = 1e4 in random spheres of radius 0.02-0.08 filling 30 %
    of the volume, 1 outside), source U[0,1]. The network is trained on the
    GPU on (residual, error) pairs harvested from plain FP64 AMG runs of
    `--train-instances` seeded instances (seeds 1000, 1001, ...), with the
    residual objective, then evaluated on `--held-out` other seeds (5000,
    5001, ...) against plain FP64 AMG and against the mixed method without
    it. All instances share the mesh; each draws its own spheres and source.
    Arms per held-out seed, each one full solve to outer 1e-10: plain (the
    reference's default solver on the GPU), mixed (CG + FP32 V-cycle),
    mixed+learned as the product runs it (the network is used only when its
    measured residual reduction pays for its cost), and mixed+learned with
    the network forced on (every step that lowers the residual is kept),
    which shows what the network itself gains or costs."""
    from fvm_b200 import meshgen
    from fvm_b200.learned import LearnedCorrection

    mesh = meshgen.hex_mesh(100)
    n = mesh["nCells"]
    pts = meshgen.cell_centers(mesh)
    bc = {1: ("T", 300.0), 2: ("T", 400.0)}

    def draw(seed):
        return meshgen.sphere_inclusions(pts, seed + 100), meshgen.uniform_field(n, 0.0, 1.0, seed + 200)

    def set_fields(s, k, src):
        s.k, s.s = np.ascontiguousarray(k), np.ascontiguousarray(src)

    t0 = time.perf_counter()
    k0, s0 = draw(1000)
    lc = LearnedCorrection(seed=0)
    lc.setObjective(LearnedCorrection.RESIDUAL)
    harvester = Solve(mesh, {"k": k0, "s": s0, "bc": bc}, "plain", args.inner_rel)
    cells = harvester.m.getCells()
    per_solve = max(1, args.pairs_per_instance // 2)
    for i in range(args.train_instances):
        k, src = draw(1000 + i) if i else (k0, s0)
        set_fields(harvester, k, src)
        harvester.tm.init()
        harvester.tf.conductivity[cells] = harvester.k
        harvester.tf.source[cells] = harvester.s
        lc.harvest(harvester.tm, nOuter=2, perSolve=per_solve, relativeTolerance=1e-8, maxCycles=100)
    del harvester
    harvest_s = time.perf_counter() - t0
    before = lc.evaluate()
    t1 = time.perf_counter()
    losses = lc.train(steps=args.train_steps, lr=1e-3, seed=0)
    train_s = time.perf_counter() - t1
    after = lc.evaluate()
    factor = lc.residualFactor()
    forced = LearnedCorrection(seed=0)
    forced.setParams(lc.getParams())
    forced.setUsefulFactor(1.0)

    arms = {"plain": Solve(mesh, {"k": k0, "s": s0, "bc": bc}, "plain", args.inner_rel),
            "mixed": Solve(mesh, {"k": k0, "s": s0, "bc": bc}, "mixed", args.inner_rel),
            "mixed_learned": Solve(mesh, {"k": k0, "s": s0, "bc": bc}, "learned", args.inner_rel),
            "mixed_learned_forced": Solve(mesh, {"k": k0, "s": s0, "bc": bc}, "learned", args.inner_rel)}
    arms["mixed_learned"].tm.setLearnedCorrection(lc)
    arms["mixed_learned_forced"].tm.setLearnedCorrection(forced)
    # warm-up on a training instance (setup caches, launch plans)
    for a in arms.values():
        if a is not arms["plain"]:
            a.step()
    res = {k: {"dev_s": [], "cycles": [], "outer": [], "learned_tried": 0, "learned_kept": 0} for k in arms}
    err = {k: [] for k in arms if k != "plain"}
    dist.barrier()
    sampler = ClockSampler(dist.local)
    if sampler:
        sampler.__enter__()
    for j in range(args.held_out):
        k, src = draw(5000 + j)
        T = {}
        for name, a in arms.items():
            set_fields(a, k, src)
            d, w, rep, Tn, _, _ = a.step()
            if not rep.converged:
                raise RuntimeError("%s: held-out seed %d did not converge" % (name, 5000 + j))
            r = res[name]
            r["dev_s"].append(d)
            r["cycles"].append(rep.linearIterations)
            r["outer"].append(rep.iterations)
            r["learned_tried"] += rep.learnedSteps
            r["learned_kept"] += rep.learnedAccepted
            T[name] = Tn[:n]
        for name in err:
            err[name].append(float(np.linalg.norm(T[name] - T["plain"]) / np.linalg.norm(T["plain"])))
    if sampler:
        sampler.__exit__()
    dist.barrier()
    if dist.rank != 0:
        return

    def mean(v):
        return float(np.mean(v))

    summary = {k: {"mean_dev_s": mean(r["dev_s"]), "mean_cycles": mean(r["cycles"]), "mean_outer": mean(r["outer"]),
                   "dev_s": r["dev_s"], "cycles": r["cycles"], "learned_tried": r["learned_tried"],
                   "learned_kept": r["learned_kept"]} for k, r in res.items()}
    head = summary["mixed_learned"]
    line = {
        "metric": METRIC, "value": head["mean_dev_s"], "unit": "s", "n_gpus": args.gpus, "steps": args.held_out,
        "warmup": 1, "ms_per_step": head["mean_dev_s"] * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 V-cycle / f64 refinement", "data": "synthetic",
        "config": {"workload": "config3 learned protocol: steady 3D heat conduction, 100^3 hexes, two-phase k = 1e4 "
                               "in random spheres (r 0.02-0.08, 30% volume), 1 outside",
                   "cells": n, "train_instances": args.train_instances,
                   "pairs_per_instance": 2 * per_solve, "held_out_seeds": args.held_out, "outer_rel": 1e-10,
                   "inner_rel": args.inner_rel,
                   "value": "mean device time of advance() over the held-out seeds, mixed + learned as the product "
                            "runs it",
                   "subsample": "the stated protocol is 200 instances, 20k pairs and 50 held-out seeds; 20k pairs of "
                                "1M-cell FP64 residual/error vectors are 320 GB, more than the GPU holds, so the pairs "
                                "and seeds here are a stated subsample"},
        "plain_fp64_s": summary["plain"]["mean_dev_s"], "mixed_without_learned_s": summary["mixed"]["mean_dev_s"],
        "speedup_vs_plain_fp64": summary["plain"]["mean_dev_s"] / head["mean_dev_s"],
        "forced_learned_vs_mixed": summary["mixed_learned_forced"]["mean_dev_s"] / summary["mixed"]["mean_dev_s"],
        "arms": summary,
        "field_rel_l2_vs_plain": {k: max(v) for k, v in err.items()},
        "learned_training": {"objective": "residual |r + A d|^2 / |r|^2", "pairs": lc.numPairs(),
                             "instances": args.train_instances, "train_steps": args.train_steps,
                             "loss_before": before, "loss_after": after, "residual_factor": factor,
                             "useful_factor": 0.5, "used_in_solve": bool(0 <= factor <= 0.5),
                             "loss_first50": mean(losses[:50]), "loss_last50": mean(losses[-50:]),
                             "harvest_seconds": harvest_s, "train_seconds": train_s},
        "clocks": sampler.summary() if sampler else None,
    }
    print(json.dumps(line))


def cpu_reference_transient(mesh, fields, inner_rel, n_steps):
    """The compiled reference (one thread) on the first n_steps backward-Euler
    steps of the same 8M-cell problem, each to outer 1e-10: a bounded sample
    of the 50-step run, stated as such."""
    from oracle import ref
    from fvm_b200.meshgen import extend_to_ghosts

    if not ref.available() or n_steps <= 0:
        return None
    r = ref.RefThermal(mesh)
    r.set_options(n_pre=1, n_post=1, max_iter=200, lin_rel=inner_rel, rel=1e-10, transient=True, dt=1e-3)
    for gid, (kind, val) in fields["bc"].items():
        r.set_bc(gid, 0 if kind == "T" else 1, [val] if kind == "T" else [None, val])
    r.init()
    r.set_field(1, extend_to_ghosts(mesh, fields["k"]))
    r.set_field(2, extend_to_ghosts(mesh, fields["s"]))
    r.set_field(3, extend_to_ghosts(mesh, fields["rc"]))
    secs = []
    for _ in range(n_steps):
        _, sec = r.advance(200)
        secs.append(sec)
        r.update_time()
    del r
    return {"value": float(sum(secs)), "unit": "s", "cores": 1, "kind": "reference",
            "sample": ("the compiled reference (ThermalModel<double> + AMG V(1,1), one thread, host %s) on the first "
                       "%d of the backward-Euler steps, each to outer 1e-10: %s s per step (a bounded sample of the "
                       "run)" % (_host_cpu(), n_steps, ", ".join("%.1f" % x for x in secs)))}


def cpu_reference_batch(ms, inner_rel, sample=6):
    """The reference solves each mesh with its own ThermalModel<double>
    (one core). Bounded sample: full solves (to 1e-10) of `sample` meshes
    spread over the size range; the batch time is extrapolated by cells."""
    from oracle import ref
    from fvm_b200.meshgen import extend_to_ghosts

    if not ref.available():
        return None
    order = sorted(range(len(ms)), key=lambda i: ms[i][0]["nCells"])
    pick = [order[int(q * (len(order) - 1) / (sample - 1))] for q in range(sample)]
    t_sum, c_sum = 0.0, 0
    for i in pick:
        mesh, f = ms[i]
        r = ref.RefThermal(mesh)
        r.set_options(n_pre=1, n_post=1, max_iter=200, lin_rel=inner_rel, rel=1e-10)
        for gid, (kind, val) in f["bc"].items():
            r.set_bc(gid, 0 if kind == "T" else 1, [val] if kind == "T" else [None, val])
        r.init()
        r.set_field(1, extend_to_ghosts(mesh, f["k"]))
        r.set_field(2, extend_to_ghosts(mesh, f["s"]))
        _, sec = r.advance(500)
        t_sum += sec
        c_sum += mesh["nCells"]
        del r
    total_cells = sum(m["nCells"] for m, _ in ms)
    est = t_sum / c_sum * total_cells
    return {"value": est, "unit": "s", "cores": 1, "kind": "reference",
            "sample": ("reference ThermalModel<double>+AMG per mesh (1 pre/1 post GS): full solves to 1e-10 of %d "
                       "meshes (%d cells, %.2f s), extrapolated by cells to the %d-mesh batch (%d cells)"
                       % (len(pick), c_sum, t_sum, len(ms), total_cells))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--workload", default="config1")
    ap.add_argument("--inner-rel", type=float, default=1e-1,
                    help="inner AMG relative tolerance (ThermalModel default 0.1)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-reps", type=int, default=5)
    ap.add_argument("--variants", default="plain,plain-cg,mixed,learned",
                    help="comma list of plain, plain-cg, mixed, learned (mixed + learned correction)")
    ap.add_argument("--train-steps", type=int, default=600)
    ap.add_argument("--batch-meshes", type=int, default=512, help="config2: number of meshes")
    ap.add_argument("--time-steps", type=int, default=50, help="config4: backward-Euler steps")
    ap.add_argument("--ref-time-steps", type=int, default=1,
                    help="config4: steps of the CPU reference sample")
    ap.add_argument("--learned-protocol", action="store_true",
                    help="config3: train the learned correction on --train-instances seeded instances and evaluate "
                         "it on --held-out other seeds")
    ap.add_argument("--train-instances", type=int, default=100)
    ap.add_argument("--pairs-per-instance", type=int, default=10)
    ap.add_argument("--held-out", type=int, default=10)
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch every kernel on its own instead of replaying CUDA graphs (ncu does not profile the "
                         "kernels of a graph with conditional nodes, which the CG solves use)")
    ap.add_argument("--outer-accel", type=int, default=None,
                    help="mixed solver: Anderson depth of the outer iteration (default per workload: 2 on the tet "
                         "meshes, 0 elsewhere)")
    ap.add_argument("--mixed-inner-rel", type=float, default=None,
                    help="mixed solver: inner CG relative tolerance (default per workload: 0.05 with the outer "
                         "acceleration, else --inner-rel)")
    ap.add_argument("--host-setup", action="store_true",
                    help="mixed path: AMG levels by the reference's greedy aggregation on the host instead of the "
                         "GPU-built hierarchy")
    args = ap.parse_args()
    global HOST_SETUP, USE_GRAPHS
    HOST_SETUP = args.host_setup
    USE_GRAPHS = not args.no_graphs

    dist = Dist()
    peaks, peak_kind = load_peaks()
    if args.workload == "config2" and args.impl == "product":
        bench_batch(args, dist, peaks, peak_kind)
        dist.close()
        return
    if args.workload == "config4" and args.impl == "product":
        bench_transient(args, dist, peaks, peak_kind)
        dist.close()
        return
    if args.workload == "config3" and args.learned_protocol and args.impl == "product":
        bench_learned_protocol(args, dist, peaks, peak_kind)
        dist.close()
        return
    if args.workload == "config2":
        if dist.rank == 0:
            from fvm_b200 import meshgen

            ms = meshgen.config2(n_meshes=args.batch_meshes)
            base = cpu_reference_batch(ms, args.inner_rel)
            if base is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfvmref.so not built"}))
            else:
                v = base["value"]
                print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "s",
                                  "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": v * 1e3,
                                  "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                                  "data": "synthetic", "config": {"workload": "config2 batch", "meshes": len(ms)},
                                  "cpu_baseline": base,
                                  "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        dist.close()
        return
    mesh, fields, desc, gen, seed = make_workload(args.workload)
    n_cells = mesh["nCells"]

    if args.impl == "reference":
        if dist.rank != 0:
            dist.close()
            return
        # One complete reference solve, measured (a full solve of the 1.5M-cell
        # workload takes about two minutes on one core, so the requested
        # --steps / --warmup are not repeated: `steps` reports the solves run).
        res = reference_solve(args.workload, seed, mesh, fields, args.inner_rel, use_cache=False)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfvmref.so not built"}))
            return
        v = res["seconds"]
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
                "steps": 1, "warmup": 0, "requested_steps": args.steps, "requested_warmup": args.warmup,
                "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": desc, "cells": n_cells, "solver": "AMG, 1 pre + 1 post GS sweep",
                           "inner_rel": args.inner_rel, "outer_rel": 1e-10},
                "outer_iterations": res["outer"], "final_outer_ratio": res["ratio"],
                "cpu_baseline": reference_baseline(res, n_cells),
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import ctypes  # noqa: F401

    results = {}
    variants = [v for v in args.variants.split(",") if v]
    accel, mixed_inner = MIXED_OUTER.get(args.workload, (0, args.inner_rel))
    if args.outer_accel is not None:
        accel = args.outer_accel
    if args.mixed_inner_rel is not None:
        mixed_inner = args.mixed_inner_rel
    if accel > 0 and "mixed" in variants and "plain" in variants and "mixed-plain-outer" not in variants:
        variants.insert(variants.index("mixed") + 1, "mixed-plain-outer")  # the same solver, plain outer loop
    lc, learned_info = None, None
    if "learned" in variants:
        try:
            lc, learned_info = train_learned(gen, args.inner_rel, steps=args.train_steps)
        except Exception as e:
            # the learned correction is an optional step of the mixed solve (it
            # is used only when its measured residual reduction pays); a failed
            # training is reported in the line and the mixed solve measured
            # without it
            lc, learned_info = None, {"failed": "%s: %s" % (type(e).__name__, e), "used_in_solve": False}
            variants = [v for v in variants if v != "learned"]
    for variant in variants:
        if variant in ("mixed", "learned"):
            solve = Solve(mesh, fields, variant, mixed_inner, accel=accel)
        else:
            solve = Solve(mesh, fields, variant, args.inner_rel)
        if variant == "learned":
            solve.tm.setLearnedCorrection(lc)
        for _ in range(args.warmup):
            solve.step()
        dev_t, wall_t, reps = [], [], []
        dist.barrier()
        sampler = ClockSampler(dist.local)
        if sampler:
            sampler.__enter__()
        T_last = None
        h2d = d2h = 0
        for _ in range(args.steps):
            d, w, rep, T, h2d, d2h = solve.step()
            dev_t.append(d)
            wall_t.append(w)
            reps.append(rep)
            T_last = T
        if sampler:
            sampler.__exit__()
        dist.barrier()
        prof = solve.tm.profile(args.profile_reps)
        plans = solve.tm.getLaunchPlans()
        results[variant] = {
            "dev": dist.max(statistics.median(dev_t)),
            "wall": dist.max(statistics.median(wall_t)),
            "outer": reps[-1].iterations,
            "cycles": reps[-1].linearIterations,
            "launches": reps[-1].launches,
            "learned_steps": reps[-1].learnedSteps,
            "learned_kept": reps[-1].learnedAccepted,
            "converged": bool(reps[-1].converged),
            "setup": reps[-1].setupSeconds,
            "T": T_last[:n_cells],
            "profile": prof,
            "plans": plans,
            "clocks": sampler.summary() if sampler else None,
            "h2d": h2d,
            "d2h": d2h,
        }
        del solve

    if "plain" not in results or "mixed" not in results:
        v = results[variants[0]]
        if dist.rank == 0:
            print(json.dumps({"partial": variants[0], "dev_s": v["dev"], "outer": v["outer"], "cycles": v["cycles"],
                              "profile": v["profile"]}))
        dist.close()
        return
    plain, mixed = results["plain"], results["mixed"]
    head = results.get("learned", mixed)  # the metric's mixed+learned solve
    rel_err = float(np.linalg.norm(head["T"] - plain["T"]) / np.linalg.norm(plain["T"]))

    # dominant kernel of the product path: the finest-level FP32 GS pass
    pm = mixed["profile"]
    gs_ms = pm["gs_pass_ms"]
    achieved = pm["gs_pass_bytes"] / (gs_ms * 1e-3) / 1e9
    peak = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    pp = plain["profile"]
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (NCU_TRAFFIC_RATIO[args.workload] * pm["gs_pass_bytes"]
                            if args.workload in NCU_TRAFFIC_RATIO else None),
                "traffic_note": ("ncu DRAM read+write of captured colour launches of this pass (caches cold before "
                                 "each launch) over their algorithmic bytes, %.3f, times the pass's algorithmic "
                                 "bytes" % NCU_TRAFFIC_RATIO[args.workload])
                if args.workload in NCU_TRAFFIC_RATIO else None,
                "kernel": "k_gs_color_ell%s<float, W> (one pass over all colours of the finest level, the autotuned "
                          "plan: %s)" % ("2" if mixed["plans"][0][1] == -2 else "",
                                         plan_name(mixed["plans"][0])),
                "peak_kind": peak_kind,
                "fp64_gs_pass": {"achieved": pp["gs_pass_bytes"] / (pp["gs_pass_ms"] * 1e-3) / 1e9,
                                 "frac": pp["gs_pass_bytes"] / (pp["gs_pass_ms"] * 1e-3) / 1e9 / peak},
                "fp64_residual": {"achieved": pp["residual_bytes"] / (pp["residual_ms"] * 1e-3) / 1e9,
                                  "frac": pp["residual_bytes"] / (pp["residual_ms"] * 1e-3) / 1e9 / peak},
                "whole_cycle": {"bytes": pm["cycle_bytes"], "ms": pm["cycle_ms"],
                                "achieved": pm["cycle_bytes"] / (pm["cycle_ms"] * 1e-3) / 1e9,
                                "frac": pm["cycle_bytes"] / (pm["cycle_ms"] * 1e-3) / 1e9 / peak,
                                "note": "algorithmic bytes of one FP32 cycle from a zero guess over its CUDA-event "
                                        "time after an L2 flush (coarse levels L2-resident within the cycle)"},
                "face_flux": {"bytes": pm["face_flux_bytes"], "ms": pm["face_flux_ms"],
                              "achieved": pm["face_flux_bytes"] / (pm["face_flux_ms"] * 1e-3) / 1e9,
                              "frac": pm["face_flux_bytes"] / (pm["face_flux_ms"] * 1e-3) / 1e9 / peak,
                              "note": "face loop of the linearization (k_face_flux), once per outer iteration"}}
    try:
        copy_gbs = dist.max(size_matched_copy_gbs(pp["residual_bytes"])) if dist.world == 1 else None
    except Exception:  # context only
        copy_gbs = None
    if copy_gbs:
        roofline["size_matched_copy"] = {
            "bytes": pp["residual_bytes"], "gbs": copy_gbs, "frac_of_peak": copy_gbs / peak,
            "fp64_residual_vs_copy": roofline["fp64_residual"]["achieved"] / copy_gbs,
            "fp64_gs_pass_vs_copy": roofline["fp64_gs_pass"]["achieved"] / copy_gbs}
        # the Gauss-Seidel pass is one launch per colour: copies of the same
        # bytes split into as many launches
        colors = int(pp.get("colors", 0))
        try:
            split_gbs = dist.max(size_matched_copy_gbs(pp["gs_pass_bytes"], launches=colors)) if colors > 1 else None
        except Exception:  # context only
            split_gbs = None
        if split_gbs:
            roofline["size_matched_copy"]["per_colour_copies"] = {
                "launches": colors, "bytes": pp["gs_pass_bytes"], "gbs": split_gbs,
                "fp64_gs_pass_vs_copies": roofline["fp64_gs_pass"]["achieved"] / split_gbs}

    # the reference's own FP64 solve of the same workload: the CPU baseline
    # and the oracle every field here is stated against (measured once per
    # run: cached by the reference arm, or solved now, after the timed work)
    cpu, vs_ref = None, {}
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            res = reference_solve(args.workload, seed, mesh, fields, args.inner_rel)
        except Exception as e:  # the baseline is reported, never required
            res = None
            cpu = {"value": None, "unit": "s", "cores": 1, "kind": "reference", "sample": "failed: %s" % e}
        if res is not None:
            cpu = reference_baseline(res, n_cells)
            Tr = res["T"]
            vs_ref = {"%s_vs_reference_rel_l2" % ("mixed_learned" if v == "learned" else v.replace("-", "_")):
                      float(np.linalg.norm(r["T"] - Tr) / np.linalg.norm(Tr)) for v, r in results.items()}

    if dist.rank == 0:
        line = {
            "metric": METRIC,
            "value": head["dev"],
            "unit": "s",
            "n_gpus": args.gpus,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": head["dev"] * 1e3,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 V-cycle / f64 refinement",
            "data": "synthetic",
            "config": {
                "workload": desc,
                "cells": n_cells,
                "solver": ("mixed+learned: flexible CG (FP64, fused iteration, each linear solve one CUDA graph) "
                           "preconditioned by an FP32 AMG V(0,2) on a hierarchy built on the GPU (pairs of pairs, "
                           "matchBeta 0.5) -- two multicolour GS sweeps on the finest level, one damped-Jacobi sweep "
                           "(w=2/3) below, "
                           "dense FP64 inverse (FP32 copy) on the coarsest level (<= 4096 rows) -- with the learned "
                           "post-correction of each preconditioner application when its measured residual reduction "
                           "pays; %s; plain: standalone FP64 AMG V(1,1) on the reference's aggregation, multicolour "
                           "GS on every level, coarsest <= 100 rows smoothed (the reference's default solver), the "
                           "reference's plain outer loop" % (
                               "outer iteration with Anderson acceleration of depth %d, inner CG to %g" % (
                                   accel, mixed_inner) if accel > 0 else
                               "the reference's plain outer loop, inner CG to %g" % mixed_inner)),
                "outer_rel": 1e-10,
                "inner_rel": args.inner_rel,
                "mixed_inner_rel": mixed_inner,
                "outer_acceleration": accel,
                "l2": "working set > 126 MB L2 (kernel timings flush L2 with a 512 MB write)",
                "parallelism": "replicas" if args.gpus > 1 else "single GPU",
            },
            "plain_fp64_s": plain["dev"],
            "plain_fp64_cg_s": results["plain-cg"]["dev"] if "plain-cg" in results else None,
            "mixed_without_learned_s": mixed["dev"],
            "mixed_plain_outer_s": results["mixed-plain-outer"]["dev"] if "mixed-plain-outer" in results else None,
            "speedup_vs_plain_fp64": plain["dev"] / head["dev"],
            "mixed_vs_plain_rel_l2": rel_err,
            "error_vs_reference": vs_ref or None,
            "cells_per_s": n_cells * head["outer"] / head["dev"] * args.gpus,
            "counts": {k: {"outer": v["outer"], "cycles": v["cycles"], "setup_s": v["setup"],
                           "learned_steps": v["learned_steps"], "learned_kept": v["learned_kept"]}
                       for k, v in results.items()},
            "learned_training": learned_info,
            "levels": int(pm["levels"]),
            "kernels_per_cycle": int(pm["kernels_per_cycle"]),
            "launch_plans": {v: [plan_name(p) for p in r["plans"]]
                             for v, r in results.items()},
            "kernel_timings": {
                v: {"gs_pass_ms": r["profile"]["gs_pass_ms"],
                    "gs_pass_gbs": r["profile"]["gs_pass_bytes"] / (r["profile"]["gs_pass_ms"] * 1e-3) / 1e9,
                    "residual_ms": r["profile"]["residual_ms"],
                    "residual_gbs": r["profile"]["residual_bytes"] / (r["profile"]["residual_ms"] * 1e-3) / 1e9,
                    "cycle_ms": r["profile"]["cycle_ms"], "kernels_per_cycle": int(r["profile"]["kernels_per_cycle"])}
                for v, r in results.items()},
            "gpu_launches": int(head["launches"]) * args.steps,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": head["wall"], "unit": "s", "h2d_bytes_per_step": head["h2d"],
                    "d2h_bytes_per_step": head["d2h"]},
            "clocks": head["clocks"],
        }
        print(json.dumps(line))
    dist.close()


if __name__ == "__main__":
    main()
