#!/usr/bin/env python
"""Benchmark: time to a 1e-10 relative composite residual of the FAC Poisson
solve on B200, with the smoother's achieved HBM bandwidth.

One step = one CellPoissonFACSolver::solveSystem of every problem of the
workload from a zero initial guess (u, f, D resident in HBM for ``value``;
host buffers with the copies inside the timed region for ``e2e``).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c5|c2|c1|c3] [--nprob P]

Multi-GPU (torchrun, one rank per GPU): nprob x N independent problems are
spread over the ranks by samrai_b200.parallel.partition (cell-balanced, about
nprob per rank: weak scaling, no data-path collective); the step time is the
maximum over ranks.

``--impl reference`` times the reference's own FAC solver on all host cores:
its C++ built from its sources with its Fortran kernels translated to C
(oracle/_ref, kind "reference"), or the oracle's restatement of it (kind
"port") where that build is absent.
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
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms to 1e-10 residual: mixed+learned vs plain FP64 FAC on B200; smoother GB/s"

# Solver settings of the benchmark stopping rule (plain variant = the
# reference's FAC semantics).  coarse_solver_tolerance is tightened from the
# reference default 1e-8, with which the plain solve stalls above the 1e-10
# relative target: the coarse red-black solve stops as soon as the last
# coarse patch's max residual is below it.  At 1e-300 every coarse solve runs
# its 500 sweeps.
PARAMS = dict(max_cycles=100, residual_tol=1e-300, relative_residual_tol=1e-10,
              pre_sweeps=2, post_sweeps=2, coarse_tol=1e-300, coarse_max_it=500, ewing=1)
# Fast variant: the same FAC cycle on the hierarchy extended by fully
# covered coarser levels (multigrid coarsest-level solve), with the sweep
# counts tuned for it on this workload (measured over pre/post sweeps 0..3
# and 10..60 coarsest-level sweeps): no pre-smoothing, 3 post-smoothing
# sweeps, 40 red-black sweeps on the coarsest extension level.
PARAMS_MG = dict(PARAMS, pre_sweeps=0, post_sweeps=3, coarse_max_it=40)
MG_LEVELS = {"c5": 3, "c2": 4, "c1": 3, "c3": 3}
# headline: FGMRES(KRYLOV) with one FAC cycle as the flexible preconditioner
KRYLOV = 20
# DRAM bytes per algorithmic byte of the FP32 staged colour pass, from one ncu
# capture of the pass on the finest level of 8 config-5 problems (67.2 MB read
# + write for 54.6 MB algorithmic on 2.48 M cells); traffic per launch is this
# times the launch's algorithmic bytes (scaling by cells processed)
STAGED_F32_TRAFFIC_RATIO = 67.2 / 54.6


def workload_desc(name, nprob):
    return {"c5": (f"config5: {nprob} independent 3-D variable-coefficient problems "
                   f"(3 levels, coarse 64^3..128^3, D=exp(g) contrast 1e3)"),
            "c2": "config2: 3-D 128^3 coarse + 2 random-box levels, f = 4 Gaussian bumps",
            "c3": "config3: 2-D 64^2 + 64^2 fine, D = exp(g) contrast 1e3",
            "c1": "config1: 2-D sine, 64^2 coarse + 64^2 fine box"}[name]


def workload_seeds(name, nprob, rank, world=1):
    """Seeds of this rank's problems.  Config 5: nprob x world problems
    (weak scaling: nprob per GPU) spread over the ranks by
    parallel.partition, longest first by coarse cells."""
    if name != "c5":
        return [rank]
    from samrai_b200 import configs, parallel
    seeds = list(range(nprob * world))
    return [seeds[i] for i in parallel.shard([configs.config5_cost(x) for x in seeds], rank,
                                             world)]


def make_workload(name, nprob, rank, world=1):
    from samrai_b200 import configs
    if name == "c5":
        probs = configs.config5(seeds=workload_seeds(name, nprob, rank, world))
    else:
        probs = [_make_problem(name, rank)]
    return probs, workload_desc(name, nprob)


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the
    timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = []
        with open(self.file.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        out.update(sm_mhz=statistics.median(sm) if sm else None,
                   sm_max_mhz=max(mx) if mx else None, reasons=sorted(reasons),
                   samples=len(rows))
        return out


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline (oracle = CPU restatement of the reference path)
# ---------------------------------------------------------------------------

# Plain FAC cycle counts of the config-5 problems to the 1e-10 relative
# residual (capped at max_cycles = 100), per seed.
PLAIN_CYCLES_FILE = os.path.join(ROOT, "oracle", "c5_plain_cycles.json")


def _make_problem(name, seed):
    from samrai_b200 import configs
    if name == "c5":
        return configs.config5_problem(seed)
    if name == "c2":
        return configs.config2(seed=2 + seed)
    if name == "c3":
        return configs.config3()
    return configs.config1()


def _ref_init(lib_path):
    """Pool initializer: every worker loads the timing build of the oracle
    (when the port is timed) and keeps numpy to one thread (one worker per
    core)."""
    sys.path.insert(0, ROOT)
    if lib_path:
        from oracle import oracle
        oracle.use_library(lib_path)
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(1)
    except ImportError:
        pass


def _ref_sample(job):
    """CPU seconds of one plain FAC cycle of one problem on one core.

    The plain cycle's coarsest solve runs exactly coarse_max_it red-black
    sweeps (tolerance 1e-300), each the same work, so the cycle is timed in
    parts: T(c cycles, m coarse sweeps) for (1, m0), (2, m0) and (1, m0 +
    sweeps); the cycle is T(2, m0) - T(1, m0) plus (coarse_max_it - m0) x
    one sweep, a sweep being (T(1, m0 + sweeps) - T(1, m0)) / sweeps.
    kind "reference" runs the reference's own CellPoissonFACSolver
    (oracle/_ref/fac_ref_driver, solveSystem timed inside; the reference
    needs m0 >= 1), kind "port" the oracle's restatement of it (m0 = 0)."""
    name, seed, sweeps, kind = job
    p = _make_problem(name, seed)
    m0 = 1 if kind == "reference" else 0

    def solve_seconds(cyc, m):
        prm = dict(PARAMS, max_cycles=cyc, coarse_max_it=m)
        if kind == "reference":
            from oracle.ref import refio
            return float(refio.run_reference(p, prm, solution=False)["seconds"][1])
        from oracle.oracle import Oracle
        o = Oracle(p, params=prm)
        t0 = time.perf_counter()
        o.solve()
        return time.perf_counter() - t0

    t_a = solve_seconds(1, m0)
    t_b = solve_seconds(2, m0)
    t_c = solve_seconds(1, m0 + sweeps)
    t_sweep = max(t_c - t_a, 0.0) / sweeps
    t_rest = max(t_b - t_a, 0.0)
    return {"seed": seed, "cells": p.num_cells(), "t_rest": t_rest, "t_sweep": t_sweep,
            "t_cycle": t_rest + (PARAMS["coarse_max_it"] - m0) * t_sweep}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def plain_cycles(name, seeds):
    """Cycle counts of the plain variant per seed: config 5 from the table
    measured by the plain FP64 path (its counts equal the oracle's cycle for
    cycle, by the parity tests); seeds missing from it get the table's mean.
    Returns (counts, number of seeds found in the table)."""
    table = {}
    if name == "c5" and os.path.exists(PLAIN_CYCLES_FILE):
        with open(PLAIN_CYCLES_FILE) as fh:
            table = {int(k): int(v) for k, v in json.load(fh)["cycles"].items()}
    mean = statistics.mean(table.values()) if table else 50.0
    return [table.get(s, mean) for s in seeds], sum(1 for s in seeds if s in table)


def lpt_makespan(costs, workers):
    """Wall time of independent jobs on `workers` processes, longest first."""
    import heapq
    heap = [0.0] * max(1, workers)
    for c in sorted(costs, reverse=True):
        heapq.heappush(heap, heapq.heappop(heap) + c)
    return max(heap)


CPU_KIND_TEXT = {
    "reference": "the reference's CellPoissonFACSolver built from its sources (g++ -O2 "
                 "-ffp-contract=off, Fortran kernels translated to C)",
    "port": "the oracle's C restatement of the reference FAC (gcc -O3 -march=native "
            "-ffp-contract=off)"}


class CpuReference:
    """Times the reference's plain FAC on the CPU -- its own solver built
    from its sources (oracle/_ref, g++ -O2) when present, else the oracle's
    restatement (timing build, gcc -O3 -march=native) -- one process per
    core, on samples of the workload, and turns them into the time to solve
    the whole workload on those cores."""

    def __init__(self, name, seeds, workers=None, sweeps=20):
        import multiprocessing as mp
        from oracle import oracle
        from oracle.ref import refio
        self.name, self.seeds, self.sweeps = name, list(seeds), sweeps
        self.workers = max(1, min(workers or host_cores(), len(self.seeds)))
        # the reference's own solver when its build is present, else the port
        self.kind = "reference" if refio.available() else "port"
        self.lib_path = oracle.build_timing() if self.kind == "port" else None
        self.pool = mp.get_context("spawn").Pool(self.workers, initializer=_ref_init,
                                                 initargs=(self.lib_path,))
        self.samples = {}
        self.next = 0

    def round(self, keep=True):
        """One sampling round: every worker times one cycle of the next
        problem in turn; returns the round's wall seconds."""
        jobs = []
        for _ in range(self.workers):
            jobs.append((self.name, self.seeds[self.next % len(self.seeds)], self.sweeps,
                         self.kind))
            self.next += 1
        t0 = time.perf_counter()
        res = self.pool.map(_ref_sample, jobs)
        wall = time.perf_counter() - t0
        if keep:
            for r in res:
                self.samples.setdefault(r["seed"], []).append(r)
        return wall

    def estimate(self, cells=None):
        """(ms to solve every problem, details): per problem the mean
        sampled cycle time times its plain cycle count; the problems spread
        over the worker processes longest first.  Problems without a sample
        (only when `cells`, seed -> cells, is given) take the sampled
        problems' seconds per cell times their cells."""
        tc = {x: statistics.mean(r["t_cycle"] for r in rs) for x, rs in self.samples.items()}
        per_cell = sum(tc.values()) / sum(rs[0]["cells"] for rs in self.samples.values())
        missing = [x for x in self.seeds if x not in tc]
        if missing and cells is None:
            raise RuntimeError(f"problems without a sample: {missing}")
        for x in missing:
            tc[x] = per_cell * cells[x]
        cyc, known = plain_cycles(self.name, self.seeds)
        costs = [tc[x] * c for x, c in zip(self.seeds, cyc)]
        ms = lpt_makespan(costs, self.workers) * 1e3
        return ms, {"problems": len(self.seeds), "sampled": len(self.samples),
                    "cycles_from_table": known,
                    "cycles_total": float(sum(cyc)), "core_seconds": round(sum(costs), 1),
                    "samples": sum(len(v) for v in self.samples.values())}

    def close(self):
        self.pool.close()
        self.pool.join()


def regrid_measure(ctx, probs, target=0.02):
    """The regrid step on the finest level of every problem after the
    solve: device tagging of the solution by the adaption estimate
    (fac_tag_gradient) and Berger-Rigoutsos clustering of each problem's
    tags within its level's bounding box (fac_cluster_tags_all: all
    problems' trees walked together, device histograms, host decisions;
    min box 4, efficiency 0.8, combine 0.8).
    The threshold is the one that tags about `target` of the cells (found
    by bisection before the timing).  Wall time of one tagging plus the
    clustering of every problem, synchronised."""
    from samrai_b200 import fac
    ln = ctx.nlev - 1
    cells = sum(int(np.prod(p.levels[-1].boxes[:, 3:] - p.levels[-1].boxes[:, :3] + 1, axis=1).sum())
                for p in probs)
    lo_t, hi_t = 0.0, 1.0
    while ctx.tag_gradient(fac.U, ln, hi_t).sum() > target * cells:
        hi_t *= 4.0
    for _ in range(24):
        mid = 0.5 * (lo_t + hi_t)
        if ctx.tag_gradient(fac.U, ln, mid).sum() > target * cells:
            lo_t = mid
        else:
            hi_t = mid
    thr = hi_t
    bounds = []
    for p in probs:
        b = p.levels[-1].boxes
        bounds.append([[int(b[:, 0].min()), int(b[:, 1].min()), int(b[:, 2].min()),
                        int(b[:, 3].max()), int(b[:, 4].max()), int(b[:, 5].max())]])
    ctx.tag_gradient(fac.U, ln, thr)  # warm-up
    ctx.cluster_tags_all(ln, bounds, (4, 4, 4))
    t0 = time.perf_counter()
    tags = ctx.tag_gradient(fac.U, ln, thr)
    nbox = sum(len(b) for b in ctx.cluster_tags_all(ln, bounds, (4, 4, 4)))
    ms = (time.perf_counter() - t0) * 1e3
    return {"ms": round(ms, 2), "level": "finest", "cells": cells, "tagged": int(tags.sum()),
            "boxes": nbox, "threshold": thr,
            "what": "fac_tag_gradient (AdaptivePoisson adaption estimate > threshold) and "
                    "fac_cluster_tags_all (Berger-Rigoutsos, min box 4, efficiency 0.8, "
                    "combine 0.8) of every problem's finest level, wall time"}


def cpu_small_solves(names=("c1", "c3")):
    """Full plain FAC solves of the small 2-D configurations on one core,
    measured, not scaled: the reference's own CellPoissonFACSolver
    (oracle/_ref, solveSystem timed inside the driver) when it is built,
    else the oracle's restatement.  Returns (kind, results)."""
    from oracle.ref import refio
    kind = "reference" if refio.available() else "port"
    out = {}
    for n in names:
        p = _make_problem(n, 0)
        if kind == "reference":
            r = refio.run_reference(p, dict(PARAMS), solution=False)
            ms = float(r["seconds"][1]) * 1e3
            its, ok = int(r["iterations"][0]), bool(r["converged"][0])
        else:
            from oracle.oracle import Oracle
            o = Oracle(p, params=dict(PARAMS))
            t0 = time.perf_counter()
            ok, its, res, _ = o.solve()
            ms = (time.perf_counter() - t0) * 1e3
        out[n] = {"cpu_ms": round(ms, 2), "cycles": int(its), "converged": bool(ok)}
    return kind, out


# ---------------------------------------------------------------------------
# main
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c5", choices=["c5", "c2", "c1", "c3"])
    ap.add_argument("--nprob", type=int, default=64)
    ap.add_argument("--plain-problems", type=int, default=64,
                    help="problems of the workload the plain variant is timed on")
    ap.add_argument("--plain-cycles-out", default=None, metavar="PATH",
                    help="write the plain variant's cycle count per seed to PATH (JSON)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-regrid", dest="regrid", action="store_false",
                    help="skip the regrid-step measurement (tagging and clustering)")
    ap.add_argument("--no-cnn", dest="cnn", action="store_false",
                    help="skip the learned part's training-throughput measurement")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="precision of the headline (multigrid-extended) variant")
    ap.add_argument("--smoother-only", type=int, default=0, metavar="SWEEPS",
                    help="only run SWEEPS red-black sweeps on the largest level (for ncu)")
    ap.add_argument("--krylov", type=int, default=KRYLOV,
                    help="FGMRES restart length of the headline solve (0: stationary FAC)")
    ap.add_argument("--cnn-only", type=int, default=0, metavar="BATCH",
                    help="only time training steps of the learned part's network on BATCH "
                         "samples (--steps of them, for kernel captures)")
    ap.add_argument("--cycles", type=int, default=0, metavar="N",
                    help="only run one solve of the headline variant stopped after N cycles "
                         "(a short, fixed launch sequence for kernel captures)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        return run_reference(args, world)

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))

    from samrai_b200 import configs, fac
    if args.cnn_only:
        from samrai_b200 import learned
        net = fac.CNN(max_batch=args.cnn_only, device=local_rank, seed=1)
        r = learned.training_throughput(net, batch=args.cnn_only, steps=max(1, args.steps),
                                        device=local_rank)
        net.close()
        print(json.dumps({"cnn_only": args.cnn_only, **r}), flush=True)
        return 0
    probs, desc = make_workload(args.config, args.nprob, rank, world)
    mg = [configs.extend_hierarchy(p, k=MG_LEVELS[args.config]) for p in probs]
    ctx = fac.FacContext(mg, params=PARAMS_MG, device=local_rank, precision=args.precision)
    ctx.set_krylov(args.krylov)
    cells = sum(p.num_cells() for p in probs)
    npatch = sum(p.num_patches() for p in probs)
    if args.smoother_only:
        # smoothing sweeps on the largest level only: a short, fixed launch
        # sequence for kernel captures
        k = MG_LEVELS[args.config]
        sizes = [sum(int(np.prod(b[3:] - b[:3] + 1)) for b in mg[0].levels[ln].boxes)
                 for ln in range(mg[0].nlev)]
        ln = int(np.argmax(sizes))
        for fid in (fac.E, fac.R):
            for ip in range(len(mg)):
                ctx.upload(fid, ip, ln, np.random.default_rng(ip).standard_normal(
                    ctx.size(fid, ip, ln)))
        ctx.timer_start()
        ctx.smooth(fac.E, fac.R, ln, args.smoother_only, -1.0)
        ms = ctx.timer_stop()
        print(json.dumps({"smoother_only": args.smoother_only, "level": ln, "cells": sizes[ln],
                          "ms": ms}), flush=True)
        ctx.close()
        return 0

    if args.cycles:
        ctx.close()
        ctx = fac.FacContext(mg, params=dict(PARAMS_MG, max_cycles=args.cycles),
                             device=local_rank, precision=args.precision)
        ctx.set_krylov(args.krylov)
        ctx.timer_start()
        conv, its, res = ctx.solve()
        ms = ctx.timer_stop()
        print(json.dumps({"cycles": args.cycles, "problems": len(mg), "cells": cells,
                          "ms": ms, "launches": fac.kernel_launches()}), flush=True)
        ctx.close()
        return 0

    def barrier():
        torch.cuda.synchronize(local_rank)
        if dist:
            dist.barrier()

    def step(c):
        c.zero(fac.U)
        return c.solve()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], device=f"cuda:{local_rank}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # autotuner: stage size of the staged smoother, timed on this workload
    tuned, tune_ms = ctx.autotune()
    for _ in range(args.warmup):
        conv, its, res = step(ctx)
    barrier()
    launches0 = fac.kernel_launches()
    sampler = ClockSampler(local_rank)
    sampler.start()
    ctx.timer_start()
    for _ in range(args.steps):
        conv, its, res = step(ctx)
    dev_ms = ctx.timer_stop()
    clocks = sampler.stop()
    launches = fac.kernel_launches() - launches0
    barrier()
    ms_per_step = max_over_ranks(dev_ms / args.steps)

    # one more step with CUDA events around every colour pass and ghost fill
    ctx.profile(True)
    ctx.timer_start()
    step(ctx)
    prof_ms = ctx.timer_stop()
    kind_rb, kind_fill = (2, 3) if args.precision == "mixed" else (0, 1)
    rb_n, rb_ms, rb_bytes = ctx.profile_read(kind_rb)
    fl_n, fl_ms, fl_bytes = ctx.profile_read(kind_fill)
    rb64 = ctx.profile_read(0)
    ctx.profile(False)

    # end to end through the host-buffer entry point (pinned buffers)
    nlev = mg[0].nlev
    f_host, u_host, u0_host = [], [], []
    h2d = d2h = 0
    for ip, p in enumerate(mg):
        for ln in range(nlev):
            f_t = torch.from_numpy(np.ascontiguousarray(p.f[ln])).pin_memory()
            u_t = torch.empty(ctx.size(fac.U, ip, ln), dtype=torch.float64).pin_memory()
            u0_t = torch.zeros(ctx.size(fac.U, ip, ln), dtype=torch.float64).pin_memory()
            f_host.append(f_t.numpy())
            u_host.append(u_t.numpy())
            u0_host.append(u0_t.numpy())
            h2d += f_t.numel() * 8 + u0_t.numel() * 8
            d2h += u_t.numel() * 8
    e2e_steps = max(1, min(args.steps, 2))
    barrier()
    t = time.perf_counter()
    for _ in range(e2e_steps):
        conv_e, its_e, res_e = ctx.solve_host(f_host, u_host, u0_host)
    barrier()
    e2e_ms = max_over_ranks((time.perf_counter() - t) * 1e3 / e2e_steps)

    # the same context without the Krylov acceleration (stationary FAC cycles)
    fac_only = None
    if args.krylov > 0:
        ctx.set_krylov(0)
        step(ctx)
        ctx.timer_start()
        conv_s, its_s, _ = step(ctx)
        ms_s = ctx.timer_stop()
        ctx.set_krylov(args.krylov)
        fac_only = {"ms": round(max_over_ranks(ms_s), 1), "converged": int(np.sum(conv_s)),
                    "cycles_max": int(np.max(its_s)), "cycles_mean": float(np.mean(its_s))}

    # the same multigrid-extended FAC all in FP64 (one timed solve)
    fp64_mg = None
    k = MG_LEVELS[args.config]
    if args.precision == "mixed":
        c64 = fac.FacContext(mg, params=PARAMS_MG, device=local_rank, precision="fp64")
        c64.set_krylov(args.krylov)
        c64.autotune()
        step(c64)
        c64.profile(True)
        c64.timer_start()
        conv64, its64, _ = step(c64)
        ms64 = c64.timer_stop()
        r64 = c64.profile_read(0)
        c64.profile(False)
        num = den = 0.0
        for i in range(len(probs)):
            for ln in range(probs[i].nlev):
                a = ctx.download(fac.U, i, ln + k)
                b = c64.download(fac.U, i, ln + k)
                num += float(np.sum((a - b) ** 2))
                den += float(np.sum(b ** 2))
        fp64_mg = {"ms": round(max_over_ranks(ms64), 1), "converged": int(np.sum(conv64)),
                   "cycles_max": int(np.max(its64)), "cycles_mean": float(np.mean(its64)),
                   "mixed_vs_fp64_rel_l2": math.sqrt(num / max(den, 1e-300)),
                   "rbgs_fp64_gbs": round(r64[2] / max(r64[1], 1e-9) / 1e6, 1),
                   "rbgs_fp64_launches": int(r64[0])}
        c64.close()

    # plain FP64 FAC (reference semantics) on a subset of the problems
    plain = None
    if not args.no_plain:
        sub = probs[:max(1, min(args.plain_problems, len(probs)))]
        pctx = fac.FacContext(sub, params=PARAMS, device=local_rank)
        pctx.timer_start()
        pconv, pits, pres = step(pctx)
        p_ms = pctx.timer_stop()
        sub_cells = sum(p.num_cells() for p in sub)
        # solution agreement of the two variants where the plain one converged
        diffs = []
        for i in range(len(sub)):
            if not pconv[i]:
                continue
            num = den = 0.0
            for ln in range(sub[i].nlev):
                a = ctx.download(fac.U, i, ln + k)
                b = pctx.download(fac.U, i, ln)
                num += float(np.sum((a - b) ** 2))
                den += float(np.sum(b ** 2))
            diffs.append(math.sqrt(num / max(den, 1e-300)))
        if args.plain_cycles_out and rank == 0:
            seeds = workload_seeds(args.config, args.nprob, rank, world)
            with open(args.plain_cycles_out, "w") as fh:
                json.dump({"what": "plain FAC cycles to a 1e-10 relative composite residual "
                                   "(max_cycles 100, 500-sweep coarsest solve) per seed",
                           "workload": desc,
                           "cycles": {str(x): int(c) for x, c in zip(seeds, pits)}}, fh,
                          indent=1)
        plain = {"ms": round(p_ms, 1), "problems": len(sub), "cells": sub_cells,
                 "ms_scaled_to_workload": round(p_ms * cells / sub_cells, 1),
                 "converged": int(np.sum(pconv)), "cycles": [int(x) for x in pits],
                 "coarse_sweeps_total": int(np.sum(pctx.coarse_sweeps())),
                 "mg_vs_plain_rel_l2_max": max(diffs) if diffs else None}
        pctx.close()

    regrid = regrid_measure(ctx, probs) if args.regrid else None
    cnn = None
    if args.cnn:
        # training throughput of the learned part's kernels (BF16 tensor
        # cores, FP32 accumulation) against the measured BF16 GEMM peak
        from samrai_b200 import learned
        net = fac.CNN(max_batch=256, device=local_rank, seed=1)
        cnn = learned.training_throughput(net, batch=256, steps=10, device=local_rank)
        net.close()
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
                bf16 = float(json.load(fh)["bf16_tflops"])
            cnn["peak_tflops"], cnn["peak_kind"] = bf16, "measured bf16 burst"
        except Exception:
            cnn["peak_tflops"], cnn["peak_kind"] = 1590.0, "fallback"
        cnn["train_frac"] = round(cnn["train_tflops"] / cnn["peak_tflops"], 4)
        for kk in ("train_ms", "forward_ms", "train_tflops", "forward_tflops"):
            cnn[kk] = round(cnn[kk], 3)
    peak, peak_kind = measured_peaks()
    achieved = rb_bytes / (rb_ms * 1e-3) / 1e9 if rb_ms > 0 else 0.0
    out = {
        "metric": METRIC,
        "value": round(ms_per_step, 3),
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 smoothing / f64 residual" if args.precision == "mixed" else "f64",
        "data": "synthetic",
        "config": {
            "workload": desc,
            "variant": ((f"FGMRES({args.krylov}) preconditioned by one " if args.krylov else "")
                        + f"{args.precision} FAC cycle on the hierarchy extended by {k} fully "
                        f"covered coarser levels (multigrid coarsest solve; "
                        f"{PARAMS_MG['pre_sweeps']} pre / {PARAMS_MG['post_sweeps']} post "
                        f"smoothing sweeps, {PARAMS_MG['coarse_max_it']} coarsest sweeps)"),
            "problems_per_gpu": len(probs),
            "cells_per_gpu": cells,
            "patches_per_gpu": npatch,
            "stopping": "relative composite RMS residual <= 1e-10, max 100 cycles, "
                        "2/2 red-black sweeps, Ewing, linear refine",
            "l2": "inputs larger than L2 (no flush needed)",
            "parallelism": f"problem shards x{world}",
            "autotuned_stage_bytes": int(tuned),
            "autotuned_stage_depth": int(ctx.stage_depth),
            "autotune_sweep_ms": [round(float(x), 3) for x in tune_ms],
        },
        "converged": int(np.sum(conv)),
        "cycles_max": int(np.max(its)),
        "cycles_mean": float(np.mean(its)),
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": {
            "kernel": ("k_rb_staged<3,D var,float> (red-black colour pass on TMA-staged "
                       "units, FP32)" if args.precision == "mixed" else
                       "k_rb_staged<3,D var,double> (red-black colour pass on TMA-staged units)"),
            "bound": "hbm",
            "achieved": round(achieved, 1),
            "peak": peak,
            "peak_kind": peak_kind,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "traffic": (round(STAGED_F32_TRAFFIC_RATIO * rb_bytes / max(rb_n, 1) / 1e6, 2)
                        if args.precision == "mixed" else None),
            "traffic_unit": "MB per launch",
            "launches": int(rb_n),
            "avg_launch_us": round(rb_ms * 1e3 / max(rb_n, 1), 2),
            "share_of_step": round(rb_ms / max(prof_ms, 1e-9), 4),
        },
        "ghost_fill": {"launches": int(fl_n), "ms": round(fl_ms, 3),
                       "gbs": round(fl_bytes / max(fl_ms, 1e-9) / 1e6, 1),
                       "share_of_step": round(fl_ms / max(prof_ms, 1e-9), 4)},
        "fp64_multigrid": fp64_mg,
        "stationary_fac": fac_only,
        "plain_fp64": plain,
        "regrid": regrid,
        "cnn_training": cnn,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference arm's estimate on a bounded sample: one round of one
        # problem per core (unsampled problems scaled by their cells)
        seeds = workload_seeds(args.config, args.nprob, 0)
        ref = CpuReference(args.config, seeds)
        wall = ref.round()
        ms_est, info = ref.estimate(cells={x: p.num_cells() for x, p in zip(seeds, probs)})
        ref.close()
        out["cpu_baseline"] = {
            "value": round(ms_est, 1), "unit": "ms", "cores": ref.workers, "kind": ref.kind,
            "sample": (f"{CPU_KIND_TEXT[ref.kind]}, plain semantics, one process per core: "
                       f"one plain cycle of each of {info['sampled']} problems timed "
                       f"({wall:.1f} s wall), "
                       f"the rest scaled by cells; each problem's plain cycle count "
                       f"({info['cycles_from_table']} of {info['problems']} from the measured "
                       f"table), problems spread over {ref.workers} processes"),
        }
        # measured full solves of the small 2-D configurations, CPU and GPU
        small_kind, small = cpu_small_solves()
        for n in small:
            sp = [_make_problem(n, 0)]
            sctx = fac.FacContext(sp, params=PARAMS, device=local_rank)
            sctx.solve()
            sctx.zero(fac.U)
            sctx.timer_start()
            _, sits, _ = sctx.solve()
            small[n]["gpu_plain_fp64_ms"] = round(sctx.timer_stop(), 3)
            small[n]["gpu_cycles"] = int(sits[0])
            sctx.close()
        out["cpu_small_configs"] = {"kind": small_kind, "measured": True, "cores": 1,
                                    "cpu": CPU_KIND_TEXT[small_kind], "configs": small}
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def run_reference(args, world):
    """CPU reference arm: the reference's plain FAC on all host cores, one
    process per core -- its own CellPoissonFACSolver built from its sources
    (oracle/_ref) when present, else the oracle's restatement (-O3
    -march=native).  A step is one sampling round, in which every process
    times one plain cycle of the next problem in turn (`_ref_sample`); the
    rounds run until every problem of the workload has a sample.  The value
    is the time to solve the workload: per problem its mean cycle time times
    its plain cycle count, the problems spread over the processes longest
    first.  Configs 1 and 3 are solved outright on one core."""
    seeds = workload_seeds(args.config, args.nprob, 0)
    desc = workload_desc(args.config, args.nprob)
    if args.config in ("c1", "c3"):
        # small enough to solve outright
        vals = []
        for it in range(args.warmup + args.steps):
            kind, rs = cpu_small_solves((args.config,))
            r = rs[args.config]
            if it >= args.warmup:
                vals.append(r["cpu_ms"])
        value, cores = statistics.mean(vals), 1
        sample = f"full plain FAC solve, {r['cycles']} cycles, one core, measured"
        info = {}
    else:
        ref = CpuReference(args.config, seeds)
        for _ in range(args.warmup):
            ref.round(keep=False)
        rounds = max(args.steps, -(-len(seeds) // ref.workers))
        walls = [ref.round() for _ in range(rounds)]
        value, info = ref.estimate()
        ref.close()
        cores, kind = ref.workers, ref.kind
        sample = (f"{rounds} rounds of one plain cycle per process ({sum(walls):.1f} s wall): "
                  f"cycle = outer-loop work + 500 x one coarse red-black sweep, timed per "
                  f"problem; per-problem plain cycle counts ({info['cycles_from_table']} of "
                  f"{info['problems']} from the measured table); problems spread over "
                  f"{cores} processes longest first")
    out = {
        "metric": METRIC,
        "impl": "reference",
        "value": round(value, 1),
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(value, 1),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": desc,
                   "variant": f"{CPU_KIND_TEXT[kind]}: plain cycle, 500-sweep red-black "
                              f"coarsest solve",
                   **info},
        "cpu_baseline": {"value": round(value, 1), "unit": "ms", "cores": cores,
                         "kind": kind, "sample": sample},
        "e2e": {"value": round(value, 1), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
