#!/usr/bin/env python
"""Benchmark: time to a 1e-10 relative composite residual of the FAC Poisson
solve on B200, with the smoother's achieved HBM bandwidth.

One step = one CellPoissonFACSolver::solveSystem of every problem of the
workload from a zero initial guess (u, f, D resident in HBM for ``value``;
host buffers with the copies inside the timed region for ``e2e``).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c5|c2|c1|c3] [--nprob P]

Multi-GPU (torchrun, one rank per GPU): the independent problems are
sharded, each rank solving its own batch of the same size (weak scaling, no
data-path collective); the step time is the maximum over ranks.

``--impl reference`` times the CPU restatement of the reference's FAC path
(oracle/, kind "port") on all host cores.
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
# covered coarser levels (multigrid coarsest-level solve), 20 red-black
# sweeps on the coarsest extension level.
PARAMS_MG = dict(PARAMS, coarse_max_it=20)
MG_LEVELS = {"c5": 3, "c2": 4, "c1": 3, "c3": 3}
# headline: FGMRES(KRYLOV) with one FAC cycle as the flexible preconditioner
KRYLOV = 20
# DRAM bytes per algorithmic byte of the FP32 staged colour pass, from one ncu
# capture of the pass on the finest level of 8 config-5 problems (67.2 MB read
# + write for 54.6 MB algorithmic on 2.48 M cells); traffic per launch is this
# times the launch's algorithmic bytes (scaling by cells processed)
STAGED_F32_TRAFFIC_RATIO = 67.2 / 54.6


def make_workload(name, nprob, rank):
    from samrai_b200 import configs
    if name == "c5":
        probs = configs.config5(nprob, first_seed=rank * nprob)
        desc = (f"config5: {nprob} independent 3-D variable-coefficient problems "
                f"(3 levels, coarse 64^3..128^3, D=exp(g) contrast 1e3)")
    elif name == "c2":
        probs = [configs.config2(seed=2 + rank)]
        desc = "config2: 3-D 128^3 coarse + 2 random-box levels, f = 4 Gaussian bumps"
    elif name == "c3":
        probs = [configs.config3()]
        desc = "config3: 2-D 64^2 + 64^2 fine, D = exp(g) contrast 1e3"
    else:
        probs = [configs.config1()]
        desc = "config1: 2-D sine, 64^2 coarse + 64^2 fine box"
    return probs, desc


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

def _cpu_cycle_sample(args):
    """Time one complete FAC cycle (V-cycle with the 500-sweep coarse solve,
    u += e, restriction and the full composite residual) of one problem on
    one core; returns (seconds, cells)."""
    name, seed, nprob = args
    sys.path.insert(0, ROOT)
    from samrai_b200 import configs
    from oracle.oracle import Oracle
    if name == "c5":
        p = configs.config5_problem(seed)
    elif name == "c2":
        p = configs.config2()
    elif name == "c3":
        p = configs.config3()
    else:
        p = configs.config1()
    prm = dict(PARAMS)
    prm["max_cycles"] = 1
    o = Oracle(p, params=prm)
    t = time.perf_counter()
    o.solve()
    dt = time.perf_counter() - t
    return dt, p.num_cells()


def cpu_estimate(name, nprob, cycles, cells_total, workers, samples):
    """Oracle time for one cycle on `samples` problems (in parallel on
    `workers` processes), scaled to the whole workload: seconds per cell per
    cycle x cells x cycles / workers."""
    import multiprocessing as mp
    jobs = [(name, s, nprob) for s in range(samples)]
    t0 = time.perf_counter()
    if workers > 1:
        ctx = mp.get_context("spawn")
        with ctx.Pool(workers) as pool:
            res = pool.map(_cpu_cycle_sample, jobs)
    else:
        res = [_cpu_cycle_sample(j) for j in jobs]
    wall = time.perf_counter() - t0
    per_cell = sum(r[0] for r in res) / sum(r[1] for r in res)
    est_s = per_cell * cells_total * cycles / max(workers, 1)
    return est_s * 1e3, wall, res


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
    ap.add_argument("--plain-problems", type=int, default=8,
                    help="problems of the workload the plain variant is timed on")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="precision of the headline (multigrid-extended) variant")
    ap.add_argument("--smoother-only", type=int, default=0, metavar="SWEEPS",
                    help="only run SWEEPS red-black sweeps on the largest level (for ncu)")
    ap.add_argument("--krylov", type=int, default=KRYLOV,
                    help="FGMRES restart length of the headline solve (0: stationary FAC)")
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
    probs, desc = make_workload(args.config, args.nprob, rank)
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
        plain = {"ms": round(p_ms, 1), "problems": len(sub), "cells": sub_cells,
                 "ms_scaled_to_workload": round(p_ms * cells / sub_cells, 1),
                 "converged": int(np.sum(pconv)), "cycles": [int(x) for x in pits],
                 "coarse_sweeps_total": int(np.sum(pctx.coarse_sweeps())),
                 "mg_vs_plain_rel_l2_max": max(diffs) if diffs else None}
        pctx.close()

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
                        f"covered coarser levels (multigrid coarsest solve)"),
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
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cyc = float(np.mean(plain["cycles"])) if plain else 50.0
        ms_est, wall, res_s = cpu_estimate(args.config, args.nprob, cyc, cells, 1, 1)
        out["cpu_baseline"] = {
            "value": round(ms_est, 1), "unit": "ms", "cores": 1, "kind": "port",
            "sample": (f"CPU restatement of the reference FAC (plain semantics, gcc -O2 "
                       f"-ffp-contract=off): one full cycle of problem 0 ({res_s[0][1]} cells) "
                       f"took {res_s[0][0]:.2f} s; scaled by cells ({cells}) and the mean plain "
                       f"cycle count ({cyc:.1f})"),
        }
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def run_reference(args, world):
    """CPU reference arm: the CPU restatement of the reference FAC (plain
    semantics) on all host cores.  Each step times one full FAC cycle of as
    many problems as there are worker processes; the value is that cost
    scaled to every cell of the workload and to REFERENCE_CYCLES cycles
    (the plain cycle count, identical on CPU and GPU by the parity tests)."""
    workers = os.cpu_count() or 1
    probs, desc = make_workload(args.config, args.nprob, 0)
    cells = sum(p.num_cells() for p in probs)
    cycles = REFERENCE_CYCLES.get(args.config, 50.0)
    samples = max(1, min(workers, len(probs), 16))
    vals = []
    for it in range(args.warmup + args.steps):
        ms_est, wall, res = cpu_estimate(args.config, args.nprob, cycles, cells, samples,
                                         samples)
        if it >= args.warmup:
            vals.append(ms_est)
    value = statistics.mean(vals)
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
        "config": {"workload": desc, "variant": "CPU FAC, reference semantics (oracle port)",
                   "cycles_assumed": cycles},
        "cpu_baseline": {"value": round(value, 1), "unit": "ms", "cores": samples,
                         "kind": "port",
                         "sample": (f"one full FAC cycle of {samples} problems on {samples} "
                                    f"processes, scaled to {cells} cells and {cycles} cycles")},
        "e2e": {"value": round(value, 1), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0


# Plain-FAC cycle counts per workload (mean over problems), as measured on
# the GPU path whose cycle counts equal the CPU oracle's (parity tests).
REFERENCE_CYCLES = {"c5": 50.0, "c2": 72.0, "c1": 20.0, "c3": 48.0}


if __name__ == "__main__":
    sys.exit(main())
