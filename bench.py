"""Benchmark: cell-steps/s of the FRiBoIS2D fluid time step on B200.

One step is one full time step of the reference's main loop (three RK3
substeps of fluid_tsch, loads, rigid-body update; src/main.F90:85-97).
Workload: the rotational-galloping rectangle on 1024 (z) x 768 (y) cells,
1200 markers, plain FP64 (synthetic deck written by fribois2d_b200.case).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs one independent replica per GPU (the single-case path does not
shard); launch with torch.distributed.run.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes
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

METRIC = "cell-steps/s (plain FP64 fluid time step, galloping rectangle 1024x768)"
# Poisson transform forms: the plain FP64 path computes them on the INT8
# tensor cores to FP64 accuracy (the default); "fp64" runs them as cuBLAS
# DGEMMs, the comparison arm
FORMS = {"int8x8": "plain FP64", "fp64": "plain FP64 with cuBLAS DGEMM transforms",
         "tf32x3": "3xTF32 tensor-core Poisson transforms + FP64 refinement"}
POISSON_IDS = {"int8x8": 2, "fp64": 0, "tf32x3": 1}
DTYPES = {"int8x8": "f64 (Poisson transforms: exact int8 digit products)", "fp64": "f64",
          "tf32x3": "f64 (Poisson transforms: 3xtf32)"}


def metric_name(args) -> str:
    if args.poisson == "int8x8" and args.config == "galloping_rectangle_1024x768":
        return METRIC
    return f"cell-steps/s ({FORMS[args.poisson]} fluid time step, {args.config.replace('_', ' ')})"
UNIT = "cell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="galloping_rectangle_1024x768",
                    choices=["viv_cylinder_384x256", "galloping_rectangle_1024x768", "viv_cylinder_2048x1536"])
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--batch", type=int, default=0,
                    help="advance N independent VIV cases (grid sizes 256x192..768x512 drawn by seed) "
                         "with one graph launch per step instead of the single case")
    ap.add_argument("--sweeps", type=int, default=2, help="FP64 refinement sweeps of the tf32x3 form")
    ap.add_argument("--coupling", default="loose", choices=["loose", "strong", "learned"],
                    help="with --batch: strong fluid-structure coupling, with the plain or the learned initial guess")
    ap.add_argument("--train-cases", type=int, default=256, help="sweep cases generating the predictor's samples")
    ap.add_argument("--train-steps", type=int, default=4000, help="coupled steps per sweep case")
    ap.add_argument("--train-epochs", type=int, default=20)
    ap.add_argument("--windows", type=int, default=4,
                    help="windows in which the batched coupled arms alternate over one stretch of the trajectory")
    ap.add_argument("--accuracy-steps", type=int, default=2000,
                    help="steps of the tf32x3 form's accuracy comparison with the FP64 path")
    ap.add_argument("--poisson", default="int8x8", choices=sorted(FORMS),
                    help="eigen transforms of the Poisson solve: FP64-accurate INT8 tensor-core products "
                         "(default), cuBLAS DGEMM (comparison arm), or 3xTF32 on the tensor cores")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(dist, x: float, device) -> float:
    """Largest value of x over all ranks (every rank takes this collective)."""
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, cells: int, steps: int, max_ms: float) -> float:
    """Whole-job cell-steps/s: every rank advanced its own replica `steps`
    steps of `cells` cells; the job took as long as its slowest rank."""
    return world * cells * steps / (max_ms * 1e-3)


def profiled_traffic(workload: str, kernel: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum of one
    ncu capture) from the '| workload | kernel | bytes |' rows of the ncu
    summaries under profiles/, or None."""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for ln in f:
                cells = [x.strip() for x in ln.strip().strip("|").split("|")]
                if len(cells) == 3 and cells[0] == workload and cells[1] == kernel and cells[2].isdigit():
                    return int(cells[2])
    return None


def make_case(name):
    from fribois2d_b200 import case as cases
    return cases.WORKLOADS[name]()


def write_deck(c, rank=0):
    root = tempfile.mkdtemp(prefix=f"fbbench{rank}_")
    return c.write(os.path.join(root, c.name))


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU arm

def cpu_run(case_name, seconds, max_steps, warmup=1):
    """The oracle (a C restatement of the reference's CPU path) on the host
    cores with all threads, after `warmup` untimed steps (the first touches
    every array); returns (cell-steps/s, steps timed, threads, seconds)."""
    import oracle
    c = make_case(case_name)
    path = write_deck(c, 99)
    threads = os.cpu_count() or 1
    o = oracle.Oracle(oracle.parse_deck(path), threads=threads)
    o.add_v_perturbation(c.v_perturbation())
    for w in range(max(1, warmup)):
        st = o.step(w)
        if st:
            raise RuntimeError(f"oracle status {st}")
    w0 = max(1, warmup)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        if o.step(w0 + steps):
            raise RuntimeError("oracle failed")
        steps += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return c.cells * steps / dt, steps, threads, dt


def reference_arm(args, rank, world):
    if rank != 0:
        return
    try:
        import oracle
        oracle.build()
        W = max(3, args.warmup)
        value, steps, threads, secs = cpu_run(args.config, seconds=max(30.0, 3.0 * args.cpu_seconds),
                                              max_steps=max(1, args.steps), warmup=W)
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"oracle failed: {e}"}))
        return
    c = make_case(args.config)
    line = {
        "impl": "reference", "metric": metric_name(args), "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": W, "ms_per_step": 1e3 * secs / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": c.name, "cells": c.cells, "markers": c.nlm, "host": "cpu"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{steps} full time steps of {c.name} (bounded by time budget)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ------------------------------------------------------------------ device arm

def fp64_gemm_peak(torch, dev):
    """cuBLAS DGEMM throughput measured in this run (the FP64 denominator;
    the driver's measured peaks cover copy bandwidth and bf16 only)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = math.inf
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def kernel_table(fb, path, c, poisson="int8x8", sweeps=2):
    """Average device time of every kernel of one step, timed live with CUDA
    events on the launching stream, on a scratch context."""
    s = fb.Solver(path)
    s.set_poisson(POISSON_IDS[poisson])
    s.set_refinement(sweeps)
    s.autotune()   # the tile shapes the timed run uses (remembered per grid size)
    s.advance(0, 2)
    s.set_substep(1, 1)
    cells = c.cells
    B = 8.0 * cells
    n2m, n3m = c.n2m, c.n3m
    gemm = 2.0 * n2m * n3m * n3m
    # (name, stage, launches per step, algorithmic bytes or flops per launch, bound);
    # rows with 0 launches per step are comparison rows, not part of the step
    dgemm_rows = [
        ("gemm_fwd (cuBLAS DGEMM)", "gemm_fwd", 0, gemm, "tensor"),
        ("gemm_bwd (cuBLAS DGEMM)", "gemm_bwd", 0, gemm, "tensor"),
    ]
    if poisson == "int8x8":
        # 36 digit-pair products of 2*n2m*n3m^2 integer ops each; the digit cut
        # reads the FP64 operand and writes 8 int8 planes (16 B per cell)
        transform = [
            ("i8x8 GEMM (tcgen05 kind::i8, 36 digit pairs)", "i8x8_gemm", 6, 36 * gemm, "tensor_i8"),
            ("i8 digit cut (row maxima from the producers)", "i8_split", 6, 2.0 * B, "hbm"),
            ("poisson_tri", "poisson_tri", 3, 3 * B, "hbm"),
        ] + dgemm_rows
    elif poisson == "fp64":
        transform = [
            ("gemm_fwd (cuBLAS DGEMM)", "gemm_fwd", 3, gemm, "tensor"),
            ("poisson_tri", "poisson_tri", 3, 3 * B, "hbm"),
            ("gemm_bwd (cuBLAS DGEMM)", "gemm_bwd", 3, gemm, "tensor"),
        ]
    else:   # 1 + sweeps solves per substep (the later ones on the residual), two transforms each
        transform = [
            ("tf32x3 GEMM (tcgen05, 3 products)", "tf32x3_gemm", 6 * (1 + sweeps), 3 * gemm, "tensor_tf32"),
            ("poisson_tri", "poisson_tri", 3 * (1 + sweeps), 3 * B, "hbm"),
        ]
    rows = [
        ("cfl", "cfl", 1, 2 * B, "hbm"),
        ("boucdq", "boucdq", 3, 8.0 * 8 * n2m, "hbm"),
        ("nl_rhs", "nl_rhs", 3, 9 * B, "hbm"),
        ("helsolve (windowed, one launch)", "helsolve", 3, 10 * B, "hbm"),
        ("divg", "divg", 3, 3 * B, "hbm"),
    ] + transform + [
        ("updvp_prcalc", "updvp", 3, 7 * B, "hbm"),
        ("submean_boucqt", "pr_submean", 3, 2 * B, "hbm"),
        ("forcing(interp+spread)", "forcing", 2, 0.0, "latency"),
        ("loads", "loads", 1, 0.0, "latency"),
    ]
    out = []
    for name, st, per_step, work, bound in rows:
        ms = s.time_stage(st, 2 if st == "forcing" else 1, reps=20)
        out.append({"kernel": name, "ms": ms, "per_step": per_step, "work": work, "bound": bound})
    s.close()
    return out


def batch_arm(args, rank, world, local):
    """N independent VIV cases stepped together (fb_batch, grouped: one
    launch per stage over each group of equal grids, one graph launch per
    step) against the same cases stepped one after another and against one
    graph holding every case's own step."""
    import torch
    import fribois2d_b200 as fb
    from fribois2d_b200 import case as cases

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cs = cases.viv_batch(args.batch, seed=rank)
    root = tempfile.mkdtemp(prefix=f"fbbatch{rank}_")
    solvers = []
    for c in cs:
        sv = fb.Solver(c.write(os.path.join(root, c.name)), device=local)
        sv.set_poisson(POISSON_IDS[args.poisson])
        sv.set_refinement(args.sweeps)
        q2 = sv.get("q2")
        q2[1:c.n3m + 1] += c.v_perturbation()
        sv.set("q2", q2)
        solvers.append(sv)
    cells = sum(c.cells for c in cs)
    W, K = max(3, args.warmup), max(1, args.steps)
    # one after another: each case's own captured step, K steps each
    seq_ms = 0.0
    for sv in solvers:
        sv.advance(0, W)
        sv.advance(W, K, history=False)
        seq_ms += sv.last_advance_ms()
    # every case's own captured step on its own branch of one graph
    gbatch = fb.Batch(solvers, mode=fb.BATCH_GRAPH)
    gbatch.advance(W)
    gbatch.advance(K)
    graph_ms = gbatch.last_ms()
    graph_launches = gbatch.info()["launches"]
    gbatch.close()
    # grouped: one launch per stage over every group of one launch geometry
    batch = fb.Batch(solvers, mode=fb.BATCH_GROUPED)
    info = batch.info()
    batch.advance(W)
    clocks = ClockSampler(local)
    torch.cuda.synchronize(dev)
    clocks.start()
    batch.advance(K)
    clk = clocks.stop()
    ms = batch.last_ms()
    value = cells * K / (ms * 1e-3)
    line = {
        "metric": f"cell-steps/s ({FORMS[args.poisson]}, batch of {args.batch} VIV cases, "
                  "one launch per stage per group of equal grids)",
        "value": value, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES[args.poisson], "data": "synthetic",
        "config": {"workload": f"viv_batch_{args.batch}", "cells_total": cells,
                   "grids": {f"{n3}x{n2}": sum(1 for c in cs if (c.n3m, c.n2m) == (n3, n2))
                             for n3, n2, _ in cases.BATCH_GRIDS},
                   "groups": info["groups"], "cases_on_own_branch": info["singles"],
                   "poisson": args.poisson, "l2": "working set far above L2 (all cases resident)"},
        "sequential": {"value": cells * K / (seq_ms * 1e-3), "ms_per_step": seq_ms / K,
                       "note": "the same cases, each advanced alone by its own captured step graph"},
        "graph_of_cases": {"value": cells * K / (graph_ms * 1e-3), "ms_per_step": graph_ms / K,
                           "launches_per_step": graph_launches,
                           "note": "every case's own step on its own branch of one graph"},
        "speedup_vs_sequential": seq_ms / ms,
        "gpu_launches": info["launches"] * K, "clocks": clk,
    }
    batch.close()
    for sv in solvers:
        sv.close()
    if rank == 0:
        print(json.dumps(line))


def merge_clocks(a, b):
    """Clock records of two sampled windows as one: the reasons seen in
    either, the lower median SM clock, the samples of both."""
    if a is None:
        return b
    out = dict(b)
    out["reasons"] = sorted(set(a.get("reasons", [])) | set(b.get("reasons", [])))
    mhz = [x["sm_mhz"] for x in (a, b) if x.get("sm_mhz") is not None]
    out["sm_mhz"] = min(mhz) if mhz else None
    out["samples"] = a.get("samples", 0) + b.get("samples", 0)
    return out


def coupled_batch_arm(args, rank, world, local):
    """Strongly coupled batch: N VIV cases of the batching form advanced
    together with the coupling iteration on the device (a graph WHILE node;
    converged cases sit out the grouped launches), with the learned initial
    guess (or the plain one).  All arms run on one set of cases, in turn, on
    the continuing trajectory after a loosely coupled warm-up of W steps (a
    developed flow, where the predictors have a history): the plain FP64
    path with the reference's loose coupling and with strong coupling (each
    case stepped alone by its own captured graph), then the batched form
    with the plain and with the learned predictor, alternating in short
    windows so that the two predictors meet the same stretch of the flow.
    The accuracy block runs a subset from the start against the FP64 path
    with strong coupling."""
    import torch
    import fribois2d_b200 as fb
    from fribois2d_b200 import case as cases
    from fribois2d_b200 import learn

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W, K = max(3, args.warmup), max(1, args.steps)
    pred, train = None, None
    if args.coupling == "learned":
        t0 = time.perf_counter()
        x, t, plain_train = learn.generate(learn.sweep(args.train_cases, seed=1000 + rank), steps=args.train_steps,
                                           device=local)
        t1 = time.perf_counter()
        pred = learn.train(x, t, epochs=args.train_epochs, batch=1024, lr=1e-3, seed=rank, device=local)
        train = {"coupling_steps": int(x.shape[0]), "kept": float(learn.predictable(t).mean()),
                 "cases": args.train_cases, "steps_per_case": args.train_steps,
                 "generate_s": t1 - t0, "train_s": time.perf_counter() - t1, "final_loss": pred.final_loss,
                 "plain_solves_per_step": plain_train,
                 "sweep": "small VIV cylinders (48x32 cells), Re, mass ratio, reduced velocity drawn by seed"}
    cs = cases.viv_batch(args.batch, seed=rank)
    cells = sum(c.cells for c in cs)
    root = tempfile.mkdtemp(prefix=f"fbcbatch{rank}_")
    form, fp64 = POISSON_IDS[args.poisson], POISSON_IDS["int8x8"]
    svs = []
    for c in cs:
        sv = fb.Solver(c.write(os.path.join(root, c.name)), device=local)
        sv.set_refinement(args.sweeps)
        q2 = sv.get("q2")
        q2[1:c.n3m + 1] += c.v_perturbation()
        sv.set("q2", q2)
        svs.append(sv)
    done = 0

    def solves_of(before):
        after = [sv.coupling_stats() for sv in svs]
        n = sum(a["solves"] - q["solves"] for a, q in zip(after, before))
        k = sum(a["steps"] - q["steps"] for a, q in zip(after, before))
        return n / max(k, 1.0)

    def solve_count(before):
        after = [sv.coupling_stats() for sv in svs]
        return (sum(a["solves"] - q["solves"] for a, q in zip(after, before)),
                sum(a["steps"] - q["steps"] for a, q in zip(after, before)))

    def sequential():   # each case alone, its own captured graph
        nonlocal done
        ms = 0.0
        for sv in svs:
            sv.set_poisson(fp64)
            sv.advance(done, K, history=False)
            ms += sv.last_advance_ms()
        done += K
        return ms

    def batched(mode, predictor, steps):
        nonlocal done
        for sv in svs:
            sv.set_poisson(form)
            sv.set_coupling(mode, 1e-8)
            if predictor is not None:
                sv.set_predictor(predictor.mlp, predictor.norm)
        b = fb.Batch(svs)
        info = b.info()
        before = [sv.coupling_stats() for sv in svs]
        clocks = ClockSampler(local)
        torch.cuda.synchronize(dev)
        clocks.start()
        b.advance(steps)
        clk = clocks.stop()
        ms = b.last_ms()
        b.close()
        done += steps
        return ms, solve_count(before), info, clk

    # loosely coupled warm-up as a batch in the FP64 form: a developed flow
    for sv in svs:
        sv.set_poisson(fp64)
    wb = fb.Batch(svs)
    wb.advance(W)
    wb.close()
    done += W
    seq_loose_ms = sequential()
    for sv in svs:
        sv.set_coupling(fb.COUPLING_STRONG, 1e-8)
    before = [sv.coupling_stats() for sv in svs]
    seq_coupled_ms = sequential()
    seq_coupled_solves = solves_of(before)
    # the batched arms alternate in windows over the same stretch of the
    # trajectory, so that both see the same flow
    nwin = max(1, min(args.windows, K))
    bounds = [K * w // nwin for w in range(nwin + 1)]
    arms = {"plain": [0.0, 0, 0], "main": [0.0, 0, 0]}
    info = clk = None
    for w in range(nwin):
        n = bounds[w + 1] - bounds[w]
        if n == 0:
            continue
        for arm in ("plain", "main"):
            mode, pr_ = (fb.COUPLING_STRONG, None) if (arm == "plain" or pred is None) else (fb.COUPLING_LEARNED, pred)
            wms, (ns, nk), winfo, wclk = batched(mode, pr_, n)
            a = arms[arm]
            a[0] += wms
            a[1] += ns
            a[2] += nk
            if arm == "main":
                info = winfo
                clk = merge_clocks(clk, wclk)
    plain_ms, plain_solves = arms["plain"][0], arms["plain"][1] / max(arms["plain"][2], 1)
    ms, solves = arms["main"][0], arms["main"][1] / max(arms["main"][2], 1)
    for sv in svs:
        sv.close()
    # accuracy: a subset from the start against the FP64 path, each case alone
    acc = None
    mode = fb.COUPLING_LEARNED if pred is not None else fb.COUPLING_STRONG
    if args.accuracy_steps > 0:
        picks = []
        for n3, n2, _ in cases.BATCH_GRIDS:
            picks += [c for c in cs if (c.n3m, c.n2m) == (n3, n2)][:2]
        worst_f = worst_d = 0.0
        for c in picks:
            hs = []
            for pform, md, pr_ in ((fp64, fb.COUPLING_STRONG, None), (form, mode, pred)):
                sv = fb.Solver(c.write(os.path.join(root, "acc_" + c.name)), device=local)
                sv.set_poisson(pform)
                sv.set_refinement(args.sweeps)
                q2 = sv.get("q2")
                q2[1:c.n3m + 1] += c.v_perturbation()
                sv.set("q2", q2)
                sv.set_coupling(md, 1e-8)
                if pr_ is not None:
                    sv.set_predictor(pr_.mlp, pr_.norm)
                hs.append(sv.advance(0, args.accuracy_steps))
                sv.close()
            a, b_ = hs
            f_ref, d_ref = a[:, 1], a[:, 9]
            worst_f = max(worst_f, float(np.max(np.abs(b_[:, 1] - f_ref)) / max(np.ptp(f_ref), 1e-300)))
            worst_d = max(worst_d, float(np.max(np.abs(b_[:, 9] - d_ref)) / max(np.ptp(d_ref), 1e-300)))
        acc = {"cases": len(picks), "steps": args.accuracy_steps, "lift_rel_of_range": worst_f,
               "displacement_rel_of_range": worst_d,
               "reference": "FP64 device path (INT8-exact transforms), strong coupling, plain predictor; "
                            "its coupled steps follow the oracle's fbo_coupled_step to round-off (tests)"}
    value = cells * K / (ms * 1e-3)
    seq_loose = cells * K / (seq_loose_ms * 1e-3)
    seq_coupled = cells * K / (seq_coupled_ms * 1e-3)
    line = {
        "metric": f"cell-steps/s (batch of {args.batch} VIV cases, {FORMS[args.poisson]}, strong coupling, "
                  f"{'learned' if pred is not None else 'plain'} predictor)",
        "value": value, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES[args.poisson], "data": "synthetic",
        "config": {"workload": f"viv_batch_{args.batch}_coupled", "cells_total": cells,
                   "grids": {f"{n3}x{n2}": sum(1 for c in cs if (c.n3m, c.n2m) == (n3, n2))
                             for n3, n2, _ in cases.BATCH_GRIDS},
                   "groups": info["groups"], "poisson": args.poisson, "coupling": args.coupling,
                   "tol": 1e-8, "l2": "working set far above L2 (all cases resident)",
                   "warmup": f"{W} loosely coupled steps as a batch, then the sequential arms {K} steps each, "
                             f"then the two batched arms alternating in {nwin} windows ({K} steps each in all)"},
        "fluid_solves_per_step": solves,
        "plain_fp64_sequential": {"value": seq_loose, "ms_per_step": seq_loose_ms / K,
                                  "note": "the same cases, FP64 (INT8-exact transforms), loose coupling as the "
                                          "reference, each advanced alone by its own captured step"},
        "plain_fp64_coupled_sequential": {"value": seq_coupled, "ms_per_step": seq_coupled_ms / K,
                                          "fluid_solves_per_step": seq_coupled_solves,
                                          "note": "the same cases, FP64, strong coupling with the plain "
                                                  "predictor, each advanced alone"},
        "speedup_vs_plain_fp64": value / seq_loose,
        "speedup_vs_plain_fp64_coupled": value / seq_coupled,
        "batched_plain_predictor": {"value": cells * K / (plain_ms * 1e-3), "ms_per_step": plain_ms / K,
                                    "fluid_solves_per_step": plain_solves},
        "training": train, "accuracy": acc,
        "gpu_launches": info["launches"] * K, "clocks": clk,
    }
    if pred is not None:
        pred.mlp.close()
    if rank == 0:
        print(json.dumps(line))


def precision_error(fb, path, c, steps, sweeps):
    """The precision form against the plain FP64 path (itself within 1e-10
    per step of the oracle) on the same case and inputs: lift, displacement
    and post-projection divergence over `steps` steps."""
    runs = {}
    for mode in (fb.POISSON_INT8X8, fb.POISSON_TF32X3):
        s = fb.Solver(path)
        s.set_poisson(mode)
        s.set_refinement(sweeps)
        s.set_report(True)
        q2 = s.get("q2")
        q2[1:c.n3m + 1] += c.v_perturbation()
        s.set("q2", q2)
        runs[mode] = s.advance(0, steps)
        s.close()
    a, b = runs[fb.POISSON_INT8X8], runs[fb.POISSON_TF32X3]
    col = {n: fb.HIST_NAMES.index(n) for n in ("Fy", "Fz", "py", "pa", "dmax")}
    def rel(x, y):
        return float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))
    return {"steps": steps, "lift_rel": rel(b[:, col["Fy"]], a[:, col["Fy"]]),
            "drag_rel": rel(b[:, col["Fz"]], a[:, col["Fz"]]),
            "displacement_abs": float(np.max(np.abs(b[:, col["py"]] - a[:, col["py"]]))),
            "divergence_max_fp64": float(np.max(a[:, col["dmax"]])),
            "divergence_max_tf32x3": float(np.max(b[:, col["dmax"]])),
            "refinement_sweeps": sweeps, "resid": 1e-7,
            "reference": "plain FP64 device path (parity with the oracle: 1e-10 per step)"}


def device_arm(args, rank, world, local):
    import torch
    import fribois2d_b200 as fb

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
        dist = dist_mod
    c = make_case(args.config)
    path = write_deck(c, rank)
    s = fb.Solver(path, device=local)
    s.set_poisson(POISSON_IDS[args.poisson])
    s.set_refinement(args.sweeps)
    tiles = s.autotune()   # tile shapes for this grid size (state preserved)
    pert = c.v_perturbation()
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += pert
    s.set("q2", q2)
    W, K = max(3, args.warmup), max(1, args.steps)
    s.advance(0, W)
    per_step_kernels = s.kernel_count()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    t_wall0 = time.perf_counter()
    dev_ms = 0.0
    for i in range(K):
        flush.zero_()                     # L2 flushed between timed steps
        s.advance(W + i, 1, history=False)  # device-timed (events on the step's stream)
        dev_ms += s.last_advance_ms()
    barrier()
    wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    dev_ms_max = max_over_ranks(dist, dev_ms, dev)
    value = replica_throughput(world, c.cells, K, dev_ms_max)

    # end to end through the C ABI with host buffers (loose FSI coupling as
    # the reference runs it: markers in, fluid step, rigid step, state out)
    e2e = e2e_one_call = None
    if not args.no_e2e:
        nlm = c.nlm
        pin = [torch.empty(2 * nlm, dtype=torch.float64).pin_memory() for _ in range(4)]
        fc = torch.empty(8, dtype=torch.float64).pin_memory()
        for buf, name in zip(pin, ("lmcc", "lmvel", "lmacc", "lmnor")):
            buf.copy_(torch.from_numpy(s.get(name)))
        L = fb.lib()
        ptr = [ctypes.cast(b.data_ptr(), ctypes.POINTER(ctypes.c_double)) for b in pin]
        fptr = ctypes.cast(fc.data_ptr(), ctypes.POINTER(ctypes.c_double))
        ns0 = W + K
        Ke = max(3, min(K, 20))

        def e2e_step(ns):
            assert L.fb_set_markers(s.ctx, *ptr) == 0
            assert L.fb_fluid_tsch(s.ctx, ns) == 0
            assert L.fb_rigid(s.ctx, ns, fptr) == 0
            assert L.fb_get_markers(s.ctx, *ptr) == 0

        # warm-up: the first fb_fluid_tsch captures and instantiates its graph
        We = max(3, W)
        for i in range(We):
            e2e_step(ns0 + i)
        ns0 += We
        barrier()
        te0 = time.perf_counter()
        for i in range(Ke):
            e2e_step(ns0 + i)
        barrier()
        te = time.perf_counter() - te0
        te_max = max_over_ranks(dist, te, dev)
        e2e = {"value": replica_throughput(world, c.cells, Ke, 1e3 * te_max), "unit": UNIT,
               "h2d_bytes_per_step": 4 * 2 * nlm * 8, "d2h_bytes_per_step": 4 * 2 * nlm * 8 + 8 * 8,
               "steps": Ke, "warmup": We, "timing": "host wall clock, per-step synchronous C-ABI calls"}
        # the same step through the combined call (one wait per step)
        ns0 += Ke
        for i in range(We):
            assert L.fb_step_markers(s.ctx, ns0 + i, *ptr, fptr) == 0
        ns0 += We
        barrier()
        te0 = time.perf_counter()
        for i in range(Ke):
            assert L.fb_step_markers(s.ctx, ns0 + i, *ptr, fptr) == 0
        barrier()
        te1_max = max_over_ranks(dist, time.perf_counter() - te0, dev)
        e2e_one_call = {"value": replica_throughput(world, c.cells, Ke, 1e3 * te1_max), "unit": UNIT,
                        "h2d_bytes_per_step": 4 * 2 * nlm * 8, "d2h_bytes_per_step": 4 * 2 * nlm * 8 + 8 * 8,
                        "steps": Ke, "warmup": We,
                        "timing": "host wall clock, fb_step_markers: markers in, fluid step, rigid update, "
                                  "markers and the forcecomp row out, one wait per step"}

    result = None
    if rank == 0:
        table = kernel_table(fb, path, c, args.poisson, args.sweeps)
        peak_fp64 = fp64_gemm_peak(torch, dev)
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except OSError:
            pass
        hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
        hbm_src = "of measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "of fallback 6.65 TB/s"
        step_ms = dev_ms_max / K
        for r in table:
            r["share"] = r["ms"] * r["per_step"] / step_ms
        # the dominant kernel of this library (library kernels are comparison rows)
        dom = max((r for r in table if r["bound"] in ("hbm", "tensor", "tensor_tf32", "tensor_i8")
                   and "cuBLAS" not in r["kernel"] and r["per_step"] > 0),
                  key=lambda r: r["ms"] * r["per_step"])
        traffic = profiled_traffic(c.name, dom["kernel"])
        if dom["bound"] == "tensor_i8":
            # dense INT8 runs at twice the bf16 rate on these tensor cores; the
            # measured bf16 burst figure doubled is the denominator
            peak_i8 = float(peaks.get("bf16_tflops", 1590.0)) * 2.0
            achieved = dom["work"] / (dom["ms"] * 1e-3) / 1e12
            roof = {"kernel": dom["kernel"], "bound": "tensor", "achieved": achieved, "peak": peak_i8,
                    "unit": "TFLOP/s", "frac": achieved / peak_i8, "traffic": traffic,
                    "peak_source": ("of measured: MEASURED_PEAKS.json bf16_tflops x 2 (dense INT8 rate; "
                                    "integer ops counted as flop)" if "bf16_tflops" in peaks
                                    else "of fallback 1.59 PFLOP/s bf16 x 2"),
                    "work_per_launch": f"36 digit pairs x 2*n2m*n3m^2 = {dom['work']:.4g} integer ops",
                    "fp64_equivalent_tflops": dom["work"] / 36.0 / (dom["ms"] * 1e-3) / 1e12}
        elif dom["bound"] == "tensor":
            achieved = dom["work"] / (dom["ms"] * 1e-3) / 1e12
            roof = {"kernel": dom["kernel"], "bound": "tensor", "achieved": achieved, "peak": peak_fp64,
                    "unit": "TFLOP/s", "frac": achieved / peak_fp64, "traffic": traffic,
                    "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run (no FP64 entry in MEASURED_PEAKS.json)",
                    "work_per_launch": f"2*n2m*n3m^2 = {dom['work']:.4g} flop"}
        elif dom["bound"] == "tensor_tf32":
            # dense TF32 runs at half the bf16 rate on these tensor cores; the
            # measured bf16 burst figure halved is the denominator
            peak_tf32 = float(peaks.get("bf16_tflops", 1590.0)) / 2.0
            achieved = dom["work"] / (dom["ms"] * 1e-3) / 1e12
            roof = {"kernel": dom["kernel"], "bound": "tensor", "achieved": achieved, "peak": peak_tf32,
                    "unit": "TFLOP/s", "frac": achieved / peak_tf32, "traffic": traffic,
                    "peak_source": ("of measured: MEASURED_PEAKS.json bf16_tflops / 2 (dense TF32 rate)"
                                    if "bf16_tflops" in peaks else "of fallback 1.59 PFLOP/s bf16 / 2"),
                    "work_per_launch": f"3 products x 2*n2m*n3m^2 = {dom['work']:.4g} flop"}
        else:
            achieved = dom["work"] / (dom["ms"] * 1e-3) / 1e9
            roof = {"kernel": dom["kernel"], "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                    "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": hbm_src}
        accuracy = None
        if args.poisson == "tf32x3" and args.accuracy_steps > 0:
            accuracy = precision_error(fb, path, c, steps=args.accuracy_steps, sweeps=args.sweeps)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            v, steps, threads, secs = cpu_run(args.config, seconds=args.cpu_seconds, max_steps=1000)
            cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{steps} full time steps of {c.name} on the oracle ({secs:.1f} s)"}
        result = {
            "metric": metric_name(args), "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPES[args.poisson], "data": "synthetic",
            "config": {"workload": c.name, "poisson": args.poisson, "cells": c.cells, "markers": c.nlm, "dt": c.params.dt,
                       "parallelism": f"replicas x{world}" if world > 1 else "single case",
                       "tiles": {"helsolve_rows": tiles[0], "gemm_cols": tiles[1] if args.poisson == "tf32x3" else None},
                       "l2": "flushed (256 MB write) between timed steps"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "e2e_one_call": e2e_one_call,
            "accuracy": accuracy,
            "gpu_launches": per_step_kernels * K, "clocks": clk,
            "fp64_gemm_peak_tflops": peak_fp64,
            "kernels": [{k: (round(v, 6) if isinstance(v, float) else v) for k, v in r.items()} for r in table],
            "wall_s": wall,
        }
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result))


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.batch and args.coupling != "loose":
        coupled_batch_arm(args, rank, world, local)
        return
    if args.batch:
        batch_arm(args, rank, world, local)
        return
    device_arm(args, rank, world, local)


if __name__ == "__main__":
    main()
