"""Benchmark: FMM evaluations per second on one B200 (or N replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 1048576] [--P 10] [--precision fp64|mixed]

Workload (default): 3D free-space Laplace FMM, N = 1,048,576 bodies uniform
in [-pi, pi]^3 with charges uniform in [-0.5, 0.5] (neutralised), generated
exactly like the reference driver (srand48(0)/drand48), P = 10, theta = 0.4,
ncrit = 64.  One step is one complete evaluation -- tree build, interaction
lists, upward pass, M2L + P2P, downward pass -- from the unsorted bodies
already resident in HBM.  Between timed steps the L2 is flushed by writing a
256 MB buffer (outside the timed events).

Printed: one JSON line (rank 0) with the driver's keys plus the e2e number
(Body records in pinned host memory -> set_bodies -> evaluate -> get_bodies
back to host, per step), the roofline of the dominant kernel, the reference's
own CPU build timed on this host's cores, per-phase times and the error of
the result against FP64 direct summation on 1000 sampled bodies.

--impl reference times the reference itself (its own headers compiled by
oracle/Makefile into oracle/_ref, lazy traversal, OpenMP on all host cores)
on the same workload and prints the same line with "impl": "reference".

Multi-GPU: the evaluation does not shard across GPUs in this build; with
--gpus N (under torchrun) every rank evaluates its own independent system of
the same size ("replicas"), so value = N / max-over-ranks time per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FMM evals/s at 1M bodies P=10: mixed vs FP64 GPU at ≤1e-5 rel. force error"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--P", type=int, default=10)
    ap.add_argument("--theta", type=float, default=0.4)
    ap.add_argument("--ncrit", type=int, default=64)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=40.0, help="seconds of reference CPU work at most")
    return ap.parse_args()


def workload(a):
    return {"workload": f"3d free-space Laplace FMM, {a.n} uniform bodies in [-pi,pi]^3 (drand48 seed 0), "
                        f"P={a.P}, theta={a.theta}, ncrit={a.ncrit}",
            "n_bodies": a.n, "P": a.P, "theta": a.theta, "ncrit": a.ncrit,
            "l2": "flushed between steps (256 MB write)"}


# ---------------------------------------------------------------- roofline
def m2l_flops_per_pair(P):
    """Real flops of one M2L with the reference's truncation (degree j+n < P,
    3d/kernel.h:83-116 fills only n < P): per output (j,k) and input (n,|m|)
    with n <= P-1-j one 2x2 real block, 4 multiply-adds = 8 flops."""
    blocks = sum((j + 1) * (n + 1) for j in range(P) for n in range(P - j))
    return 8 * blocks


def pair_count(fmm):
    """Body-pair interactions of the P2P lists (self pairs included)."""
    t = fmm.tree()
    lists = fmm.lists()
    nb = t["nbody"].astype(np.int64)
    off = lists["p2p_off"]
    tgt = np.repeat(np.arange(len(off) - 1), np.diff(off))
    return int((nb[tgt] * nb[lists["p2p_src"]]).sum()), len(lists["m2l_src"])


# ---------------------------------------------------------------- clocks
class Clocks:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = f"/tmp/exafmm_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- reference arm
def reference_eval(xq, a, threads):
    import oracle

    ref = oracle.Ref("3d", "lazy")
    ref.set_threads(threads)
    t0 = time.perf_counter()
    ref.fmm(xq, a.P, a.ncrit, a.theta)
    return time.perf_counter() - t0, ref


def cpu_baseline(xq, a):
    """The reference's own CPU build on all host cores: one full evaluation
    of the same workload (about 15 s on 8 cores)."""
    threads = os.cpu_count() or 1
    dt, _ = reference_eval(xq, a, threads)
    return {"value": 1.0 / dt, "unit": "evals/s", "cores": threads, "kind": "reference",
            "sample": f"one full evaluation of the same {a.n}-body workload (reference lazy traversal, "
                      f"OpenMP {threads} threads), {dt:.2f} s"}


def run_reference(a, rank, world):
    if rank != 0:
        return
    from minimal_b200.bodies import drand48_bodies

    xq = drand48_bodies(a.n, 0)
    threads = os.cpu_count() or 1
    times = []
    t_start = time.perf_counter()
    steps_done = 0
    for s in range(a.warmup + a.steps):
        if s < a.warmup and s > 0 and time.perf_counter() - t_start > a.cpu_budget / 4:
            continue  # keep the warm-up bounded: one evaluation is enough to warm caches
        dt, _ = reference_eval(xq, a, threads)
        if s >= a.warmup:
            times.append(dt)
            steps_done += 1
        if time.perf_counter() - t_start > 4 * a.cpu_budget and len(times) >= 1:
            break
    t = statistics.mean(times)
    v = 1.0 / t
    line = {"metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": 0, "steps": steps_done, "warmup": a.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (drand48 seed 0, the reference driver's generator)",
            "config": workload(a), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": threads, "kind": "reference",
                             "sample": f"{steps_done} full evaluations of the workload (bounded to ~{4 * a.cpu_budget:.0f} s)"},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def run_ours(a, rank, world, local_rank):
    import torch

    import minimal_b200
    from minimal_b200 import FMM, drand48_bodies

    dist = world > 1
    if dist:
        import datetime

        import torch.distributed as td

        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    def barrier_max(x):
        if not dist:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        import torch.distributed as td

        td.all_reduce(t, op=td.ReduceOp.MAX)
        return float(t.item())

    # each rank: its own system (seed = rank), the reference's generator
    xq = drand48_bodies(a.n, rank)
    rec = np.zeros((a.n, 8))
    rec[:, :4] = xq
    d_rec = torch.from_numpy(rec).to(dev)
    fmm = FMM(P=a.P, ncrit=a.ncrit, theta=a.theta, precision=a.precision, device=local_rank)
    torch.cuda.synchronize()
    fmm.set_bodies_device(d_rec.data_ptr(), a.n)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    for _ in range(a.warmup):
        fmm.evaluate()

    clocks = Clocks(local_rank)
    phase = {k: [] for k in minimal_b200.PHASES}
    launches = 0
    torch.cuda.synchronize()
    if dist:
        import torch.distributed as td

        td.barrier()
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize()
        fmm.evaluate()
        launches += fmm.last_launches()
        for k, v in fmm.timings().items():
            phase[k].append(v)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    if dist:
        td.barrier()
    clk = clocks.stop()
    ms_dev = statistics.mean(phase["total"])
    ms_max = barrier_max(ms_dev)
    value = world * 1e3 / ms_max

    # e2e: host Body records (pinned) -> C ABI -> host results, every step
    h_in = torch.from_numpy(rec).pin_memory()
    h_out = torch.empty((a.n, 8), dtype=torch.float64).pin_memory()
    lib = fmm.lib
    e2e = []
    for s in range(max(2, min(a.steps, 5)) + 1):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        fmm._check(lib.exafmm_b200_set_bodies(fmm.h, h_in.data_ptr(), a.n, minimal_b200.HOST))
        fmm._check(lib.exafmm_b200_evaluate(fmm.h))
        fmm._check(lib.exafmm_b200_get_bodies(fmm.h, h_out.data_ptr(), minimal_b200.HOST))
        dt = time.perf_counter() - t1
        if s > 0:
            e2e.append(dt)
    e2e_ms = barrier_max(statistics.mean(e2e) * 1e3)

    if rank != 0:
        fmm.close()
        if dist:
            td.destroy_process_group()
        return

    # accuracy on 1000 sampled tree positions vs FP64 direct summation
    out = h_out.numpy().copy()
    sample = np.arange(0, a.n, max(1, a.n // 1000))[:1000]
    tgt = out[sample].copy()
    res = tgt.copy()
    tgt[:, 4:] = 0
    d = fmm.direct(tgt)
    err_p = float(np.sqrt(((res[:, 4] - d[:, 4]) ** 2).sum() / (d[:, 4] ** 2).sum()))
    err_f = float(np.sqrt(((res[:, 5:] - d[:, 5:]) ** 2).sum() / (d[:, 5:] ** 2).sum()))

    # roofline of the dominant kernel (one launch per phase for m2l and p2p)
    pairs, n_m2l = pair_count(fmm)
    peak64 = fmm.fma_peak("fp64")
    m2l_ms = statistics.mean(phase["m2l"])
    p2p_ms = statistics.mean(phase["p2p"])
    m2l_tf = n_m2l * m2l_flops_per_pair(a.P) / (m2l_ms * 1e-3) / 1e12
    p2p_tf = pairs * 20 / (p2p_ms * 1e-3) / 1e12
    if m2l_ms >= p2p_ms:
        dom = {"kernel": "k_m2l (M2L, FP64)", "achieved": m2l_tf, "flops_per_launch": n_m2l * m2l_flops_per_pair(a.P)}
    else:
        dom = {"kernel": "k_p2p (P2P, FP64)", "achieved": p2p_tf, "flops_per_launch": pairs * 20}
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(dom["kernel"].split()[0])
    roof = {"bound": "fp64", "kernel": dom["kernel"], "achieved": dom["achieved"], "peak": peak64,
            "unit": "TFLOP/s", "frac": dom["achieved"] / peak64, "traffic": traffic,
            "peak_source": "measured FP64 FMA-pipe microbenchmark on this GPU (exafmm_b200_fma_peak)",
            "flops_per_launch": dom["flops_per_launch"],
            "other": {"k_m2l_tflops": m2l_tf, "k_p2p_tflops": p2p_tf}}

    cpu = None
    if not a.no_cpu_baseline:
        try:
            cpu = cpu_baseline(xq, a)
        except Exception as e:  # the reference build missing is reported, not hidden
            cpu = {"unavailable": str(e)}

    line = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "mixed",
            "data": "synthetic (drand48, the reference driver's generator; seed = rank)",
            "config": dict(workload(a), parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                           precision=a.precision),
            "e2e": {"value": world * 1e3 / e2e_ms, "unit": "evals/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": a.n * 64, "d2h_bytes_per_step": a.n * 64},
            "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            "phases_ms": {k: statistics.mean(v) for k, v in phase.items()},
            "wall_ms_per_step": wall * 1e3 / a.steps,
            "error_vs_direct": {"p": err_p, "F": err_f, "targets": len(sample)},
            "work": {"cells": fmm.num_cells(), "m2l_pairs": n_m2l, "p2p_body_pairs": pairs}}
    print(json.dumps(line), flush=True)
    fmm.close()
    if dist:
        td.destroy_process_group()


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ["WORLD_SIZE"]) if "WORLD_SIZE" in os.environ else 1
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    run_ours(a, rank, world, local_rank)


if __name__ == "__main__":
    main()
