"""Benchmark: FMM evaluations per second on one B200 (or N replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 1048576] [--P 10] [--precision mixed|fp64] [--legs all|fp64|none]

Headline workload: 3D free-space Laplace FMM, N = 1,048,576 bodies uniform in
[-pi, pi]^3 with charges uniform in [-0.5, 0.5] (neutralised), generated
exactly like the reference driver (srand48(0)/drand48), P = 10, theta = 0.4,
ncrit = 64, in the mixed-precision form (FP32 near field with compensated
sums, tensor-core M2L).  One step is one complete evaluation -- tree build,
interaction lists, upward pass, M2L + P2P, downward pass -- from the unsorted
bodies already resident in HBM.  Between timed steps the L2 is flushed by
writing a 256 MB buffer (outside the timed events).

Printed: one JSON line (rank 0) with the driver's keys; the e2e number (Body
records in pinned host memory -> set_bodies -> evaluate -> get_bodies back to
host, per step); the roofline of the dominant kernel (the FP32 near field)
and of the tensor-core M2L; the reference's own CPU build timed on this
host's cores; per-phase times; the error against FP64 direct summation on
1000 sampled bodies; and, beside the headline, the same workload in the FP64
form (the ratio the metric names), the P = 12 point (where 1e-5 force error
is reachable), the batched form (2048 uneven systems, batched vs one system
at a time) and the periodic form (1M bodies, 3 image layers, checked against
the GPU Ewald sum).  --legs fp64 keeps only the FP64 leg, --legs none only
the headline (for profiling).

--impl reference times the reference itself (its own headers compiled by
oracle/Makefile into oracle/_ref, lazy traversal, OpenMP on all host cores)
on the same workload and prints the same line with "impl": "reference".

Multi-GPU: one evaluation does not shard across GPUs in this build; with
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
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--bodies", dest="n", type=int, default=1 << 20)  # --bodies under torchrun
    ap.add_argument("--P", type=int, default=10)
    ap.add_argument("--theta", type=float, default=0.4)
    ap.add_argument("--ncrit", type=int, default=64)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--legs", default="all", choices=["all", "fp64", "none"],
                    help="side legs: all (FP64, P=12, batched, periodic), fp64 only, or none (profiling)")
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
def max_over_ranks(x, device):
    """Max of x over the ranks of the default process group (a replica
    time: the job takes as long as its slowest replica); x itself without a
    group.  `device` holds the reduction tensor: the rank's GPU under NCCL,
    "cpu" under gloo."""
    import torch
    import torch.distributed as td

    if not (td.is_available() and td.is_initialized()) or td.get_world_size() == 1:
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def timed_steps(fmm, steps, flush, torch):
    """Per-phase device times (library CUDA events) of `steps` evaluations,
    each after an L2 flush; returns (phase lists, kernel launches)."""
    import minimal_b200

    phase = {k: [] for k in minimal_b200.PHASES}
    launches = 0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        fmm.evaluate()
        launches += fmm.last_launches()
        for k, v in fmm.timings().items():
            phase[k].append(v)
    return phase, launches


def isolated_phases(fmm, reps, flush, torch):
    """Per-phase device times of `reps` evaluations through the step API, in
    which each phase runs alone on the GPU (a whole evaluation runs the near
    field beside the far field): the kernel durations for the roofline."""
    phase = {"p2p": [], "m2l": []}
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        fmm.build_tree()
        fmm.build_lists()
        fmm.upward()
        fmm.horizontal()
        fmm.downward()
        t = fmm.timings()
        phase["p2p"].append(t["p2p"])
        phase["m2l"].append(t["m2l"])
    return phase


def errors_vs_direct(fmm, n, out=None):
    """Relative L2 error of p and F on 1000 stride-sampled tree positions
    against FP64 direct summation on the GPU."""
    out = fmm.bodies() if out is None else out
    sample = np.arange(0, n, max(1, n // 1000))[:1000]
    tgt = out[sample].copy()
    res = tgt.copy()
    tgt[:, 4:] = 0
    d = fmm.direct(tgt)
    ep = float(np.sqrt(((res[:, 4] - d[:, 4]) ** 2).sum() / (d[:, 4] ** 2).sum()))
    ef = float(np.sqrt(((res[:, 5:] - d[:, 5:]) ** 2).sum() / (d[:, 5:] ** 2).sum()))
    return {"p": ep, "F": ef, "targets": len(sample)}


def form_leg(FMM, d_rec, n, P, a, precision, flush, torch, local_rank, steps=3, warmup=2):
    fmm = FMM(P=P, ncrit=a.ncrit, theta=a.theta, precision=precision, device=local_rank)
    fmm.set_bodies_device(d_rec.data_ptr(), n)
    for _ in range(warmup):
        fmm.evaluate()
    phase, _ = timed_steps(fmm, steps, flush, torch)
    ms = statistics.mean(phase["total"])
    err = errors_vs_direct(fmm, n)
    fmm.close()
    return {"evals_per_s": 1e3 / ms, "ms_per_eval": ms, "error_vs_direct": err,
            "phases_ms": {k: statistics.mean(v) for k, v in phase.items()}}


def plummer_leg(FMM, flush, torch, local_rank, n=1 << 22, orders=(6, 8, 10, 12), steps=3, warmup=2):
    """Non-uniform bodies: 4,194,304 bodies of a Plummer sphere (scale radius
    1, radii above 10 rejected, equal charges 1/N; positions and charges
    rounded to FP32 values).  Per order P: the mixed form with its leaf size
    autotuned, timed, and its error against FP64 direct summation on 1,000
    sampled targets, beside the FP64 form's error with the same leaf size
    (the same tree, so the same sampled bodies)."""
    from minimal_b200 import plummer_bodies

    xq = plummer_bodies(n, 7).astype(np.float32).astype(np.float64)
    res = {"workload": f"{n} bodies, Plummer sphere (a=1, r<=10), charges 1/N, positions and charges FP32 "
                       "values; theta=0.4; mixed form with ncrit autotuned; errors vs FP64 direct on 1000 "
                       "targets"}
    for P in orders:
        f = FMM(P=P, ncrit=64, theta=0.4, precision="mixed", device=local_rank)
        f.set_bodies(xq)
        ncrit, _ = f.autotune(repeats=2)
        ts = []
        for s in range(warmup + steps):
            flush.zero_()
            torch.cuda.synchronize()
            f.evaluate()
            if s >= warmup:
                ts.append(f.timings()["total"])
        err = errors_vs_direct(f, n)
        f.close()
        g = FMM(P=P, ncrit=ncrit, theta=0.4, precision="fp64", device=local_rank)
        g.set_bodies(xq)
        g.evaluate()
        err64 = errors_vs_direct(g, n)
        g.close()
        ms = statistics.mean(ts)
        res[f"P{P}"] = {"ncrit": ncrit, "ms_per_eval": ms, "evals_per_s": 1e3 / ms, "error_vs_direct": err,
                        "fp64_error_vs_direct": err64}
    return res


def reevaluate_leg(fmm, n, flush, torch, full_ms, steps=5, warmup=3):
    """Fixed positions, new charges every evaluation (an FMM matrix-vector
    product): set_charges keeps the tree and the lists, reevaluate runs the
    passes over them.  Device time of the passes; the charge upload (8 B per
    body) happens before each timed evaluation."""
    rng = np.random.default_rng(1)
    ts = []
    for s in range(warmup + steps):
        q = rng.uniform(-0.5, 0.5, n)
        fmm.set_charges(q - q.mean())
        flush.zero_()
        torch.cuda.synchronize()
        fmm.reevaluate()
        if s >= warmup:
            ts.append(fmm.timings()["total"])
    ms = statistics.mean(ts)
    return {"workload": f"the same {n} positions, new neutral charges U[-0.5,0.5) each evaluation; tree and "
                        "lists kept (set_charges + reevaluate)",
            "ms_per_eval": ms, "evals_per_s": 1e3 / ms, "full_evaluate_ms": full_ms,
            "speedup_vs_full_evaluate": full_ms / ms}


def batched_leg(FMM, torch, dev, local_rank, nsys=2048):
    """Batched configuration: 2048 independent systems, sizes log-uniform in
    [1000, 65536] (seeded), each uniform in [-pi, pi]^3, P=6, theta=0.5,
    mixed, ncrit picked by the autotuner; one batched evaluation vs the same
    systems one at a time (same ncrit), host clock around each."""
    from minimal_b200.bodies import uniform_bodies

    rng = np.random.default_rng(2048)
    sizes = np.exp(rng.uniform(np.log(1000), np.log(65536), nsys)).astype(np.int64)
    offs = np.zeros(nsys + 1, np.int64)
    offs[1:] = np.cumsum(sizes)
    N = int(offs[-1])
    rec = np.zeros((N, 8))
    for q in range(nsys):
        rec[offs[q]:offs[q + 1], :4] = uniform_bodies(int(sizes[q]), q)
    d = torch.from_numpy(rec).to(dev)
    f = FMM(P=6, ncrit=64, theta=0.5, precision="mixed", device=local_rank)
    f.set_batch_device(d.data_ptr(), offs)
    f.evaluate()
    t64 = []
    for _ in range(2):
        f.evaluate()
        t64.append(f.timings()["total"])
    ncrit, tuned_ms = f.autotune(repeats=2)  # the project's autotuner over the leaf size
    tb = []
    for _ in range(3):
        torch.cuda.synchronize()
        t = time.perf_counter()
        f.set_batch_device(d.data_ptr(), offs)
        f.evaluate()
        torch.cuda.synchronize()
        tb.append(time.perf_counter() - t)
    phases = f.timings()
    # spot check: one system of the batch against its own evaluation
    out = f.bodies()
    q = int(np.argmax(sizes))
    f.close()
    g = FMM(P=6, ncrit=ncrit, theta=0.5, precision="mixed", device=local_rank)
    g.set_bodies_device(d[offs[q]:].data_ptr(), int(sizes[q]))
    g.evaluate()
    alone = g.bodies()
    mine = out[offs[q]:offs[q + 1]]
    same_order = bool(np.array_equal(mine[:, :4], alone[:, :4]))
    dev_f = float(np.sqrt(((mine[:, 5:] - alone[:, 5:]) ** 2).sum() / (alone[:, 5:] ** 2).sum()))
    for k in range(8):  # warm the one-at-a-time path
        g.set_bodies_device(d[offs[k]:].data_ptr(), int(sizes[k]))
        g.evaluate()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for k in range(nsys):
        g.set_bodies_device(d[offs[k]:].data_ptr(), int(sizes[k]))
        g.evaluate()
    torch.cuda.synchronize()
    t1 = time.perf_counter() - t
    g.close()
    t_b = min(tb)
    return {"workload": f"{nsys} systems, sizes log-uniform in [1000, 65536] (seeded), {N} bodies, "
                        f"uniform in [-pi,pi]^3, P=6, theta=0.5, mixed, ncrit autotuned -> {ncrit}",
            "autotune": {"ncrit": ncrit, "tuned_device_ms": tuned_ms, "device_ms_at_ncrit_64": min(t64)},
            "bodies": N, "batched_ms": t_b * 1e3, "batched_bodies_per_s": N / t_b,
            "one_at_a_time_ms": t1 * 1e3, "one_at_a_time_bodies_per_s": N / t1, "speedup": t1 / t_b,
            "batched_phases_ms": phases,
            "check_largest_system": {"same_tree_order": same_order, "rel_force_diff_vs_alone": dev_f}}


def periodic_leg(FMM, torch, dev, local_rank, n):
    """Periodic configuration: N bodies uniform in a cube of side 2 pi
    (neutralised), P=10, theta=0.4, ncrit=64, 3 image layers, both forms
    (root images in FP64).  After the dipole correction each form is checked
    by the reference's own measures (3dp/fmm.cxx:96-111) over ALL N bodies:
    the relative error of the energy sum q.p and the relative L2 error of
    the forces, against one GPU FP64 Ewald sum of all N bodies (ksize=11,
    sigma=1/(4 pi), cutoff=cycle/2, alpha=ksize/cycle as the reference's
    driver sets it, 3dp/fmm.cxx:20-23).  A second Ewald sum with the
    alpha=10/(2 pi) of the benchmark's configuration shows how far the Ewald
    check itself moves with alpha."""
    from minimal_b200 import drand48_bodies

    cyc = 2 * np.pi
    xq = drand48_bodies(n, 0, "3dp", cyc)
    rec = np.zeros((n, 8))
    rec[:, :4] = xq
    d = torch.from_numpy(rec).to(dev)
    res, outs = {}, {}
    ewald_handle = None
    for prec in ("mixed", "fp64"):
        f = FMM(P=10, ncrit=64, theta=0.4, images=3, cycle=cyc, precision=prec, device=local_rank)
        f.set_bodies_device(d.data_ptr(), n)
        f.evaluate()
        ts = []
        for _ in range(3):
            f.evaluate()
            ts.append(f.timings()["total"])
        f.dipole_correction()
        outs[prec] = f.bodies()
        res[prec] = {"ms_per_eval": statistics.mean(ts), "evals_per_s": 1e3 / statistics.mean(ts)}
        if prec == "fp64":
            ewald_handle = f
        else:
            f.close()
    assert np.array_equal(outs["mixed"][:, :4], outs["fp64"][:, :4])  # same tree, same body order
    tgt = outs["fp64"].copy()
    tgt[:, 4:] = 0
    ewald = {}
    for name, alpha in (("alpha_ksize_over_cycle", 11 / cyc), ("alpha_10_over_2pi", 10 / cyc)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ewald[name] = ewald_handle.ewald(tgt, ksize=11, alpha=alpha)
        ewald[name + "_s"] = time.perf_counter() - t0
    ewald_handle.close()

    def measures(o, ew):
        e, e0 = float((o[:, 4] * o[:, 3]).sum()), float((ew[:, 4] * ew[:, 3]).sum())
        return {"energy_rel_err": abs(e - e0) / abs(e0),
                "force_rel_l2": float(np.sqrt(((o[:, 5:] - ew[:, 5:]) ** 2).sum() / (ew[:, 5:] ** 2).sum()))}

    ew = ewald["alpha_ksize_over_cycle"]
    for prec in ("mixed", "fp64"):
        m = measures(outs[prec], ew)
        res[prec]["energy_rel_err_vs_ewald"] = m["energy_rel_err"]
        res[prec]["force_rel_l2_vs_ewald"] = m["force_rel_l2"]
    res["mixed_over_fp64_speedup"] = res["fp64"]["ms_per_eval"] / res["mixed"]["ms_per_eval"]
    res["ewald"] = {"targets": n, "alpha": 11 / cyc, "ksize": 11, "cutoff": cyc / 2,
                    "seconds": ewald["alpha_ksize_over_cycle_s"],
                    "vs_alpha_10_over_2pi": measures(ewald["alpha_10_over_2pi"], ew)}
    res["workload"] = (f"{n} bodies uniform in a cube of side 2 pi, P=10, theta=0.4, ncrit=64, images=3; errors "
                       "over all bodies against the GPU FP64 Ewald sum, as 3dp/fmm.cxx:96-111 measures them")
    return res


def two_d_leg(FMM, torch, flush, local_rank, n=1 << 20, P=10, ncrit=8, steps=3, warmup=2):
    """The 2D variant (2d/: log kernel, complex series of P terms,
    quadtree), FP64: N bodies as the reference's 2d driver makes them
    (drand48 seed 0, uniform in [-pi, pi]^2, 2d/fmm.cxx:21-35), its P = 10 and
    ncrit = 8, theta = 0.4.  Device ms per evaluation, error against the GPU
    FP64 direct sum on 1000 targets, and the reference's own 2d build (lazy
    traversal, all host cores) on the same bodies, timed here on the host."""
    import oracle

    xyq = oracle.reference_bodies_2d(n, 0)
    f = FMM(P=P, ncrit=ncrit, theta=0.4, dim=2, device=local_rank)
    f.set_bodies(xyq)
    ts = []
    for s in range(warmup + steps):
        flush.zero_()
        torch.cuda.synchronize()
        f.evaluate()
        if s >= warmup:
            ts.append(f.timings()["total"])
    out = f.bodies()
    sample = np.arange(0, n, max(1, n // 1000))[:1000]
    tgt = out[sample].copy()
    tgt[:, 3:] = 0
    d = f.direct(tgt)
    err = {"p": float(np.sqrt(((out[sample, 3] - d[:, 3]) ** 2).sum() / (d[:, 3] ** 2).sum())),
           "F": float(np.sqrt(((out[sample, 4:] - d[:, 4:]) ** 2).sum() / (d[:, 4:] ** 2).sum()))}
    f.close()
    ms = statistics.mean(ts)
    res = {"workload": f"2d: {n} bodies (drand48 seed 0) in [-pi,pi]^2, P={P}, ncrit={ncrit}, theta=0.4, FP64",
           "ms_per_eval": ms, "evals_per_s": 1e3 / ms, "error_vs_direct": err}
    threads = os.cpu_count() or 1
    try:
        ref = oracle.Fmm2D("ref")
        t0 = time.perf_counter()
        ref.fmm(xyq, P, ncrit, 0.4, 0, 0.0)
        dt = time.perf_counter() - t0
        rb = ref.bodies()
        res["cpu_reference"] = {"value": 1.0 / dt, "unit": "evals/s", "cores": threads, "kind": "reference",
                                "sample": f"one evaluation of the same {n}-body 2d workload (reference lazy "
                                          f"traversal, OpenMP {threads} threads), {dt:.2f} s"}
        res["gpu_over_cpu_reference"] = dt * 1e3 / ms
        res["rel_l2_p_vs_reference_fmm"] = float(np.sqrt(((out[:, 3] - rb[:, 3]) ** 2).sum() / (rb[:, 3] ** 2).sum()))
    except Exception as e:  # the reference build missing is reported, not hidden
        res["cpu_reference"] = {"unavailable": str(e)}
    return res


def run_ours(a, rank, world, local_rank):
    import torch

    import minimal_b200
    from minimal_b200 import FMM, drand48_bodies

    dist = world > 1
    if dist:
        import datetime

        import torch.distributed as td

        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    def barrier_max(x):
        return max_over_ranks(x, dev)

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
    torch.cuda.synchronize()
    if dist:
        import torch.distributed as td

        td.barrier()
    clocks.start()
    t0 = time.perf_counter()
    phase, launches = timed_steps(fmm, a.steps, flush, torch)
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

    # The same steps pipelined: a second handle on a second host thread, so
    # that one handle's host copies run while the other evaluates (each step
    # still copies its own records in and its results out).  Reported beside
    # the serial figure above, which stays the e2e number.
    pipe_local = -1.0
    try:
        import threading

        fmm2 = FMM(P=a.P, ncrit=a.ncrit, theta=a.theta, precision=a.precision, device=local_rank)
        h_in2 = torch.from_numpy(rec).pin_memory()
        h_out2 = torch.empty((a.n, 8), dtype=torch.float64).pin_memory()
        per_thread = max(2, min(a.steps, 5))
        errs = []

        def drive(f, hin, hout, k):
            try:
                for _ in range(k):
                    f._check(lib.exafmm_b200_set_bodies(f.h, hin.data_ptr(), a.n, minimal_b200.HOST))
                    f._check(lib.exafmm_b200_evaluate(f.h))
                    f._check(lib.exafmm_b200_get_bodies(f.h, hout.data_ptr(), minimal_b200.HOST))
            except Exception as e:
                errs.append(e)

        drive(fmm2, h_in2, h_out2, 1)  # warm the second handle
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ths = [threading.Thread(target=drive, args=(fmm, h_in, h_out, per_thread)),
               threading.Thread(target=drive, args=(fmm2, h_in2, h_out2, per_thread))]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        pipe_local = (time.perf_counter() - t1) * 1e3 / (2 * per_thread) if not errs else -1.0
        fmm2.close()
    except Exception:
        pipe_local = -1.0
    # every rank takes part in both reductions (a rank that failed reports -1)
    failed_any = barrier_max(1.0 if pipe_local < 0 else 0.0) > 0.5
    pipe_ms = barrier_max(pipe_local)
    if failed_any:
        pipe_ms = None

    if rank != 0:
        fmm.close()
        if dist:
            td.barrier()
            td.destroy_process_group()
        return

    err = errors_vs_direct(fmm, a.n, h_out.numpy().copy())

    # roofline: the near field (FP32 pipe in the mixed form, FP64 in the
    # plain form) dominates; the tensor-core M2L is reported beside it
    pairs, n_m2l = pair_count(fmm)
    mixed = a.precision == "mixed"
    peak_fma = fmm.fma_peak("mixed" if mixed else "fp64")
    iso = isolated_phases(fmm, 3, flush, torch)
    m2l_ms = statistics.mean(iso["m2l"])
    p2p_ms = statistics.mean(iso["p2p"])
    p2p_flops = pairs * 20
    m2l_flops = n_m2l * m2l_flops_per_pair(a.P)
    p2p_tf = p2p_flops / (p2p_ms * 1e-3) / 1e12
    m2l_tf = m2l_flops / (m2l_ms * 1e-3) / 1e12
    peaks = {}
    ppath = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(ppath):
        peaks = json.load(open(ppath))
    traffic = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath))
    kern = "k_p2p_cta<1>" if mixed else "k_p2p_cta<0>"
    roof = {"bound": "fp32" if mixed else "fp64", "kernel": kern + " (P2P near field)", "achieved": p2p_tf,
            "peak": peak_fma, "unit": "TFLOP/s", "frac": p2p_tf / peak_fma,
            "traffic": traffic.get(kern, {}).get("bytes_per_launch_1M"),
            "peak_source": ("measured FP32" if mixed else "measured FP64") +
                           " FMA-pipe peak on this GPU (dependent-chain microbenchmark, exafmm_b200_fma_peak); "
                           "the pool's MEASURED_PEAKS.json has no FP32/FP64 figure",
            "flops_per_launch": p2p_flops, "flops_per_unit": "20 per body pair (3d/kernel.h:133-142)",
            "time": "P2P phase events of 3 step-API evaluations after the timed region, the near field "
                    "alone on the GPU (source conversion + near-field kernel)",
            "in_step_ms": statistics.mean(phase["p2p"]),
            "in_step_note": "P2P phase events inside the timed evaluations, where the near field shares the "
                            "SMs with the far field on a second stream"}
    roof_m2l = None
    if mixed and peaks.get("bf16_tflops"):
        roof_m2l = {"bound": "tensor", "kernel": "k_m2l_tc (grouped M2L, tcgen05 split-FP16) + grouping",
                    "achieved": m2l_tf, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                    "frac": m2l_tf / peaks["bf16_tflops"], "peak_source": "MEASURED_PEAKS.json bf16 burst",
                    "flops_per_launch": m2l_flops,
                    "flops_per_unit": f"{m2l_flops_per_pair(a.P)} per M2L pair (dense realified, truncated)",
                    "time": "M2L phase events of 3 step-API evaluations after the timed region (grouping "
                            "kernels + contraction + residual, alone on the GPU)",
                    "traffic": traffic.get("k_m2l_tc", {}).get("bytes_per_launch_1M")}

    extra = {}
    other = "fp64" if mixed else "mixed"
    if a.legs != "none":
        extra[f"{other}_same_workload"] = form_leg(FMM, d_rec, a.n, a.P, a, other, flush, torch, local_rank)
        if mixed:
            extra["mixed_over_fp64_speedup"] = extra["fp64_same_workload"]["ms_per_eval"] / ms_dev
    if a.legs == "all" and world == 1:  # the side legs run at N = 1 only
        extra["p12"] = {prec: form_leg(FMM, d_rec, a.n, 12, a, prec, flush, torch, local_rank)
                        for prec in ("mixed", "fp64")}
        extra["p12"]["mixed_over_fp64_speedup"] = (extra["p12"]["fp64"]["ms_per_eval"] /
                                                   extra["p12"]["mixed"]["ms_per_eval"])
        extra["same_positions_new_charges"] = reevaluate_leg(fmm, a.n, flush, torch, ms_dev)
        extra["batched"] = batched_leg(FMM, torch, dev, local_rank)
        extra["periodic"] = periodic_leg(FMM, torch, dev, local_rank, a.n)
        try:  # a side leg: its failure is reported, the headline line still prints
            extra["plummer_4M"] = plummer_leg(FMM, flush, torch, local_rank)
        except Exception as e:
            extra["plummer_4M"] = {"error": f"{type(e).__name__}: {e}"}
        try:
            extra["two_d"] = two_d_leg(FMM, torch, flush, local_rank)
        except Exception as e:
            extra["two_d"] = {"error": f"{type(e).__name__}: {e}"}

    cpu = None
    if not a.no_cpu_baseline and world == 1:
        try:
            cpu = cpu_baseline(xq, a)
        except Exception as e:  # the reference build missing is reported, not hidden
            cpu = {"unavailable": str(e)}

    line = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f16x3 tensor (mixed), f64 root/coefficients" if mixed else "f64",
            "data": "synthetic (drand48, the reference driver's generator; seed = rank)",
            "config": dict(workload(a), parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                           precision=a.precision),
            "e2e": {"value": world * 1e3 / e2e_ms, "unit": "evals/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": a.n * 64, "d2h_bytes_per_step": a.n * 64},
            "e2e_pipelined": None if pipe_ms is None else {
                "value": world * 1e3 / pipe_ms, "unit": "evals/s", "ms_per_step": pipe_ms,
                "h2d_bytes_per_step": a.n * 64, "d2h_bytes_per_step": a.n * 64,
                "mode": "two handles on two host threads, each step set_bodies (pinned host -> device), "
                        "evaluate, get_bodies (device -> pinned host); one handle's copies run during the "
                        "other's evaluation; wall clock over all steps"},
            "gpu_launches": launches, "roofline": roof, "roofline_m2l": roof_m2l, "cpu_baseline": cpu,
            "clocks": clk, "phases_ms": {k: statistics.mean(v) for k, v in phase.items()},
            "wall_ms_per_step": wall * 1e3 / a.steps, "error_vs_direct": err,
            "work": {"cells": fmm.num_cells(), "m2l_pairs": n_m2l, "p2p_body_pairs": pairs}}
    line.update(extra)
    print(json.dumps(line), flush=True)
    fmm.close()
    if dist:
        td.barrier()
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
