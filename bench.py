#!/usr/bin/env python
"""Benchmark: TEBD two-site updates/s at chi=256.

Workload: the n=128 chain with couplings to neighbours at distances 1..4 (J ~ U(-1,1), h = 0,
linear schedule T=50, dt=0.02 -> 2500 steps), chi=256, complex128, each ZZ edge through the
swap network in the reference's order (1998 two-site updates per Trotter step).  Every
timed update is a saturated chi=256 update: each MPS starts as a seeded random state with
every bond at its cap min(256, 2^i, 2^(n-i)).

Default (--batch 148): 148 independent instances of that workload (seeds 2..149, one per
SM) in one batched session; a bench step is 8 consecutive gate slots of the ZZ block of the
Trotter step at s = 0.5 on every instance (148 x 8 two-site updates, each instance in its
own reference gate order).  --batch 1 runs the plain single-instance engine, whose SVDs use
all SMs cooperatively; its rate is also reported beside the batched line.

  python bench.py [--gpus N --steps K --warmup W]            # libtessera_qa.so
  python bench.py --impl reference [...]                     # the reference's CPU engine

Printed: one JSON line on rank 0.  `value` = updates/s over all ranks with the MPS resident
in HBM (CUDA events on the session stream, max over ranks); `e2e` = the same metric through
the host-buffer C ABI call tessera_qa_session_run_host (per step: h, J and the schedule
copied from pinned host memory, run, statistics read back); `roofline` = the Jacobi-SVD
kernel's algorithmic bytes per launch over its average launch time; `cpu_baseline` = the
reference engine timed on this host's cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TEBD two-site updates/s at chi=256"
UNIT = "two-site updates/s"
MID_STEP = 1250  # s = 1250/2499 ~ 0.5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=148, help="instances per GPU (1 = plain single-instance engine)")
    ap.add_argument("--gates", type=int, default=8, help="gate slots per bench step")
    ap.add_argument("--impl", choices=["tessera", "reference"], default="tessera")
    ap.add_argument("--ref-chi", type=int, default=64,
                    help="bond dimension the reference arm times (scaled to --chi when smaller)")
    ap.add_argument("--precision", choices=["c128", "c64"], default="c128")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--dmax", type=int, default=4)
    ap.add_argument("--chi", type=int, default=256)
    ap.add_argument("--jacobi-block", type=int, default=0)
    ap.add_argument("--graded-decay", type=float, default=24.0,
                    help="also time the step on random MPS with graded spectra (site column b scaled by "
                         "exp(-b/decay)); 0 = skip")
    ap.add_argument("--no-c64", action="store_true", help="skip the complex64 leg of a complex128 run")
    ap.add_argument("--precondition", choices=["on", "off"], default="on",
                    help="pivoted LQ of theta before the batched Jacobi (fewer sweeps)")
    ap.add_argument("--theta-tc", action="store_true",
                    help="complex64: bond contraction on the tcgen05 tensor cores (split-TF32)")
    ap.add_argument("--autotune", action="store_true",
                    help="time the batched Jacobi kernels (and, in complex64, the tensor-core contraction) on a "
                         "slice of this workload first and run the fastest (tessera_b200.autotune)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solves", action="store_true", help="skip the solves/s (chosen vs plain) measurement")
    ap.add_argument("--solve-instances", type=int, default=296, help="held-out instances for solves/s")
    ap.add_argument("--solve-T", type=float, default=10.0, help="anneal time of the solves/s workload")
    ap.add_argument("--solve-dt", type=float, default=0.1)
    ap.add_argument("--solve-chi", type=int, default=32)
    ap.add_argument("--solve-nmin", type=int, default=12, help="held-out instances: n from nmin to nmax")
    ap.add_argument("--solve-nmax", type=int, default=14)
    ap.add_argument("--solve-train", type=int, default=160, help="training instances, n from 8 to --solve-train-nmax")
    ap.add_argument("--solve-train-nmax", type=int, default=12)
    ap.add_argument("--solve-train-T", type=float, default=None, help="anneal time of the labels (default --solve-T)")
    ap.add_argument("--plain-sample", type=int, default=8, help="plain instances timed one call each")
    ap.add_argument("--plain-steps", type=int, default=None,
                    help="time the plain calls on the first k schedule steps and scale to the full schedule")
    ap.add_argument("--solves-only", action="store_true", help="run only the solves/s study; print its JSON")
    ap.add_argument("--profile-run", action="store_true",
                    help="one untimed step only (for ncu); prints no bench line")
    ap.add_argument("--profile-sv", action="store_true",
                    help="one exact state-vector anneal, n=24 (a 256 MiB state), 4 steps (the tiled gate passes, "
                         "for ncu); prints no bench line")
    ap.add_argument("--profile-anneal", action="store_true",
                    help="one batched anneal of 148 dense ER instances n=12, chi=32, T=0.3 (the small-bond resident "
                         "kernel, for ncu); prints no bench line")
    return ap.parse_args()


def workload(args, rank=0):
    from tessera_b200 import instances
    p = instances.chain_range(n=args.n, dmax=args.dmax, seed=2 + rank, T=50.0, dt=0.02, chi=args.chi)
    return p


def shard(rank: int, per_rank: int):
    """Instance indices of one rank: disjoint contiguous blocks, no data-path exchange."""
    return [rank * per_rank + b for b in range(per_rank)]


def max_over_ranks(ms: float, world: int, device: str = "cuda") -> float:
    """The step time of the job: the slowest rank's CUDA-event time (all-reduce MAX)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_status(status: int, world: int, device: str = "cuda") -> int:
    """Nonzero on every rank when any rank's run reported status bits (the largest value), so
    all ranks stop together instead of some waiting at the next collective."""
    if world <= 1:
        return int(status)
    return int(max_over_ranks(float(status), world, device=device))


def fp64_peak_tflops(dtype=None) -> float:
    """FP64 (or, with dtype=float32, FP32 CUDA-core) peak of this GPU as cuBLAS reaches it: best of
    5 GEMMs of 4096^3 (CUDA events; TF32 is off for float32 matmuls by default)."""
    import torch
    dtype = dtype or torch.float64
    a = torch.randn(4096, 4096, dtype=dtype, device="cuda")
    b = torch.randn(4096, 4096, dtype=dtype, device="cuda")
    torch.matmul(a, b)
    best = None
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    return 2.0 * 4096 ** 3 / (best / 1e3) / 1e12


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ------------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.dev), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------------
# reference CPU engine (oracle/_ref: the reference's own sources compiled here)
# ------------------------------------------------------------------------------------
def ref_update_sample(chi: int, threads: int, seed: int = 0):
    """Wall time of `threads` concurrent saturated-bond updates through the reference's own
    MPS::apply_adjacent (cuda/src/mps.cpp:41-100), one per thread on a (2 chi) x (2 chi) theta
    (ctypes releases the GIL); returns (wall seconds, per-update seconds)."""
    from oracle.oracle import Reference
    R = Reference()
    per = [0.0] * threads

    def one(k):
        sec, _ = R.saturated_update(chi, 1, seed + k)
        per[k] = float(sec[0])

    ths = [threading.Thread(target=one, args=(k,)) for k in range(threads)]
    t0 = time.perf_counter()
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return time.perf_counter() - t0, per


REF_DIRECT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "reference_update_chi256.json")


class RefModel:
    """Reference cost of saturated chi=256 updates on the host cores.  A direct chi=256 update
    (512 x 512 theta, MPS::apply_adjacent) takes about 17 minutes per thread with 16 threads
    busy, so it is measured once per pool (--ref-chi 256; profiles/reference_update_chi256.json)
    together with the same concurrency's chi=64 time.  A default step times one chi=64 update on
    every host thread at once and scales it to chi=256 by that recorded ratio, i.e. the direct
    chi=256 rate corrected by how fast this box's cores run the chi=64 update.  Without the
    record, the cost exponent between chi=64 and chi=128, timed at the same concurrency, is
    used instead."""

    def __init__(self, chi: int = 64, target: int = 256):
        self.threads = max(1, min(len(os.sched_getaffinity(0)), 64))
        self.chi, self.target = chi, target
        self.cal = None
        self.p = None
        self.t_lo = None
        if chi >= target:
            return
        if os.path.exists(REF_DIRECT):
            with open(REF_DIRECT) as f:
                rd = json.load(f)
            c = rd.get("calibration", {})
            key = f"chi{chi}_seconds"
            if rd.get("chi") == target and key in c:
                self.cal = {"t_target": rd["seconds"], "t_chi": c[key], "threads": rd["threads"],
                            "value": rd["value"]}
        if self.cal is None:
            self.t_lo, _ = ref_update_sample(chi // 2, self.threads, seed=1)

    def step(self, seed=3):
        import math
        t, _ = ref_update_sample(self.chi, self.threads, seed=seed)
        if self.chi >= self.target:
            return t, self.threads / t
        if self.cal is not None:
            return t, self.threads / (t * self.cal["t_target"] / self.cal["t_chi"])
        self.p = math.log2(t / self.t_lo)
        return t, self.threads / (t * (self.target / self.chi) ** self.p)

    def describe(self, t):
        if self.chi >= self.target:
            return (f"{self.threads} concurrent reference MPS::apply_adjacent updates of a saturated chi={self.chi} "
                    f"bond ({2 * self.chi}x{2 * self.chi} complex128 theta), measured directly: {t:.1f} s")
        head = (f"{self.threads} concurrent reference MPS::apply_adjacent updates of a saturated chi={self.chi} bond "
                f"({2 * self.chi}x{2 * self.chi} complex128 theta) took {t:.1f} s; ")
        if self.cal is not None:
            c = self.cal
            return head + (f"scaled to chi={self.target} by the ratio measured directly on this pool with "
                           f"{c['threads']} threads (chi={self.target}: {c['t_target']:.0f} s, chi={self.chi}: "
                           f"{c['t_chi']:.2f} s; the direct chi={self.target} rate was {c['value']:.4g} updates/s)")
        return head + (f"extrapolated to chi={self.target} with the cost exponent {self.p:.2f} measured between "
                       f"chi={self.chi // 2} ({self.t_lo:.2f} s) and chi={self.chi} at the same concurrency")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtessera_ref.so was not built"}))
        return
    model = RefModel(chi=min(args.ref_chi, args.chi), target=args.chi)
    for w in range(args.warmup):
        model.step(seed=10 + w)
    vals, walls = [], []
    for k in range(args.steps):
        t, v = model.step(seed=100 + k)
        vals.append(v)
        walls.append(t)
    value = statistics.mean(vals)
    p = workload(args)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(args, p),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": model.threads, "kind": "reference",
                             "sample": model.describe(statistics.mean(walls))},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def config_dict(args, p):
    return {"workload": f"chain n={args.n}, couplings at distances 1..{args.dmax}, J~U(-1,1), h=0, "
                        f"linear schedule T=50 dt=0.02, chi={args.chi}, one Trotter step at s=0.5",
            "n": args.n, "dmax": args.dmax, "chi": args.chi, "precision": args.precision,
            "updates_per_trotter_step": p.updates_per_step(), "logical_zz_per_trotter_step": p.m,
            "gate_order": "reference (edges in order, swap network, truncation after every swap)",
            "l2": "inputs larger than L2 (MPS of 2*chi^2*16 B per site x n sites)",
            "parallelism": "instance replicas (no data-path collective)"}


# ------------------------------------------------------------------------------------
# tessera engine
# ------------------------------------------------------------------------------------
def plain_rate(args, local, peak_gbs=None, peak_tflops=None):
    """Plain single-instance engine (cooperative SVD over all SMs) on one instance, same gates;
    returns (updates/s, ms per update, roofline of its SVD kernel or None)."""
    from tessera_b200 import ffi
    p = workload(args, 0)
    s = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=args.chi, precision=args.precision,
                    kernel_timing=True, device=local, jacobi_precondition=1 if args.precondition == "on" else 2)
    s.randomize(1234)
    lo = 16 * min(32, args.n // 4)
    s.run_gates(MID_STEP, lo, lo + 2)
    r0 = s.sync()
    g = max(2, args.gates // 2)
    s.run_gates(MID_STEP, lo + 2, lo + 2 + g)
    r = s.sync()
    s.close()
    n = r.svd_launches - r0.svd_launches
    ms = r.svd_ms - r0.svd_ms
    roof = None
    if n and ms > 0:
        gbs = (r.svd_bytes - r0.svd_bytes) / (ms / 1e3) / 1e9
        tfl = (r.svd_flops - r0.svd_flops) / (ms / 1e3) / 1e12
        roof = {"kernel": "k_svd (cooperative column-pair Jacobi, 512x512 theta)", "avg_launch_ms": ms / n,
                "sweeps_per_update": (r.svd_sweeps - r0.svd_sweeps) / max(r.two_site_updates - r0.two_site_updates, 1),
                "hbm": {"achieved": gbs, "unit": "GB/s", "peak": peak_gbs,
                        "frac": gbs / peak_gbs if peak_gbs else None},
                "compute": {"achieved": tfl, "unit": "TFLOP/s", "peak": peak_tflops,
                            "frac": tfl / peak_tflops if peak_tflops else None},
                "precond_avg_launch_ms": (r.precond_ms - r0.precond_ms) / n,
                "precond": "k_lq_coop (cooperative pivoted LQ, 8 rows of theta per CTA)"
                           if args.precondition == "on" else "off"}
    return g / (r.device_ms / 1e3), r.device_ms / g, roof


def c64_leg(args, probs, window, rank, world, local, peak_gbs):
    """The same timed step in complex64 (FP32 storage and rotations, FP64 reductions): the same
    instances, random start, warm-up and timed gate windows, on a complex64 batched session.
    Returns its updates/s over all ranks (device time, max over ranks), its Jacobi sweeps and
    the roofline of its Jacobi kernel against the FP32 GEMM rate measured here."""
    import torch
    import torch.distributed as dist
    from tessera_b200 import ffi
    sess = ffi.Session.batch(probs, chi=args.chi, precision="c64", kernel_timing=True, device=local,
                             jacobi_precondition=1 if args.precondition == "on" else 2)
    try:
        sess.randomize(1234 + 1000 * rank)
        for w in range(args.warmup):
            q0, q1 = window(w)
            sess.run_gates(MID_STEP, q0, q1)
        r0 = sess.sync()
        stream = torch.cuda.ExternalStream(sess.stream)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(args.steps):
            q0, q1 = window(args.warmup + k)
            sess.run_gates(MID_STEP, q0, q1)
        e1.record(stream)
        r1 = sess.sync()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        st = job_status(r1.status, world)
        if st:
            raise RuntimeError(f"engine status bits {st} in the complex64 steps (largest over ranks)")
    finally:
        sess.close()
    upd = r1.two_site_updates - r0.two_site_updates
    n = max(r1.svd_launches - r0.svd_launches, 1)
    svd_ms = r1.svd_ms - r0.svd_ms
    flops = r1.svd_flops - r0.svd_flops
    byts = r1.svd_bytes - r0.svd_bytes
    try:
        p32 = fp64_peak_tflops(torch.float32)
    except Exception:
        p32 = None
    ach = flops / (svd_ms / 1e3) / 1e12 if svd_ms else 0.0
    gbs = byts / (svd_ms / 1e3) / 1e9 if svd_ms else 0.0
    return {"value": upd * world / (ms / 1e3), "unit": UNIT, "dtype": "f32", "ms_per_step": ms / args.steps,
            "avg_sweeps": (r1.svd_sweeps - r0.svd_sweeps) / max(upd, 1),
            "precond_avg_launch_ms": (r1.precond_ms - r0.precond_ms) / n,
            "roofline": {"kernel": "k_svd_batch (complex64 column-pair Jacobi in blocks of 16)", "bound": "fp32",
                         "achieved": ach, "peak": p32, "unit": "TFLOP/s", "frac": ach / p32 if p32 else None,
                         "peak_kind": "cuBLAS SGEMM 4096^3 measured in this run (best of 5)",
                         "avg_launch_ms": svd_ms / n, "hbm_achieved_gbs": gbs,
                         "hbm_frac": gbs / peak_gbs if peak_gbs else None},
            "workload": "the headline's instances, random start, warm-up and timed gate windows in complex64 "
                        "(FP32 storage, contraction and rotations; FP64 convergence test, discarded weight, "
                        "entropy and norms)"}


def solves(args):
    """Second half of the metric: solves/s at <= 1% energy gap, chosen vs plain.

    Dense Erdos-Renyi instances (p = 0.5, J ~ U(-1,1), h ~ U(-0.2,0.2)).  The schedule GNN is
    trained here, on the GPU, from labels the engine itself generates: --solve-train training
    instances, n from 8 to --solve-train-nmax, each annealed under 16 candidate schedules
    (batched, complex64) and scored by the exact ground energy.  Then on --solve-instances
    held-out instances, n from --solve-nmin to --solve-nmax: chosen = learned knots + warm-start
    bias, batched complex64, with the linear-schedule fallback judged by the engine's own final
    energy; plain = linear schedule, complex128, one instance per call (timed on --plain-sample
    instances, over the first --plain-steps steps when given and scaled to the whole schedule;
    energies of all instances from the bit-identical batched complex128 run).  Scores are
    against the exact ground energy for n <= 24, else against the best of a large simulated-
    annealing budget on the GPU.  The learned and the linear runs are also reported each on
    their own (no fallback): the network's gain over the method without it."""
    from tessera_b200 import instances, learned
    cfg = learned.LearnConfig(T=args.solve_T, dt=args.solve_dt, chi=args.solve_chi, precision="c64")
    tcfg = learned.LearnConfig(T=args.solve_train_T or args.solve_T, dt=args.solve_dt, chi=min(args.solve_chi, 32),
                               precision="c64")
    ns = list(range(8, args.solve_train_nmax + 1))
    train = [instances.dense_er(n, 1000 + i, T=1.0) for i, n in
             enumerate((ns * (args.solve_train // len(ns) + 1))[:args.solve_train])]
    hs = list(range(args.solve_nmin, args.solve_nmax + 1))
    held = [instances.dense_er(n, 50000 + i, T=1.0) for i, n in
            enumerate((hs * (args.solve_instances // len(hs) + 1))[:args.solve_instances])]
    t0 = time.perf_counter()
    tk, _, gs, gaps = learned.label(train, tcfg, learned.candidates(count=16))
    t_label = time.perf_counter() - t0
    net = learned.ScheduleGNN(seed=1)
    t0 = time.perf_counter()
    losses = learned.train(net, train, tk, gs, epochs=100, batch=32, lr=2e-3)
    t_train = time.perf_counter() - t0
    ev = learned.evaluate(net, held, cfg, plain_sample=args.plain_sample, plain_steps=args.plain_steps)
    net.close()
    out = {"metric": "solves/s at <=1% energy gap, chosen vs plain", "unit": "solves/s",
           "chosen": ev["chosen_solves_per_s"], "plain": ev["plain_solves_per_s"],
           "ratio": ev["chosen_solves_per_s"] / ev["plain_solves_per_s"] if ev["plain_solves_per_s"] else None}
    out.update({k: v for k, v in ev.items() if k not in ("chosen_solves_per_s", "plain_solves_per_s")})
    out["train"] = {"instances": len(train), "n": [8, args.solve_train_nmax], "candidates": 16, "T": tcfg.T,
                    "chi": tcfg.chi, "label_seconds": t_label, "train_seconds": t_train, "loss_first": losses[0],
                    "loss_last": losses[-1], "best_candidate_solved": int((gaps.min(axis=1) <= 0.01).sum()),
                    "linear_solved": int((gaps[:, 0] <= 0.01).sum())}
    out["workload"] = (f"dense ER p=0.5, train {len(train)} instances n 8..{args.solve_train_nmax} (labels at "
                       f"T={tcfg.T}, chi={tcfg.chi}), held-out {len(held)} instances n {args.solve_nmin}.."
                       f"{args.solve_nmax}, T={cfg.T}, dt={cfg.dt}, chi={cfg.chi}; the full learned-schedule study "
                       "is 20k train n 8..20 and 1024 eval n 24..48 at chi=128, T=30")
    return out


def profile_anneal():
    from tessera_b200 import ffi, instances
    probs = [instances.dense_er(12, 100 + i, T=0.3, dt=0.1, chi=32) for i in range(148)]
    res = ffi.anneal_batch(probs, precision="c64", raise_on_status=False)
    print(f"profile anneal: {sum(r.two_site_updates for r in res)} updates, status "
          f"{sorted(set(r.status for r in res))}, {res[0].device_ms:.1f} ms")


def profile_sv():
    from tessera_b200 import ffi, instances
    p = instances.chain_range(n=24, dmax=2, seed=5, T=0.4, dt=0.1)
    r = ffi.sv_anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, mode=1)
    # steps + 1 sweeps of 3 tiled passes (read + write 16 B per amplitude each), the ZZ diagonal
    # read once per step (8 B, fused into a sweep), the diagonals' set-up (32 B written) and the
    # readout (24 B read)
    bytes_run = ((p.steps + 1) * 3 * 32 + p.steps * 8 + 32 + 24) * float(1 << 24)
    print(f"profile sv: n=24, {p.steps} steps, {r.device_ms:.2f} ms, norm {r.norm2:.12f}, "
          f"{bytes_run / (r.device_ms / 1e3) / 1e9:.0f} GB/s algorithmic")


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.profile_anneal:
        profile_anneal()
        return
    if args.profile_sv:
        profile_sv()
        return
    if args.solves_only:
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"solves": solves(args)}))
        return
    import numpy as np
    import torch
    import torch.distributed as dist

    from tessera_b200 import ffi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    B = max(1, args.batch)
    probs = [workload(args, i) for i in shard(rank, B)]
    p = probs[0]
    tuned = None
    if args.autotune and B > 1:
        from tessera_b200 import autotune
        ch = autotune.tune(probs, args.chi, args.precision)
        args.jacobi_block, args.theta_tc = ch.jacobi_block, ch.theta_tensor_cores
        args.precondition = "on" if ch.jacobi_precondition == 1 else "off"
        tuned = {"jacobi_block": ch.jacobi_block, "theta_tensor_cores": ch.theta_tensor_cores,
                 "jacobi_precondition": args.precondition,
                 "measured_ms_per_update": {k: v["ms_per_update"] for k, v in ch.measured.items()}}
    upd_per_step_inst = min(args.gates, p.updates_per_step())
    if B == 1:
        sess = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=args.chi, precision=args.precision,
                           jacobi_block=args.jacobi_block, kernel_timing=True, device=local,
                           jacobi_precondition=1 if args.precondition == "on" else 2)
    else:
        sess = ffi.Session.batch(probs, chi=args.chi, precision=args.precision, jacobi_block=args.jacobi_block,
                                 kernel_timing=True, device=local, theta_tensor_cores=args.theta_tc,
                                 jacobi_precondition=1 if args.precondition == "on" else 2)
    sess.randomize(1234 + 1000 * rank)
    G = upd_per_step_inst
    # Gate slots of edges (i, i+d) with 32 <= i < 96: every bond they touch sits at chi = 256
    # (the chain's bond i is capped by 2^min(i, n-i)); each edge i owns 16 consecutive slots.
    lo = 16 * min(32, args.n // 4)
    span = max(G, 16 * (args.n // 2))

    def window(i):
        q0 = lo + (i * G) % max(1, span - G + 1)
        return q0, min(q0 + G, p.updates_per_step())

    def step(i):
        q0, q1 = window(i)
        sess.run_gates(MID_STEP, q0, q1)

    if args.profile_run:
        step(0)
        r = sess.sync()
        print(f"profile run: {r.two_site_updates} updates, status {r.status}, {r.device_ms:.1f} ms")
        return
    for w in range(args.warmup):
        step(w)
    r0 = sess.sync()
    stream = torch.cuda.ExternalStream(sess.stream)
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        step(args.warmup + k)
    e1.record(stream)
    r1 = sess.sync()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world)
    updates = r1.two_site_updates - r0.two_site_updates
    assert updates == B * G * args.steps, (updates, B, G)
    st = job_status(r1.status, world)
    if st:
        raise RuntimeError(f"engine status bits {st} during the timed steps (largest over ranks)")
    value = updates * world / (ms_max / 1e3)
    svd_n = r1.svd_launches - r0.svd_launches
    svd_ms = r1.svd_ms - r0.svd_ms
    lq_ms = r1.precond_ms - r0.precond_ms
    svd_bytes = r1.svd_bytes - r0.svd_bytes
    svd_flops = r1.svd_flops - r0.svd_flops
    launches = r1.kernel_launches - r0.kernel_launches
    sweeps = (r1.svd_sweeps - r0.svd_sweeps) / max(updates, 1)
    peak, peak_kind = peaks()
    achieved = (svd_bytes / svd_n) / (svd_ms / svd_n / 1e3) / 1e9 if svd_n else 0.0
    traffic = None
    tf = os.path.join(ROOT, "profiles", "k_svd_traffic.json")
    if os.path.exists(tf):
        try:
            with open(tf) as f:
                d = json.load(f)
            if (d.get("chi") == args.chi and d.get("precision") == args.precision and d.get("batch") == B
                    and d.get("jacobi_precondition", "off") == args.precondition):
                traffic = d.get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    if B == 1:
        kname = "k_svd (cooperative column-pair Jacobi, 512x512 theta)"
    elif args.jacobi_block == 32:
        kname = "k_svd_bgj_batch (block-Gram Jacobi, one CTA per 512x512 theta)"
    else:
        bw = args.jacobi_block or (16 if args.precision == "c64" else 8)
        kname = f"k_svd_batch (column-pair Jacobi in blocks of {max(4, bw)}, one CTA per 512x512 theta)"
    roofline = {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": traffic, "avg_launch_ms": svd_ms / max(svd_n, 1),
                "algorithmic_bytes_per_launch": svd_bytes / max(svd_n, 1), "avg_sweeps": sweeps,
                "svd_share_of_step": svd_ms / ms if ms else None}

    # the Jacobi arithmetic against the peak of the pipe it runs on: complex128 computes its dot
    # products and rotations in FP64; complex64 in FP32 (FP64 only for the per-pair cross-lane sums,
    # the convergence test and the rotation angle)
    c64 = args.precision == "c64"
    try:
        p64 = fp64_peak_tflops(torch.float32 if c64 else None)
    except Exception:
        p64 = None
    ach64 = svd_flops / (svd_ms / 1e3) / 1e12 if svd_ms else 0.0
    compute_roofline = {"kernel": kname, "bound": "fp32" if c64 else "fp64", "achieved": ach64, "peak": p64,
                        "unit": "TFLOP/s", "frac": ach64 / p64 if p64 else None,
                        "peak_kind": f"cuBLAS {'SGEMM' if c64 else 'DGEMM'} 4096^3 measured in this run (best of 5)",
                        "flops_per_launch": svd_flops / max(svd_n, 1)}

    # the pivoted-LQ preconditioner (k_lq_batch): its own launches, timed apart from the Jacobi;
    # algorithmic bytes per theta: one read for the row norms, then per elimination step one read
    # of the trailing block and one write of column k, and per panel of 8 steps one read and one
    # write of the trailing block (the delayed updates)
    precond = None
    if B > 1 and args.precondition == "on" and lq_ms > 0:
        R = Nc = 2 * args.chi
        esz = 16 if args.precision == "c128" else 8
        km = min(R, Nc)
        lq_bytes = esz * (R * Nc + sum((R - k) * (Nc - k) + (R - k) for k in range(km))
                          + sum(2 * (R - k) * (Nc - k) for k in range(8, km + 1, 8)))
        lq_per_launch = B * lq_bytes
        lq_avg = lq_ms / max(svd_n, 1)
        precond = {"kernel": "k_lq_batch (row-pivoted Householder LQ, one CTA per 512x512 theta)",
                   "avg_launch_ms": lq_avg, "share_of_step": lq_ms / ms if ms else None,
                   "algorithmic_bytes_per_launch": lq_per_launch,
                   "achieved": lq_per_launch / (lq_avg / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                   "frac": lq_per_launch / (lq_avg / 1e3) / 1e9 / peak}

    # ---- e2e: host-buffer ABI call per step (values from pinned host memory, stats back) ----
    e2e = None
    if not args.no_e2e:
        pinned = []
        for q in probs:
            cp = type(q)(*(torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
                           if isinstance(x, np.ndarray) else x for x in
                           (q.h, q.ei, q.ej, q.ew, q.sa, q.sb, q.dt, q.chi, q.name)))
            pinned.append(cp)
        h2d = sum(q.h.nbytes + q.ew.nbytes + 2 * q.ei.nbytes + q.sa.nbytes + q.sb.nbytes for q in pinned)
        # the same work as the device-timed region: the same random start, the same warm-up
        # windows (untimed), then the same timed windows, each step one host-buffer call
        sess.randomize(1234 + 1000 * rank)
        for w in range(args.warmup):
            step(w)
        sess.sync()
        walls = []
        e2e_status = 0
        for i in range(args.steps):
            q0, q1 = window(args.warmup + i)
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            rr = sess.run_host(pinned, MID_STEP, q0, q1)
            walls.append(time.perf_counter() - t0)
            e2e_status |= rr.status
        st = job_status(e2e_status, world)
        if st:
            raise RuntimeError(f"engine status bits {st} in the e2e step (largest over ranks)")
        wall = max_over_ranks(1e3 * sum(walls), world) / 1e3  # the slowest rank's calls
        e2e = {"value": B * G * world * args.steps / wall, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": 128 * B,
               "api": "tessera_qa_session_run_host (h, J, schedule of every instance from pinned host memory -> "
                      f"{G} gate slots -> run statistics to host)"}

    # ---- the same step on states whose spectra fall off like a TEBD state's Schmidt values ----
    graded = None
    if args.graded_decay > 0 and B > 1:
        sess.randomize(1234 + 1000 * rank, decay=args.graded_decay)
        for w in range(args.warmup):
            step(w)
        g0 = sess.sync()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for k in range(args.steps):
            step(args.warmup + k)
        e1.record(stream)
        g1 = sess.sync()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        gms = max_over_ranks(e0.elapsed_time(e1), world)
        gup = g1.two_site_updates - g0.two_site_updates
        st = job_status(g1.status, world)
        if st:
            raise RuntimeError(f"engine status bits {st} in the graded-spectrum steps (largest over ranks)")
        gn = g1.svd_launches - g0.svd_launches
        graded = {"value": gup * world / (gms / 1e3), "unit": UNIT, "decay": args.graded_decay,
                  "avg_sweeps": (g1.svd_sweeps - g0.svd_sweeps) / max(gup, 1),
                  "svd_avg_launch_ms": (g1.svd_ms - g0.svd_ms) / max(gn, 1),
                  "precond_avg_launch_ms": (g1.precond_ms - g0.precond_ms) / max(gn, 1),
                  "workload": "the headline's instances, gate windows and step count on seeded random MPS whose "
                              f"site column b is scaled by exp(-b/{args.graded_decay:g}): each theta's singular "
                              "values fall off like a TEBD state's Schmidt values (the 256th ~1e-7 of the largest "
                              "before the gate) instead of staying flat"}

    c64_line = None
    if B > 1 and args.precision == "c128" and not args.no_c64:
        sess.close()  # the complex64 session takes the memory the complex128 one held
        sess = None
        c64_line = c64_leg(args, probs, window, rank, world, local, peak)

    plain = None
    if B > 1 and rank == 0:
        if sess is not None:
            sess.close()
        try:
            pr, pms, proof = plain_rate(args, local, peak, p64)
            plain = {"value": pr, "unit": UNIT, "ms_per_update": pms,
                     "engine": "plain single-instance, cooperative SVD across all SMs", "roofline": proof}
        except Exception as exc:
            plain = {"value": None, "error": str(exc)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle.oracle import Reference
            if Reference.available():
                model = RefModel(chi=min(args.ref_chi, args.chi), target=args.chi)
                tw, v = model.step()
                cpu = {"value": v, "unit": UNIT, "cores": model.threads, "kind": "reference",
                       "sample": model.describe(tw)}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {exc}"}

    sol = None
    if rank == 0 and world == 1 and not args.no_solves:
        try:
            sol = solves(args)
        except Exception as exc:
            sol = {"value": None, "error": str(exc)}

    if rank == 0:
        cfg = config_dict(args, p)
        cfg.update({"jacobi_block": args.jacobi_block, "theta_tensor_cores": bool(args.theta_tc), "autotune": tuned,
                    "jacobi_precondition": args.precondition})
        cfg.update({"instances_per_gpu": B, "gates_per_step": G,
                    "step": f"{G} consecutive gate slots of the Trotter step at s=0.5 on each of {B} instances"})
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "c128" else "f32",
                "data": "synthetic: seeded Ising instances (PCG64 seeds 2..) and seeded random MPS with every "
                        "bond at its cap",
                "config": cfg, "roofline": roofline, "compute_roofline": compute_roofline, "preconditioner": precond,
                "graded_spectra": graded, "complex64": c64_line,
                "cpu_baseline": cpu,
                "e2e": e2e,
                "gpu_launches": launches, "clocks": ck, "plain_single_instance": plain, "solves": sol,
                "max_trunc_in_timed_steps": r1.max_trunc}
        print(json.dumps(line))
    if sess is not None and (B == 1 or rank != 0):
        sess.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
