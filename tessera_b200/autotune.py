"""Measured choice of the batched Jacobi kernel for a workload (the engine's autotuner).

The batched engine has three SVD kernels for a large theta (the block-row-cyclic column-pair
Jacobi with blocks of 4 or 8 columns, and the block-Gram Jacobi), the column-pair Jacobi with or
without its pivoted-LQ preconditioner, and, for complex64, two bond contractions (CUDA cores or
tcgen05 tensor cores).  Which is fastest depends on the bond dimension, the precision, the
spectra and how many instances share the GPU.  ``tune`` times each candidate
on the workload itself: a batched session of the given instances, each MPS a seeded random state
with every bond at its cap, a few interior gate slots per candidate, CUDA events around them.
The choice is cached in a JSON file keyed by (chi, precision, instance count, GPU name), so a
later run of the same workload reuses it without measuring.

Every candidate computes the same rotations to rounding; the choice changes speed, not results
beyond rounding.
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import asdict, dataclass

from . import ffi

CACHE = os.path.join(os.path.expanduser("~"), ".cache", "tessera_b200", "autotune.json")


@dataclass
class Choice:
    jacobi_block: int
    theta_tensor_cores: bool
    ms_per_update: float
    measured: dict
    jacobi_precondition: int = 1  # 1 on, 2 off (tessera_qa_config.jacobi_precondition)


def _gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


def candidates(precision: str):
    """(jacobi_block, theta_tensor_cores, jacobi_precondition) triples; the block-Gram kernel (32)
    takes no preconditioner."""
    out = [(8, False, 1), (8, False, 2), (4, False, 1), (32, False, 2)]
    if precision == "c64":
        out += [(16, False, 1), (16, False, 2), (16, True, 1)]
    return out


def _time_candidate(problems, chi, precision, block, tc, q0, gates, seed=1234, precond=1):
    s = ffi.Session.batch(problems, chi=chi, precision=precision, jacobi_block=block, theta_tensor_cores=tc,
                          jacobi_precondition=precond)
    try:
        s.randomize(seed)
        k = problems[0].steps // 2
        s.run_gates(k, q0, q0 + 1)  # warm-up slot (kernel load, caches)
        s.sync()
        s.run_gates(k, q0 + 1, q0 + 1 + gates)
        r = s.sync()
        if r.status:
            return None
        return r.device_ms / max(1, gates * len(problems))
    finally:
        s.close()


def tune(problems, chi: int, precision: str = "c128", gates: int = 2, q0: int | None = None, cache: str | None = CACHE,
         force: bool = False) -> Choice:
    """Fastest (jacobi_block, theta_tensor_cores, jacobi_precondition) for a batched run of
    `problems` at bond cap `chi`."""
    key = f"chi={chi}|{precision}|B={len(problems)}|{_gpu_name()}|lq"
    if cache and not force and os.path.exists(cache):
        try:
            with open(cache) as f:
                d = json.load(f)
            if key in d:
                return Choice(**d[key])
        except Exception:
            pass
    n = problems[0].n
    if q0 is None:
        q0 = 16 * min(32, n // 4)  # interior gate slots (saturated bonds for long chains)
    ups = min(p.updates_per_step() for p in problems)
    q0 = max(0, min(q0, ups - 1 - gates))
    gates = min(gates, ups - 1 - q0)
    measured = {}
    for block, tc, pc in candidates(precision):
        t0 = time.perf_counter()
        ms = _time_candidate(problems, chi, precision, block, tc, q0, gates, precond=pc)
        measured[f"block={block},tc={int(tc)},lq={int(pc == 1)}"] = {"ms_per_update": ms,
                                                                   "wall_s": time.perf_counter() - t0}
    ok = {k: v["ms_per_update"] for k, v in measured.items() if v["ms_per_update"] is not None}
    if not ok:
        raise RuntimeError("no Jacobi kernel candidate ran cleanly on this workload")
    best = min(ok, key=ok.get)
    f = dict(kv.split("=") for kv in best.split(","))
    choice = Choice(int(f["block"]), f["tc"] == "1", ok[best], measured, 1 if f["lq"] == "1" else 2)
    if cache:
        try:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            d = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    d = json.load(f)
            d[key] = asdict(choice)
            with open(cache, "w") as f:
                json.dump(d, f, indent=1)
        except Exception:
            pass
    return choice
