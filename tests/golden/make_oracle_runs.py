"""Generate oracle runs too long to repeat inside the test suite.

    make -C oracle oracle && python tests/golden/make_oracle_runs.py

Writes oracle_chain16_chi32.json: config 1 end to end (the n=16 chain of
tessera_b200.instances.chain_nn(n=16, seed=1), J ~ N(0, 1), h ~ N(0, 0.5), linear schedule,
T=20, dt=0.05: 400 second-order steps at chi=32) through the oracle's accurate-SVD mode,
which is the reference's MPS-TEBD algorithm (cuda/src/mps.cpp:295-381: keep rule, gauge, gate
order) with a one-sided Jacobi SVD.  It stores the readout spins and energy, <H>, max_trunc
and the per-step qubit-0 entropy, and the run's own sensitivity: the largest change of <H>
and of the entropy trace over three re-runs with h, J and B(s) moved by +4, -4 and +8 ulps.
A run takes about two minutes on one core; the four run in parallel processes.
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def _run(eps: float):
    from oracle.oracle import Instance, Oracle
    from tessera_b200 import instances
    p = instances.chain_nn(n=16, seed=1, T=20.0, dt=0.05, chi=32)
    inst = Instance(p.h * (1 + eps), p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew * (1 + eps))
    o = Oracle().mps_anneal(inst, p.sa, p.sb * (1 + eps), p.dt, 32, accurate_svd=True)
    return {"spins": [int(x) for x in o.spins], "energy": o.energy, "expected_energy": o.expected_energy,
            "max_trunc": o.max_trunc, "updates": o.updates, "entropy": [float(x) for x in o.entropy]}


def main() -> None:
    eps = [0.0, 4e-16, -4e-16, 8e-16]
    with mp.get_context("spawn").Pool(len(eps)) as pool:
        runs = pool.map(_run, eps)
    base = runs[0]
    dh = max(abs(r["expected_energy"] - base["expected_energy"]) for r in runs[1:])
    ds = max(float(np.max(np.abs(np.array(r["entropy"]) - np.array(base["entropy"])))) for r in runs[1:])
    out = {"workload": "chain_nn(n=16, seed=1), linear T=20 dt=0.05 (400 steps), chi=32, accurate-SVD oracle",
           "out": base, "sensitivity": {"expected_energy": dh, "entropy": ds},
           "spins_stable": all(r["spins"] == base["spins"] for r in runs[1:])}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_chain16_chi32.json")
    with open(path, "w") as f:
        json.dump(out, f)
    print(f"wrote {path}: <H> {base['expected_energy']:.12f} (sensitivity {dh:.2e}), entropy sensitivity {ds:.2e}")


if __name__ == "__main__":
    main()
