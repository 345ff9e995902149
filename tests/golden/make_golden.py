"""Generate the golden fixtures in this folder from the reference engine itself.

Run where the reference sources are mounted (they are compiled by oracle/Makefile into
oracle/_ref/libtessera_ref.so):

    TESSERA_REF_ROOT=<reference checkout> make -C oracle && python tests/golden/make_golden.py

Writes reference_cases.json: every case holds its inputs (instance, schedule, dt, chi,
zz_substeps) and the reference's outputs (spins, energy, expected_energy, prob,
max_trunc, entropy trace), plus reference SVD spectra and the reference's linalg
known-answer values.  Each case also records whether the reference's Gram-matrix SVD
reconstructed every theta to 1e-8 on that run ("reference_svd_sound"): where it did not,
the reference's outputs carry its SVD errors and parity is checked against the exact
state vector and the oracle's accurate-SVD mode instead.  Cases follow the reference's own tests
(cuda/tests/test_mps.cpp:55-174, cuda/tests/test_linalg.cpp:29-98) and add
below-exact-chi chains, where the truncation rule and the gate order matter.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Instance, Oracle, Reference, smooth_schedule  # noqa: E402
from tessera_b200 import instances  # noqa: E402


def inst_dict(inst):
    return {"h": list(map(float, inst.h)), "ei": list(map(int, inst.ei)), "ej": list(map(int, inst.ej)),
            "ew": list(map(float, inst.ew))}


def schedule_of(spec):
    kind, steps = spec
    return smooth_schedule(steps) if kind == "smooth" else instances.linear(steps)


ORACLE = None


def run_case(R, name, inst, spec, dt, chi, zz=1, tags=()):
    sa, sb = schedule_of(spec)
    t0 = time.time()
    r = R.mps_anneal(inst, sa, sb, dt, chi, zz)
    dtm = time.time() - t0
    # Soundness of the reference's Gram-matrix SVD on this run, measured by the oracle's
    # bit-identical restatement: every update's ||U S Vh - theta|| / ||theta|| <= 1e-8.
    o = ORACLE.mps_anneal(inst, sa, sb, dt, chi, zz)
    sound = o.extra["bad_updates"] == 0
    print(f"  {name}: E={r.energy:.6f} <H>={r.expected_energy:.6f} trunc={r.max_trunc:.2e} sound={sound} "
          f"({dtm:.1f}s)")
    return {"name": name, "tags": list(tags), "instance": inst_dict(inst), "schedule": list(spec), "dt": dt,
            "chi": chi, "zz_substeps": zz, "reference_svd_sound": bool(sound),
            "reference_svd_max_recon_err": float(o.extra["max_recon"]),
            "out": {"spins": list(map(int, r.spins)), "energy": r.energy,
                    "expected_energy": r.expected_energy, "prob": r.prob, "max_trunc": r.max_trunc,
                    "entropy": list(map(float, r.entropy))}}


def main():
    global ORACLE
    R = Reference()
    O = Oracle()
    ORACLE = O
    cases = []
    # cuda/tests/test_mps.cpp:79-94 -- single spin, ferromagnetic pair.
    cases.append(run_case(R, "single_spin", Instance(np.array([1.0]), np.zeros(0, int), np.zeros(0, int),
                                                     np.zeros(0)), ("smooth", 300), 0.1, 16, tags=("kat",)))
    cases.append(run_case(R, "ferro_pair", Instance(np.zeros(2), np.array([0]), np.array([1]),
                                                    np.array([1.0])), ("smooth", 400), 0.1, 16, tags=("kat",)))
    # cuda/tests/test_mps.cpp:99-123 -- n=6 dense, mt19937_64(123), exact chi = 8.
    for t in range(6):
        inst = O.mt_dense_instance(123, 6, 6, t)
        cases.append(run_case(R, f"dense6_seed123_t{t}", inst, ("smooth", 1200), 0.08, 8, tags=("exact_chi",)))
    # cuda/tests/test_mps.cpp:127-141 -- frustrated 3-ring (edge (2,0) given reversed).
    ring = Instance(np.array([0.5, -0.3, 0.2]), np.array([0, 1, 2]), np.array([1, 2, 0]),
                    np.array([-1.0, -1.0, -1.0]))
    for T in (20.0, 80.0, 320.0):
        cases.append(run_case(R, f"ring3_T{int(T)}", ring, ("smooth", int(T / 0.1)), 0.1, 4, tags=("ring",)))
    # cuda/tests/test_mps.cpp:144-152 -- entanglement peak.
    cases.append(run_case(R, "entropy_pair", Instance(np.array([0.3, -0.3]), np.array([0]), np.array([1]),
                                                      np.array([-1.0])), ("smooth", 400), 0.1, 16,
                          tags=("entropy",)))
    # cuda/tests/test_mps.cpp:157-174 -- KNOWN_LIMIT n=8 dense, mt19937_64(7).
    cases.append(run_case(R, "known_limit_n8", O.mt_dense_instance(7, 8, 1, 0), ("smooth", 1000), 0.1, 16,
                          tags=("known_limit",)))
    # Below exact chi: truncation active, long-range swaps, zz_substeps 1 and 2.
    p = instances.chain_range(n=8, dmax=3, seed=11, T=4.0, dt=0.05, chi=4, dist="normal", hzero=False)
    inst = Instance(p.h, p.ei, p.ej, p.ew)
    cases.append(run_case(R, "range8_d3_chi4", inst, ("linear", p.steps), p.dt, 4, tags=("truncating",)))
    cases.append(run_case(R, "range8_d3_chi4_zz2", inst, ("linear", p.steps), p.dt, 4, zz=2,
                          tags=("truncating",)))
    p = instances.chain_nn(n=10, seed=1, T=5.0, dt=0.05, chi=4)
    cases.append(run_case(R, "chain10_chi4", Instance(p.h, p.ei, p.ej, p.ew), ("linear", p.steps), p.dt, 4,
                          tags=("truncating",)))
    p = instances.chain_range(n=10, dmax=4, seed=2, T=3.0, dt=0.02, chi=8)
    cases.append(run_case(R, "range10_d4_chi8", Instance(p.h, p.ei, p.ej, p.ew), ("linear", p.steps), p.dt,
                          8, tags=("truncating", "hzero")))
    # Nearest-neighbour chains below exact chi on which the reference's SVD stays sound
    # (every update reconstructs theta to 1e-8): truncation is active and the reference's
    # outputs carry only its rounding noise.
    for seed, n in ((1, 8), (2, 8), (2, 10)):
        p = instances.chain_range(n=n, dmax=1, seed=seed, T=4.0, dt=0.05, chi=4, dist="normal", hzero=False)
        cases.append(run_case(R, f"chain{n}_seed{seed}_chi4", Instance(p.h, p.ei, p.ej, p.ew), ("linear", p.steps),
                              p.dt, 4, tags=("truncating", "sound")))
    # The reference's own C ABI (dt fixed at 0.1, cuda/src/ffi.cpp:28).
    inst = O.mt_dense_instance(123, 6, 6, 1)
    a, b = smooth_schedule(100)
    e, spins, ent = R.legacy_anneal(inst, a, b, 8)
    legacy = {"instance": inst_dict(inst), "schedule": ["smooth", 100], "chi": 8,
              "energy": e, "spins": list(map(int, spins)), "entropy": list(map(float, ent))}
    # Reference SVD spectra (cuda/src/linalg.cpp:107-172) of seeded random matrices.
    rng = np.random.Generator(np.random.PCG64(99))
    svds = []
    for (r, c) in [(4, 6), (8, 8), (6, 3), (16, 16), (32, 24)]:
        A = rng.normal(size=(r, c)) + 1j * rng.normal(size=(r, c))
        _, s, _ = R.svd(A)
        svds.append({"rows": r, "cols": c, "re": A.real.ravel().tolist(), "im": A.imag.ravel().tolist(),
                     "s": list(map(float, s))})
    # cuda/tests/test_linalg.cpp known answers, evaluated by the reference.
    X = np.array([[0, 1], [1, 0]], complex)
    H3 = np.array([[2, 1 + 2j, -0.5 + 1j], [1 - 2j, -1, -1j], [-0.5 - 1j, 1j, 0.5]], complex)
    w3, _ = R.hermitian_eig(H3)
    E = R.hermitian_expm(X, complex(0, -np.pi / 2))
    linalg = {"eig_H3": list(map(float, w3)), "expm_X_re": E.real.ravel().tolist(),
              "expm_X_im": E.imag.ravel().tolist()}
    out = {"generator": "tests/golden/make_golden.py", "cases": cases, "legacy_abi": legacy, "svd": svds,
           "linalg": linalg}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
