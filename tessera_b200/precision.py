"""Precision study: the engine's complex128, complex64 and complex64-with-tensor-core modes against
the exact FP64 state vector, on the same instances.

For each instance the final MPS is contracted to its 2^n amplitudes and compared with the GPU
state vector in the engine's splitting (tessera_qa_sv_anneal, mode 1); at exact chi the only
difference is arithmetic.  Reported per mode: the relative error of <H>, the infidelity, and the
largest deviation of the Schmidt spectrum across the central cut (singular values of the
amplitudes reshaped 2^(n/2) x 2^(n/2), relative to the largest).
"""
from __future__ import annotations

import numpy as np

from . import ffi, instances


def _schmidt(psi, n):
    a = psi.reshape(2 ** (n - n // 2), 2 ** (n // 2))  # bit i = spin i: low bits are the first sites
    return np.linalg.svd(a, compute_uv=False)


def study(count=64, n=12, dmax=3, T=2.0, dt=0.1, seed0=100):
    chi = 1 << (n // 2)
    probs = [instances.chain_range(n=n, dmax=dmax, seed=seed0 + k, T=T, dt=dt, chi=chi, dist="normal", hzero=False)
             for k in range(count)]
    refs = [ffi.sv_anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=dt, mode=1, want_state=True) for p in probs]
    modes = {"c128": dict(precision="c128"), "c64": dict(precision="c64"),
             "c64_tensor_cores": dict(precision="c64", theta_tensor_cores=True)}
    out = {"instances": count, "n": n, "chi": chi, "dmax": dmax, "steps": probs[0].steps, "dt": dt}
    for name, kw in modes.items():
        res = ffi.anneal_batch(probs, want_checkpoint=True, **kw)
        de, inf, dsig = [], [], []
        for r, ref in zip(res, refs):
            psi = ffi.sites_to_dense(ffi.checkpoint_to_sites(r.checkpoint)[1])
            de.append(abs(r.expected_energy - ref.expected_energy) / max(abs(ref.expected_energy), 1e-12))
            f = abs(np.vdot(psi, ref.state)) ** 2 / (np.vdot(psi, psi).real * np.vdot(ref.state, ref.state).real)
            inf.append(1.0 - f)
            s1 = _schmidt(psi / np.sqrt(np.vdot(psi, psi).real), n)
            s0 = _schmidt(ref.state / np.sqrt(np.vdot(ref.state, ref.state).real), n)
            dsig.append(float(np.max(np.abs(s1 - s0)) / s0[0]))
        out[name] = {"energy_rel_err_max": float(np.max(de)), "energy_rel_err_mean": float(np.mean(de)),
                     "infidelity_max": float(np.max(inf)), "infidelity_mean": float(np.mean(inf)),
                     "schmidt_dev_max": float(np.max(dsig)), "status": sorted({int(r.status) for r in res})}
    return out




def mps_fidelity(a, b):
    """|<a|b>|^2 / (<a|a><b|b>) of two MPS given as site lists (Dl, 2, Dr), by left transfer
    matrices rescaled at every site."""
    def overlap(x, y):
        e = np.ones((1, 1), np.complex128)
        logs = 0.0
        for A, B in zip(x, y):
            e = sum(A[:, s, :].conj().T @ e @ B[:, s, :] for s in range(2))
            m = np.max(np.abs(e))
            e /= m
            logs += np.log(m)
        return e[0, 0], logs
    ab, lab = overlap(a, b)
    aa, laa = overlap(a, a)
    bb, lbb = overlap(b, b)
    return float(abs(ab) ** 2 / (aa.real * bb.real) * np.exp(2 * lab - laa - lbb))


MODES = {"c128": dict(precision="c128"), "c64": dict(precision="c64"),
         "c64_tensor_cores": dict(precision="c64", theta_tensor_cores=True)}


def study_exact_chi1024(count=4, n=20, dmax=2, steps=12, dt=0.25, s=0.5, seed0=400):
    """The precision study's exact-oracle half at its own size: n = 20 chains with couplings to
    distance dmax (J ~ N(0, 1), h = 0), exact chi = 1024, a window of `steps` Trotter steps at
    fixed s (the window saturates the central bond at 1024, so the central updates are
    1024 x 1024 theta through the cooperative SVD), each mode against the GPU state vector in
    the engine's splitting."""
    import time
    chi = 1 << (n // 2)
    probs = [instances.chain_range(n=n, dmax=dmax, seed=seed0 + k, T=1.0, dt=dt, chi=chi, dist="normal", hzero=True)
             for k in range(count)]
    sa = np.full(steps, 1.0 - s)
    sb = np.full(steps, s)
    refs = [ffi.sv_anneal(p.h, p.ei, p.ej, p.ew, sa, sb, dt=dt, mode=1, want_state=True) for p in probs]
    out = {"instances": count, "n": n, "chi": chi, "dmax": dmax, "steps": steps, "dt": dt, "s": s}
    for name, kw in MODES.items():
        de, inf, dsig, ms, upd, bonds = [], [], [], 0.0, 0, []
        for p, ref in zip(probs, refs):
            t0 = time.perf_counter()
            r = ffi.anneal(p.h, p.ei, p.ej, p.ew, sa, sb, dt=dt, chi=chi, want_checkpoint=True,
                           raise_on_status=False, **kw)
            ms += (time.perf_counter() - t0) * 1e3
            upd += r.two_site_updates
            bonds.append(int(r.max_bond))
            psi = ffi.sites_to_dense(ffi.checkpoint_to_sites(r.checkpoint)[1])
            de.append(abs(r.expected_energy - ref.expected_energy) / max(abs(ref.expected_energy), 1e-12))
            f = abs(np.vdot(psi, ref.state)) ** 2 / (np.vdot(psi, psi).real * np.vdot(ref.state, ref.state).real)
            inf.append(1.0 - f)
            s1 = _schmidt(psi / np.sqrt(np.vdot(psi, psi).real), n)
            s0 = _schmidt(ref.state / np.sqrt(np.vdot(ref.state, ref.state).real), n)
            dsig.append(float(np.max(np.abs(s1 - s0)) / s0[0]))
        out[name] = {"energy_rel_err_max": float(np.max(de)), "infidelity_max": float(np.max(inf)),
                     "infidelity_mean": float(np.mean(inf)), "schmidt_dev_max": float(np.max(dsig)),
                     "max_bond": max(bonds), "wall_ms_per_update": ms / max(upd, 1)}
    return out


def study_chi512(n=64, dmax=2, slots=6, seed=4):
    """The precision study's large half: the n = 64 chain with couplings to distance dmax
    (J ~ N(0, 1), h = 0), a random MPS with every interior bond at chi = 512, and `slots`
    consecutive truncating gate slots of the s = 0.5 step on interior bonds (1024 x 1024 theta),
    in each mode from the same start; each mode's state against the complex128 one (infidelity
    by MPS overlap), with the discarded weight and the device time per update."""
    p = instances.chain_range(n=n, dmax=dmax, seed=seed, T=40.0, dt=0.02, chi=512, dist="normal", hzero=True)
    step = len(p.sa) // 2
    bonds = []
    for i, j in zip(p.ei, p.ej):
        bonds += [k - 1 for k in range(int(j), int(i) + 1, -1)] + [int(i)] + [k for k in range(int(i) + 1, int(j))]
    q0 = next(q for q, b in enumerate(bonds) if b >= n // 2)
    out = {"n": n, "chi": 512, "dmax": dmax, "slots": slots, "first_slot": q0}
    states = {}
    for name, kw in MODES.items():
        sess = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=512, **kw)
        sess.randomize(seed)
        sess.run_gates(step, q0, q0 + slots)
        r = sess.sync()
        states[name] = ffi.checkpoint_to_sites(sess.save())[1]
        sess.close()
        out[name] = {"status": int(r.status), "max_trunc": float(r.max_trunc), "device_ms_per_update": r.device_ms / slots,
                     "max_sweeps": int(r.max_sweeps)}
    for name in ("c64", "c64_tensor_cores"):
        out[name]["infidelity_vs_c128"] = 1.0 - mps_fidelity(states["c128"], states[name])
    return out


if __name__ == "__main__":
    import json
    import sys
    which = sys.argv[1] if len(sys.argv) > 1 else "small"
    if which == "chi1024":
        print(json.dumps(study_exact_chi1024()))
    elif which == "chi512":
        print(json.dumps(study_chi512()))
    else:
        print(json.dumps(study()))
