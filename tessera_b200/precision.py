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


if __name__ == "__main__":
    import json
    print(json.dumps(study()))
