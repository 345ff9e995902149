"""tessera_qa_sa_solve, the GPU simulated-annealing scorer, against the oracle and brute force.

The kernel restates the reference's best-of-restarts SA (rust/src/ising.rs:64-136) with a
counter-based random stream that the oracle (orc_sa_solve) draws from too, so a batch on the GPU
must reproduce the oracle's runs draw for draw: the same best energies, bit for bit, and the
same spin patterns.  With a large budget it must also reach the exact ground energy
(tessera_qa_exact_ground) on dense instances up to n = 20, which is what makes it the
best-known-energy scorer for the held-out instances beyond brute force.
"""
import numpy as np
import pytest

from oracle.oracle import Instance
from tessera_b200 import ffi, instances, learned

pytestmark = pytest.mark.gpu


def _inst(p):
    return Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)


def test_sa_matches_the_oracle_draw_for_draw(oracle):
    probs = [instances.dense_er(n, 40 + n, T=1.0, dt=0.1, chi=8) for n in (5, 9, 13, 20)]
    probs += instances.batch_3_regular(count=2, T=0.2, dt=0.05, nmin=32, nmax=40)
    probs.append(instances.chain_range(n=70, dmax=3, seed=3, T=1.0, dt=0.1, chi=8, dist="normal", hzero=False))
    en, spins = ffi.sa_solve(probs, restarts=150, sweeps=120, seed=11)
    for b, p in enumerate(probs):
        s_o, e_o = oracle.sa_solve(_inst(p), 150, 120, seed=11, index=b)
        assert en[b] == e_o, (b, p.name, en[b], e_o)
        assert list(spins[b]) == list(s_o), (b, p.name)
        assert p.energy(spins[b]) == pytest.approx(en[b], abs=1e-12)


def test_sa_reaches_the_exact_ground_energy_up_to_n20():
    probs = [instances.dense_er(n, 900 + n, T=1.0, dt=0.1, chi=8) for n in range(12, 21)] * 2
    en, spins = ffi.sa_solve(probs, restarts=256, sweeps=2000, seed=5)
    for b, p in enumerate(probs):
        e_ex, _ = learned.exact_ground(p)
        assert en[b] == pytest.approx(e_ex, abs=1e-9), (p.name, en[b], e_ex)
