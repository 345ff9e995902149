"""CPU check of the step order the GPU state vector (tessera_b200/csrc/statevector.cu) runs.

In the engine's splitting (mode 1) a step is G(k) Z(k) G(k): single-qubit half steps G(k) on
every qubit around the exact ZZ phase Z(k) (cuda/src/mps.cpp:309-356).  The GPU merges the
closing G(k) of one step with the opening G(k+1) of the next into one gate per qubit,
G(k+1) G(k), and reads the step's qubit-0 entropy from the state after that product, before
Z(k+1).  This is exact because G(k+1) is a product of one-qubit unitaries, which leave the
Schmidt spectrum across the qubit-0 cut unchanged.  The test restates that merged order in
numpy and compares it with the oracle's plain order (every step in full, entropy after it).
"""
import numpy as np
import pytest
from scipy.linalg import expm

from oracle.oracle import Instance
from tessera_b200 import instances


def _gate(A, B, hi, dt, C=0.0, bi=0.0):
    # exp(-i dt/2 g), g = -A X - (B h_i + C b_i) Z (engine basis: bit set <-> spin -1)
    z = B * hi + C * bi
    g = np.array([[-z, -A], [-A, z]], dtype=np.complex128)
    return expm(-0.5j * dt * g)


def _apply(psi, n, i, G):
    v = psi.reshape(-1, 2, 1 << i)  # axis 1 is bit i
    a, b = v[:, 0, :].copy(), v[:, 1, :].copy()
    v[:, 0, :] = G[0, 0] * a + G[0, 1] * b
    v[:, 1, :] = G[1, 0] * a + G[1, 1] * b


def _entropy0(psi):
    u, v = psi[0::2], psi[1::2]
    r00, r11 = np.vdot(u, u).real, np.vdot(v, v).real
    r01 = np.sum(u * np.conj(v))
    tot = r00 + r11
    p, q, off2 = r00 / tot, r11 / tot, abs(r01) ** 2 / tot ** 2
    mid, rad = 0.5 * (p + q), np.sqrt(max(0.0, 0.25 * (p - q) ** 2 + off2))
    s = 0.0
    for lam in (min(1.0, max(0.0, mid + rad)), min(1.0, max(0.0, mid - rad))):
        if lam > 1e-12:
            s -= lam * np.log2(lam)
    return s


def merged_mode1(inst, sa, sb, dt, bias=None, sc=None):
    """Final state and per-step qubit-0 entropies in the GPU's merged order."""
    n, steps = inst.n, len(sa)
    dim = 1 << n
    x = np.arange(dim)
    z = 1 - 2 * ((x[:, None] >> np.arange(n)[None, :]) & 1)  # spin of every qubit
    ezz = -np.sum(inst.ew[None, :] * z[:, inst.ei] * z[:, inst.ej], axis=1)
    psi = np.full(dim, 1.0 / np.sqrt(dim), np.complex128)

    def gates(k):
        if bias is None:
            return [_gate(sa[k], sb[k], inst.h[i], dt) for i in range(n)]
        return [_gate(sa[k], sb[k], inst.h[i], dt, sc[k], bias[i]) for i in range(n)]

    ent = np.zeros(steps)
    for i, G in enumerate(gates(0)):
        _apply(psi, n, i, G)
    psi *= np.exp(-1j * dt * sb[0] * ezz)
    for k in range(steps):
        g = gates(k)
        if k + 1 < steps:
            g = [gn @ gk for gn, gk in zip(gates(k + 1), g)]
        for i, G in enumerate(g):
            _apply(psi, n, i, G)
        ent[k] = _entropy0(psi)
        if k + 1 < steps:
            psi *= np.exp(-1j * dt * sb[k + 1] * ezz)
    return psi, ent


def _inst(p):
    return Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)


@pytest.mark.parametrize("kind,n,seed", [("chain", 6, 1), ("dense", 7, 2), ("dense", 8, 3)])
def test_merged_half_steps_equal_the_plain_order(oracle, kind, n, seed):
    p = (instances.chain_range(n=n, dmax=2, seed=seed, T=2.0, dt=0.1, hzero=False) if kind == "chain"
         else instances.dense_er(n, seed, T=2.0, dt=0.1))
    inst = _inst(p)
    ref = oracle.sv_anneal(inst, p.sa, p.sb, p.dt, mode=1, want_state=True)
    psi, ent = merged_mode1(inst, p.sa, p.sb, p.dt)
    fid = abs(np.vdot(psi, ref.state)) ** 2 / (np.vdot(psi, psi).real * np.vdot(ref.state, ref.state).real)
    assert 1.0 - fid < 1e-12
    assert np.max(np.abs(ent - ref.entropy)) < 1e-10
    assert np.max(ent) > 0.05  # the anneal entangles qubit 0, so the entropy check has teeth


def test_merged_half_steps_with_warm_start_field(oracle):
    p = instances.dense_er(7, 5, T=2.0, dt=0.1)
    inst = _inst(p)
    rng = np.random.default_rng(5)
    bias = rng.uniform(-1.0, 1.0, p.n)
    s = np.linspace(0.0, 1.0, len(p.sa))
    sc = 0.3 * 4.0 * s * (1.0 - s)
    ref = oracle.sv_anneal(inst, p.sa, p.sb, p.dt, mode=1, want_state=True, bias=bias, sc=sc)
    psi, ent = merged_mode1(inst, p.sa, p.sb, p.dt, bias=bias, sc=sc)
    fid = abs(np.vdot(psi, ref.state)) ** 2 / (np.vdot(psi, psi).real * np.vdot(ref.state, ref.state).real)
    assert 1.0 - fid < 1e-12
    assert np.max(np.abs(ent - ref.entropy)) < 1e-10


def test_entropy_is_not_blind_to_a_two_qubit_phase():
    # the merge is exact only for one-qubit unitaries: a ZZ phase between qubit 0 and another
    # qubit does change the qubit-0 entropy, which is why the entropy is read before Z(k+1)
    n = 3
    psi = np.full(1 << n, 1.0 / np.sqrt(1 << n), np.complex128)
    s0 = _entropy0(psi)
    x = np.arange(1 << n)
    z0, z1 = 1 - 2 * (x & 1), 1 - 2 * ((x >> 1) & 1)
    psi2 = psi * np.exp(-1j * 0.7 * z0 * z1)
    rng = np.random.default_rng(0)
    psi3 = psi2.copy()
    for i in range(n):
        q, _ = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))
        _apply(psi3, n, i, q)
    assert abs(s0) < 1e-12 and _entropy0(psi2) > 0.1
    assert abs(_entropy0(psi3) - _entropy0(psi2)) < 1e-12
