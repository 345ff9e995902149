"""The exact state-vector anneal on the GPU (tessera_qa_sv_anneal) against the CPU state-vector
oracle (rust/src/quantum.rs:63-207 restated), both splittings, with and without the warm-start
field; the assertions of rust/src/quantum.rs:229-296 on the GPU; and the MPS engine at exact chi
against it.  Tolerances: state fidelity 1e-12, energies 1e-10, entropy 1e-10, patterns equal."""
import numpy as np
import pytest

from oracle.oracle import Instance, smooth_schedule
from tessera_b200 import ffi, instances

pytestmark = pytest.mark.gpu


def _fid(x, y):
    return abs(np.vdot(x, y)) ** 2 / (np.vdot(x, x).real * np.vdot(y, y).real)


def _rand(n, seed, p=0.5):
    rng = np.random.Generator(np.random.PCG64(seed))
    h = rng.uniform(-1, 1, n)
    ei, ej, ew = [], [], []
    for i in range(n):
        for k in range(i + 1, n):
            if rng.random() < p:
                ei.append(i); ej.append(k); ew.append(rng.uniform(-1, 1))
    return Instance(h, np.array(ei, np.int32), np.array(ej, np.int32), np.array(ew))


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("n,seed", [(1, 1), (2, 2), (3, 3), (5, 4), (9, 5), (12, 6)])
def test_gpu_statevector_matches_cpu_oracle(oracle, n, seed, mode):
    m = _rand(n, seed) if n > 1 else Instance(np.array([0.7]), np.zeros(0, np.int32), np.zeros(0, np.int32),
                                             np.zeros(0))
    sa, sb = instances.linear(80)
    g = ffi.sv_anneal(m.h, m.ei, m.ej, m.ew, sa, sb, dt=0.1, mode=mode, want_state=True)
    o = oracle.sv_anneal(m, sa, sb, 0.1, mode=mode, want_state=True)
    assert 1 - _fid(g.state, o.state) < 1e-12
    assert np.linalg.norm(g.state - o.state) < 1e-10
    assert g.expected_energy == pytest.approx(o.expected_energy, abs=1e-10)
    assert np.max(np.abs(g.entropy - o.entropy)) < 1e-10
    assert list(g.spins) == list(o.spins) and g.energy == pytest.approx(o.energy, abs=1e-12)
    assert list(g.sign_spins) == list(o.extra["sign_spins"])
    assert g.prob == pytest.approx(o.prob, rel=1e-10)


def test_gpu_statevector_bias_field(oracle):
    m = _rand(8, 9)
    sa, sb = instances.linear(60)
    rng = np.random.Generator(np.random.PCG64(3))
    bias = rng.uniform(-1, 1, 8)
    sc = 0.5 * 4 * sb * (1 - sb)
    g = ffi.sv_anneal(m.h, m.ei, m.ej, m.ew, sa, sb, dt=0.1, mode=1, bias=bias, sc=sc, want_state=True)
    o = oracle.sv_anneal(m, sa, sb, 0.1, mode=1, want_state=True, bias=bias, sc=sc)
    assert 1 - _fid(g.state, o.state) < 1e-12
    assert np.max(np.abs(g.entropy - o.entropy)) < 1e-10


def test_gpu_statevector_rust_assertions():
    """rust/src/quantum.rs:229-296 on the GPU state vector (own seeded instances)."""
    a, b = smooth_schedule(400)
    r = ffi.sv_anneal([1.0], [], [], [], a, b, dt=0.1)
    assert list(r.spins) == [1] and abs(r.energy + 1) < 1e-9 and r.prob > 0.9
    a, b = smooth_schedule(500)
    assert abs(ffi.sv_anneal([0.0, 0.0], [0], [1], [1.0], a, b, dt=0.1).energy + 1) < 1e-9
    a, b = smooth_schedule(400)
    tr = ffi.sv_anneal([0.3, -0.3], [0], [1], [-1.0], a, b, dt=0.1).entropy
    assert tr.max() > 0.05 and tr.max() > tr[0] and tr.max() >= tr[-1] and tr.max() <= 1 + 1e-9


def test_gpu_statevector_equals_mps_engine_at_exact_chi():
    m = _rand(10, 11)
    sa, sb = instances.linear(100)
    g = ffi.sv_anneal(m.h, m.ei, m.ej, m.ew, sa, sb, dt=0.1, mode=1, want_state=True)
    r = ffi.anneal(m.h, m.ei, m.ej, m.ew, sa, sb, dt=0.1, chi=32, want_checkpoint=True)
    psi = ffi.sites_to_dense(ffi.checkpoint_to_sites(r.checkpoint)[1])
    assert 1 - _fid(psi, g.state) < 1e-8
    assert r.expected_energy == pytest.approx(g.expected_energy, abs=1e-8)


def test_gpu_statevector_large_tiles():
    """n = 20: three tiled passes per half step (qubits 0-10, 11-16, 17-19); norm kept, the
    pattern and energy consistent."""
    p = instances.chain_range(n=20, dmax=4, seed=2, T=1.0, dt=0.02)
    g = ffi.sv_anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, mode=1)
    assert g.norm2 == pytest.approx(1.0, abs=1e-10)
    assert len(g.entropy) == p.steps and np.all(g.entropy >= 0) and np.all(g.entropy <= 1 + 1e-12)
    e = -sum(w * g.spins[i] * g.spins[j] for i, j, w in zip(p.ei, p.ej, p.ew)) - float(np.dot(p.h, g.spins))
    assert g.energy == pytest.approx(e, abs=1e-9)
