"""Pins the CPU oracle (test infrastructure) before anything is checked against it.

* The MPS-TEBD restatement must reproduce every golden case written by the reference
  engine itself (tests/golden/make_golden.py), to rounding.
* The reference's linalg known answers (cuda/tests/test_linalg.cpp:29-98) hold.
* The state-vector oracle satisfies the assertions of rust/src/quantum.rs:229-296 (on our
  own seeded instances: the Rust StdRng instances cannot be regenerated here), and in
  the engine's Trotter splitting it equals the exact-chi MPS state.
"""
import numpy as np
import pytest

from oracle.oracle import Instance, Reference, smooth_schedule
from tessera_b200 import instances


def schedule_of(spec):
    kind, steps = spec
    return smooth_schedule(steps) if kind == "smooth" else instances.linear(steps)


def inst_of(d):
    return Instance(np.array(d["h"]), np.array(d["ei"], dtype=np.int32), np.array(d["ej"], dtype=np.int32),
                    np.array(d["ew"]))


def test_oracle_reproduces_every_golden_case(oracle, golden):
    for case in golden["cases"]:
        sa, sb = schedule_of(case["schedule"])
        r = oracle.mps_anneal(inst_of(case["instance"]), sa, sb, case["dt"], case["chi"], case["zz_substeps"])
        ref = case["out"]
        assert list(r.spins) == ref["spins"], case["name"]
        assert r.energy == pytest.approx(ref["energy"], rel=1e-12, abs=1e-12), case["name"]
        assert r.expected_energy == pytest.approx(ref["expected_energy"], rel=1e-9, abs=1e-10), case["name"]
        assert r.prob == pytest.approx(ref["prob"], rel=1e-9, abs=1e-12), case["name"]
        assert r.max_trunc == pytest.approx(ref["max_trunc"], rel=1e-6, abs=1e-20), case["name"]
        assert np.max(np.abs(r.entropy - np.array(ref["entropy"]))) < 1e-9, case["name"]


def test_reference_test_mps_claims_hold_in_golden(golden):
    """cuda/tests/test_mps.cpp:79-152 assertions, on the reference's own outputs."""
    by = {c["name"]: c for c in golden["cases"]}
    assert by["single_spin"]["out"]["spins"] == [1]
    assert abs(by["single_spin"]["out"]["energy"] + 1.0) < 1e-9
    assert abs(by["ferro_pair"]["out"]["energy"] + 1.0) < 1e-9
    for t in range(6):
        c = by[f"dense6_seed123_t{t}"]
        assert c["out"]["max_trunc"] < 1e-9
    ring = by["ring3_T320"]["out"]
    assert abs(ring["expected_energy"] - (-2.0)) < 0.05
    ent = by["entropy_pair"]["out"]["entropy"]
    assert max(ent) > 0.05 and max(ent) <= 1.0 + 1e-9


def test_exact_chi_hits_ground_state(oracle, golden):
    hits = 0
    for t in range(6):
        c = next(x for x in golden["cases"] if x["name"] == f"dense6_seed123_t{t}")
        _, e = oracle.exact_ground(inst_of(c["instance"]))
        hits += abs(c["out"]["energy"] - e) < 1e-6
    assert hits >= 5  # cuda/tests/test_mps.cpp:121


def test_linalg_known_answers(oracle, golden):
    Z = np.diag([1.0, -1.0]).astype(complex)
    w, _ = oracle.hermitian_eig(Z)
    assert sorted(np.round(w, 9)) == [-1.0, 1.0]
    Y = np.array([[0, -1j], [1j, 0]])
    w, _ = oracle.hermitian_eig(Y)
    assert abs(abs(w[0]) - 1) < 1e-9 and abs(w[0] + w[1]) < 1e-9
    X = np.array([[0, 1], [1, 0]], complex)
    U = oracle.hermitian_expm(X, complex(0, -np.pi / 2))
    assert np.linalg.norm(U - (-1j) * X) < 1e-9
    E = np.array(golden["linalg"]["expm_X_re"]) + 1j * np.array(golden["linalg"]["expm_X_im"])
    assert np.linalg.norm(U.ravel() - E) < 1e-12
    H3 = np.array([[2, 1 + 2j, -0.5 + 1j], [1 - 2j, -1, -1j], [-0.5 - 1j, 1j, 0.5]], complex)
    w, V = oracle.hermitian_eig(H3)
    assert np.linalg.norm(V @ np.diag(w) @ V.conj().T - H3) < 1e-7
    assert np.allclose(w, golden["linalg"]["eig_H3"], atol=1e-12)
    H = np.array([[1, 0.3 + 0.7j, 0], [0.3 - 0.7j, 2, -0.2 + 0.5j], [0, -0.2 - 0.5j, -1]])
    U = oracle.hermitian_expm(H, complex(0, -0.83))
    assert np.linalg.norm(U @ U.conj().T - np.eye(3)) < 1e-9


def test_oracle_svd_matches_reference_spectra(oracle, golden):
    for c in golden["svd"]:
        A = (np.array(c["re"]) + 1j * np.array(c["im"])).reshape(c["rows"], c["cols"])
        _, s, _ = oracle.svd(A)
        assert np.allclose(s, c["s"], rtol=1e-12, atol=1e-13)
        assert np.allclose(s, np.linalg.svd(A, compute_uv=False), rtol=1e-8)


def _rand_small(n, rng):
    h = rng.uniform(-1, 1, n)
    ei, ej, ew = [], [], []
    for i in range(n):
        for k in range(i + 1, n):
            if rng.random() < 0.5:
                ei.append(i); ej.append(k); ew.append(rng.uniform(-1, 1))
    return Instance(h, np.array(ei, np.int32), np.array(ej, np.int32), np.array(ew))


def test_statevector_oracle_rust_assertions(oracle):
    """rust/src/quantum.rs:229-296, restated."""
    one = Instance(np.array([1.0]), np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0))
    a, b = smooth_schedule(400)
    r = oracle.sv_anneal(one, a, b, 0.1)
    assert list(r.spins) == [1] and abs(r.energy + 1) < 1e-9 and r.prob > 0.9
    pair = Instance(np.zeros(2), np.array([0], np.int32), np.array([1], np.int32), np.array([1.0]))
    a, b = smooth_schedule(500)
    assert abs(oracle.sv_anneal(pair, a, b, 0.1).energy + 1) < 1e-9
    fr = Instance(np.array([0.3, -0.3]), np.array([0], np.int32), np.array([1], np.int32), np.array([-1.0]))
    a, b = smooth_schedule(400)
    tr = oracle.sv_anneal(fr, a, b, 0.1).entropy
    assert len(tr) == 400 and tr.max() > 0.05 and tr.max() > tr[0] and tr.max() >= tr[-1] and tr.max() <= 1 + 1e-9
    p3 = Instance(np.array([0.5, -0.5, 0.2]), np.array([0], np.int32), np.array([1], np.int32), np.array([0.4]))
    a, b = smooth_schedule(50)
    assert oracle.sv_anneal(p3, a, b, 0.1).entropy[0] < 0.2
    rng = np.random.Generator(np.random.PCG64(5))
    a, b = smooth_schedule(1500)
    hits = 0
    for _ in range(8):
        m = _rand_small(6, rng)
        _, e = oracle.exact_ground(m)
        out = oracle.sv_anneal(m, a, b, 0.1)
        assert out.energy >= e - 1e-9
        hits += abs(out.energy - e) < 1e-6
    assert hits >= 5


def _fid(x, y):
    return abs(np.vdot(x, y)) ** 2 / (np.vdot(x, x).real * np.vdot(y, y).real)


def test_statevector_engine_splitting_equals_exact_chi_mps(oracle):
    """Mode 1 of the state-vector oracle is the MPS engine's own Trotter splitting: at exact chi
    the MPS algorithm with an accurate SVD and the state vector agree state-for-state."""
    rng = np.random.Generator(np.random.PCG64(21))
    for n in (4, 5, 6, 7):
        m = _rand_small(n, rng)
        a, b = instances.linear(60)
        mp = oracle.mps_anneal(m, a, b, 0.1, 1 << (n // 2 + 1), want_state=True, accurate_svd=True)
        sv = oracle.sv_anneal(m, a, b, 0.1, mode=1, want_state=True)
        assert 1 - _fid(mp.state, sv.state) < 1e-12, n
        assert mp.expected_energy == pytest.approx(sv.expected_energy, abs=1e-10)
        assert np.max(np.abs(mp.entropy - sv.entropy)) < 1e-9
        assert mp.extra["norm2"] == pytest.approx(1.0, abs=1e-10)


def test_accurate_mode_equals_reference_where_its_svd_is_sound(oracle, golden):
    """The oracle's accurate-SVD mode changes nothing but the SVD: on every golden case whose
    reference run reconstructed each theta to 1e-8, it reproduces the reference."""
    for case in golden["cases"]:
        if not case["reference_svd_sound"]:
            continue
        sa, sb = schedule_of(case["schedule"])
        r = oracle.mps_anneal(inst_of(case["instance"]), sa, sb, case["dt"], case["chi"], case["zz_substeps"],
                              accurate_svd=True)
        ref = case["out"]
        assert list(r.spins) == ref["spins"], case["name"]
        assert r.expected_energy == pytest.approx(ref["expected_energy"], rel=1e-4), case["name"]
        assert r.max_trunc == pytest.approx(ref["max_trunc"], rel=1e-3, abs=1e-20), case["name"]
        assert np.max(np.abs(r.entropy - np.array(ref["entropy"]))) < 1e-4, case["name"]


def test_reference_gram_svd_defect_is_reproduced(oracle, golden):
    """The reference's Gram-matrix SVD (cuda/src/linalg.cpp:56-172) mis-factorises theta when
    singular values are degenerate; its own exact-chi test instance (cuda/tests/test_mps.cpp:99-123)
    drifts off the exact evolution.  The oracle's reference mode reproduces that drift bit for bit
    (previous test); the accurate mode follows the exact state vector."""
    c = next(x for x in golden["cases"] if x["name"] == "dense6_seed123_t0")
    assert not c["reference_svd_sound"] and c["reference_svd_max_recon_err"] > 1e-2
    sa, sb = schedule_of(c["schedule"])
    inst = inst_of(c["instance"])
    ref_mode = oracle.mps_anneal(inst, sa, sb, c["dt"], c["chi"], want_state=True)
    acc_mode = oracle.mps_anneal(inst, sa, sb, c["dt"], c["chi"], want_state=True, accurate_svd=True)
    sv = oracle.sv_anneal(inst, sa, sb, c["dt"], mode=1, want_state=True)
    assert 1 - _fid(ref_mode.state, sv.state) > 1e-3
    assert 1 - _fid(acc_mode.state, sv.state) < 1e-12
    assert acc_mode.extra["bad_updates"] == 0


def test_reference_live_matches_oracle_when_built(oracle):
    if not Reference.available():
        pytest.skip("oracle/_ref not built here")
    R = Reference()
    p = instances.chain_range(n=7, dmax=3, seed=3, T=2.0, dt=0.05, chi=4, dist="normal", hzero=False)
    inst = Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)
    r1 = R.mps_anneal(inst, p.sa, p.sb, p.dt, 4)
    r2 = oracle.mps_anneal(inst, p.sa, p.sb, p.dt, 4)
    assert r1.energy == r2.energy and r1.max_trunc == pytest.approx(r2.max_trunc, rel=1e-9)
    assert np.max(np.abs(r1.entropy - r2.entropy)) < 1e-10


def test_apply_slots_equals_zz_phases_on_the_dense_state(oracle):
    """orc_mps_apply_slots (gate slots of one step's ZZ block on a given MPS) at exact bond
    dimension: the swap network moves sites and moves them back, so after all slots of the block
    the state is the input times exp(-i theta_e Z_i Z_j) for every edge, theta_e = -B w_e dt
    (cuda/src/mps.cpp:116-145, 330-341).  A random MPS of 7 sites, couplings to distance 3."""
    from tessera_b200 import ffi
    rng = np.random.default_rng(5)
    n = 7
    dims = [1] + [2 ** min(i, n - i) for i in range(1, n)] + [1]
    sites = [rng.normal(size=(dims[i], 2, dims[i + 1])) + 1j * rng.normal(size=(dims[i], 2, dims[i + 1]))
             for i in range(n)]
    p = instances.chain_range(n=n, dmax=3, seed=4, T=1.0, dt=0.1, chi=8, dist="normal")
    inst = Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)
    nslots = sum(2 * abs(int(j) - int(i)) - 1 for i, j in zip(p.ei, p.ej))
    B, dt = 0.7, 0.1
    out, st = oracle.apply_slots(inst, sites, B, dt, 8, 0, nslots)
    assert st["updates"] == nslots and st["max_trunc"] < 1e-28
    psi = ffi.sites_to_dense(sites)
    x = np.arange(1 << n)
    z = 1 - 2 * ((x[:, None] >> np.arange(n)) & 1)  # physical index 0 <-> spin +1
    phase = np.zeros(1 << n)
    for i, j, w in zip(p.ei, p.ej, p.ew):
        phase += -B * w * dt * z[:, i] * z[:, j]
    want = psi * np.exp(-1j * phase)
    got = ffi.sites_to_dense(out)
    assert np.linalg.norm(got - want) < 1e-12 * np.linalg.norm(want)
    # slots 2..4 are updates on bonds 0, 1, 2 (edges (0,2) and (0,3)): sites 4.. are untouched
    part, st2 = oracle.apply_slots(inst, sites, B, dt, 8, 2, 5)
    assert st2["updates"] == 3
    assert all(np.array_equal(part[i], sites[i]) for i in range(4, n))


def _rand_instance(n, p, rng):
    """rust/src/ising.rs:143-153 (random_instance): h ~ U(-1, 1), each pair an edge with
    probability p, J ~ U(-1, 1) -- drawn here from numpy's PCG64 (StdRng is not reproducible)."""
    h = rng.uniform(-1, 1, n)
    ei, ej, ew = [], [], []
    for i in range(n):
        for k in range(i + 1, n):
            if rng.random() < p:
                ei.append(i); ej.append(k); ew.append(rng.uniform(-1, 1))
    return Instance(h, np.array(ei, np.int32), np.array(ej, np.int32), np.array(ew))


def test_oracle_sa_reaches_exact_ground_state_on_small_instances(oracle):
    """The reference's own SA claim (rust/src/ising.rs:156-174): best of 40 restarts x 400 sweeps,
    t0 = 5, t_end = 0.01, reaches the exact ground energy on at least 19 of 20 random n=12, p=0.5
    instances; and its returned energy is the energy of its returned pattern."""
    rng = np.random.Generator(np.random.PCG64(1))
    hits = 0
    for k in range(20):
        m = _rand_instance(12, 0.5, rng)
        _, e_exact = oracle.exact_ground(m)
        s, e_sa = oracle.sa_solve(m, 40, 400, seed=1, index=k)
        assert e_sa == pytest.approx(m.energy(s), abs=1e-12)
        hits += abs(e_sa - e_exact) < 1e-6
    assert hits >= 19


def test_oracle_single_sa_run_beats_a_random_pattern(oracle):
    """rust/src/ising.rs:176-183: one run of 400 sweeps (t0 = 3) ends below a random pattern."""
    rng = np.random.Generator(np.random.PCG64(2))
    m = _rand_instance(16, 0.5, rng)
    rand_s = rng.choice([-1, 1], 16)
    _, e = oracle.sa_solve(m, 1, 400, t0=3.0, seed=2)
    assert e < m.energy(rand_s)
