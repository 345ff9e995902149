"""Parity of the CUDA engine (through the C ABI) with the oracle and the reference.

Tolerances (complex128 unless stated):
* reference golden cases whose reference SVD is sound and which never truncate: energy,
  <H>, prob rel 1e-9; entropy abs 1e-9.
* reference golden cases whose reference SVD is sound and that truncate (chi below exact):
  <H> rel 1e-4, entropy abs 1e-4, max_trunc rel 1e-2 -- the reference's own Gram-SVD
  rounding (up to 1e-8 per update) accumulates to that level over the run.
* every golden case against the oracle's accurate-SVD mode (same algorithm, keep rule,
  gauge, gate order): <H> and entropy within 1e-6 plus ten times the case's own
  sensitivity, the largest change over oracle re-runs with schedule and couplings moved by
  +4, -4 and +8 ulps.  Truncated TEBD can amplify rounding exponentially in time (observed: x1000
  per two steps at chi=8, n=8, d<=3), so two correct implementations agree only as well
  as the run is conditioned; spins must agree where the run is well conditioned.
* exact chi against the exact state vector (engine's Trotter splitting): fidelity within 1e-8,
  and the most probable bit pattern equal.
* complex64 mode: <H> within 1e-4 relative of the complex128 engine, fidelity within 1e-6.
"""
import numpy as np
import pytest

from oracle.oracle import Instance, smooth_schedule
from tessera_b200 import ffi, instances

pytestmark = pytest.mark.gpu


def schedule_of(spec):
    kind, steps = spec
    return smooth_schedule(steps) if kind == "smooth" else instances.linear(steps)


def spins_agree(r, ref_spins, floor=1e-8):
    """Readout spins agree wherever the sign of <Z_i> is resolved (|<Z_i>| > floor); with h = 0 the
    exact <Z_i> vanish and the sign is rounding noise in both implementations."""
    z = r.z_expect
    return all(int(a) == int(b) for a, b, zz in zip(r.spins, ref_spins, z) if abs(zz) > floor)


def run_case(case, **kw):
    d = case["instance"]
    sa, sb = schedule_of(case["schedule"])
    return ffi.anneal(d["h"], d["ei"], d["ej"], d["ew"], sa, sb, dt=case["dt"], chi=case["chi"],
                      zz_substeps=case["zz_substeps"], **kw)


def inst_of(d):
    return Instance(np.array(d["h"]), np.array(d["ei"], dtype=np.int32), np.array(d["ej"], dtype=np.int32),
                    np.array(d["ew"]))


def fidelity(x, y):
    return abs(np.vdot(x, y)) ** 2 / (np.vdot(x, x).real * np.vdot(y, y).real)


def test_svd_kernel_matches_reference_spectra(golden):
    for c in golden["svd"]:
        A = (np.array(c["re"]) + 1j * np.array(c["im"])).reshape(c["rows"], c["cols"])
        u, s, vh = ffi.svd(A)
        assert np.allclose(s, c["s"], rtol=1e-10, atol=1e-12)
        k = len(s)
        assert np.linalg.norm(u.conj().T @ u - np.eye(k)) < 1e-12
        assert np.linalg.norm(u @ np.diag(s) @ vh - A) < 1e-12 * np.linalg.norm(A) * max(A.shape)


@pytest.mark.parametrize("shape", [(64, 64), (128, 96), (512, 512), (200, 300), (2048, 256), (1024, 1024)])
def test_svd_kernel_large_random(shape):
    """Random unitary factors around a TEBD-like spectrum exp(-k/20).  Values above the
    kernel's noise floor (8 sqrt(R) ulps of ||A||_F) are resolved to 1e-9 relative or 1% of the
    floor absolute; those under it come back under twice it.  At 1024 x 1024, 437 of the values lie under the floor, and
    columns whose norm dips under it mid-sweep must still be orthogonalised against the resolved
    ones (the early, mixed phase of the freeze rule), else values a few times the floor come
    back at it and U loses orthogonality."""
    rng = np.random.Generator(np.random.PCG64(sum(shape)))
    A = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    U, s, Vh = np.linalg.svd(A, full_matrices=False)
    s = np.exp(-np.arange(len(s)) / 20.0)
    A = (U * s) @ Vh
    u, sg, vh = ffi.svd(A)
    floor = 8.0 * np.sqrt(max(shape)) * np.finfo(np.float64).eps * np.linalg.norm(A)
    assert np.allclose(sg, s, rtol=1e-9, atol=floor)
    # resolved: off by a small fraction of the floor (a frozen column is off by ~ the floor), plus
    # 1e-12 relative: the rotations' coefficients come from FP64 rsqrt, whose rounding moves every
    # column norm the same way by a fraction of an ulp per rotation (measured 1.9e-13 relative at
    # 512 x 512 and 3.7e-13 at 1024 x 1024 on the largest values)
    above = s > 4 * floor
    assert np.all(np.abs(sg[above] - s[above]) < 0.01 * floor + 1e-12 * s[above])
    assert np.max(sg[s < floor]) <= 2 * floor if np.any(s < floor) else True
    assert np.linalg.norm(u.conj().T @ u - np.eye(len(s))) < 1e-9
    assert np.linalg.norm(u @ np.diag(sg) @ vh - A) < 1e-11 * np.linalg.norm(A)


def test_sound_reference_cases_match_the_reference(golden):
    for case in golden["cases"]:
        if not case["reference_svd_sound"]:
            continue
        r = run_case(case)
        ref = case["out"]
        truncating = "truncating" in case["tags"]
        assert spins_agree(r, ref["spins"]), case["name"]
        if all(abs(z) > 1e-8 for z in r.z_expect):
            assert r.energy == pytest.approx(ref["energy"], rel=1e-12, abs=1e-12), case["name"]
        rt = 1e-4 if truncating else 1e-9
        assert r.expected_energy == pytest.approx(ref["expected_energy"], rel=rt, abs=1e-10), case["name"]
        assert np.max(np.abs(r.entropy - np.array(ref["entropy"]))) < (1e-4 if truncating else 1e-9), case["name"]
        if truncating:
            assert r.max_trunc == pytest.approx(ref["max_trunc"], rel=1e-2), case["name"]
        else:
            assert r.max_trunc < 1e-12 and ref["max_trunc"] < 1e-12
        assert r.status == 0


def perturbed(inst, sa, sb, eps=4e-16):
    return (Instance(inst.h * (1 + eps), inst.ei, inst.ej, inst.ew * (1 + eps)), sa, sb * (1 + eps))


def oracle_with_sensitivity(oracle, inst, sa, sb, dt, chi, zz=1):
    """The oracle's accurate-SVD run and its spread: the largest change of <H> and of the entropy
    trace over three runs with inputs moved by a few ulps (+4, -4, +8 ulps)."""
    o = oracle.mps_anneal(inst, sa, sb, dt, chi, zz, accurate_svd=True)
    dh = ds = 0.0
    for eps in (4e-16, -4e-16, 8e-16):
        i2, a2, b2 = perturbed(inst, sa, sb, eps)
        p = oracle.mps_anneal(i2, a2, b2, dt, chi, zz, accurate_svd=True)
        dh = max(dh, abs(o.expected_energy - p.expected_energy))
        ds = max(ds, float(np.max(np.abs(o.entropy - p.entropy))))
    return o, dh, ds


def test_every_golden_case_matches_the_accurate_oracle(oracle, golden):
    for case in golden["cases"]:
        sa, sb = schedule_of(case["schedule"])
        o, dh, ds = oracle_with_sensitivity(oracle, inst_of(case["instance"]), sa, sb, case["dt"], case["chi"],
                                            case["zz_substeps"])
        r = run_case(case)
        tol_h = 1e-6 * abs(o.expected_energy) + 1e-9 + 10 * dh
        assert abs(r.expected_energy - o.expected_energy) <= tol_h, (case["name"], r.expected_energy,
                                                                     o.expected_energy, dh)
        assert np.max(np.abs(r.entropy - o.entropy)) <= 1e-6 + 10 * ds, case["name"]
        if dh < 1e-9:
            assert spins_agree(r, o.spins), case["name"]
            if o.max_trunc > 1e-12:
                assert r.max_trunc == pytest.approx(o.max_trunc, rel=1e-4), case["name"]
            else:
                assert r.max_trunc < 1e-12, case["name"]


@pytest.mark.parametrize("dmax,chi", [(1, 4), (2, 4), (3, 8)])
def test_truncating_chain_tracks_the_oracle_step_by_step(oracle, dmax, chi):
    """n=8, chi below exact: state fidelity to the oracle after every few steps, within the run's
    own sensitivity (the d<=3, chi=8 run is chaotic after ~10 steps)."""
    p = instances.chain_range(n=8, dmax=dmax, seed=9 if dmax > 1 else 1, T=2.0, dt=0.05, chi=chi, dist="normal",
                              hzero=False)
    inst = Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)
    for steps in (2, 4, 8):
        sa, sb = p.sa[:steps], p.sb[:steps]
        r = ffi.anneal(p.h, p.ei, p.ej, p.ew, sa, sb, dt=p.dt, chi=chi, want_checkpoint=True)
        o = oracle.mps_anneal(inst, sa, sb, p.dt, chi, want_state=True, accurate_svd=True)
        _, sites = ffi.checkpoint_to_sites(r.checkpoint)
        assert 1 - fidelity(ffi.sites_to_dense(sites), o.state) < 1e-8, (dmax, chi, steps)
        # the largest discarded ratio of the run sits at a heavy cut, where the 1e-8 state
        # difference of the chaotic chi=8 run moves it by up to a few 1e-4 relative
        assert r.max_trunc == pytest.approx(o.max_trunc, rel=1e-3, abs=1e-20)
        assert r.min_cut_gap == pytest.approx(o.extra["min_cut_gap"], rel=1e-3)


def _rand_small(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    h = rng.uniform(-1, 1, n)
    ei, ej, ew = [], [], []
    for i in range(n):
        for k in range(i + 1, n):
            if rng.random() < 0.5:
                ei.append(i); ej.append(k); ew.append(rng.uniform(-1, 1))
    return Instance(h, np.array(ei, np.int32), np.array(ej, np.int32), np.array(ew))


@pytest.mark.parametrize("n,seed", [(6, 1), (8, 2), (10, 3)])
def test_exact_chi_state_matches_statevector(oracle, n, seed):
    m = _rand_small(n, seed)
    sa, sb = instances.linear(120)
    chi = 1 << (n // 2)
    r = ffi.anneal(m.h, m.ei, m.ej, m.ew, sa, sb, dt=0.1, chi=chi, want_checkpoint=True)
    _, sites = ffi.checkpoint_to_sites(r.checkpoint)
    psi = ffi.sites_to_dense(sites)
    sv = oracle.sv_anneal(m, sa, sb, 0.1, mode=1, want_state=True)
    assert 1 - fidelity(psi, sv.state) < 1e-8
    assert r.expected_energy == pytest.approx(sv.expected_energy, abs=1e-8)
    assert np.max(np.abs(r.entropy - sv.entropy)) < 1e-7
    # most probable bit pattern (quantum.rs readout) equals the oracle's
    best = int(np.argmax(np.abs(psi) ** 2))
    spins = np.array([-1 if (best >> i) & 1 else 1 for i in range(n)])
    assert list(spins) == list(sv.spins)
    assert r.max_trunc < 1e-20
    assert r.norm2 == pytest.approx(1.0, abs=1e-9)


def test_legacy_symbol_through_rust_style_wrapper(oracle, golden):
    lg = golden["legacy_abi"]
    d = lg["instance"]
    sa, sb = smooth_schedule(lg["schedule"][1])
    model = ffi.Ising(d["h"], list(zip(d["ei"], d["ej"], d["ew"])))
    res = ffi.quantum_anneal(model, ffi.Schedule(list(sa), list(sb)), lg["chi"])
    o = oracle.mps_anneal(inst_of(d), sa, sb, 0.1, lg["chi"], accurate_svd=True)
    assert list(res.spins) == list(o.spins)  # h != 0: every <Z_i> is resolved
    assert res.energy == pytest.approx(o.energy, abs=1e-10)
    assert np.max(np.abs(res.entropy - o.entropy)) < 1e-6


def test_complex64_mode_error_is_bounded(oracle):
    m = _rand_small(8, 7)
    sa, sb = instances.linear(150)
    r64 = ffi.anneal(m.h, m.ei, m.ej, m.ew, sa, sb, dt=0.1, chi=16, precision="c64", want_checkpoint=True)
    sv = oracle.sv_anneal(m, sa, sb, 0.1, mode=1, want_state=True)
    _, sites = ffi.checkpoint_to_sites(r64.checkpoint)
    psi = ffi.sites_to_dense(sites)
    assert 1 - fidelity(psi, sv.state) < 1e-6
    assert r64.expected_energy == pytest.approx(sv.expected_energy, rel=1e-4)


def test_jacobi_sweep_cap_reports_not_converged():
    """The give-up path: with the sweep cap forced to 1 the Jacobi cannot converge, the call
    returns TESSERA_QA_ESTATUS with status bit 1 and still fills the result; the default cap
    converges on the same input."""
    from tessera_b200 import _lib
    p = instances.chain_range(n=8, dmax=2, seed=9, T=1.0, dt=0.1, chi=8, dist="normal", hzero=False)
    args = (p.h, p.ei, p.ej, p.ew, p.sa, p.sb)
    with pytest.raises(_lib.EngineError) as err:
        ffi.anneal(*args, dt=p.dt, chi=8, jacobi_max_sweeps=1)
    assert err.value.code == _lib.ESTATUS
    r = ffi.anneal(*args, dt=p.dt, chi=8, jacobi_max_sweeps=1, raise_on_status=False)
    assert r.status & 1 and r.max_sweeps == 1 and r.two_site_updates > 0
    ok = ffi.anneal(*args, dt=p.dt, chi=8)
    assert ok.status == 0 and 1 < ok.max_sweeps < 60


def test_checkpoint_resume_equals_straight_run():
    p = instances.chain_range(n=12, dmax=2, seed=5, T=3.0, dt=0.05, chi=8, dist="normal", hzero=False)
    full = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=8)
    half = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=8, step_end=30, skip_observables=True,
                      want_checkpoint=True)
    rest = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=8, step_begin=30,
                      initial_mps=half.checkpoint)
    assert rest.expected_energy == pytest.approx(full.expected_energy, rel=1e-9)
    assert spins_agree(rest, full.spins)
    assert np.max(np.abs(np.concatenate([half.entropy, rest.entropy]) - full.entropy)) < 1e-9


def test_chain16_chi32_against_statevector(oracle):
    """Config-1 shape (n=16 chain, chi=32, linear schedule, dt=0.05) over the first 100 of its
    400 steps, against the exact 2^16 state vector in the engine's splitting."""
    p = instances.chain_nn(n=16, seed=1, T=20.0, dt=0.05, chi=32)
    sa, sb = p.sa[:100], p.sb[:100]
    r = ffi.anneal(p.h, p.ei, p.ej, p.ew, sa, sb, dt=p.dt, chi=32, want_checkpoint=True)
    sv = oracle.sv_anneal(Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew), sa, sb, p.dt,
                          mode=1, want_state=True)
    _, sites = ffi.checkpoint_to_sites(r.checkpoint)
    psi = ffi.sites_to_dense(sites)
    assert 1 - fidelity(psi, sv.state) < 1e-6
    assert r.expected_energy == pytest.approx(sv.expected_energy, rel=1e-6)
    assert np.max(np.abs(r.entropy - sv.entropy)) < 1e-6


def test_batched_anneal_equals_single_instance_runs():
    """tessera_qa_anneal_batch: ragged instances (different n, edges, chi) give the same results as
    one tessera_qa_anneal_ex call each.  With every theta of at most 64 rows both run the same
    resident anneal kernel for each instance, so the results are bit for bit equal."""
    probs = [instances.chain_range(n=8, dmax=2, seed=5, T=2.0, dt=0.05, chi=4, dist="normal", hzero=False),
             instances.chain_range(n=10, dmax=3, seed=6, T=2.0, dt=0.05, chi=8, dist="normal", hzero=False),
             instances.chain_nn(n=12, seed=7, T=2.0, dt=0.05, chi=16),
             instances.dense_er(n=7, seed=8, T=2.0, dt=0.05, chi=8)]
    for prec in ("c128", "c64"):
        batch = ffi.anneal_batch(probs, precision=prec)
        for p, rb in zip(probs, batch):
            rs = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=p.chi, precision=prec)
            assert rb.two_site_updates == rs.two_site_updates
            assert rb.expected_energy == rs.expected_energy, (p.name, prec)
            assert np.array_equal(rb.entropy, rs.entropy), (p.name, prec)
            assert list(rb.spins) == list(rs.spins) and rb.max_trunc == rs.max_trunc
            assert rb.status == 0


def test_batch_session_gate_slots_match_single_sessions():
    """Batched session (resident MPS of several instances, random saturated start): a run of gate
    slots updates every instance exactly like a single-instance session does."""
    probs = [instances.chain_range(n=12, dmax=3, seed=s, T=1.0, dt=0.05, chi=16) for s in (1, 2, 3)]
    sb = ffi.Session.batch(probs, chi=16, kernel_timing=True)
    sb.randomize(5)
    sb.run_gates(3, 0, 10)
    rb = sb.sync()
    assert rb.two_site_updates == 30 and rb.status == 0 and rb.svd_launches == 10
    tr = []
    for b, p in enumerate(probs):
        s1 = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=16)
        s1.randomize(5 + 7919 * b)
        s1.run_gates(3, 0, 10)
        r1 = s1.sync()
        tr.append(r1.max_trunc)
        s1.close()
    assert rb.max_trunc == pytest.approx(max(tr), rel=1e-9)
    r2 = sb.run_host(probs, 4, 0, 5)
    assert r2.status == 0
    sb.close()


def test_resident_whole_anneal_matches_gate_slot_path():
    """Small bonds run the whole batch in one launch (one CTA per instance, instances taken
    longest first from a work counter); an explicit Jacobi block width forces the per-gate-slot
    launches.  Both give the same anneals, also when instances outnumber the resident CTAs."""
    # chi at or above the exact bond dimension: no truncation, so the two paths (the same Jacobi,
    # different contraction and absorption kernels) agree to rounding; truncated dense instances
    # amplify rounding differences chaotically
    probs = [instances.dense_er(n, 300 + i, T=1.0, dt=0.1, chi=chi)
             for i, (n, chi) in enumerate([(10, 32), (8, 16), (9, 16), (11, 32), (5, 4), (7, 8)] * 3)]
    probs += [instances.dense_er(4 + i % 3, 900 + i, T=1.0, dt=0.1, chi=8) for i in range(330)]
    # complex64 rounds differently on the two paths; over ~1000 unitary updates its own error
    # against complex128 reaches ~1e-4 relative on these dense instances
    for prec, tol in (("c128", 1e-9), ("c64", 2e-3)):
        res = ffi.anneal_batch(probs, precision=prec)
        slot = ffi.anneal_batch(probs, precision=prec, jacobi_block=8)
        for p, a, b in zip(probs, res, slot):
            assert a.status == 0 and b.status == 0, p.name
            assert a.two_site_updates == b.two_site_updates, p.name
            assert a.expected_energy == pytest.approx(b.expected_energy, rel=tol, abs=tol), (p.name, prec)
            assert np.max(np.abs(a.entropy - b.entropy)) < 10 * tol, (p.name, prec)
            if prec == "c64":
                ref = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=p.chi, precision="c128") \
                    if p.n >= 9 else None
                if ref is not None:
                    assert a.expected_energy == pytest.approx(ref.expected_energy, rel=tol), p.name
            assert a.max_trunc < 1e-9 and b.max_trunc < 1e-9, (p.name, prec)


@pytest.mark.parametrize("block", [0, 32])
@pytest.mark.parametrize("prec,n,chi,q0,tol", [("c128", 12, 64, 36, 1e-10), ("c64", 16, 128, 54, 1e-4)])
def test_large_theta_batch_matches_cooperative_sessions(prec, n, chi, q0, tol, block):
    """Large theta in a batch (128 x 128 complex128 or 256 x 256 complex64: too big for the
    resident kernel) runs the block-row-cyclic column-pair Jacobi (jacobi_block 0) or the
    block-Gram Jacobi (32); the same gate slots on single-instance sessions run the cooperative
    column-pair kernel.  Random saturated MPS, interior bonds, truncating updates: the states
    agree to rounding and the runs are clean."""
    probs = [instances.chain_range(n=n, dmax=3, seed=s, T=1.0, dt=0.05, chi=chi) for s in (4, 5)]
    sb = ffi.Session.batch(probs, chi=chi, precision=prec, jacobi_block=block)
    sb.randomize(11)
    sb.run_gates(7, q0, q0 + 12)
    rb = sb.sync()
    assert rb.status == 0 and rb.two_site_updates == 24
    for b, p in enumerate(probs):
        s1 = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=chi, precision=prec)
        s1.randomize(11 + 7919 * b)
        s1.run_gates(7, q0, q0 + 12)
        r1 = s1.sync()
        assert r1.status == 0
        x = ffi.sites_to_dense(ffi.checkpoint_to_sites(s1.save())[1])
        s1.close()
        y = ffi.sites_to_dense(ffi.checkpoint_to_sites(sb.save_instance(b))[1])
        assert 1 - fidelity(x, y) < tol, (prec, b)
        assert np.vdot(y, y).real == pytest.approx(np.vdot(x, x).real, rel=tol)
    sb.close()


@pytest.mark.parametrize("batched", [False, True])
def test_tensor_core_theta_matches_cuda_core_theta(batched):
    """complex64 with theta_tensor_cores: the bond contraction runs on tcgen05 (split-TF32, FP32
    accumulators in tensor memory).  Same gate slots on the same random saturated MPS (chi=128:
    full 64 x 64 contraction tiles, and ragged ones on the chi-limited edge bonds), every update
    truncating.  Measured against the complex128 run, the tensor-core contraction is as accurate
    as the CUDA-core FP32 one (within a factor of 10 of its infidelity, and below 1e-5)."""
    p = instances.chain_range(n=16, dmax=3, seed=6, T=1.0, dt=0.05, chi=128)

    def run(prec, tc):
        if batched:
            s = ffi.Session.batch([p], chi=128, precision=prec, theta_tensor_cores=tc)
        else:
            s = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=128, precision=prec,
                            theta_tensor_cores=tc)
        s.randomize(21)
        s.run_gates(5, 0, 72)
        r = s.sync()
        ck = s.save_instance(0) if batched else s.save()
        s.close()
        assert r.status == 0 and r.two_site_updates == 72
        return ffi.sites_to_dense(ffi.checkpoint_to_sites(ck)[1])

    ref = run("c128", False)
    cuda_core = run("c64", False)
    tensor_core = run("c64", True)
    d_cc = 1 - fidelity(ref, cuda_core)
    d_tc = 1 - fidelity(ref, tensor_core)
    assert d_tc < 1e-5
    assert d_tc <= 10 * max(d_cc, 1e-9), (d_tc, d_cc)


@pytest.mark.parametrize("batched", [False, True])
def test_exact_chi256_state_matches_statevector(oracle, batched):
    """The large-theta kernels against the exact state vector: n=16 chain with couplings to
    distance 4, chi = 256 = 2^(n/2) (no truncation), so bonds reach 256 and every central update
    is a 512 x 512 theta -- the cooperative column-pair SVD for a single instance, the batched
    block-row-cyclic one for a batch.  A few steps of the anneal: state fidelity within 1e-8 of
    the oracle in the engine's splitting, the oracle's most probable pattern most probable in the
    MPS too."""
    p = instances.chain_range(n=16, dmax=4, seed=12, T=0.3, dt=0.1, chi=256)
    inst = Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)
    if batched:
        r = ffi.anneal_batch([p], want_checkpoint=True)[0]
    else:
        r = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=256, want_checkpoint=True)
    assert r.status == 0 and r.max_trunc < 1e-20
    psi = ffi.sites_to_dense(ffi.checkpoint_to_sites(r.checkpoint)[1])
    sv = oracle.sv_anneal(inst, p.sa, p.sb, p.dt, mode=1, want_state=True)
    assert 1 - fidelity(psi, sv.state) < 1e-8
    assert r.expected_energy == pytest.approx(sv.expected_energy, abs=1e-8)
    # h = 0 here: x and its complement are equally probable, so compare the maximum itself
    p_mps, p_sv = np.abs(psi) ** 2 / np.vdot(psi, psi).real, np.abs(sv.state) ** 2
    assert p_mps[int(np.argmax(p_sv))] == pytest.approx(p_mps.max(), rel=1e-9)


def test_autotuner_times_every_candidate_and_picks_the_fastest():
    from tessera_b200 import autotune
    probs = [instances.chain_range(n=24, dmax=2, seed=s, T=1.0, dt=0.05, chi=64) for s in (1, 2, 3)]
    # complex128 chi=64: a 128 x 128 theta is too big for the resident kernel, so the candidates
    # really are different kernels
    ch = autotune.tune(probs, 64, "c128", gates=2, cache=None)
    assert len(ch.measured) == len(autotune.candidates("c128"))
    times = {k: v["ms_per_update"] for k, v in ch.measured.items() if v["ms_per_update"] is not None}
    assert len(times) == len(ch.measured) and ch.ms_per_update == min(times.values())
    assert (ch.jacobi_block, ch.theta_tensor_cores, ch.jacobi_precondition) in autotune.candidates("c128")


def test_mps_sampling_matches_state_probabilities():
    """tessera_qa_session_sample draws patterns with the MPS's own probabilities: on an n=8
    exact-chi anneal the empirical frequencies of the most probable patterns agree with
    |<x|psi>|^2 / <psi|psi> within 5 standard errors, the total variation distance is small,
    the energies belong to the patterns, and a seed reproduces its draw."""
    m = _rand_small(8, 4)
    sa, sb = instances.linear(60)
    s = ffi.Session(m.h, m.ei, m.ej, m.ew, sa, sb, dt=0.1, chi=16)
    s.run(0, 60)
    s.sync()
    psi = ffi.sites_to_dense(ffi.checkpoint_to_sites(s.save())[1])
    prob = np.abs(psi) ** 2 / np.vdot(psi, psi).real
    N = 40000
    spins, en = s.sample(N, seed=7)
    idx = ((spins == -1).astype(np.int64) << np.arange(8)).sum(axis=1)
    freq = np.bincount(idx, minlength=256) / N
    for x in np.argsort(prob)[-10:]:
        assert abs(freq[x] - prob[x]) < 5 * np.sqrt(prob[x] * (1 - prob[x]) / N) + 1e-3, (x, freq[x], prob[x])
    assert 0.5 * np.abs(freq - prob).sum() < 0.05
    for k in range(20):
        x = spins[k]
        e = -sum(w * x[i] * x[j] for i, j, w in zip(m.ei, m.ej, m.ew)) - float(np.dot(m.h, x))
        assert en[k] == pytest.approx(e, abs=1e-12)
    again, _ = s.sample(100, seed=7)
    assert np.array_equal(again, spins[:100])
    s.close()


def test_precision_study_against_exact_state_vector():
    """The three arithmetic modes against the FP64 state vector at exact chi (16 instances, n=12):
    complex128 to rounding, complex64 (CUDA cores or split-TF32 tensor cores) to FP32 accuracy."""
    from tessera_b200 import precision
    r = precision.study(count=16)
    assert r["c128"]["infidelity_max"] < 1e-10 and r["c128"]["energy_rel_err_max"] < 1e-9
    for mode in ("c64", "c64_tensor_cores"):
        assert r[mode]["infidelity_max"] < 1e-4, (mode, r[mode])
        assert r[mode]["energy_rel_err_max"] < 1e-3, (mode, r[mode])
        assert r[mode]["schmidt_dev_max"] < 1e-3, (mode, r[mode])
    assert all(r[m]["status"] == [0] for m in ("c128", "c64", "c64_tensor_cores"))


def test_ragged_three_regular_batch_with_mixed_chi():
    """The batching workload's shape: random 3-regular graphs of uneven n (32..40) with bond caps
    chi = 64 or 128 in one batched session (complex64, long-range edges through the swap network,
    random saturated MPS).  Each instance's state after a window of gate slots, loaded into a
    single-instance session, has the same <H> as the same slots run on that instance alone."""
    probs = instances.batch_3_regular(count=6, T=0.2, dt=0.05, nmin=32, nmax=40)
    assert len({p.chi for p in probs}) == 2 and len({p.n for p in probs}) > 1
    sb = ffi.Session.batch(probs, precision="c64")
    sb.randomize(17)
    sb.run_gates(2, 10, 16)
    rb = sb.sync()
    assert rb.status == 0 and rb.two_site_updates == 6 * len(probs)
    for b, p in enumerate(probs):
        s1 = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=p.chi, precision="c64")
        s1.randomize(17 + 7919 * b)
        s1.run_gates(2, 10, 16)
        assert s1.sync().status == 0
        e_single = s1.observe().expected_energy
        s1.load(sb.save_instance(b))
        e_batch = s1.observe().expected_energy
        s1.close()
        assert e_batch == pytest.approx(e_single, rel=1e-3, abs=1e-4), (b, p.n, p.chi)
    sb.close()


def test_exact_chi1024_n20_matches_statevector(oracle):
    """Config 2b: the n=20 chain with couplings to distance 4 (J ~ U(-1, 1), h = 0) at exact
    chi = 1024 = 2^(n/2), against the exact state vector in the engine's splitting, on the CPU
    oracle and on the GPU (tessera_qa_sv_anneal).  The stated window is 12 Trotter steps at
    fixed s = 0.5 with dt = 0.25: from |+>^n that saturates the central bond at 1024 (its
    1024th Schmidt value is 3e-10 there, far above the noise floor), so the central updates
    run the 1024 x 1024 theta through the cooperative column-pair SVD.  Fidelity within 1e-8,
    <H> within 1e-8, the entropy trace within 1e-7, and the oracle's most probable pattern most
    probable in the MPS too (h = 0: a pattern and its complement tie)."""
    p = instances.chain_range(n=20, dmax=4, seed=2, T=1.0, dt=0.25, chi=1024)
    sa = np.full(12, 0.5)
    sb = np.full(12, 0.5)
    inst = Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)
    r = ffi.anneal(p.h, p.ei, p.ej, p.ew, sa, sb, dt=0.25, chi=1024, want_checkpoint=True)
    assert r.status == 0 and r.max_trunc < 1e-20
    assert r.max_bond == 1024
    psi = ffi.sites_to_dense(ffi.checkpoint_to_sites(r.checkpoint)[1])
    sv = oracle.sv_anneal(inst, sa, sb, 0.25, mode=1, want_state=True)
    gsv = ffi.sv_anneal(p.h, p.ei, p.ej, p.ew, sa, sb, dt=0.25, mode=1, want_state=True)
    for ref in (sv.state, gsv.state):
        assert 1 - fidelity(psi, ref) < 1e-8
    assert r.expected_energy == pytest.approx(sv.expected_energy, abs=1e-8)
    assert np.max(np.abs(r.entropy - sv.entropy)) < 1e-7
    p_mps, p_sv = np.abs(psi) ** 2 / np.vdot(psi, psi).real, np.abs(sv.state) ** 2
    assert p_mps[int(np.argmax(p_sv))] == pytest.approx(p_mps.max(), rel=1e-9)


def test_chain16_chi32_full_run_tracks_the_oracle():
    """Config 1 end to end: the n=16 chain (J ~ N(0, 1), h ~ N(0, 0.5)), linear schedule, T=20,
    dt=0.05, all 400 steps at chi=32 (truncating), against the oracle's accurate-SVD mode (the
    reference's algorithm: keep rule, gauge, gate order), whose run is stored in
    tests/golden/oracle_chain16_chi32.json (tests/golden/make_oracle_runs.py; two minutes of CPU).
    Over 400 truncating steps the run amplifies rounding: moving the inputs by 4 ulps moves the
    oracle's own <H> by about 7e-3.  So <H> and the entropy trace are held to ten times that
    sensitivity plus 1e-6; the readout spins, which the perturbed runs all share, and the
    readout energy are held exactly."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "oracle_chain16_chi32.json")) as f:
        g = json.load(f)
    o, sens = g["out"], g["sensitivity"]
    p = instances.chain_nn(n=16, seed=1, T=20.0, dt=0.05, chi=32)
    assert p.steps == 400
    r = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=32)
    assert r.status == 0 and r.two_site_updates == o["updates"]
    assert abs(r.expected_energy - o["expected_energy"]) <= 1e-6 * abs(o["expected_energy"]) + \
        10 * sens["expected_energy"]
    assert np.max(np.abs(r.entropy - np.array(o["entropy"]))) <= 1e-6 + 10 * sens["entropy"]
    assert g["spins_stable"] and list(r.spins) == o["spins"]
    assert r.energy == pytest.approx(o["energy"], abs=1e-9)


def mps_fidelity(a, b):
    """|<a|b>|^2 / (<a|a><b|b>) of two MPS given as site lists (Dl, 2, Dr), by left transfer
    matrices rescaled at every site (the random MPS here are far from normalised)."""
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


def left_norms(site):
    """Norm of every left-bond slice A[a, :, :]: the kept singular values for a site that an
    update last wrote as S Vh, and invariant under the SVD's phase freedom for every site."""
    return np.sqrt(np.sum(np.abs(site) ** 2, axis=(1, 2)))


@pytest.fixture(scope="module")
def chi256_window(oracle):
    """The headline update against the oracle: the bench's generator (chain with couplings to
    distance 4, J ~ U(-1, 1), h = 0) at n = 40, a random MPS with every interior bond at
    chi = 256, and three consecutive gate slots of the s = 0.5 step on interior bonds (swaps on
    bonds 16, 15, 14): three truncating 512 x 512 updates.  The oracle applies the same slots
    to the same MPS with the reference's update (keep rule, gauge A <- U, C <- S Vh) and an
    accurate SVD."""
    p = instances.chain_range(n=40, dmax=4, seed=2, T=50.0, dt=0.02, chi=256)
    step = len(p.sa) // 2
    bonds = []
    for i, j in zip(p.ei, p.ej):
        bonds += [k - 1 for k in range(int(j), int(i) + 1, -1)] + [int(i)] + [k for k in range(int(i) + 1, int(j))]
    q0 = next(q for q, b in enumerate(bonds) if b >= 16)
    s = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=256)
    s.randomize(31)
    start = ffi.checkpoint_to_sites(s.save())[1]
    s.close()
    inst = Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)
    o_sites, st = oracle.apply_slots(inst, start, float(p.sb[step]), p.dt, 256, q0, q0 + 3)
    return p, step, q0, start, o_sites, st


@pytest.mark.parametrize("batched,precond", [(False, 1), (False, 2), (True, 1), (True, 2)])
def test_truncating_chi256_updates_match_the_oracle(chi256_window, batched, precond):
    """Three truncating chi=256 updates (512 x 512 theta) through the cooperative single-instance
    SVD and the batched block-row-cyclic SVD, each with (1) and without (2) the pivoted-LQ
    preconditioner (cooperative or one CTA per theta), against the oracle.  The cut is well conditioned
    (relative gap at the cut above 1e-4 in every update), so two accurate SVDs differ there by
    rounding over the gap: the states agree to infidelity 1e-12, the discarded-weight ratio to
    1e-6 relative, and the kept singular values (left-slice norms of the sites last written as
    S Vh, and the same norms of every other site) to 1e-10 relative."""
    p, step, q0, start, o_sites, st = chi256_window
    assert st["updates"] == 3 and st["min_cut_gap"] > 1e-4 and st["max_trunc"] > 1e-3
    if batched:
        s = ffi.Session.batch([p], chi=256, jacobi_precondition=precond)
    else:
        s = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=256, jacobi_precondition=precond)
    s.randomize(31)
    s.run_gates(step, q0, q0 + 3)
    r = s.sync()
    ck = s.save_instance(0) if batched else s.save()
    s.close()
    assert r.status == 0 and r.two_site_updates == 3
    g_sites = ffi.checkpoint_to_sites(ck)[1]
    assert [t.shape for t in g_sites] == [t.shape for t in o_sites]
    assert 1 - mps_fidelity(g_sites, o_sites) < 1e-12
    assert r.max_trunc == pytest.approx(st["max_trunc"], rel=1e-6)
    for i, (g, o) in enumerate(zip(g_sites, o_sites)):
        ng, no = left_norms(g), left_norms(o)
        assert np.max(np.abs(ng - no) / no) < 1e-10, i


@pytest.mark.parametrize("precond", [1, 2])
def test_graded_chi256_updates_match_the_oracle(oracle, precond):
    """The bench's second input: a random MPS whose site columns fall off as exp(-b/24), so
    each theta's spectrum is graded like a TEBD state's Schmidt values (tessera_qa_session_
    randomize_graded).  Three chi=256 updates (512 x 512 theta) through the batched Jacobi with
    and without the pivoted-LQ preconditioner, against the oracle on the same start: infidelity
    under 1e-12, the (tiny) discarded weights equal to 1e-12 absolute, the left-slice norms of
    every site within 1e-10 relative where they exceed 1e-3 of the site's largest and within
    1e-12 of it elsewhere (the graded tail reaches the rounding floor)."""
    p = instances.chain_range(n=40, dmax=4, seed=2, T=50.0, dt=0.02, chi=256)
    step = len(p.sa) // 2
    bonds = []
    for i, j in zip(p.ei, p.ej):
        bonds += [k - 1 for k in range(int(j), int(i) + 1, -1)] + [int(i)] + [k for k in range(int(i) + 1, int(j))]
    q0 = next(q for q, b in enumerate(bonds) if b >= 16)
    s = ffi.Session.batch([p], chi=256, jacobi_precondition=precond)
    s.randomize(31, decay=24.0)
    start = ffi.checkpoint_to_sites(s.save_instance(0))[1]
    s.run_gates(step, q0, q0 + 3)
    r = s.sync()
    ck = s.save_instance(0)
    s.close()
    assert r.status == 0 and r.two_site_updates == 3
    inst = Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)
    o_sites, st = oracle.apply_slots(inst, start, float(p.sb[step]), p.dt, 256, q0, q0 + 3)
    g_sites = ffi.checkpoint_to_sites(ck)[1]
    assert [t.shape for t in g_sites] == [t.shape for t in o_sites]
    assert 1 - mps_fidelity(g_sites, o_sites) < 1e-12
    assert abs(r.max_trunc - st["max_trunc"]) < 1e-12
    for i, (g, o) in enumerate(zip(g_sites, o_sites)):
        ng, no = left_norms(g), left_norms(o)
        big = no > 1e-3 * no.max()
        assert np.max(np.abs(ng[big] - no[big]) / no[big]) < 1e-10, i
        assert np.max(np.abs(ng - no)) < 1e-12 * no.max(), i


def test_chi512_updates_with_and_without_the_preconditioner_agree():
    """1024 x 1024 theta in a single instance: the cooperative LQ runs on 128 CTAs before the
    cooperative Jacobi.  Three truncating chi=512 updates from the same random MPS (the
    precision study's generator, n=24, couplings to distance 2) with and without it: the states
    agree to infidelity 1e-11, the discarded weights to 1e-6 relative, and the preconditioned run
    takes fewer sweeps.  Without the preconditioner this path is the one the 1024 x 1024 SVD test
    and the exact chi=1024 anneal check."""
    from tessera_b200.precision import mps_fidelity as mfid
    p = instances.chain_range(n=24, dmax=2, seed=4, T=40.0, dt=0.02, chi=512, dist="normal", hzero=True)
    step = len(p.sa) // 2
    bonds = []
    for i, j in zip(p.ei, p.ej):
        bonds += [k - 1 for k in range(int(j), int(i) + 1, -1)] + [int(i)] + [k for k in range(int(i) + 1, int(j))]
    q0 = next(q for q, b in enumerate(bonds) if b >= 11)
    out = {}
    for precond in (1, 2):
        s = ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=512, jacobi_precondition=precond)
        s.randomize(4)
        s.run_gates(step, q0, q0 + 3)
        r = s.sync()
        out[precond] = (ffi.checkpoint_to_sites(s.save())[1], r)
        s.close()
        assert r.status == 0 and r.two_site_updates == 3
    (a, ra), (b, rb) = out[1], out[2]
    assert ra.max_bond == 512 and ra.max_trunc > 1e-6
    assert 1 - mfid(a, b) < 1e-11
    assert ra.max_trunc == pytest.approx(rb.max_trunc, rel=1e-6)
    assert ra.max_sweeps < rb.max_sweeps


def test_graph_captured_steps_equal_launched_steps():
    """The batched slot path captures one Trotter step into a CUDA graph and replays it for every
    step when no per-launch timing is asked for; with kernel timing it launches kernel by
    kernel. Same batch (128-row theta: too big for the resident kernel), same steps: the states,
    the discarded weight and the launch counts are identical."""
    probs = [instances.chain_range(n=12, dmax=3, seed=s, T=1.0, dt=0.05, chi=64) for s in (1, 2)]
    out = []
    for timing in (False, True):
        sb = ffi.Session.batch(probs, chi=64, kernel_timing=timing)
        sb.run(0, 6)
        r = sb.sync()
        assert r.status == 0
        out.append(([sb.save_instance(b) for b in range(len(probs))], r.max_trunc, r.two_site_updates,
                    r.svd_launches))
        sb.close()
    assert out[0][0] == out[1][0]
    assert out[0][1:] == out[1][1:]
    assert out[0][3] == 6 * max(p.updates_per_step() for p in probs)
