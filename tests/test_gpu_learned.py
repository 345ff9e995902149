"""The learned-schedule layer on the GPU: exact ground state, GNN forward/backward against the
float64 CPU oracle (oracle/gnn_oracle.py), the warm-start bias field, and the gain of training.

Tolerances: exact ground energy and spins bit-exact (same enumeration order and tie rule as
rust/src/ising.rs:46-61); GNN with FP32 weights: outputs within 1e-4 and gradient within 2e-3
relative (L2) of float64 autograd; BF16 weights: knots within 3e-2 of the FP32 network; bias
field at exact chi: state fidelity within 1e-8 of the exact state vector.
"""
import numpy as np
import pytest

from oracle import gnn_oracle
from oracle.oracle import Instance
from tessera_b200 import ffi, instances, learned

pytestmark = pytest.mark.gpu


def _inst(p):
    return Instance(p.h, p.ei.astype(np.int32), p.ej.astype(np.int32), p.ew)


def test_exact_ground_matches_oracle(oracle):
    for n, seed in ((6, 1), (9, 2), (12, 3), (16, 4)):
        p = instances.dense_er(n, seed, T=1.0)
        e, s = learned.exact_ground(p)
        s_ref, e_ref = oracle.exact_ground(_inst(p))
        assert e == e_ref
        assert list(s) == list(s_ref)


def test_gnn_gradient_matches_float64_oracle():
    probs = [instances.dense_er(n, 10 + n, T=1.0) for n in (5, 7, 8)]
    H, L, K = 16, 2, 8
    g = learned.ScheduleGNN(hidden=H, layers=L, knots=K, seed=3, bf16=False)
    theta = g.get_params().astype(np.float64)
    rng = np.random.Generator(np.random.PCG64(0))
    tk = np.sort(rng.random((len(probs), K)), axis=1)
    tk[:, 0], tk[:, -1] = 0.0, 1.0
    ts = np.concatenate([rng.integers(0, 2, p.n).astype(np.float32) for p in probs])
    ts[1] = -1.0  # an unlabelled node
    kn, pp = g.forward(probs)
    loss, grad = g.train_step(probs, tk, ts, lr=0.0, lambda_knots=1.0, lambda_spins=0.5, want_grads=True)
    l_ref, g_ref, kn_ref, p_ref = gnn_oracle.loss_and_grad(theta, probs, tk, ts, H, L, K, 1.0, 0.5)
    assert np.max(np.abs(kn - kn_ref)) < 1e-4
    assert np.max(np.abs(pp - p_ref)) < 1e-4
    assert loss == pytest.approx(l_ref, rel=1e-4)
    assert np.linalg.norm(grad - g_ref) <= 2e-3 * np.linalg.norm(g_ref)
    g.close()


def test_gnn_bf16_forward_close_to_fp32():
    probs = [instances.dense_er(n, 20 + n, T=1.0) for n in (8, 10, 12)]
    a = learned.ScheduleGNN(seed=5, bf16=False)
    b = learned.ScheduleGNN(seed=5, bf16=True)
    ka, pa = a.forward(probs)
    kb, pb = b.forward(probs)
    assert np.all(np.diff(kb, axis=1) >= -1e-6) and np.allclose(kb[:, [0, -1]], [0.0, 1.0], atol=1e-6)
    assert np.max(np.abs(ka - kb)) < 3e-2
    assert np.max(np.abs(pa - pb)) < 3e-2


def test_bias_field_matches_statevector(oracle):
    p = instances.dense_er(8, 31, T=3.0, dt=0.1)
    rng = np.random.Generator(np.random.PCG64(1))
    bias = rng.uniform(-1, 1, p.n)
    sc = 0.5 * 4 * p.sb * (1 - p.sb)
    r = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=16, bias=bias, sc=sc, want_checkpoint=True)
    sv = oracle.sv_anneal(_inst(p), p.sa, p.sb, p.dt, mode=1, want_state=True, bias=bias, sc=sc)
    _, sites = ffi.checkpoint_to_sites(r.checkpoint)
    psi = ffi.sites_to_dense(sites)
    fid = abs(np.vdot(psi, sv.state)) ** 2 / (np.vdot(psi, psi).real * np.vdot(sv.state, sv.state).real)
    assert 1 - fid < 1e-8
    # and the bias really changes the dynamics
    r0 = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=16)
    assert abs(r0.expected_energy - r.expected_energy) > 1e-6


def test_training_reduces_loss_and_beats_the_untrained_network():
    """The gain test: on held-out instances, schedules from the trained network reach lower
    energies than those of the same network untrained; the learned schedule on its own, without
    the fallback, beats the linear schedule it replaces (same batch, same precision, mean gap to
    the exact ground energy); and with the fallback rule the chosen result is never worse than
    the plain linear schedule."""
    cfg = learned.LearnConfig(T=4.0, dt=0.1, chi=16, precision="c64")
    train_p = [instances.dense_er(n, 1000 + i, T=1.0) for i, n in enumerate([8, 9, 10] * 16)]
    test_p = [instances.dense_er(n, 5000 + i, T=1.0) for i, n in enumerate([10, 11] * 6)]
    cands = learned.candidates(count=16)
    tk, e0, gs, gaps = learned.label(train_p, cfg, cands)
    assert np.all(gaps.min(axis=1) <= gaps[:, 0] + 1e-12)  # the label is at least as good as linear
    net = learned.ScheduleGNN(seed=11)
    untrained = learned.ScheduleGNN(seed=11)
    losses = learned.train(net, train_p, tk, gs, epochs=40, batch=16, lr=3e-3)
    assert np.mean(losses[-5:]) < 0.6 * np.mean(losses[:5])
    e0_test = np.array([learned.exact_ground(p)[0] for p in test_p])

    def mean_gap(model):
        kn, bias = model.predict(test_p)
        res = ffi.anneal_batch([learned.with_schedule(p, kn[g], cfg, bias[g]) for g, p in enumerate(test_p)],
                               precision=cfg.precision, raise_on_status=False)
        return float(np.mean([(r.energy - e) / abs(e) for r, e in zip(res, e0_test)]))

    assert mean_gap(net) <= mean_gap(untrained) + 1e-12
    ev = learned.evaluate(net, test_p, cfg)
    assert ev["reference_energy"] == {"exact": len(test_p), "sa": 0}
    assert ev["learned_mean_gap_no_fallback"] < ev["linear_c64_mean_gap"], ev
    assert ev["chosen_solved"] >= ev["plain_solved"]
    assert ev["chosen_mean_gap"] <= ev["plain_mean_gap"] + 1e-9


def test_apply_grads_is_an_adam_step_on_the_given_gradient():
    """tessera_qa_gnn_apply_grads (the data-parallel path's optimizer step) applies Adam
    (beta 0.9 / 0.999, eps 1e-8, bias-corrected, the update train_step makes) to exactly the
    gradient it is given: two steps checked against a float64 restatement."""
    probs = [instances.dense_er(n, 40 + n, T=1.0) for n in (6, 8, 9)]
    rng = np.random.Generator(np.random.PCG64(2))
    tk = np.sort(rng.random((len(probs), 16)), axis=1)
    tk[:, 0], tk[:, -1] = 0.0, 1.0
    ts = np.concatenate([rng.integers(0, 2, p.n).astype(np.float32) for p in probs])
    net = learned.ScheduleGNN(seed=4, bf16=False)
    p = net.get_params().astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    lr = 1e-2
    for step in (1, 2):
        _, g = net.train_step(probs, tk, ts, lr=0.0, want_grads=True)  # lr = 0: no optimizer step
        net.apply_grads(g, lr=lr)
        g = g.astype(np.float64)
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g * g
        p = p - lr * (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8)
        assert np.allclose(net.get_params(), p, rtol=1e-5, atol=2e-6), step
