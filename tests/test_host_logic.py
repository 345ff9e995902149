"""Host-side logic that needs no GPU: instance generators, schedules, the learned layer's
candidate family, warm-start schedule and targets, and the bench's instance sharding."""
import numpy as np
import pytest

from tessera_b200 import instances, learned


def test_three_regular_batch_shape():
    probs = instances.batch_3_regular(count=8, T=0.5, dt=0.05, nmin=32, nmax=48)
    for p in probs:
        assert p.n % 2 == 0 and 32 <= p.n <= 48 and p.chi in (64, 128)
        deg = np.bincount(np.concatenate([p.ei, p.ej]), minlength=p.n)
        assert np.all(deg == 3)
        pairs = set(zip(np.minimum(p.ei, p.ej).tolist(), np.maximum(p.ei, p.ej).tolist()))
        assert len(pairs) == p.m and all(i != j for i, j in pairs)
        assert list(zip(p.ei, p.ej)) == sorted(zip(p.ei, p.ej))  # lexicographic edge order
    assert len({p.steps for p in probs}) == 1


def test_linear_schedule_includes_both_ends():
    sa, sb = instances.linear(400)
    assert sb[0] == 0.0 and sb[-1] == 1.0 and np.allclose(sa + sb, 1.0)
    assert np.all(np.diff(sb) > 0)


def test_candidates_are_monotone_knot_schedules():
    c = learned.candidates(count=24)
    assert c.shape == (24, learned.K_KNOTS)
    assert np.all(c[:, 0] == 0.0) and np.all(c[:, -1] == 1.0)
    assert np.all(np.diff(c, axis=1) >= 0)
    assert np.allclose(c[0], np.linspace(0, 1, learned.K_KNOTS))  # candidate 0 is linear


def test_from_knots_interpolates_the_knots():
    kn = np.linspace(0, 1, 16) ** 2
    sa, sb = instances.from_knots(kn, 151)
    t = np.arange(151) / 150
    assert np.allclose(sb, np.interp(t, np.linspace(0, 1, 16), kn)) and np.allclose(sa, 1 - sb)


def test_warm_start_field_vanishes_at_both_ends():
    p = instances.dense_er(8, 3, T=1.0)
    cfg = learned.LearnConfig(T=2.0, dt=0.1, chi=16, bias_strength=0.7)
    q = learned.with_schedule(p, np.linspace(0, 1, 16), cfg, bias=np.ones(8))
    assert q.steps == 20 and q.sc[0] == 0.0 and q.sc[-1] == 0.0
    assert np.max(q.sc) == pytest.approx(0.7, rel=0.02)
    plain = learned.plain_problem(p, cfg)
    assert plain.bias is None and np.array_equal(plain.sb, instances.linear(20)[1])


def test_spin_targets_map_spins_to_probabilities():
    t = learned.spin_targets([np.array([1, -1, 1], np.int8), np.array([-1], np.int8)])
    assert t.tolist() == [1.0, 0.0, 1.0, 0.0] and t.dtype == np.float32
