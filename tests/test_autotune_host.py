"""Host logic of the autotuner (no GPU): it picks the fastest candidate, skips failed ones,
caches the choice per workload key and reuses it without measuring."""
import json

import pytest

from tessera_b200 import autotune, instances


def test_tune_picks_fastest_and_caches(tmp_path, monkeypatch):
    probs = [instances.chain_range(n=40, dmax=2, seed=s, T=1.0, dt=0.05, chi=64) for s in (1, 2)]
    calls = []
    times = {(8, False, 1): 3.0, (8, False, 2): 3.5, (4, False, 1): 2.0, (32, False, 2): None,
             (16, False, 1): 2.2, (16, False, 2): 1.9, (16, True, 1): 2.5}

    def fake(problems, chi, precision, block, tc, q0, gates, seed=1234, precond=1):
        calls.append((block, tc, q0, gates))
        ups = min(p.updates_per_step() for p in problems)
        assert 0 <= q0 and q0 + 1 + gates <= ups
        return times[(block, tc, precond)]

    monkeypatch.setattr(autotune, "_time_candidate", fake)
    monkeypatch.setattr(autotune, "_gpu_name", lambda: "test-gpu")
    cache = str(tmp_path / "tune.json")
    ch = autotune.tune(probs, 64, "c64", cache=cache)
    assert (ch.jacobi_block, ch.theta_tensor_cores, ch.jacobi_precondition) == (16, False, 2)
    assert ch.ms_per_update == 1.9
    assert len(calls) == len(autotune.candidates("c64"))
    with open(cache) as f:
        d = json.load(f)
    assert any(k.startswith("chi=64|c64|B=2|test-gpu") for k in d)
    calls.clear()
    again = autotune.tune(probs, 64, "c64", cache=cache)
    assert calls == [] and again.jacobi_block == 16 and again.jacobi_precondition == 2
    forced = autotune.tune(probs, 64, "c64", cache=cache, force=True)
    assert len(calls) == len(autotune.candidates("c64")) and forced.jacobi_block == 16


def test_tune_fails_loudly_when_nothing_runs(monkeypatch):
    probs = [instances.chain_range(n=40, dmax=2, seed=1, T=1.0, dt=0.05, chi=64)]
    monkeypatch.setattr(autotune, "_time_candidate", lambda *a, **k: None)
    with pytest.raises(RuntimeError):
        autotune.tune(probs, 64, "c128", cache=None)
