"""The JSON line of `bench.py --impl reference` on CPU: its keys, units and the scaling.

The reference's own update sample (concurrent MPS::apply_adjacent calls on saturated bonds,
a few seconds per step at chi=64) is replaced by a stub that returns fixed wall times, so only
the line's assembly is under test: rank 0 alone prints one line; other ranks print nothing;
value = threads / (t64 * t256 / t64') with the direct chi=256 measurement and its chi=64 time
t64' recorded in profiles/reference_update_chi256.json; without that record, value = threads /
(t64 * 4^p) with p = log2(t64 / t32), both at the same concurrency; with --ref-chi 256 the
chi=256 time is used directly.
"""
import io
import json
import math
import sys
from contextlib import redirect_stdout

import pytest

import bench


def _run(monkeypatch, argv, rank="0"):
    from oracle import oracle as orc
    monkeypatch.setattr(sys, "argv", ["bench.py"] + argv)
    monkeypatch.setenv("RANK", rank)
    monkeypatch.setattr(orc.Reference, "available", staticmethod(lambda: True))
    times = {32: 0.01, 64: 0.05, 128: 0.8, 256: 9.0}
    monkeypatch.setattr(bench, "ref_update_sample", lambda chi, threads, seed=0: (times[chi], [times[chi]] * threads))
    out = io.StringIO()
    with redirect_stdout(out):
        bench.run_reference(bench.parse())
    return out.getvalue()


def test_reference_line_keys_and_value(monkeypatch):
    text = _run(monkeypatch, ["--impl", "reference", "--steps", "2", "--warmup", "1"])
    lines = [l for l in text.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["higher_is_better"] is True and d["vs_baseline"] is None
    cal = json.load(open(bench.REF_DIRECT))
    threads = d["cpu_baseline"]["cores"]
    assert threads >= 1
    ratio = cal["seconds"] / cal["calibration"]["chi64_seconds"]
    assert d["value"] == pytest.approx(threads / (0.05 * ratio))
    assert d["ms_per_step"] == pytest.approx(50.0)
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["unit"] == bench.UNIT
    assert "measured directly on this pool" in cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["config"]["chi"] == 256 and d["config"]["updates_per_trotter_step"] == 1998


def test_reference_line_only_on_rank_zero(monkeypatch):
    assert _run(monkeypatch, ["--impl", "reference", "--steps", "1", "--warmup", "0"], rank="1") == ""


def test_reference_line_direct_chi256(monkeypatch):
    text = _run(monkeypatch, ["--impl", "reference", "--steps", "1", "--warmup", "0", "--ref-chi", "256"])
    d = json.loads(text.strip())
    assert d["value"] == pytest.approx(d["cpu_baseline"]["cores"] / 9.0)
    assert "measured directly" in d["cpu_baseline"]["sample"]


def test_reference_line_without_the_direct_record(monkeypatch, tmp_path):
    monkeypatch.setattr(bench, "REF_DIRECT", str(tmp_path / "absent.json"))
    d = json.loads(_run(monkeypatch, ["--impl", "reference", "--steps", "1", "--warmup", "0"]).strip())
    p = math.log2(0.05 / 0.01)
    assert d["value"] == pytest.approx(d["cpu_baseline"]["cores"] / (0.05 * 4.0 ** p))
    assert "extrapolated" in d["cpu_baseline"]["sample"] and "same concurrency" in d["cpu_baseline"]["sample"]
