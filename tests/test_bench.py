"""Host-side logic of bench.py: the reference arm's JSON line, the roofline arithmetic and the clock
record.  No GPU, no CPU solve (the pooled oracle sample is replaced by a canned record)."""
import json
import sys
from pathlib import Path
from types import SimpleNamespace

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def canned_sample(workers=16):
    return {"workers": workers, "iterations_mean": 12.9, "text": "canned sample"}


def test_reference_arm_prints_one_contract_line(monkeypatch, capsys):
    calls = []

    def fake_samples(system, density, count=1, block=3, cores=None):
        calls.append(count)
        return [(30.0 + i, canned_sample()) for i in range(count)]

    monkeypatch.setattr(bench, "cpu_samples", fake_samples)
    monkeypatch.delenv("RANK", raising=False)
    args = SimpleNamespace(config="plate_96x96x16", warmup=3, steps=2, gpus=1)
    line = bench.reference(args)
    printed = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert printed == json.loads(json.dumps(line))
    assert calls == [5]                                  # warm-up and timed steps, one pool
    assert printed["impl"] == "reference" and printed["value"] == pytest.approx(33.5)   # mean of the timed steps
    assert printed["unit"] == "s" and printed["higher_is_better"] is False and printed["metric"] == bench.METRIC
    assert printed["config"]["workload"] == "plate_96x96x16" and printed["config"]["ndof"] == 479859
    cpu = printed["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] == 16 and cpu["value"] == printed["value"] and cpu["sample"]
    assert printed["e2e"] == {"value": printed["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_nothing(monkeypatch, capsys):
    monkeypatch.setattr(bench, "cpu_samples", lambda *a, **k: pytest.fail("rank 1 must not sample"))
    monkeypatch.setenv("RANK", "1")
    assert bench.reference(SimpleNamespace(config="plate_96x96x16", warmup=3, steps=2, gpus=2)) is None
    assert capsys.readouterr().out == ""


def test_reference_arm_retries_with_fewer_workers_then_reports_unavailable(monkeypatch, capsys):
    tried = []

    def broken(system, density, count=1, block=3, cores=None):
        tried.append(cores)
        raise RuntimeError("worker died")

    monkeypatch.setattr(bench, "cpu_samples", broken)
    monkeypatch.delenv("RANK", raising=False)
    import oracle.baseline
    monkeypatch.setattr(oracle.baseline, "host_cores", lambda: 8)
    assert bench.reference(SimpleNamespace(config="plate_96x96x16", warmup=0, steps=1, gpus=1)) is None
    out = json.loads(capsys.readouterr().out.strip())
    assert out["impl"] == "reference" and "worker died" in out["unavailable"]
    assert tried == [None, 4, 2]


def test_fma_roof_arithmetic():
    r = bench.fma_roof("fp32", 1152.0 * 159953 * 42, 0.283, sm_mhz=1342.0, sm_max_mhz=1965.0)
    assert r["peak"] == pytest.approx(148 * 128 * 2 * 1.965e-3, rel=1e-3)      # 74.4 TFLOP/s
    assert r["achieved"] == pytest.approx(1152.0 * 159953 * 42 / 0.283e-3 / 1e12, abs=0.01)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"], rel=1e-3)
    assert r["frac_at_sampled_clock"] == pytest.approx(r["frac"] * 1965.0 / 1342.0, rel=1e-3)
    d = bench.fma_roof("fp64", 1e9, 1.0)
    assert d["peak"] == pytest.approx(148 * 64 * 2 * 1.965e-3, rel=1e-3) and "frac_at_sampled_clock" not in d


def test_clock_summary_reads_reasons():
    c = bench.Clocks(0)
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1900, 1965, 990.5, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1800, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active",
               "garbage line"]
    s = c.summary()
    assert s["sm_mhz"] == 1900.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]
