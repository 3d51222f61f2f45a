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


def test_gpu_arm_line_from_a_device_result(monkeypatch, capsys):
    """main() assembles the contract line from what ours() measured (a canned device result here,
    shaped like the plate's) plus the CPU leg: every required key, the roofline arithmetic and
    the errors against the FP64 oracle fixture."""
    import numpy as np
    ref = np.load(ROOT / "tests" / "golden" / "plate_96x96x16.npz")
    nodes, cols = 159953, 84
    result = {"rank": 0, "world": 1, "ms": 93.6, "dominant": "fine_work", "nodes": nodes, "cols": cols, "columns": [42, 42],
              "smoother": {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0, "tensor_cores": False},
              "dominant_per_launch_ms": 0.2832, "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 5},
              "ndof": 479859, "levels": 4, "coarsest_dofs": 1521, "iterations_max": [18, 18], "tuning": None,
              "launches_per_step": 2075.0, "breakdown": {"fine_work": {"ms": 20.4, "launches": 72}}, "converged": True,
              "e2e": {"ms": 95.8, "h2d_bytes_per_step": 2359296, "d2h_bytes_per_step": 2359312},
              "solve_api": {"ms": 267.2, "h2d_bytes_per_step": 1, "d2h_bytes_per_step": 1},
              "measure_api": {"ms": 97.0, "h2d_bytes_per_step": 1179648, "d2h_bytes_per_step": 2373480},
              "tr": float(ref["tr"]) * (1 + 1e-10), "lambda_max": float(ref["lambda_max"]),
              "grad_mean": ref["grad_mean"], "grad_worst": ref["grad_worst"] * (1 + 1e-9)}
    monkeypatch.setattr(bench, "ours", lambda args: (result, SimpleNamespace(), None, None))
    monkeypatch.setattr(bench, "cpu_samples", lambda system, density, **k: [(32.08, {"workers": 16, "text": "canned"})])
    monkeypatch.setattr(sys, "argv", ["bench.py", "--steps", "5", "--warmup", "3", "--schedule", "1,2"])
    bench.main()
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "clocks", "gpu_launches", "roofline", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] == pytest.approx(0.0936) and line["n_gpus"] == 1 and line["gpu_launches"] == 10375
    assert line["config"]["workload"] == "plate_96x96x16" and line["config"]["smoother_choice"] == "fixed by --schedule"
    roof = line["roofline"]
    # degree-1 schedule: every finest launch a residual apply, 9 words per node and column + the moduli
    algorithmic = nodes * 42 * 36 + nodes * 4
    assert roof["algorithmic_bytes_per_launch"] == algorithmic and roof["traffic"] == bench.FINE_TRAFFIC["resid"]
    assert roof["achieved"] == pytest.approx(algorithmic / 0.2832e-3 / 1e9, abs=0.1) and roof["frac"] == pytest.approx(roof["achieved"] / roof["peak"], abs=1e-4)
    assert roof["compute"]["flops_per_launch"] == int(1152 * nodes * 42)
    assert line["cpu_baseline"] == {"value": 32.08, "unit": "s", "cores": 16, "kind": "port", "sample": "canned"}
    assert line["e2e"]["value"] == pytest.approx(0.0958) and line["e2e"]["h2d_bytes_per_step"] == 2359296
    assert line["e2e_measure_api"]["value"] == pytest.approx(0.097) and line["e2e_measure_api"]["call"].startswith("InterfaceCovariance")
    errors = line["results"]["vs_fp64_oracle"]
    assert errors["tr_rel"] == pytest.approx(1e-10, rel=1e-3) and errors["lambda_max_rel"] == 0.0
    assert errors["grad_mean_rel"] == 0.0 and errors["grad_worst_rel"] == pytest.approx(1e-9, rel=1e-3)
