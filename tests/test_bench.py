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

    def fake_samples(system, density, count=1, cores=None):
        calls.append(count)
        return [(30.0 + i, canned_sample()) for i in range(count)]

    monkeypatch.setattr(bench, "cpu_samples", fake_samples)
    monkeypatch.delenv("RANK", raising=False)
    args = SimpleNamespace(config="plate_96x96x16", warmup=3, steps=5, gpus=1)
    line = bench.reference(args)
    printed = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert printed == json.loads(json.dumps(line))
    assert calls == [4]                                  # one warm-up and at most three timed evaluations, one pool
    assert printed["steps"] == 3 and printed["warmup"] == 1 and printed["steps_requested"] == 5
    assert printed["impl"] == "reference" and printed["value"] == pytest.approx(32.0)   # mean of the timed evaluations
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

    def broken(system, density, count=1, cores=None):
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


def test_reference_arm_reports_a_problem_beyond_the_host_as_unavailable(monkeypatch, capsys):
    """The 352 x 352 x 48 plate (18.3 M dofs) is beyond the oracle's CPU budget: one line with the
    reason and the workload, no sampling, no extrapolated number."""
    monkeypatch.setattr(bench, "cpu_samples", lambda *a, **k: pytest.fail("must not sample"))
    monkeypatch.delenv("RANK", raising=False)
    line = bench.reference(SimpleNamespace(config="plate_352x352x48", warmup=5, steps=20, gpus=1))
    printed = json.loads(capsys.readouterr().out.strip())
    assert printed == line and printed["impl"] == "reference" and "value" not in printed
    assert "budget" in printed["unavailable"] and printed["config"] == {"workload": "plate_352x352x48", "ndof": 18317523}


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
    shaped like the 96 x 96 x 16 plate's) plus the CPU leg: every required key, the roofline
    arithmetic, the plain FP64 arm and the errors against the FP64 oracle fixture."""
    import numpy as np
    import torch
    ref = np.load(ROOT / "tests" / "golden" / "plate_96x96x16.npz")
    nodes, cols = 159953, 84

    def rows(scale_tr, scale_grad):
        return [{"name": "load_mean", "value": float(ref["tr"]) * scale_tr, "gradient": torch.as_tensor(ref["grad_mean"])},
                {"name": "load_worst", "value": float(ref["lambda_max"]), "gradient": torch.as_tensor(ref["grad_worst"] * scale_grad),
                 "info": {"ks_n_mm": float(ref["ks"])}}]

    result = {"rank": 0, "world": 1, "ms": 93.6, "dominant": "fine_work", "nodes": nodes, "cols": cols, "columns": [42, 42],
              "smoother": {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0, "tensor_cores": False, "precision": "float32",
                           "pcg_precision": "float64"},
              "dominant_per_launch_ms": 0.2832, "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 5},
              "ndof": 479859, "levels": 4, "coarsest_dofs": 1521, "iterations_max": [18, 18], "tuning": None,
              "launches_per_step": 2075.0, "breakdown": {"fine_work": {"ms": 20.4, "launches": 72}}, "converged": True,
              "e2e": {"ms": 95.8, "steps": 3, "h2d_bytes_per_step": 1179648, "d2h_bytes_per_step": 2373480},
              "rows": rows(1 + 1e-10, 1 + 1e-9),
              "plain": {"ms": 140.4, "steps": 3, "rows": rows(1.0, 1.0), "clocks": None, "iterations_max": [18, 18], "converged": True}}
    monkeypatch.setattr(bench, "ours", lambda args: (result, SimpleNamespace(ndof=479859), None, None))
    monkeypatch.setattr(bench, "cpu_samples", lambda system, density, **k: [(45.5, {"workers": 16, "text": "canned"})])
    monkeypatch.setattr(sys, "argv", ["bench.py", "--steps", "5", "--warmup", "3", "--config", "plate_96x96x16"])
    bench.main()
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "clocks", "gpu_launches", "roofline", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] == pytest.approx(0.0936) and line["n_gpus"] == 1 and line["gpu_launches"] == 10375
    assert line["config"]["workload"] == "plate_96x96x16" and line["config"]["outer"] == "fp64 PCG"
    roof = line["roofline"]
    # degree-1 schedule: every finest launch a residual apply, 9 words per node and column + the moduli
    algorithmic = nodes * 42 * 36 + nodes * 4
    assert roof["algorithmic_bytes_per_launch"] == algorithmic and roof["traffic"] == pytest.approx(bench.FINE_TRAFFIC["resid"])
    assert roof["achieved"] == pytest.approx(algorithmic / 0.2832e-3 / 1e9, abs=0.1) and roof["frac"] == pytest.approx(roof["achieved"] / roof["peak"], abs=1e-4)
    assert roof["compute"]["flops_per_launch"] == int(1152 * nodes * 42)
    cpu = line["cpu_baseline"]
    assert cpu["value"] == 45.5 and cpu["cores"] == 16 and cpu["kind"] == "port" and cpu["workload"] == "plate_96x96x16"
    assert line["e2e"]["value"] == pytest.approx(0.0958) and line["e2e"]["call"].startswith("InterfaceCovariance")
    plain = line["results"]["plain_fp64"]
    assert plain["s"] == pytest.approx(0.1404) and plain["speedup_of_value"] == pytest.approx(1.5, abs=1e-3)
    assert plain["fast_vs_plain"]["tr_rel"] == pytest.approx(1e-10, rel=1e-3) and plain["fast_vs_plain"]["lambda_max_rel"] == 0.0
    errors = line["results"]["vs_fp64_oracle"]
    assert errors["tr_rel"] == pytest.approx(1e-10, rel=1e-3) and errors["lambda_max_rel"] == 0.0
    assert errors["grad_mean_rel"] == 0.0 and errors["grad_worst_rel"] == pytest.approx(1e-9, rel=1e-3)


def test_cpu_leg_of_a_workload_beyond_the_host_measures_the_small_plate(monkeypatch, capsys):
    """On the 352 x 352 x 48 plate the GPU line's cpu_baseline is a full measured evaluation of the
    96 x 96 x 16 plate, and says so."""
    import torch
    seen = []
    rows = [{"name": "load_mean", "value": 1.0, "gradient": torch.ones(3)},
            {"name": "load_worst", "value": 0.5, "gradient": torch.ones(3), "info": {"ks_n_mm": 0.6}}]
    result = {"rank": 0, "world": 1, "ms": 2000.0, "dominant": "fine_work", "nodes": 10, "cols": 84, "columns": [42, 42],
              "smoother": {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0}, "clocks": None, "ndof": 18317523,
              "levels": 6, "coarsest_dofs": 4000, "iterations_max": [23, 23], "tuning": None, "launches_per_step": 10.0,
              "breakdown": {}, "converged": True, "rows": rows}
    monkeypatch.setattr(bench, "ours", lambda args: (result, SimpleNamespace(ndof=18317523), None, None))
    monkeypatch.setattr(bench, "cpu_problem", lambda config: (None, SimpleNamespace(ndof=479859, name=config), None, "density"))

    def fake(system, density, **k):
        seen.append(system.name)
        return [(45.5, {"workers": 16, "text": "canned"})]

    monkeypatch.setattr(bench, "cpu_samples", fake)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--steps", "2", "--warmup", "3"])
    bench.main()
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert seen == ["plate_96x96x16"] and line["config"]["workload"] == "plate_352x352x48"
    assert line["cpu_baseline"]["workload"] == "plate_96x96x16" and "not plate_352x352x48" in line["cpu_baseline"]["sample"]


def test_options_of_the_side_benchmarks():
    """The batch, tile-height and coarsest-size options parse and reach the solver settings."""
    args = bench.parse(["--instances", "32", "--instance-sizes", "small", "--fine-tz", "7", "--coarsest-dofs", "80000"])
    assert args.instances == 32 and args.instance_sizes == "small" and args.fine_tz == 7 and args.coarsest_dofs == 80000
    assert bench.fast_settings(args)["fine_tz"] == 7
    schedule = bench.schedule_settings(args.schedule, args.coarsest_dofs)
    assert schedule["coarsest_dofs"] == 80000 and schedule["smoother"] == "chebyshev"
    assert "coarsest_dofs" not in bench.schedule_settings(args.schedule, 0)
    defaults = bench.parse([])
    assert defaults.instance_sizes == "plate" and defaults.fine_tz == 0 and defaults.learned_epochs == 4
    with pytest.raises(SystemExit):
        bench.parse(["--fine-tz", "6"])
