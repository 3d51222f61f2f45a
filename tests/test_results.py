"""Result and checkpoint files (deep_frame_b200/results.py) in the reference's formats, on the CPU.

The layouts follow deep_frame/topology_pipeline.py:44-71,192-219,309 (fields.npz, result.json,
artifact digests) and tools/formulation_study.py:1066,1109,1216-1227 (design.npz, checkpoint and
best-feasible files).
"""
import json

import numpy as np
import pytest

from deep_frame_b200 import results


def outcome(shape=(4, 3, 2)):
    rng = np.random.default_rng(0)
    return {"status": "ok", "density": rng.uniform(size=shape), "design_density": rng.uniform(size=shape),
            "summary": {"iterations": np.int64(3), "objective_final": np.float64(0.5), "robust": {"thresholds": {"eroded": 0.75}}},
            "history": [{"iteration": 1, "maximum_design_change": np.float32(0.25), "compliances_n_mm": {"tip": 1.5}},
                        {"iteration": 2, "maximum_design_change": None}],
            "diagnostics": ["Density iteration stopped at max_iterations; convergence is not claimed"]}


def domain(shape=(4, 3, 2)):
    allowed = np.ones(shape, dtype=bool)
    allowed[0, 0, 0] = False
    preserve = np.zeros(shape, dtype=bool)
    preserve[-1] = True
    return {"allowed": allowed, "preserve": preserve, "forbidden": ~allowed}


def test_outcome_round_trip_and_artifact_digests(tmp_path):
    out = outcome()
    record = results.write_outcome(tmp_path, domain(), out, name="simp")
    assert record["status"] == "ok" and set(record["artifacts"]) == {"fields", "result"}
    assert record["artifacts"]["fields"]["path"] == "fields.npz" and record["artifacts"]["result"]["size_bytes"] > 0
    back = results.read_outcome(tmp_path, record)
    assert np.array_equal(back["density"], out["density"]) and np.array_equal(back["design_density"], out["design_density"])
    assert back["summary"] == {"iterations": 3, "objective_final": 0.5, "robust": {"thresholds": {"eroded": 0.75}}}
    assert back["history"][0]["maximum_design_change"] == 0.25 and back["history"][1]["maximum_design_change"] is None
    with np.load(tmp_path / "fields.npz") as fields:
        assert fields["allowed"].dtype == bool and np.array_equal(fields["forbidden"], ~fields["allowed"])
    raw = json.loads((tmp_path / "result.json").read_text())
    assert "density" not in raw and raw["status"] == "ok"
    (tmp_path / "result.json").write_text(json.dumps({**raw, "status": "failed"}))
    assert results.read_outcome(tmp_path, record) is None          # digest no longer matches


def test_json_rejects_nan_and_leaves_no_partial_file(tmp_path):
    with pytest.raises(ValueError):
        results.save_json(tmp_path / "r.json", {"x": float("nan")})
    assert not (tmp_path / "r.json").exists()


def test_design_checkpoint_and_best_files(tmp_path):
    grid = {"shape": [4, 3, 2], "spacing_mm": [1.0, 1.0, 1.0], "origin_mm": [0.0, 0.0, 0.0]}
    design = np.linspace(0, 1, 24)
    results.save_design(tmp_path, design, grid, {"status": "ok"})
    back, back_grid = results.load_design(tmp_path)
    assert np.array_equal(back, design) and back_grid == grid
    save = results.checkpoint(tmp_path / "ck.npz")
    save(design, [{"level": 0}, {"level": 2}], [])
    with np.load(tmp_path / "ck.npz") as ck:
        assert int(ck["level"]) == 2 and int(ck["iteration"]) == 2 and np.array_equal(ck["design"], design)
    keep = results.keep_best(tmp_path)
    keep(design, {"iteration": 7, "level": 1, "beta": 4.0, "f0": 0.3, "mass_g": 12.5, "max_violation": -1e-4})
    with np.load(tmp_path / "best_beta4.npz") as best:
        assert int(best["iteration"]) == 7 and float(best["mass_g"]) == 12.5


def test_mma_state_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    state = {"iteration": 5, "old1": rng.uniform(size=10), "old2": rng.uniform(size=10), "low": -rng.uniform(size=10),
             "upp": 1 + rng.uniform(size=10), "objective_scale": 123.25}
    x = rng.uniform(size=16)
    results.save_mma_state(tmp_path / "mma.npz", x, state, [{"iteration": 4, "tr": np.float64(1.5)}])
    back_x, back, history = results.load_mma_state(tmp_path / "mma.npz")
    assert np.array_equal(back_x, x) and back["iteration"] == 5 and back["objective_scale"] == 123.25
    for key in ("old1", "old2", "low", "upp"):
        assert np.array_equal(back[key], state[key])
    assert history == [{"iteration": 4, "tr": 1.5}]
