"""Device OC driver and update (tf_oc_update, tf_filter_volume) against the reference's own runs.

Mirrors the reference's tests/test_topology_optimization.py: CPU = GPU densities
to 1e-7 after 3 OC updates (:491-521), robust continuation CPU = GPU (:523-535),
determinism (:109-118, :304-322), the OC bisection bar and the lowest-design
shortcut (:231-245), invalid sensitivities (:214-229).  Golden values come from
tests/golden/oc.npz (the reference's optimize_topology / _oc_update on the CPU).
"""
import json
from copy import deepcopy
from pathlib import Path

import numpy as np
import pytest

from oracle import density as oden

from test_oracle_oc import GOLDEN, beam_domain

pytestmark = pytest.mark.gpu


def run(name, **extra):
    from deep_frame_b200.topology_optimization import optimize_topology
    shape = tuple(int(s) for s in GOLDEN[f"{name}_shape"])
    settings = {**json.loads(str(GOLDEN[f"{name}_settings"])), **extra}
    result = optimize_topology(beam_domain(shape, tuple(GOLDEN[f"{name}_spacing"])), settings)
    assert result["status"] == "ok", result["diagnostics"]
    return result


def test_single_projection_three_updates_match_reference(cuda):
    result = run("single")
    assert np.max(np.abs(result["density"].ravel() - GOLDEN["single_density"])) < 1e-7
    assert np.max(np.abs(result["design_density"].ravel() - GOLDEN["single_design"])) < 1e-7
    assert result["summary"]["objective_final"] == pytest.approx(GOLDEN["single_objective"][-1], rel=1e-8)
    assert not result["summary"]["converged"] and result["summary"]["stop_reason"] == "max_iterations"
    assert len(result["history"]) == 4 and result["history"][-1]["final_evaluation"]


def test_robust_continuation_matches_reference(cuda):
    result = run("robust")
    assert [entry["projection_beta"] for entry in result["history"]] == GOLDEN["robust_beta"].tolist()
    for key, golden in (("density", "robust_density"), ("design_density", "robust_design"), ("eroded_density", "robust_eroded"),
                        ("dilated_density", "robust_dilated")):
        assert np.max(np.abs(result[key].ravel() - GOLDEN[golden])) < 1e-7, key
    names = json.loads(str(GOLDEN["robust_case_names"]))
    for entry, row in zip(result["history"], GOLDEN["robust_compliance"], strict=True):
        assert max(abs(entry["compliances_n_mm"][case] / value - 1) for case, value in zip(names, row)) < 1e-6
    assert abs(result["summary"]["objective_final"] / GOLDEN["robust_objective"][-1] - 1) < 1e-6
    assert np.allclose([e["dilated_volume_target"] for e in result["history"][:-1]], GOLDEN["robust_volume_target"][:-1], rtol=1e-9)


def test_multigrid_solver_path_matches_reference(cuda):
    result = run("robust", linear_solver="multigrid")
    assert np.max(np.abs(result["density"].ravel() - GOLDEN["robust_density"])) < 1e-6
    assert abs(result["summary"]["objective_final"] / GOLDEN["robust_objective"][-1] - 1) < 1e-6


def test_optimizer_is_bitwise_deterministic(cuda):
    first, second = run("robust"), run("robust")
    for key in ("density", "design_density", "eroded_density", "dilated_density", "filtered_density"):
        assert np.array_equal(first[key], second[key]), key
    strip = lambda history: [{k: v for k, v in entry.items() if k != "elapsed_s"} for entry in history]
    assert strip(first["history"]) == strip(second["history"])


def robust_map():
    from deep_frame_b200.density import DensityMap
    from deep_frame_b200.topology_optimization import _settings
    domain = beam_domain((6, 4, 4), (1.0, 1.0, 1.0))
    mapping = DensityMap(domain, _settings({"projection": "robust", "filter_radius_mm": 2.6}))
    mapping.beta = 4.0
    oracle = oden.DensityMapOracle((6, 4, 4), (1.0, 1.0, 1.0), 2.6, GOLDEN["update_allowed"], GOLDEN["update_preserve"], beta=4.0,
                                   eta=0.5, robust=True, delta=0.25)
    return mapping, oracle


def test_device_update_matches_reference_update(cuda):
    from deep_frame_b200.density import _oc_update
    mapping, oracle = robust_map()
    design, objective, volume = GOLDEN["update_design"], GOLDEN["update_objective"], GOLDEN["update_volume_derivative"]
    assert mapping.volume(design) == pytest.approx(oracle.volume(design), rel=1e-13)
    target = float(GOLDEN["update_target"])
    candidate = _oc_update(design, objective, volume, mapping, target, mapping.settings, 0.2)
    assert np.max(np.abs(candidate - GOLDEN["update_candidate"])) < 1e-7
    assert target * (1 - 1e-6) <= oracle.volume(candidate) <= target * (1 + 1e-12)
    assert np.max(np.abs(candidate - design)) <= 0.2 + 1e-15
    lowest = _oc_update(design, objective, volume, mapping, float(GOLDEN["update_lowest_target"]), mapping.settings, 0.05)
    assert np.array_equal(lowest, GOLDEN["update_lowest"])
    _, report = mapping.oc_update_device(mapping._dev(design), mapping._dev(objective), mapping._dev(volume), target, 0.2)
    assert not report["lowest"] and 3 <= report["evaluations"] <= 171
    bad = volume.copy()
    bad[np.flatnonzero(mapping.free)[0]] = -1e-9
    with pytest.raises(RuntimeError, match="OC sensitivities"):
        _oc_update(design, objective, bad, mapping, target, mapping.settings, 0.2)
    bad[np.flatnonzero(mapping.free)[0]] = np.nan
    with pytest.raises(RuntimeError, match="OC sensitivities"):
        _oc_update(design, objective, bad, mapping, target, mapping.settings, 0.2)
    mapping.close()


@pytest.mark.parametrize("beta", [32.0, 64.0])
def test_high_beta_saturated_volume_derivative_is_accepted(cuda, beta):
    from deep_frame_b200.density import _oc_update
    mapping, oracle = robust_map()
    mapping.beta = oracle.beta = beta
    design = np.ones(mapping.n)
    design[mapping.free] = 0.3
    fields, _ = mapping.fields(design)
    saturated = mapping.pullback(np.ones(mapping.n), fields["dilated"][1])
    saturated[np.flatnonzero(mapping.free)[::2]] = 0
    objective = -np.ones(mapping.n)
    target = 0.9 * mapping.volume(design)
    candidate = _oc_update(design, objective, saturated, mapping, target, mapping.settings, 0.2)
    expected = oden.oc_update(design, objective, saturated, oracle, target, 0.2)
    assert np.all(np.isfinite(candidate)) and mapping.volume(candidate) <= target
    assert np.max(np.abs(candidate - expected)) < 1e-7
    mapping.close()


def test_device_fields_are_ordered_and_respect_masks(cuda):
    from deep_frame_b200.density import DensityMap
    from deep_frame_b200.topology_optimization import _settings
    domain = beam_domain((6, 4, 4), (1.0, 1.0, 1.0))
    domain["allowed"][2:4, 1, 1] = False
    domain["forbidden"] = ~domain["allowed"]
    for beta in (1.0, 16.0, 64.0):
        mapping = DensityMap(domain, _settings({"projection": "robust", "filter_radius_mm": 2.6}))
        mapping.beta = beta
        oracle = oden.DensityMapOracle((6, 4, 4), (1, 1, 1), 2.6, domain["allowed"], domain["preserve"] & domain["allowed"], beta=beta,
                                       robust=True)
        design = np.random.default_rng(int(beta)).uniform(0, 1, mapping.n)
        fields, filtered = mapping.fields(design)
        ref, ref_filtered = oracle.fields(design)
        assert np.allclose(filtered, ref_filtered, rtol=0, atol=1e-14)
        for name in ("eroded", "intermediate", "dilated"):
            assert np.allclose(fields[name][0], ref[name][0], rtol=0, atol=1e-12)
            assert np.allclose(fields[name][1], ref[name][1], rtol=1e-12, atol=1e-12)
        assert np.all(fields["eroded"][0] <= fields["intermediate"][0]) and np.all(fields["intermediate"][0] <= fields["dilated"][0])
        mapping.close()


def test_outcome_files_round_trip(cuda, tmp_path):
    from deep_frame_b200 import results
    result = run("single")
    shape = tuple(int(s) for s in GOLDEN["single_shape"])
    dom = beam_domain(shape, tuple(GOLDEN["single_spacing"]))
    record = results.write_outcome(tmp_path, dom, result, name="single")
    back = results.read_outcome(tmp_path, record)
    assert np.array_equal(back["density"], result["density"]) and np.array_equal(back["design_density"], result["design_density"])
    assert back["summary"]["objective_final"] == result["summary"]["objective_final"]
    assert [e["objective"] for e in back["history"]] == [e["objective"] for e in result["history"]]
