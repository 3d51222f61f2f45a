"""SIMP + optimality-criteria topology optimisation (the reference's OC driver), device resident.

Drop-in for ``deep_frame.topology_optimization``'s optimisation entry points:
``optimize_topology(domain, settings, progress_callback=None)``
(topology_optimization.py:1265-1406), its settings (``DEFAULT_SETTINGS`` /
``_settings``, :969-1054), ``continuation_decision`` (:17-25), the case
normalisation and history records (:1235-1263), plus re-exports of the
element, system and density classes under the reference's names.

Per iteration: the density fields (single intermediate projection, or robust
eroded / intermediate / dilated) come from the device cone filter; the
stiffness field goes through ``HexElasticity.solve`` (multigrid PCG or the
device Cholesky); the compliance gradient and the volume gradient are pulled
back through the filter on the device; the OC multiplier search runs on the
device (``tf_oc_update``).  Robust runs use beta continuation with the
reference's level rules and the relaxed dilated-volume target.  Modal
constraints, corridor blends and prop-disc volume weights are not part of
this library and are rejected as invalid settings.
"""
from copy import deepcopy
from time import perf_counter

import numpy as np

from .density import ConeFilter, DensityMap, _oc_update
from .elasticity import HexElasticity
from .elements import elasticity_matrix, hexahedron_matrices, regular_grid

__all__ = ["DEFAULT_SETTINGS", "LINEAR_SOLVERS", "DENSITY_FILTERS", "ConeFilter", "DensityMap", "HexElasticity", "_oc_update",
           "_settings", "continuation_decision", "elasticity_matrix", "hexahedron_matrices", "optimize_topology", "regular_grid",
           "validate_masks"]

LINEAR_SOLVERS = ("auto", "cpu_superlu", "cuda_cudss", "multigrid")
DENSITY_FILTERS = ("auto", "sparse", "convolution")
SOLVER_CHOICE = {"multigrid_below_mm": 1.1}

DEFAULT_SETTINGS = {
    "volume_fraction": 0.20,
    "filter_radius_mm": 6.0,
    "penalization": 3.0,
    "min_stiffness_ratio": 1e-6,
    "max_iterations": 60,
    "minimum_iterations": 10,
    "change_tolerance": 0.01,
    "move_limit": 0.15,
    "projection_beta": 1.0,
    "projection_eta": 0.5,
    "minimum_design_density": 1e-3,
    "case_weights": {},
    "max_runtime_s": None,
    "interface_node_policy": "allowed_adjacent",
    "linear_solver": "auto",
    "projection": "single",
    "robust_delta": 0.25,
    "beta_schedule": None,
    "beta_interval": 50,
    "beta_minimum_iterations": 20,
    "beta_change_tolerance": 0.01,
    "move_limit_late": None,
    "move_limit_late_beta": 8.0,
    "volume_target_relaxation": 0.2,
    "objective_window": 10,
    "gpu_solver_residency": "resident",
    "prop_discs": None,
    "modal": None,
    "feasibility_tolerance": 1e-3,
    "solver_choice": SOLVER_CHOICE,
    "density_filter": "auto",
    "corridor": None,
}


def _positive_integer(value):
    return not isinstance(value, bool) and int(value) == value and value >= 1


def _is_positive_finite(value):
    return bool(np.isfinite(value)) and value > 0


def _robust_ok(s):
    delta, eta = s["robust_delta"], s["projection_eta"]
    return s["projection"] != "robust" or (np.isfinite(delta) and delta > 0 and 0 < eta - delta < eta + delta < 1)


def _schedule_ok(schedule):
    if schedule is None:
        return True
    values = [float(beta) for beta in schedule]
    return bool(values) and all(np.isfinite(values)) and values[0] > 0 and all(b > a for a, b in zip(values, values[1:]))


# The reference's settings rules in its order, each with its message (topology_optimization.py:993-1054).
_RULES = (
    [(lambda s, n=name: _is_positive_finite(s[n]), f"{name} must be finite and positive")
     for name in ("filter_radius_mm", "penalization", "min_stiffness_ratio", "change_tolerance", "move_limit", "minimum_design_density")]
    + [(lambda s, n=name: _positive_integer(s[n]), f"{name} must be a positive integer") for name in ("max_iterations", "minimum_iterations")]
    + [(lambda s: bool(np.isfinite(s["volume_fraction"])) and 0 < s["volume_fraction"] <= 1, "volume_fraction must be in (0, 1]"),
       (lambda s: s["penalization"] >= 1 and 0 < s["min_stiffness_ratio"] < 1 and s["minimum_design_density"] < 1 and s["move_limit"] <= 1,
        "Invalid SIMP or OC settings"),
       (lambda s: bool(np.isfinite(s["projection_beta"])) and s["projection_beta"] >= 0 and 0 < s["projection_eta"] < 1,
        "Invalid density projection settings"),
       (lambda s: s["max_runtime_s"] is None or _is_positive_finite(s["max_runtime_s"]), "max_runtime_s must be positive or None"),
       (lambda s: s["interface_node_policy"] in ("allowed_adjacent", "preserve_adjacent"), "Invalid topology interface_node_policy"),
       (lambda s: s["linear_solver"] in LINEAR_SOLVERS, "Invalid topology linear_solver"),
       (lambda s: s["gpu_solver_residency"] in ("resident", "transient"), "Invalid topology gpu_solver_residency"),
       (lambda s: s["density_filter"] in DENSITY_FILTERS, "Invalid topology density_filter"),
       (lambda s: s["projection"] in ("single", "robust"), "Invalid topology projection"),
       (_robust_ok, "Robust projection thresholds must lie within (0, 1)")]
    + [(lambda s, n=name: _positive_integer(s[n]), f"{name} must be a positive integer") for name in ("beta_interval", "beta_minimum_iterations")]
    + [(lambda s: not isinstance(s["objective_window"], bool) and int(s["objective_window"]) == s["objective_window"] and s["objective_window"] >= 2,
        "objective_window must be an integer of at least 2"),
       (lambda s: _schedule_ok(s["beta_schedule"]), "beta_schedule must be a nonempty strictly increasing list of positive values"),
       (lambda s: s["move_limit_late"] is None or (bool(np.isfinite(s["move_limit_late"])) and 0 < s["move_limit_late"] <= 1),
        "move_limit_late must be in (0, 1] or None"),
       (lambda s: _is_positive_finite(s["beta_change_tolerance"]) and bool(np.isfinite(s["move_limit_late_beta"]))
        and bool(np.isfinite(s["volume_target_relaxation"])) and 0 < s["volume_target_relaxation"] <= 1, "Invalid beta continuation settings")]
)


def _settings(settings):
    """Defaults plus the reference's validation rules and messages, checked in the reference's order;
    the minimum iteration counts are clipped to their maxima and the beta schedule made floats.
    Options this library does not implement are rejected as invalid."""
    result = deepcopy(DEFAULT_SETTINGS)
    result.update(deepcopy(settings))
    for rule, message in _RULES:
        if not rule(result):
            raise ValueError(message)
        if message.startswith("minimum_iterations"):
            result["minimum_iterations"] = min(result["minimum_iterations"], result["max_iterations"])
        if message.startswith("beta_minimum_iterations"):
            result["beta_minimum_iterations"] = min(result["beta_minimum_iterations"], result["beta_interval"])
    if result["beta_schedule"] is not None:
        result["beta_schedule"] = [float(beta) for beta in result["beta_schedule"]]
    for name, what in (("modal", "modal constraints"), ("corridor", "corridor blends"), ("prop_discs", "prop-disc volume weights")):
        if result[name] is not None:
            raise ValueError(f"{what} are not part of this library")
    return result


def validate_masks(domain):
    """(allowed, preserve, forbidden) as flat boolean arrays after the reference's checks
    (topology_optimization.py:1056-1069): grid-shaped booleans, forbidden the complement of allowed,
    preserve inside allowed, and at least one free cell."""
    shape = tuple(domain["grid"]["shape"])
    arrays = {name: np.asarray(domain[name]) for name in ("allowed", "preserve", "forbidden")}
    for name, array in arrays.items():
        if array.dtype != bool or array.shape != shape:
            raise ValueError(f"{name} must be a boolean array with grid shape")
    allowed, preserve, forbidden = (arrays[name].ravel().copy() for name in ("allowed", "preserve", "forbidden"))
    if (forbidden != ~allowed).any() or (preserve & forbidden).any():
        raise ValueError("Forbidden must complement allowed; preserve must be allowed")
    if not (allowed & ~preserve).any():
        raise ValueError("The design domain has no free material cells")
    return allowed, preserve, forbidden


def continuation_decision(iterations, final_level, change, violation, minimum, maximum, change_tolerance, violation_tolerance):
    """The reference's stopping rule for one continuation level (topology_optimization.py:17-25):
    "converged" (final level) or "advance" once past the minimum iterations with a design change
    below tolerance and a feasible design; at the iteration cap "iteration_cap" on the final level
    (or when the cap is below the minimum), "advance" otherwise; None to keep iterating."""
    limit = 1e-3 if violation_tolerance is None else violation_tolerance
    done = (iterations >= minimum and change is not None and np.isfinite(change) and change < change_tolerance
            and np.isfinite(violation) and violation <= limit)
    if done:
        return "converged" if final_level else "advance"
    if iterations < maximum:
        return None
    return "iteration_cap" if (final_level or iterations < minimum) else "advance"


def _case_scaling(solutions, settings):
    """(objective scale per case, first compliances, normalised weights): each static case counts with
    weight / total weight / its first compliance (topology_optimization.py:1235-1245)."""
    given = settings["case_weights"]
    if not set(given) <= set(solutions):
        raise ValueError("case_weights references an unknown static load case")
    weights = {name: float(given.get(name, 1.0)) for name in solutions}
    if not all(np.isfinite(w) and w > 0 for w in weights.values()):
        raise ValueError("Every static load case requires a finite positive weight")
    total = sum(weights.values())
    first = {name: entry["compliance_n_mm"] for name, entry in solutions.items()}
    shares = {name: w / total for name, w in weights.items()}
    return {name: shares[name] / first[name] for name in solutions}, first, shares


def _history_entry(iteration, physical_sum, solutions, scales, change, elapsed, final=False):
    """One record of the OC history with the reference's keys (topology_optimization.py:1246-1256)."""
    compliances = {name: entry["compliance_n_mm"] for name, entry in solutions.items()}
    return {"iteration": iteration, "final_evaluation": final,
            "objective": float(sum(scales[name] * value for name, value in compliances.items())),
            "physical_density_sum": float(physical_sum), "compliances_n_mm": compliances,
            "maximum_design_change": change,
            "maximum_relative_residual": float(max(entry["relative_residual"] for entry in solutions.values())),
            "elapsed_s": elapsed}


def _stage_entry(mapping, sums, volume_target, move_limit):
    entry = {"projection_beta": mapping.beta, "move_limit": move_limit}
    if mapping.robust:
        entry.update({"dilated_volume_target": volume_target, "eroded_density_sum": sums["eroded"],
                      "dilated_density_sum": sums["dilated"]})
    return entry


def _sums(torch, fields):
    return {name: float(torch.sum(value)) for name, (value, _) in fields.items()}


def optimize_topology(domain, settings, *, progress_callback=None, device="cuda"):
    """The reference's OC driver; returns the same outcome dict (status ok / invalid / failed)."""
    started = perf_counter()
    history, diagnostics = [], []
    system = mapping = outcome = None
    density = np.zeros(tuple(domain.get("grid", {}).get("shape", (0, 0, 0))))
    try:
        import torch
        settings = _settings(settings)
        validate_masks(domain)
        # the reference's HexElasticity refuses a domain without a static case (topology_optimization.py:440-441);
        # this library's HexElasticity accepts one (a covariance-only plate), so the OC driver checks it here
        if not any(case.get("analysis") == "static" for case in domain.get("load_cases", [])):
            raise ValueError("Topology optimization requires at least one static case")
        mapping = DensityMap(domain, settings, device)
        grid_shape = tuple(domain["grid"]["shape"])
        target = settings["volume_fraction"] * int(np.count_nonzero(mapping.allowed))
        if np.count_nonzero(mapping.preserve) >= target:
            raise ValueError("The volume budget must exceed the preserve-cell volume")
        design = mapping._dev(mapping.initial(target))
        system = HexElasticity(domain, interface_node_policy=settings["interface_node_policy"], linear_solver=settings["linear_solver"],
                               solver_choice=settings["solver_choice"], gpu_solver_residency=settings["gpu_solver_residency"],
                               multigrid={"device": str(mapping.device)})
        weights = torch.ones(mapping.n, dtype=torch.float64, device=mapping.device)
        scales = normalization = case_weights = None
        converged, stop_reason = False, "max_iterations"
        schedule = settings["beta_schedule"] or [mapping.beta]
        staged = mapping.robust or settings["beta_schedule"] is not None
        stiffness_name, volume_name = ("eroded", "dilated") if mapping.robust else ("intermediate", "intermediate")
        minimum_iterations = max(settings["minimum_iterations"], settings["beta_minimum_iterations"]) if staged else settings["minimum_iterations"]
        level = level_iterations = 0
        volume_target = target
        iteration = 0
        for iteration in range(1, settings["max_iterations"] + 1):
            fields, _ = mapping.fields_device(design)
            sums = _sums(torch, fields)
            physical_sum = sums["intermediate"]
            density = fields["intermediate"][0].cpu().numpy().reshape(grid_shape)
            if mapping.robust:
                dilated = sums[volume_name]
                reference = dilated if level_iterations == 0 else volume_target
                volume_target = reference + settings["volume_target_relaxation"] * (target * dilated / physical_sum - reference)
            solutions = system.solve(fields[stiffness_name][0].cpu().numpy(), settings["penalization"], settings["min_stiffness_ratio"])
            if scales is None:
                scales, normalization, case_weights = _case_scaling(solutions, settings)
            physical_gradient = sum(scales[name] * result["derivative"] for name, result in solutions.items())
            gradient = mapping.pullback_device(mapping._dev(physical_gradient), fields[stiffness_name][1])
            volume_gradient = mapping.pullback_device(weights, fields[volume_name][1])
            late = settings["move_limit_late"] is not None and mapping.beta >= settings["move_limit_late_beta"]
            move_limit = settings["move_limit_late"] if late else settings["move_limit"]
            candidate, _ = mapping.oc_update_device(design, gradient, volume_gradient, volume_target, move_limit)
            change = float(torch.max(torch.abs(candidate - design)))
            history.append(_history_entry(iteration, physical_sum, solutions, scales, change, perf_counter() - started))
            history[-1].update(modal_penalty=0.0, f1_hz=None)
            if staged:
                recent = [entry["objective"] for entry in history[-min(level_iterations + 1, settings["objective_window"]):]]
                stall = (max(recent) - min(recent)) / min(recent) if len(recent) == settings["objective_window"] else None
                history[-1].update(_stage_entry(mapping, sums, volume_target, move_limit), objective_stall=stall)
            level_iterations += 1
            final_level = level == len(schedule) - 1
            violation = float(torch.dot(weights, fields[volume_name][0])) / volume_target - 1
            history[-1]["max_violation"] = violation
            if progress_callback is not None:
                progress_callback(deepcopy(history[-1]))
            decision = continuation_decision(level_iterations, final_level, change, violation,
                                             minimum_iterations if final_level else settings["beta_minimum_iterations"],
                                             float("inf") if final_level else settings["beta_interval"],
                                             settings["change_tolerance"] if final_level else settings["beta_change_tolerance"],
                                             settings["feasibility_tolerance"])
            if decision == "converged":
                converged, stop_reason = True, "change_tolerance"
                break
            if settings["max_runtime_s"] is not None and perf_counter() - started >= settings["max_runtime_s"]:
                stop_reason = "max_runtime_s"
                break
            if iteration == settings["max_iterations"]:
                break
            design = candidate
            if decision == "advance":
                level += 1
                level_iterations = 0
                mapping.beta = schedule[level]
        fields, filtered = mapping.fields_device(design)
        sums = _sums(torch, fields)
        physical = fields["intermediate"][0].cpu().numpy()
        density = physical.reshape(grid_shape)
        solutions = system.solve(fields[stiffness_name][0].cpu().numpy(), settings["penalization"], settings["min_stiffness_ratio"], metrics=True)
        final_entry = _history_entry(iteration + 1, sums["intermediate"], solutions, scales, None, perf_counter() - started, final=True)
        if staged:
            final_entry.update(_stage_entry(mapping, sums, volume_target, None))
        history.append(final_entry)
        if progress_callback is not None:
            progress_callback(deepcopy(final_entry))
        volume = float(np.sum(physical) * np.prod(system.spacing))
        allowed = int(np.count_nonzero(mapping.allowed))
        summary = {
            "method": "3D Hex8 SIMP, spatial density filter, smooth projection, normalized multi-load compliance, OC volume constraint",
            "initialization": "uniform in every free cell; fixed preserves",
            "settings": settings,
            "converged": converged,
            "stop_reason": stop_reason,
            "iterations": iteration,
            "volume_fraction": float(np.sum(physical) / allowed),
            "target_volume_fraction": settings["volume_fraction"],
            "density_volume_mm3": volume,
            "density_frame_mass_g": volume * system.density / 1000,
            "objective_initial": history[0]["objective"],
            "objective_final": final_entry["objective"],
            "normalization_compliances_n_mm": normalization,
            "normalized_case_weights": case_weights,
            "static_surrogate_metrics": {name: {key: value for key, value in result.items() if key not in ("derivative", "fields", "modulus_derivative")}
                                         for name, result in solutions.items()},
            "gray_fraction_free": float(np.mean((physical[mapping.free] > 0.1) & (physical[mapping.free] < 0.9))),
            "modal": None,
            "element_model": "three displacement DOFs/node, fully integrated trilinear 8-node 3D elasticity, 2x2x2 Gauss integration",
            "units": {"length": "mm", "force": "N", "stress": "MPa", "density": "g/cm3"},
            "system": system.diagnostics(),
            "elapsed_s": perf_counter() - started,
        }
        if staged:
            summary["continuation"] = {"beta_schedule": schedule, "beta_final": mapping.beta, "final_level_reached": level == len(schedule) - 1,
                                       "level_iterations_final": level_iterations}
        host_design = design.cpu().numpy().reshape(grid_shape)
        outcome = {"status": "ok", "density": density.copy(), "design_density": host_design, "summary": summary, "history": history,
                   "diagnostics": diagnostics}
        if mapping.robust:
            eroded, dilated = (fields[name][0].cpu().numpy() for name in ("eroded", "dilated"))
            summary["method"] = ("3D Hex8 SIMP, spatial density filter, robust eroded/intermediate/dilated Heaviside projection with beta "
                                 "continuation, eroded-design normalized multi-load compliance, OC dilated-volume constraint")
            summary["robust"] = {"thresholds": mapping.thresholds, "objective_field": "eroded", "volume_constraint_field": "dilated",
                                 "reported_density_field": "intermediate", "dilated_volume_target_final": volume_target,
                                 "eroded_volume_fraction": float(np.sum(eroded) / allowed),
                                 "dilated_volume_fraction": float(np.sum(dilated) / allowed),
                                 "dilated_frame_mass_g": float(np.sum(dilated) * np.prod(system.spacing) * system.density / 1000)}
            outcome["eroded_density"] = eroded.reshape(grid_shape)
            outcome["dilated_density"] = dilated.reshape(grid_shape)
            outcome["filtered_density"] = filtered.cpu().numpy().reshape(grid_shape)
        if not converged:
            diagnostics.append(f"Density iteration stopped at {stop_reason}; convergence is not claimed")
        return outcome
    except ValueError as error:
        outcome = {"status": "invalid", "density": density, "summary": {}, "history": history, "diagnostics": [str(error)]}
        return outcome
    except (RuntimeError, MemoryError, np.linalg.LinAlgError) as error:
        outcome = {"status": "failed", "density": density, "summary": {}, "history": history, "diagnostics": [str(error)]}
        return outcome
    finally:
        if system is not None:
            cleanup = system.close()
            if cleanup and outcome is not None:
                outcome["diagnostics"].extend(cleanup)
                outcome["status"] = "failed"
        if mapping is not None:
            mapping.close()
