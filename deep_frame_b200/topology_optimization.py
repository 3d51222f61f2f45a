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


class _Levels:
    """The projection continuation of an OC run.

    Holds the beta schedule and the current level, the iterations spent at that level, and, for
    robust runs, the dilated-volume target that relaxes toward the budget scaled by the
    dilated / intermediate volume ratio (topology_optimization.py:1296-1300).  ``rule`` gives the
    arguments of ``continuation_decision`` that end the current level: the final level runs to
    the change tolerance with the run's minimum iterations; earlier levels advance after
    beta_minimum_iterations with the beta change tolerance, or at beta_interval."""

    def __init__(self, settings, mapping, budget):
        self.settings, self.mapping, self.budget = settings, mapping, budget
        self.schedule = settings["beta_schedule"] or [mapping.beta]
        self.staged = mapping.robust or settings["beta_schedule"] is not None
        self.level, self.count, self.volume_target = 0, 0, budget
        self.minimum = (max(settings["minimum_iterations"], settings["beta_minimum_iterations"]) if self.staged
                        else settings["minimum_iterations"])

    @property
    def final(self):
        return self.level == len(self.schedule) - 1

    def relax(self, dilated, intermediate):
        anchor = dilated if self.count == 0 else self.volume_target
        self.volume_target = anchor + self.settings["volume_target_relaxation"] * (self.budget * dilated / intermediate - anchor)

    def move_limit(self):
        late = self.settings["move_limit_late"]
        return late if late is not None and self.mapping.beta >= self.settings["move_limit_late_beta"] else self.settings["move_limit"]

    def rule(self):
        if self.final:
            return self.minimum, float("inf"), self.settings["change_tolerance"]
        return self.settings["beta_minimum_iterations"], self.settings["beta_interval"], self.settings["beta_change_tolerance"]

    def stall(self, objectives):
        """Relative spread of the objective over the last objective_window iterations of this level,
        or None before the window is full."""
        window = objectives[-min(self.count + 1, self.settings["objective_window"]):]
        if len(window) < self.settings["objective_window"]:
            return None
        return (max(window) - min(window)) / min(window)

    def record(self, sums, move_limit):
        entry = {"projection_beta": self.mapping.beta, "move_limit": move_limit}
        if self.mapping.robust:
            entry.update(dilated_volume_target=self.volume_target, eroded_density_sum=sums["eroded"], dilated_density_sum=sums["dilated"])
        return entry

    def advance(self):
        self.level += 1
        self.count = 0
        self.mapping.beta = self.schedule[self.level]


class _OcRun:
    """State of one device-resident OC run: the density map and elasticity system, the design on the
    device, the case scaling fixed by the first evaluation, and the history."""

    def __init__(self, settings, started, shape):
        import torch
        self.torch, self.settings, self.started = torch, settings, started
        self.mapping = self.system = None
        self.history, self.shape, self.density = [], shape, np.zeros(shape)

    def start(self, domain, device):
        """Masks, density map, volume budget, initial design and the elasticity system."""
        settings = self.settings
        validate_masks(domain)
        # the reference's HexElasticity refuses a domain without a static case (topology_optimization.py:440-441);
        # this library's HexElasticity accepts one (a covariance-only plate), so the OC driver checks it here
        if not any(case.get("analysis") == "static" for case in domain.get("load_cases", [])):
            raise ValueError("Topology optimization requires at least one static case")
        self.mapping = DensityMap(domain, settings, device)
        self.allowed_cells = int(np.count_nonzero(self.mapping.allowed))
        budget = settings["volume_fraction"] * self.allowed_cells
        if np.count_nonzero(self.mapping.preserve) >= budget:
            raise ValueError("The volume budget must exceed the preserve-cell volume")
        self.levels = _Levels(settings, self.mapping, budget)
        self.stiffness_field, self.volume_field = ("eroded", "dilated") if self.mapping.robust else ("intermediate", "intermediate")
        self.design = self.mapping._dev(self.mapping.initial(budget))
        self.system = HexElasticity(domain, interface_node_policy=settings["interface_node_policy"], linear_solver=settings["linear_solver"],
                                    solver_choice=settings["solver_choice"], gpu_solver_residency=settings["gpu_solver_residency"],
                                    multigrid={"device": str(self.mapping.device)})
        self.unit = self.torch.ones(self.mapping.n, dtype=self.torch.float64, device=self.mapping.device)
        self.scales = self.normalization = self.shares = None

    def evaluate(self, design):
        """Density fields of ``design`` (with the filtered field) and their sums; keeps the physical
        density on the host for the outcome."""
        fields, filtered = self.mapping.fields_device(design)
        sums = {name: float(self.torch.sum(value)) for name, (value, _) in fields.items()}
        self.density = fields["intermediate"][0].cpu().numpy().reshape(self.shape)
        return fields, filtered, sums

    def solve(self, fields, metrics=False):
        return self.system.solve(fields[self.stiffness_field][0].cpu().numpy(), self.settings["penalization"],
                                 self.settings["min_stiffness_ratio"], metrics=metrics)

    def entry(self, iteration, sums, solutions, change, final=False):
        self.history.append(_history_entry(iteration, sums["intermediate"], solutions, self.scales, change,
                                           perf_counter() - self.started, final=final))
        return self.history[-1]

    def step(self, iteration):
        """One OC iteration: evaluate, scale, pull the gradients back through the filter, run the
        device multiplier search.  Returns (candidate design, history entry, design change, volume
        violation)."""
        levels, mapping = self.levels, self.mapping
        fields, _, sums = self.evaluate(self.design)
        if mapping.robust:
            levels.relax(sums[self.volume_field], sums["intermediate"])
        solutions = self.solve(fields)
        if self.scales is None:
            self.scales, self.normalization, self.shares = _case_scaling(solutions, self.settings)
        objective_gradient = mapping._dev(sum(self.scales[name] * result["derivative"] for name, result in solutions.items()))
        move_limit = levels.move_limit()
        candidate, _ = mapping.oc_update_device(self.design, mapping.pullback_device(objective_gradient, fields[self.stiffness_field][1]),
                                                mapping.pullback_device(self.unit, fields[self.volume_field][1]),
                                                levels.volume_target, move_limit)
        change = float(self.torch.max(self.torch.abs(candidate - self.design)))
        entry = self.entry(iteration, sums, solutions, change)
        entry.update(modal_penalty=0.0, f1_hz=None)
        if levels.staged:
            entry.update(levels.record(sums, move_limit), objective_stall=levels.stall([item["objective"] for item in self.history]))
        levels.count += 1
        violation = float(self.torch.dot(self.unit, fields[self.volume_field][0])) / levels.volume_target - 1
        entry["max_violation"] = violation
        return candidate, entry, change, violation

    def iterate(self, callback):
        """Iterations until a level rule converges, the runtime or iteration cap is hit.  Returns
        (iterations run, converged, stop reason)."""
        settings, levels = self.settings, self.levels
        iteration = 0
        for iteration in range(1, settings["max_iterations"] + 1):
            candidate, entry, change, violation = self.step(iteration)
            if callback is not None:
                callback(deepcopy(entry))
            minimum, maximum, tolerance = levels.rule()
            decision = continuation_decision(levels.count, levels.final, change, violation, minimum, maximum, tolerance,
                                             settings["feasibility_tolerance"])
            if decision == "converged":
                return iteration, True, "change_tolerance"
            if settings["max_runtime_s"] is not None and perf_counter() - self.started >= settings["max_runtime_s"]:
                return iteration, False, "max_runtime_s"
            if iteration == settings["max_iterations"]:
                break
            self.design = candidate
            if decision == "advance":
                levels.advance()
        return iteration, False, "max_iterations"

    def finish(self, iterations, converged, stop_reason, callback):
        """The final evaluation (with metrics) and the reference's outcome record."""
        fields, filtered, sums = self.evaluate(self.design)
        solutions = self.solve(fields, metrics=True)
        final = self.entry(iterations + 1, sums, solutions, None, final=True)
        if self.levels.staged:
            final.update(self.levels.record(sums, None))
        if callback is not None:
            callback(deepcopy(final))
        physical = fields["intermediate"][0].cpu().numpy()
        outcome = {"status": "ok", "density": self.density.copy(), "design_density": self.design.cpu().numpy().reshape(self.shape),
                   "summary": self.summary(physical, solutions, final, iterations, converged, stop_reason), "history": self.history,
                   "diagnostics": []}
        if self.mapping.robust:
            self._robust(outcome, fields, filtered)
        if not converged:
            outcome["diagnostics"].append(f"Density iteration stopped at {stop_reason}; convergence is not claimed")
        return outcome

    def summary(self, physical, solutions, final, iterations, converged, stop_reason):
        settings, system, levels = self.settings, self.system, self.levels
        cell_volume = float(np.prod(system.spacing))
        volume = float(np.sum(physical)) * cell_volume
        free = physical[self.mapping.free]
        out = {
            "method": "3D Hex8 SIMP, spatial density filter, smooth projection, normalized multi-load compliance, OC volume constraint",
            "initialization": "uniform in every free cell; fixed preserves",
            "settings": settings, "converged": converged, "stop_reason": stop_reason, "iterations": iterations,
            "volume_fraction": float(np.sum(physical) / self.allowed_cells), "target_volume_fraction": settings["volume_fraction"],
            "density_volume_mm3": volume, "density_frame_mass_g": volume * system.density / 1000,
            "objective_initial": self.history[0]["objective"], "objective_final": final["objective"],
            "normalization_compliances_n_mm": self.normalization, "normalized_case_weights": self.shares,
            "static_surrogate_metrics": {name: {key: value for key, value in result.items() if key not in ("derivative", "fields", "modulus_derivative")}
                                         for name, result in solutions.items()},
            "gray_fraction_free": float(np.mean((free > 0.1) & (free < 0.9))),
            "modal": None,
            "element_model": "three displacement DOFs/node, fully integrated trilinear 8-node 3D elasticity, 2x2x2 Gauss integration",
            "units": {"length": "mm", "force": "N", "stress": "MPa", "density": "g/cm3"},
            "system": system.diagnostics(), "elapsed_s": perf_counter() - self.started,
        }
        if levels.staged:
            out["continuation"] = {"beta_schedule": levels.schedule, "beta_final": self.mapping.beta, "final_level_reached": levels.final,
                                   "level_iterations_final": levels.count}
        return out

    def _robust(self, outcome, fields, filtered):
        """Robust runs also report the eroded / dilated / filtered fields and their volumes."""
        eroded, dilated = (fields[name][0].cpu().numpy() for name in ("eroded", "dilated"))
        mass_scale = float(np.prod(self.system.spacing)) * self.system.density / 1000
        summary = outcome["summary"]
        summary["method"] = ("3D Hex8 SIMP, spatial density filter, robust eroded/intermediate/dilated Heaviside projection with beta "
                             "continuation, eroded-design normalized multi-load compliance, OC dilated-volume constraint")
        summary["robust"] = {"thresholds": self.mapping.thresholds, "objective_field": "eroded", "volume_constraint_field": "dilated",
                             "reported_density_field": "intermediate", "dilated_volume_target_final": self.levels.volume_target,
                             "eroded_volume_fraction": float(np.sum(eroded) / self.allowed_cells),
                             "dilated_volume_fraction": float(np.sum(dilated) / self.allowed_cells),
                             "dilated_frame_mass_g": float(np.sum(dilated)) * mass_scale}
        outcome["eroded_density"] = eroded.reshape(self.shape)
        outcome["dilated_density"] = dilated.reshape(self.shape)
        outcome["filtered_density"] = filtered.cpu().numpy().reshape(self.shape)

    def close(self):
        """Release the system, then the density map; the system's cleanup errors are returned."""
        errors = self.system.close() if self.system is not None else []
        if self.mapping is not None:
            self.mapping.close()
        return errors


def optimize_topology(domain, settings, *, progress_callback=None, device="cuda"):
    """The reference's OC driver (topology_optimization.py:1265-1406); returns the same outcome dict:
    status "ok", "invalid" (a ValueError: bad settings, masks or domain) or "failed" (a runtime,
    memory or linear-algebra error), with cleanup errors appended to the diagnostics and turning
    the status to "failed"."""
    started = perf_counter()
    run, outcome = None, None
    shape = tuple(domain.get("grid", {}).get("shape", (0, 0, 0)))
    try:
        run = _OcRun(_settings(settings), started, shape)
        run.start(domain, device)
        iterations, converged, stop_reason = run.iterate(progress_callback)
        outcome = run.finish(iterations, converged, stop_reason, progress_callback)
    except (ValueError, RuntimeError, MemoryError, np.linalg.LinAlgError) as error:
        status = "invalid" if isinstance(error, ValueError) else "failed"
        density, history = (run.density, run.history) if run is not None else (np.zeros(shape), [])
        outcome = {"status": status, "density": density, "summary": {}, "history": history, "diagnostics": [str(error)]}
    finally:
        if run is not None:
            cleanup = run.close()
            if cleanup and outcome is not None:
                outcome["diagnostics"].extend(cleanup)
                outcome["status"] = "failed"
    return outcome
