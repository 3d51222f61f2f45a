"""SIMP + OC driver on the CPU (oracle, test only).

Restates ``optimize_topology`` of deep_frame/topology_optimization.py
(:1265-1406) for static Dirichlet-supported cases without symmetry, modal
constraints, corridors or prop discs: density fields from the oracle cone
filter (single or robust projection with beta continuation), SIMP moduli
(:657-661), direct sparse solves of the reduced stiffness, compliance f.u and
sensitivities -dE/drho u_e^T K0 u_e (:721-734), case normalisation by the
first compliances (:1235-1245), pullback, the relaxed dilated-volume target,
``oc_update`` and ``continuation_decision`` (:17-25).  Cases are given as
(name, fixed dofs, force vector), so the oracle does not depend on the
product's node selection.
"""
import numpy as np
from scipy.sparse.linalg import spsolve

from . import density as oden
from . import operator as op


def continuation_decision(iterations, final_level, change, violation, minimum, maximum, change_tolerance, violation_tolerance):
    """Stopping rule of one continuation level (topology_optimization.py:17-25)."""
    tolerance = 1e-3 if violation_tolerance is None else violation_tolerance
    quiet = change is not None and bool(np.isfinite(change)) and change < change_tolerance
    feasible = bool(np.isfinite(violation)) and violation <= tolerance
    if quiet and feasible and iterations >= minimum:
        return ("advance", "converged")[bool(final_level)]
    if iterations < maximum:
        return None
    return "iteration_cap" if (final_level or iterations < minimum) else "advance"


def solve_cases(shape, ke, young, active, cases, density, p, eps):
    """{name: (compliance, derivative)} of every case for the stiffness density field."""
    density = np.asarray(density, dtype=float)
    moduli = np.where(active, young * (eps + (1 - eps) * density ** p), 0.0)
    slope = np.where(active, young * (1 - eps) * p * density ** (p - 1), 0.0)
    matrix = op.assemble(shape, ke, moduli).tocsc()
    out = {}
    for name, fixed, force in cases:
        live = op.live_dofs(shape, moduli, fixed)
        u = np.zeros(len(force))
        u[live] = spsolve(matrix[live][:, live].tocsc(), force[live])
        energy = op.element_energy(shape, ke, u)
        out[name] = (float(force @ u), -slope * energy)
    return out


def optimize(shape, spacing, ke, young, allowed, preserve, cases, settings):
    """Density history of the reference's OC driver: dict(density, design, fields, history)."""
    n = int(np.prod(shape))
    robust = settings["projection"] == "robust"
    schedule = settings["beta_schedule"] or [settings["projection_beta"]]
    mapping = oden.DensityMapOracle(shape, spacing, settings["filter_radius_mm"], allowed, preserve, beta=schedule[0],
                                    eta=settings["projection_eta"], robust=robust, delta=settings["robust_delta"],
                                    minimum_design_density=settings["minimum_design_density"])
    active = np.asarray(allowed, dtype=bool).ravel()
    target = settings["volume_fraction"] * int(np.count_nonzero(active))
    design = mapping.initial(target)
    staged = robust or settings["beta_schedule"] is not None
    stiffness_name, volume_name = ("eroded", "dilated") if robust else ("intermediate", "intermediate")
    minimum_iterations = max(settings["minimum_iterations"], settings["beta_minimum_iterations"]) if staged else settings["minimum_iterations"]
    level = level_iterations = 0
    volume_target = target
    scales = None
    history = []
    ones = np.ones(n)
    iteration = 0
    for iteration in range(1, settings["max_iterations"] + 1):
        fields, _ = mapping.fields(design)
        physical = fields["intermediate"][0]
        if robust:
            dilated = float(np.sum(fields[volume_name][0]))
            reference = dilated if level_iterations == 0 else volume_target
            volume_target = reference + settings["volume_target_relaxation"] * (target * dilated / float(np.sum(physical)) - reference)
        solved = solve_cases(shape, ke, young, active, cases, fields[stiffness_name][0], settings["penalization"], settings["min_stiffness_ratio"])
        if scales is None:
            scales = {name: 1.0 / len(solved) / value[0] for name, value in solved.items()}
        gradient = mapping.pullback(sum(scales[name] * value[1] for name, value in solved.items()), fields[stiffness_name][1])
        volume_gradient = mapping.pullback(ones, fields[volume_name][1])
        late = settings["move_limit_late"] is not None and mapping.beta >= settings["move_limit_late_beta"]
        move_limit = settings["move_limit_late"] if late else settings["move_limit"]
        candidate = oden.oc_update(design, gradient, volume_gradient, mapping, volume_target, move_limit)
        change = float(np.max(np.abs(candidate - design)))
        history.append({"objective": float(sum(scales[name] * value[0] for name, value in solved.items())), "beta": mapping.beta,
                        "compliances": {name: value[0] for name, value in solved.items()}, "change": change, "move_limit": move_limit,
                        "volume_target": volume_target})
        level_iterations += 1
        final_level = level == len(schedule) - 1
        violation = float(np.sum(fields[volume_name][0]) / volume_target - 1)
        decision = continuation_decision(level_iterations, final_level, change, violation,
                                         minimum_iterations if final_level else settings["beta_minimum_iterations"],
                                         float("inf") if final_level else settings["beta_interval"],
                                         settings["change_tolerance"] if final_level else settings["beta_change_tolerance"],
                                         settings["feasibility_tolerance"])
        if decision == "converged" or iteration == settings["max_iterations"]:
            break
        design = candidate
        if decision == "advance":
            level += 1
            level_iterations = 0
            mapping.beta = schedule[level]
    fields, filtered = mapping.fields(design)
    solved = solve_cases(shape, ke, young, active, cases, fields[stiffness_name][0], settings["penalization"], settings["min_stiffness_ratio"])
    history.append({"objective": float(sum(scales[name] * value[0] for name, value in solved.items())), "beta": mapping.beta,
                    "compliances": {name: value[0] for name, value in solved.items()}, "change": None})
    return {"density": fields["intermediate"][0], "design": design, "fields": {name: value[0] for name, value in fields.items()},
            "filtered": filtered, "history": history}
