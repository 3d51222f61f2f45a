"""Inertia-relief (free-flying) load cases: host set-up against the reference's own cases.

tests/golden/inertia_relief.npz holds the reference's HexElasticity on the tiny half-model domain of
its tests/test_topology_problem.py:156-172 and on the full / half relief domain of
tests/test_topology_optimization.py:585-612 (SuperLU solves): the determinate support dofs, every
part's fixed dofs, force (applied + d'Alembert loads) and support, the relief mass summary, and the
compliances / sensitivities.  The product's set-up must reproduce the dofs and forces exactly; the
oracle's direct solve of those parts must reproduce the compliances (the reference's floating solve
and the solve with the support held are the same problem).
"""
import json
from pathlib import Path

import numpy as np
import pytest
from scipy.sparse.linalg import spsolve

from oracle import operator as op

GOLDEN = np.load(Path(__file__).parent / "golden" / "inertia_relief.npz")
NAMES = ("tiny", "relief_full", "relief_half")


def domain_of(name):
    domain = json.loads(str(GOLDEN[f"{name}_domain"]))
    for key in ("allowed", "preserve", "forbidden"):
        domain[key] = np.asarray(domain[key], dtype=bool)
    return domain


def parts_of(name, case):
    k, parts = 0, []
    while f"{name}_{case}_part{k}_fixed" in GOLDEN:
        parts.append({key: GOLDEN[f"{name}_{case}_part{k}_{key}"] for key in ("fixed", "force", "support")})
        k += 1
    return parts


@pytest.mark.parametrize("name", NAMES)
def test_support_parts_and_relief_loads_match_reference(name):
    from deep_frame_b200.elasticity import HexElasticity
    system = HexElasticity(domain_of(name), linear_solver="cuda_cudss")
    assert np.array_equal(np.sort(system.support[1]), np.sort(GOLDEN[f"{name}_support"]))
    for case_name in GOLDEN[f"{name}_cases"]:
        case = next(c for c in system.cases if c["name"] == case_name)
        expected = parts_of(name, case_name)
        assert len(case["parts"]) == len(expected)
        for part, ref in zip(case["parts"], expected):
            assert np.array_equal(part["fixed"], ref["fixed"]) and np.array_equal(part["support"], ref["support"])
            assert np.allclose(part["force"], ref["force"], rtol=0, atol=1e-12 * np.abs(ref["force"]).max())
        if f"{name}_{case_name}_mass_g" in GOLDEN:
            relief = case["inertia_relief"]
            assert relief["mass_g"] == pytest.approx(float(GOLDEN[f"{name}_{case_name}_mass_g"]), rel=1e-12)
            assert np.allclose(relief["center_of_mass_mm"], GOLDEN[f"{name}_{case_name}_center"], rtol=1e-12, atol=1e-12)
            assert np.allclose(relief["acceleration_n_per_g"], GOLDEN[f"{name}_{case_name}_acceleration"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", NAMES)
def test_relief_cases_are_balanced_and_oracle_compliance_matches(name):
    from deep_frame_b200.elasticity import HexElasticity
    system = HexElasticity(domain_of(name), linear_solver="cuda_cudss")
    density = GOLDEN[f"{name}_density"]
    moduli = np.where(system.active_elements, system.young * (1e-6 + (1 - 1e-6) * density ** 3), 0.0)
    matrix = op.assemble(system.shape, system.ke, moduli).tocsc()
    factor = 1.0 if system.symmetry is None else 2.0
    for case_name in GOLDEN[f"{name}_cases"]:
        case = next(c for c in system.cases if c["name"] == case_name)
        compliance = 0.0
        for part in case["parts"]:
            free = part["free"]
            u = np.zeros(system.ndof)
            u[free] = spsolve(matrix[free][:, free], part["force"][free])
            compliance += factor * float(part["force"] @ u)
            if "inertia_relief" in case:
                reaction = matrix @ u - part["force"]
                assert np.max(np.abs(reaction[part["support"]])) < 1e-9 * np.abs(part["force"]).sum()
        assert compliance == pytest.approx(float(GOLDEN[f"{name}_{case_name}_compliance"]), rel=1e-9)


@pytest.mark.parametrize("name", ["relief_full", "relief_half"])
def test_balanced_relief_cases_leave_the_support_unloaded(name):
    """support_reactions (the reference's check, topology_optimization.py:570-580) on the relief
    domains, with a SciPy stand-in for the device direct solver: the d'Alembert loads balance every
    part, so its determinate support carries (numerically) nothing."""
    from scipy.sparse.linalg import splu
    from deep_frame_b200.elasticity import HexElasticity

    class HostSolver:
        def __init__(self, matrix, rhs):
            self.lu = splu(matrix.tocsc())

        def solve(self, matrix, rhs):
            return self.lu.solve(rhs)

        def close(self):
            return []

    system = HexElasticity(domain_of(name))
    density = GOLDEN[f"{name}_density"]
    for case in system.cases:
        if "inertia_relief" not in case:
            continue
        for row in system.support_reactions(density, case["name"], solver=HostSolver):
            assert row["support_dofs"] >= 3
            assert row["max_reaction_n"] < 1e-9 * row["nodal_force_sum_n"]
