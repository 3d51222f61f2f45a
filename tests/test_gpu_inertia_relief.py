"""Device solves of the inertia-relief domains vs the reference's SuperLU results (tests/golden/inertia_relief.npz).

Mirrors tests/test_topology_multigrid.py:74-99 of the reference (multigrid = direct to 1e-7 on
compliance, sensitivities and max displacement) for the free-flying cases, through both device
solvers: GMG-PCG and the dense Cholesky.
"""
import numpy as np
import pytest

from test_inertia_relief import GOLDEN, NAMES, domain_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver", ["multigrid", "cuda_cudss"])
@pytest.mark.parametrize("name", NAMES)
def test_relief_solves_match_reference(cuda, name, solver):
    from deep_frame_b200.elasticity import HexElasticity
    settings = {"coarsest_dofs": 200, "tolerance": 1e-10}
    system = HexElasticity(domain_of(name), linear_solver=solver, multigrid=settings)
    result = system.solve(GOLDEN[f"{name}_density"], metrics=True)
    for case_name in GOLDEN[f"{name}_cases"]:
        entry = result[str(case_name)]
        assert entry["compliance_n_mm"] == pytest.approx(float(GOLDEN[f"{name}_{case_name}_compliance"]), rel=1e-7)
        ref = GOLDEN[f"{name}_{case_name}_derivative"]
        assert np.linalg.norm(entry["derivative"] - ref) <= 1e-7 * np.linalg.norm(ref)
        assert entry["max_displacement_mm"] == pytest.approx(float(GOLDEN[f"{name}_{case_name}_max_displacement"]), rel=1e-7)
    assert not system.close()


@pytest.mark.parametrize("name", NAMES)
def test_support_reactions_vanish_with_the_default_device_solver(cuda, name):
    """HexElasticity.support_reactions with its default solver (the device direct solver, banded
    for these grids): the d'Alembert loads balance every free-flying case, so the largest support
    reaction is negligible against the applied nodal forces (the reference's check,
    topology_optimization.py:570-580)."""
    from deep_frame_b200.elasticity import HexElasticity
    system = HexElasticity(domain_of(name))
    for case_name in GOLDEN[f"{name}_cases"]:
        case = next(c for c in system.cases if c["name"] == str(case_name))
        if "inertia_relief" not in case:
            continue
        for part in system.support_reactions(GOLDEN[f"{name}_density"], str(case_name)):
            assert part["max_reaction_n"] <= 1e-8 * part["nodal_force_sum_n"], part
    assert not system.close()
