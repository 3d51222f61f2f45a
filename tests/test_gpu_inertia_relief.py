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
