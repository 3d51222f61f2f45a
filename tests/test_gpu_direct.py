"""Dense device direct solver (CudaDirectSolver drop-in) and the HexElasticity solve paths.

Mirrors the reference's cuDSS tests (tests/test_topology_optimization.py:451-553):
direct = CPU sparse solve, symbolic reuse, invalid input, cleanup; and the
multigrid HexElasticity solve = direct solve on compliance, sensitivities and max
displacement (tests/test_topology_multigrid.py:74-86, rel 1e-7).
"""
import numpy as np
import pytest
from scipy.sparse.linalg import spsolve

pytestmark = pytest.mark.gpu


def _system(shape=(12, 6, 6), seed=0, solver="cuda_cudss", multigrid=None):
    from deep_frame_b200 import problems
    from deep_frame_b200.elasticity import HexElasticity
    domain, density = problems.cantilever(shape, seed)
    return HexElasticity(domain, linear_solver=solver, multigrid=multigrid), density


def test_direct_solver_matches_sparse_solve_and_reuses_structure(cuda):
    from deep_frame_b200.direct import CudaDirectSolver
    system, density = _system()
    moduli, _ = system.moduli(density, 3.0, 1e-9)
    full = system.matrix(1e-9 + (1 - 1e-9) * density ** 3)
    free = next(iter(system.groups.values()))[0][1]["free"]
    reduced = full[free][:, free].tocsc()
    rhs = np.random.default_rng(1).normal(size=(len(free), 3))
    solver = CudaDirectSolver(reduced, rhs)
    x = solver.solve(reduced, rhs)
    want = spsolve(reduced, rhs)
    assert np.linalg.norm(x - want) < 1e-9 * np.linalg.norm(want)
    x2 = solver.substitute(2 * rhs)
    assert np.linalg.norm(x2 - 2 * want) < 1e-9 * np.linalg.norm(want)
    scaled = reduced * 3.0
    assert solver.same_structure(scaled)
    assert np.linalg.norm(solver.solve(scaled, rhs) - want / 3) < 1e-9 * np.linalg.norm(want)
    with pytest.raises(ValueError):
        solver.solve(reduced[:-1, :-1], rhs[:-1])
    with pytest.raises(ValueError):
        solver.substitute(rhs[:, :2])
    assert solver.close() == [] and solver.close() == []
    with pytest.raises(RuntimeError):
        solver.solve(reduced, rhs)


def test_direct_solver_rejects_indefinite_matrix(cuda):
    from scipy.sparse import csr_matrix
    from deep_frame_b200.direct import CudaDirectSolver
    m = csr_matrix(np.array([[1.0, 2.0], [2.0, 1.0]]))
    solver = CudaDirectSolver(m, np.ones((2, 1)))
    with pytest.raises(RuntimeError, match="positive definite"):
        solver.solve(m, np.ones((2, 1)))
    solver.close()


@pytest.mark.parametrize("n", [1, 5, 31, 32, 33, 64, 97, 300])
def test_direct_solver_sizes_around_panel_edges(cuda, n):
    """The fused blocked factorisation and inversion (32-wide panels, 64 x 64 update tiles, a last
    partial panel padded with the identity) against NumPy, two right-hand sides."""
    from scipy.sparse import csr_matrix
    from deep_frame_b200.direct import CudaDirectSolver
    rng = np.random.default_rng(n)
    m = rng.standard_normal((n, n)) / np.sqrt(n)
    a = m @ m.T + 0.5 * np.eye(n)
    rhs = rng.standard_normal((n, 2))
    solver = CudaDirectSolver(csr_matrix(a), rhs)
    x = solver.solve(csr_matrix(a), rhs)
    want = np.linalg.solve(a, rhs)
    assert np.linalg.norm(x - want) <= 1e-10 * np.linalg.norm(want)
    assert solver.close() == []


def test_direct_solver_reports_first_bad_pivot_beyond_first_panel(cuda):
    """A diagonally dominant matrix with one negative diagonal entry at row 40 (second panel): the
    factorisation stops being positive definite there and reports pivot 41 (1-based)."""
    from scipy.sparse import csr_matrix
    from deep_frame_b200.direct import CudaDirectSolver
    n = 70
    a = np.full((n, n), 0.01) + np.eye(n) * 4.0
    a[40, 40] = -1.0
    solver = CudaDirectSolver(csr_matrix(a), np.ones((n, 1)))
    with pytest.raises(RuntimeError, match=r"pivot 41\)"):
        solver.solve(csr_matrix(a), np.ones((n, 1)))
    solver.close()


def test_multigrid_system_solve_matches_direct_system_solve(cuda):
    direct, density = _system((16, 8, 8), 3)
    mg, _ = _system((16, 8, 8), 3, "multigrid", {"tolerance": 1e-12, "coarsest_dofs": 200, "precision": "float64"})
    a = direct.solve(density, 3.0, 1e-9, metrics=True)["tip"]
    b = mg.solve(density, 3.0, 1e-9, metrics=True)["tip"]
    assert b["compliance_n_mm"] == pytest.approx(a["compliance_n_mm"], rel=1e-7)
    assert np.linalg.norm(b["derivative"] - a["derivative"]) <= 1e-7 * np.linalg.norm(a["derivative"])
    assert b["max_displacement_mm"] == pytest.approx(a["max_displacement_mm"], rel=1e-7)
    assert direct.close() == [] and mg.close() == []


def test_system_solve_matches_reference_superlu_golden(cuda):
    """The 48 x 24 x 24 cantilever: compliance 1e-6 and sensitivities 1e-5 vs the reference's SuperLU."""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "cantilever_48x24x24.npz")
    system, _ = _system((48, 24, 24), 0, "multigrid", {"precision": "float64", "smoother": "jacobi", "sweeps": 2,
                                                      "coarsest_dofs": 400, "tolerance": 1e-10})
    result = system.solve(g["density"], 3.0, 1e-9, metrics=True)["tip"]
    assert system.multigrid.statistics[-1]["levels"] == 4
    assert result["compliance_n_mm"] == pytest.approx(float(g["compliance"]), rel=1e-6)
    assert np.linalg.norm(result["derivative"] - g["derivative"]) < 1e-5 * np.linalg.norm(g["derivative"])
    assert result["max_displacement_mm"] == pytest.approx(float(g["max_displacement"]), rel=1e-6)
    system.close()


def test_direct_system_solve_of_config_one_matches_reference_superlu(cuda):
    """linear_solver="cuda_cudss" on the 48 x 24 x 24 cantilever (91 875 dofs: the banded
    factorisation, bandwidth about 3 x 25 x 25): compliance within 1e-6 and sensitivities within
    1e-5 of the reference's SuperLU golden."""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "cantilever_48x24x24.npz")
    system, _ = _system((48, 24, 24), 0, "cuda_cudss")
    result = system.solve(g["density"], 3.0, 1e-9, metrics=True)["tip"]
    assert result["compliance_n_mm"] == pytest.approx(float(g["compliance"]), rel=1e-6)
    assert np.linalg.norm(result["derivative"] - g["derivative"]) < 1e-5 * np.linalg.norm(g["derivative"])
    assert result["max_displacement_mm"] == pytest.approx(float(g["max_displacement"]), rel=1e-6)
    assert system.diagnostics()["gpu_solver_details"][0]["shape"][0] > 32768
    assert system.close() == []


@pytest.mark.parametrize("n,bw", [(200, 3), (600, 64), (1000, 65), (4000, 130)])
def test_banded_factorisation_sizes_around_block_edges(cuda, n, bw):
    """Band matrices whose bandwidth is below, at and beyond the 64-wide block columns, with a last
    partial block: the banded path against NumPy, three right-hand sides."""
    from scipy.sparse import diags
    from deep_frame_b200.direct import CudaDirectSolver
    rng = np.random.default_rng(n + bw)
    bands = [rng.standard_normal(n - k) for k in range(bw + 1)]
    lower = diags(bands, [-k for k in range(bw + 1)], shape=(n, n)).toarray()
    a = lower @ lower.T + 0.1 * np.eye(n)
    a[np.abs(np.subtract.outer(np.arange(n), np.arange(n))) > bw] = 0.0
    a += np.diag(np.abs(a).sum(axis=1))          # diagonally dominant: SPD with the band kept
    from scipy.sparse import csr_matrix
    rhs = rng.standard_normal((n, 3))
    solver = CudaDirectSolver(csr_matrix(a), rhs)
    x = solver.solve(csr_matrix(a), rhs)
    want = np.linalg.solve(a, rhs)
    assert np.linalg.norm(x - want) <= 1e-10 * np.linalg.norm(want)
    assert solver.close() == []


def test_banded_factorisation_reports_the_failing_pivot(cuda):
    """A diagonally dominant tridiagonal matrix with one negative diagonal entry at row 150 (third
    block column of the banded path): "not positive definite (pivot 151)"."""
    from scipy.sparse import diags
    from deep_frame_b200.direct import CudaDirectSolver
    n = 300
    main = np.full(n, 4.0)
    main[150] = -1.0
    a = diags([np.full(n - 1, 0.5), main, np.full(n - 1, 0.5)], [-1, 0, 1], shape=(n, n)).tocsr()
    solver = CudaDirectSolver(a, np.ones((n, 1)))
    with pytest.raises(RuntimeError, match=r"pivot 151\)"):
        solver.solve(a, np.ones((n, 1)))
    solver.close()
