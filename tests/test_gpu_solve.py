"""GMG-PCG solves vs a direct sparse solve of the oracle's assembled matrix.

Mirrors tests/test_topology_multigrid.py:55-72 (PCG = spsolve to 1e-6) and
:178-188 (zero RHS columns skip PCG) of the reference, over the settings the
reference exposes (precision, smoother, cycle).
"""
import numpy as np
import pytest
from scipy.sparse.linalg import spsolve

from oracle import hex8, operator as op

pytestmark = pytest.mark.gpu


def cantilever(shape, seed=0):
    """x = 0 face clamped, unit -z load at the bottom-edge centre of the free end; rho ~ U[0.01, 1]."""
    k0, _, _ = hex8.element_matrices((1, 1, 1), 0.3)
    rho = np.random.default_rng(seed).uniform(0.01, 1.0, int(np.prod(shape)))
    moduli = 1e-9 + (1 - 1e-9) * rho ** 3
    points = hex8.node_points(shape, (1, 1, 1))
    fixed_nodes = np.flatnonzero(points[:, 0] == 0)
    fixed = (3 * fixed_nodes[:, None] + np.arange(3)).ravel()
    ndof = 3 * len(points)
    force = np.zeros(ndof)
    tip = np.flatnonzero((points[:, 0] == shape[0]) & (points[:, 1] == shape[1] // 2) & (points[:, 2] == 0))[0]
    force[3 * tip + 2] = -1.0
    return k0, rho, moduli, fixed, force


def direct(shape, k0, moduli, fixed, forces):
    matrix = op.assemble(shape, k0, moduli).tocsc()
    live = op.live_dofs(shape, moduli, fixed)
    out = np.zeros_like(forces)
    reduced = matrix[live][:, live].tocsc()
    sol = spsolve(reduced, forces[live])
    out[live] = sol.reshape(out[live].shape)
    return out


@pytest.mark.parametrize("settings", [
    {"precision": "float64", "smoother": "jacobi", "sweeps": 2, "tolerance": 1e-10},
    {"precision": "float32", "smoother": "chebyshev", "tolerance": 1e-10},
    {"precision": "float32", "smoother": "jacobi", "cycle": "W", "tolerance": 1e-10},
    {"precision": "float64", "smoother": "chebyshev", "cycle": "W", "tolerance": 1e-10},
])
def test_pcg_matches_direct_solution(cuda, settings):
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (16, 8, 8)
    k0, _, moduli, fixed, force = cantilever(shape)
    rng = np.random.default_rng(7)
    forces = np.column_stack([force, rng.normal(size=force.size), rng.normal(size=force.size)])
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 200, **settings})
    mg.update(moduli)
    solution, report = mg.solve("clamped", fixed, forces)
    assert report["converged"], report
    assert report["levels"] >= 3 and report["batches"] == 1
    expected = direct(shape, k0, moduli, fixed, forces)
    for c in range(forces.shape[1]):
        assert np.linalg.norm(solution[:, c] - expected[:, c]) < 1e-6 * np.linalg.norm(expected[:, c])
    # compliance to 1e-6 relative
    assert force @ solution[:, 0] == pytest.approx(force @ expected[:, 0], rel=1e-8)
    assert all(r < settings["tolerance"] for r in report["relative_residual"])
    mg.close()


def test_zero_load_columns_skip_pcg(cuda):
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (8, 4, 4)
    k0, _, moduli, fixed, force = cantilever(shape, 1)
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 200, "precision": "float64", "tolerance": 1e-12})
    mg.update(moduli)
    forces = np.column_stack([force, 1e-20 * force])
    flat, report = mg.solve("zero", fixed, forces)
    single, _ = mg.solve("zero", fixed, forces[:, :1])
    assert report["converged"] and report["zero_rhs_columns"] == 1 and report["iterations"][1] == 0
    assert not np.any(flat[:, 1]) and np.linalg.norm(flat[:, 0] - single[:, 0]) <= 1e-12 * np.linalg.norm(single[:, 0])
    mg.close()


def test_batched_columns_match_single_columns(cuda):
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (12, 6, 6)
    k0, _, moduli, fixed, force = cantilever(shape, 2)
    rng = np.random.default_rng(3)
    forces = rng.normal(size=(force.size, 5))
    forces[fixed] = 0
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 200, "tolerance": 1e-10, "batch": 2})
    mg.update(moduli)
    flat, report = mg.solve("c", fixed, forces)
    assert report["batches"] == 3 and report["converged"]
    expected = direct(shape, k0, moduli, fixed, forces)
    assert np.linalg.norm(flat - expected) < 1e-7 * np.linalg.norm(expected)
    mg.close()


def test_warm_start_matches_cold_solution_with_fewer_iterations(cuda):
    """tf_solve_guess: starting from the solution of a nearby design converges to the same answer faster."""
    import torch
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (16, 8, 8)
    k0, rho, moduli, fixed, force = cantilever(shape, 4)
    rng = np.random.default_rng(11)
    forces = np.column_stack([force, rng.normal(size=force.size), np.zeros(force.size)])
    forces[fixed] = 0
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 200, "precision": "float64", "tolerance": 1e-10})
    nearby = 1e-9 + (1 - 1e-9) * np.clip(rho * (1 + 0.02 * rng.normal(size=rho.size)), 0.01, 1.0) ** 3
    mg.update(nearby)
    f = torch.as_tensor(np.ascontiguousarray(forces.T), device="cuda")
    guess, _ = mg.solve_device("w", fixed, f)
    guess = guess.clone()
    mg.update(moduli)
    cold, cold_report = mg.solve_device("w", fixed, f)
    cold = cold.clone()
    warm, warm_report = mg.solve_device("w", fixed, f, initial=guess)
    assert warm_report["converged"] and cold_report["converged"]
    assert warm_report["zero_rhs_columns"] == 1 and not torch.any(warm[2])
    assert max(warm_report["iterations"][:2]) < max(cold_report["iterations"][:2])
    expected = direct(shape, k0, moduli, fixed, forces)
    for c in range(2):
        got = warm[c].cpu().numpy()
        assert np.linalg.norm(got - expected[:, c]) < 1e-7 * np.linalg.norm(expected[:, c])
    # a guess that is already the solution still takes one step and stays put
    again, again_report = mg.solve_device("w", fixed, f, initial=warm.clone())
    assert max(again_report["iterations"]) <= 2
    assert torch.linalg.vector_norm(again - warm) <= 1e-9 * torch.linalg.vector_norm(warm)
    with pytest.raises(ValueError):
        mg.solve_device("w", fixed, f, initial=guess[:2])
    mg.close()


@pytest.mark.parametrize("shape", [(24, 12, 10), (16, 8, 16), (12, 20, 7)])
def test_tensor_core_vcycle_matches_cuda_core_vcycle(cuda, shape):
    """settings.tensor_cores: the FP32 finest-level apply on tcgen05 (TF32 operands) solves to the same answer.

    The tensor-core apply is ~1e-3 accurate (TF32 operand rounding), so it changes the preconditioner a
    little, never the converged solution: both V-cycles must give the direct solution to the tolerance,
    similar iteration counts and the same lambda_max estimates to ~1e-2."""
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    k0, _, moduli, fixed, force = cantilever(shape, 6)
    rng = np.random.default_rng(12)
    forces = np.column_stack([force, rng.normal(size=(force.size, 4))])
    forces[fixed] = 0
    expected = direct(shape, k0, moduli, fixed, forces)
    runs = {}
    for tensor in (False, True):
        mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "precision": "float32", "tolerance": 1e-10,
                                                        "tensor_cores": tensor})
        mg.update(moduli)
        solution, report = mg.solve("c", fixed, forces)
        assert report["converged"], report
        for c in range(forces.shape[1]):
            assert np.linalg.norm(solution[:, c] - expected[:, c]) < 1e-7 * np.linalg.norm(expected[:, c])
        runs[tensor] = report
        mg.close()
    assert max(runs[True]["iterations"]) <= 1.3 * max(runs[False]["iterations"]) + 2
    lam_tc, lam_cc = np.asarray(runs[True]["lambda_max"]), np.asarray(runs[False]["lambda_max"])
    assert np.max(np.abs(lam_tc / lam_cc - 1)) < 1e-2


@pytest.mark.parametrize("shape,tolerance", [((24, 12, 10), 1e-10), ((16, 8, 16), 1e-8)])
def test_mixed_pcg_converges_on_the_fp64_true_residual(cuda, shape, tolerance):
    """pcg_precision = float32: FP32 iterations and operator with FP64 reliable residual updates.
    Convergence is still decided on the FP64 true residual, so every column meets the tolerance and
    equals the direct solution as closely as the FP64 PCG's; the iteration count stays close to the
    FP64 PCG's on the same hierarchy."""
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    k0, _, moduli, fixed, force = cantilever(shape, 3)
    rng = np.random.default_rng(5)
    forces = np.column_stack([force, rng.normal(size=(force.size, 5))])
    forces[fixed] = 0
    expected = direct(shape, k0, moduli, fixed, forces)
    runs = {}
    for pcg in ("float64", "float32"):
        mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "precision": "float32", "tolerance": tolerance,
                                                        "pcg_precision": pcg})
        mg.update(moduli)
        solution, report = mg.solve("c", fixed, forces)
        assert report["converged"] and max(report["relative_residual"]) < tolerance, report
        bar = 1e-7 if tolerance < 1e-9 else 1e-5
        for c in range(forces.shape[1]):
            assert np.linalg.norm(solution[:, c] - expected[:, c]) < bar * np.linalg.norm(expected[:, c])
        residual = op.assemble(shape, k0, moduli) @ solution - forces
        live = op.live_dofs(shape, moduli, fixed)
        assert np.all(np.linalg.norm(residual[live], axis=0) < 1.01 * tolerance * np.linalg.norm(forces[live], axis=0))
        runs[pcg] = report
        mg.close()
    assert max(runs["float32"]["iterations"]) <= 1.25 * max(runs["float64"]["iterations"]) + 2


def test_mixed_pcg_rejects_a_float64_vcycle(cuda):
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    k0 = hex8.element_matrices((1, 1, 1), 0.3)[0]
    with pytest.raises(ValueError, match="float32 work precision"):
        GeometricMultigrid((8, 4, 4), (1, 1, 1), k0, {"precision": "float64", "pcg_precision": "float32"})


@pytest.mark.parametrize("precision", ["bfloat16", "float16"])
def test_sixteen_bit_vcycle_storage_still_converges_to_the_fp64_answer(cuda, precision):
    """bfloat16 / float16 work precision: every V-cycle vector rounded to the 16-bit format when
    stored (FP32 arithmetic, FP64 outer PCG).  The preconditioner is weaker, never the answer: the
    solution still equals the direct solve to the tolerance."""
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (24, 12, 10)
    k0, _, moduli, fixed, force = cantilever(shape, 3)
    rng = np.random.default_rng(9)
    forces = np.column_stack([force, rng.normal(size=(force.size, 2))])
    forces[fixed] = 0
    expected = direct(shape, k0, moduli, fixed, forces)
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "precision": precision, "tolerance": 1e-10,
                                                    "max_iterations": 3000})
    mg.update(moduli)
    solution, report = mg.solve("c", fixed, forces)
    assert report["converged"], report
    for c in range(forces.shape[1]):
        assert np.linalg.norm(solution[:, c] - expected[:, c]) < 1e-7 * np.linalg.norm(expected[:, c])
    mg.close()


def test_sixteen_bit_storage_refuses_the_tensor_core_apply(cuda):
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    k0 = hex8.element_matrices((1, 1, 1), 0.3)[0]
    with pytest.raises(ValueError, match="tensor_cores"):
        GeometricMultigrid((8, 4, 4), (1, 1, 1), k0, {"precision": "bfloat16", "tensor_cores": True})


def test_banded_coarsest_factor(cuda):
    """A coarsest grid above the dense limit (24,000 live dofs) is factored banded.  With
    coarsest_dofs = 40,000 the 56 x 56 x 24 cantilever keeps two levels, the coarsest with about
    32,800 live dofs; its solve equals the default hierarchy's (dense coarsest factor, more levels,
    itself held to direct solves above), and a batched solve of it next to a dense-coarsest instance
    equals the two own solves."""
    import torch
    from deep_frame_b200.topology_multigrid import GeometricMultigrid, solve_batch_device
    shape = (56, 56, 24)
    k0, _, moduli, fixed, force = cantilever(shape)
    rng = np.random.default_rng(11)
    forces = np.column_stack([force, rng.normal(size=force.size)])
    band = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 40000, "tolerance": 1e-10})
    dense = GeometricMultigrid(shape, (1, 1, 1), k0, {"tolerance": 1e-10})
    for mg in (band, dense):
        mg.update(moduli)
    u_band, rep_band = band.solve("clamped", fixed, forces)
    u_dense, rep_dense = dense.solve("clamped", fixed, forces)
    assert rep_band["converged"] and rep_dense["converged"]
    assert rep_band["levels"] == 2 and rep_band["coarsest_dofs"] > 24000
    assert rep_dense["levels"] > 2 and rep_dense["coarsest_dofs"] <= 8000
    for c in range(forces.shape[1]):
        assert np.linalg.norm(u_band[:, c] - u_dense[:, c]) < 1e-7 * np.linalg.norm(u_dense[:, c])
    small_shape = (16, 8, 8)
    k1, _, m1, f1, g1 = cantilever(small_shape, seed=3)
    small = GeometricMultigrid(small_shape, (1, 1, 1), k1, {"coarsest_dofs": 200, "tolerance": 1e-10})
    small.update(m1)
    jobs = [(band, "clamped", fixed, torch.as_tensor(forces.T.copy(), device="cuda")),
            (small, "clamped", f1, torch.as_tensor(g1[None, :].copy(), device="cuda"))]
    own = [mg.solve_device(key, fx, f) for mg, key, fx, f in jobs]
    batched = solve_batch_device(jobs)
    for (a, _), (b, rep) in zip(own, batched):
        assert rep["converged"]
        assert float((a - b).norm() / a.norm()) < 1e-7
    for mg in (band, dense, small):
        mg.close()
