"""LOBPCG eigenpairs with the V-cycle preconditioner vs a shift-invert Lanczos solve of the assembled pencil.

Mirrors the reference's tests/test_topology_multigrid.py:106-138 (eigenvalues to 1e-9 relative against
scipy eigsh with sigma = 0) on a clamped cantilever with SIMP stiffness, element masses and a few
lumped nodal masses.
"""
import numpy as np
import pytest
from scipy.sparse import diags
from scipy.sparse.linalg import eigsh

from oracle import hex8, operator as op

pytestmark = pytest.mark.gpu


def problem(shape=(16, 3, 6), seed=3):
    k0, m0, _ = hex8.element_matrices((1.0, 1.0, 1.0), 0.3)
    density = np.clip(np.random.default_rng(seed).uniform(0.2, 1.3, int(np.prod(shape))), 0, 1)
    moduli = 1e-6 + (1 - 1e-6) * density ** 3
    mass = 1.09 * density
    points = hex8.node_points(shape, (1, 1, 1))
    fixed_nodes = np.flatnonzero(points[:, 0] == 0)
    fixed = (3 * fixed_nodes[:, None] + np.arange(3)).ravel()
    lumped = np.zeros(3 * len(points))
    tip = np.flatnonzero(points[:, 0] == shape[0])
    lumped[(3 * tip[:, None] + np.arange(3)).ravel()] = 0.05
    return k0, m0, moduli, mass, lumped, fixed


def shift_invert(shape, k0, m0, moduli, mass, lumped, fixed, count):
    stiffness = op.assemble(shape, k0, moduli).tocsc()
    pencil = (op.assemble(shape, m0, mass) + diags(lumped)).tocsc()
    live = op.live_dofs(shape, moduli, fixed)
    values, vectors = eigsh(stiffness[live][:, live], k=count, M=pencil[live][:, live], sigma=0.0)
    order = np.argsort(values)
    full = np.zeros((stiffness.shape[0], count))
    full[live] = vectors[:, order]
    return values[order], full, stiffness, pencil


@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_lobpcg_matches_shift_invert(cuda, precision):
    import torch
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (16, 3, 6)
    k0, m0, moduli, mass, lumped, fixed = problem(shape)
    expected, vectors, stiffness, pencil = shift_invert(shape, k0, m0, moduli, mass, lumped, fixed, 4)
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 200, "precision": precision}, m0)
    mg.update(moduli)
    values, modes, report = mg.eigenpairs("modes", fixed, mass, lumped, 4)
    assert report["converged"] and report["levels"] > 1, report
    assert np.max(np.abs(values - expected) / expected) < 1e-9
    v = modes[:4].cpu().numpy().T
    # M-orthonormal Ritz vectors with small residuals, spanning the reference modes
    assert np.allclose(v.T @ (pencil @ v), np.eye(4), atol=1e-8)
    residual = np.linalg.norm(stiffness @ v - (pencil @ v) * values, axis=0) / np.linalg.norm(stiffness @ v, axis=0)
    live = np.zeros(stiffness.shape[0], dtype=bool)
    live[op.live_dofs(shape, moduli, fixed)] = True
    residual = np.linalg.norm((stiffness @ v - (pencil @ v) * values)[live], axis=0) / np.linalg.norm((stiffness @ v)[live], axis=0)
    assert np.all(residual < 1e-7)
    overlap = np.abs(vectors[:, 0] @ (pencil @ v[:, 0])) / np.sqrt((vectors[:, 0] @ (pencil @ vectors[:, 0])) * (v[:, 0] @ (pencil @ v[:, 0])))
    assert overlap == pytest.approx(1.0, abs=1e-8)
    # a warm start from the converged block converges at once to the same values
    again, _, report2 = mg.eigenpairs("modes", fixed, mass, lumped, 4, initial=modes)
    assert report2["iterations"] <= 1 and np.max(np.abs(again - values) / values) < 1e-10
    mg.close()


def test_mass_operator_matches_assembled_mass(cuda):
    import torch
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (8, 4, 5)
    k0, m0, moduli, mass, lumped, fixed = problem(shape, 1)
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 200}, m0)
    mg.update(moduli)
    u = np.random.default_rng(4).normal(size=(2, 3 * int(np.prod(np.asarray(shape) + 1))))
    y = mg.mass_device(torch.as_tensor(u, device="cuda"), "m", fixed, torch.as_tensor(mass, device="cuda"),
                       torch.as_tensor(lumped, device="cuda")).cpu().numpy()
    pencil = (op.assemble(shape, m0, mass) + diags(lumped)).tocsc()
    live = np.zeros(pencil.shape[0])
    live[op.live_dofs(shape, moduli, fixed)] = 1
    expected = (live[:, None] * (pencil @ (live[:, None] * u.T))).T
    assert np.max(np.abs(y - expected)) < 1e-13 * np.max(np.abs(expected))
    mg.close()
