"""Fine operator, masked operator and element energies vs the oracle's assembled matrix.

Mirrors the reference's test_operator_matches_assembled_matrix
(tests/test_topology_multigrid.py:24-38): 1e-12 relative in FP64.
"""
import numpy as np
import pytest

from oracle import hex8, operator as op

pytestmark = pytest.mark.gpu


def _moduli(shape, seed, dead=0.0):
    rng = np.random.default_rng(seed)
    density = np.clip(rng.uniform(0.3, 1.2, int(np.prod(shape))), 0, 1)
    moduli = 1e-6 + (1 - 1e-6) * density ** 3
    if dead:
        moduli[rng.uniform(size=moduli.size) < dead] = 0.0
    return moduli


@pytest.mark.parametrize("shape,spacing,dead", [((8, 3, 5), (1.0, 1.0, 1.0), 0.0), ((4, 8, 4), (1.0, 1.0, 1.0), 0.0),
                                                 ((7, 6, 5), (0.747, 0.753, 0.667), 0.2), ((12, 10, 17), (1.0, 1.0, 1.0), 0.1),
                                                 ((9, 7, 1), (1.0, 1.0, 1.0), 0.0), ((5, 3, 30), (1.0, 2.0, 0.5), 0.05)])
def test_operator_matches_assembled_matrix(cuda, shape, spacing, dead):
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    k0, _, _ = hex8.element_matrices(spacing, 0.3)
    moduli = _moduli(shape, 0, dead)
    mg = GeometricMultigrid(shape, spacing, k0, {"coarsest_dofs": 200})
    mg.update(moduli)
    matrix = op.assemble(shape, k0, moduli)
    ndof = matrix.shape[0]
    vectors = np.random.default_rng(1).normal(size=(ndof, 3))
    inactive = ~op.live_dofs(shape, moduli)
    vectors[inactive] = 0
    expected = matrix @ vectors
    full = mg.product(vectors)
    assert np.linalg.norm(full - expected) < 1e-12 * np.linalg.norm(expected)
    # reduced operator with the Dirichlet mask of the x = 0 face (the PCG operator)
    nodes = np.asarray(shape) + 1
    fixed_nodes = np.flatnonzero(hex8.node_points(shape, (1, 1, 1))[:, 0] == 0)
    fixed = (3 * fixed_nodes[:, None] + np.arange(3)).ravel()
    live = op.live_dofs(shape, moduli, fixed)
    columns = mg._columns(vectors)
    reduced = mg.apply_device(columns, key="x0", fixed=fixed).T.cpu().numpy()
    exp_red = np.zeros_like(vectors)
    exp_red[live] = matrix[live][:, live] @ vectors[live]
    assert np.linalg.norm(reduced - exp_red) < 1e-12 * np.linalg.norm(exp_red)
    assert np.all(reduced[~live] == 0)
    mg.close()


def test_element_energy_matches_oracle(cuda):
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (9, 5, 6)
    k0, _, _ = hex8.element_matrices((1, 1, 1), 0.3)
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 200})
    mg.update(_moduli(shape, 2))
    u = np.random.default_rng(3).normal(size=(3 * int(np.prod(np.asarray(shape) + 1)), 4))
    expected = op.element_energy(shape, k0, u)
    columns = mg._columns(u)
    got = mg.energy_device(columns).cpu().numpy()
    assert np.max(np.abs(got - expected)) < 1e-12 * np.max(np.abs(expected))
    # weighted sum with a per-element scale, and the combination form sum_j c_j (U v_j)^T K0 (U v_j)
    import torch
    coef = np.array([0.5, 2.0, -1.0, 3.0])
    scale = np.random.default_rng(4).uniform(0.1, 2.0, mg.nelem)
    s_dev = torch.as_tensor(scale, device=cuda)
    got = mg.energy_device(columns, coefficients=coef, scale=s_dev).cpu().numpy()
    assert np.max(np.abs(got - scale * (coef @ expected))) < 1e-12 * np.max(np.abs(scale * (coef @ expected)))
    comb = np.random.default_rng(5).normal(size=(4, 2))
    got = mg.energy_device(columns, combination=comb, coefficients=[1.0, -0.5]).cpu().numpy()
    w = u @ comb
    ref = op.element_energy(shape, k0, w)
    assert np.max(np.abs(got - (ref[0] - 0.5 * ref[1]))) < 1e-11 * np.max(np.abs(ref))
    # the reference grid-layout entry point returns the padded element grid
    grid = mg.grid(u)
    padded = mg.element_energy(grid).cpu().numpy()
    assert padded.shape == (4,) + mg.padded
    assert np.max(np.abs(padded[:, :shape[0], :shape[1], :shape[2]].reshape(4, -1) - expected)) < 1e-12 * np.max(np.abs(expected))
    mg.close()


@pytest.mark.parametrize("fine_tz", [7, 8, 9])
def test_tile_heights_give_the_same_operator(cuda, fine_tz):
    """Every finest-level tile height (7, 8, 9 nodes along z; a tuning choice) applies the same
    FP64 operator (1e-12 vs the assembled matrix) and gives the same FP32-V-cycle PCG solve."""
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    shape = (12, 10, 20)
    k0, _, _ = hex8.element_matrices((1, 1, 1), 0.3)
    moduli = _moduli(shape, 4, 0.05)
    matrix = op.assemble(shape, k0, moduli)
    vectors = np.random.default_rng(5).normal(size=(matrix.shape[0], 3))
    vectors[~op.live_dofs(shape, moduli)] = 0
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "fine_tz": fine_tz, "tolerance": 1e-10})
    mg.update(moduli)
    expected = matrix @ vectors
    assert np.linalg.norm(mg.product(vectors) - expected) < 1e-12 * np.linalg.norm(expected)
    fixed_nodes = np.flatnonzero(hex8.node_points(shape, (1, 1, 1))[:, 0] == 0)
    fixed = (3 * fixed_nodes[:, None] + np.arange(3)).ravel()
    forces = np.random.default_rng(6).normal(size=(matrix.shape[0], 2))
    u, report = mg.solve("x0", fixed, forces)
    ref = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "fine_tz": 8, "tolerance": 1e-10})
    ref.update(moduli)
    u8, report8 = ref.solve("x0", fixed, forces)
    assert report["converged"] and abs(report["iterations"][0] - report8["iterations"][0]) <= 1
    assert np.linalg.norm(u - u8) < 1e-8 * np.linalg.norm(u8)
    mg.close()
    ref.close()
