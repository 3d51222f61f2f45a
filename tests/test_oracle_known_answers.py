"""Known answers the oracle must reproduce, after the reference's own physics tests.  No GPU.

* Euler-Bernoulli tip deflection (8 %) and first bending frequency (5 %) of a slender clamped
  hex8 beam (reference tests/test_topology_optimization.py:56-68);
* compliance sensitivity through SIMP, the cone filter and the projection against central
  finite differences, relative 2e-5, and the volume derivative (:70-89);
* tr(K^-1 Sigma) and the KS aggregate of the covariance eigenvalues against central finite
  differences in the physical densities, relative 1e-5 (reference
  tests/test_topology_problem.py:510-528).

The device results are held to the oracle elsewhere (the tests marked gpu), so these close the
chain from the kernels to the physics.
"""
import numpy as np
import pytest
from scipy.sparse.linalg import eigsh, splu

from oracle import covariance as ocov
from oracle import hex8, operator as op
from oracle.density import DensityMapOracle


def clamped_beam(shape):
    nodes = tuple(n + 1 for n in shape)
    i = np.indices(nodes).reshape(3, -1)
    clamp = np.flatnonzero(i[0] == 0)
    tip = np.flatnonzero(i[0] == shape[0])
    fixed = (3 * clamp[:, None] + np.arange(3)).ravel()
    free = np.setdiff1d(np.arange(3 * int(np.prod(nodes))), fixed)
    return tip, free


def test_cantilever_deflection_and_frequency_against_euler_bernoulli():
    shape, spacing = (24, 4, 4), (2.0, 1.5, 1.5)
    young, rho = 4430.0, 1.09e-9
    k0, m0, _ = hex8.element_matrices(spacing, 0.3)
    nelem = int(np.prod(shape))
    stiffness = op.assemble(shape, k0, np.full(nelem, young)).tocsc()
    mass = op.assemble(shape, m0, np.full(nelem, rho)).tocsc()
    tip, free = clamped_beam(shape)
    force = np.zeros(stiffness.shape[0])
    force[3 * tip + 2] = -1.0 / len(tip)                  # 1 N in -z spread over the end face
    u = np.zeros_like(force)
    u[free] = splu(stiffness[free][:, free]).solve(force[free])
    deflection = -np.mean(u[3 * tip + 2])
    length, width, height = np.asarray(shape) * spacing
    second_moment = width * height ** 3 / 12
    assert deflection == pytest.approx(length ** 3 / (3 * young * second_moment), rel=0.08)
    omega2 = eigsh(stiffness[free][:, free], k=1, M=mass[free][:, free], sigma=0, which="LM")[0][0]
    expected = 1.875104068711961 ** 2 / (2 * np.pi * length ** 2) * np.sqrt(young * second_moment / (rho * width * height))
    assert np.sqrt(omega2) / (2 * np.pi) == pytest.approx(expected, rel=0.05)


def test_filtered_projected_compliance_sensitivity_matches_finite_difference():
    shape, spacing = (5, 3, 3), (2.0, 2.0, 2.0)
    young, p, eps = 4430.0, 3.0, 1e-9
    preserve = np.zeros(shape, dtype=bool)
    preserve[0] = True
    preserve[-1] = True
    mapping = DensityMapOracle(shape, spacing, 3.1, np.ones(shape, dtype=bool), preserve, beta=2.0)
    k0 = hex8.element_matrices(spacing, 0.3)[0]
    tip, free = clamped_beam(shape)
    force = np.zeros(3 * int(np.prod(np.asarray(shape) + 1)))
    force[3 * tip + 2] = -1.0 / len(tip)

    def compliance(design, gradient=False):
        physical, projection = mapping.physical(design)
        moduli, slope = hex8.simp(physical, p, eps, young)
        k = op.assemble(shape, k0, moduli).tocsc()
        u = np.zeros_like(force)
        u[free] = splu(k[free][:, free]).solve(force[free])
        value = float(force @ u)
        if not gradient:
            return value
        return value, mapping.pullback(-slope * op.element_energy(shape, k0, u), projection), projection

    design = np.full(mapping.n, 0.65)
    design[mapping.preserve.ravel()] = 1.0
    _, derivative, projection = compliance(design, gradient=True)
    volume_derivative = mapping.pullback(np.ones(mapping.n), projection)
    direction = np.random.default_rng(42).normal(size=mapping.n)
    direction[~mapping.free.ravel()] = 0.0
    direction /= np.linalg.norm(direction)
    step = 1e-5
    fd = (compliance(design + step * direction) - compliance(design - step * direction)) / (2 * step)
    assert derivative @ direction == pytest.approx(fd, rel=2e-5, abs=1e-10)
    plus, minus = mapping.physical(design + step * direction)[0], mapping.physical(design - step * direction)[0]
    assert volume_derivative @ direction == pytest.approx((plus.sum() - minus.sum()) / (2 * step), rel=1e-7)


def test_covariance_trace_and_ks_gradients_match_finite_differences():
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    shape = (16, 12, 4)
    domain, density, cov = problems.plate(shape, 3)
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    index = {name: k for k, name in enumerate(model.cases)}
    halves = []
    for members in system.groups.values():
        forces = np.zeros((system.ndof, model.rank))
        for case, part in members:
            forces[:, index[case["name"]]] = part["force"]
        halves.append((forces, members[0][1]["fixed"]))

    def measure(physical):
        moduli, slope = system.moduli(physical, 3.0, 1e-9)
        k = op.assemble(shape, system.ke, moduli).tocsc()
        parts = []
        for forces, fixed in halves:
            live = op.live_dofs(shape, moduli, fixed)
            u = np.zeros_like(forces)
            u[live] = splu(k[live][:, live].tocsc()).solve(forces[live])
            parts.append((forces, u))
        # KS with a fixed scale (the constraint limit), as the reference's load_worst constraint uses
        return ocov.measure(parts, model.factor, shape, system.ke, slope, ks=5.0, limit_worst=40.0)

    rng = np.random.default_rng(5)
    physical = rng.uniform(0.3, 0.7, int(np.prod(shape)))
    direction = rng.standard_normal(physical.size)
    step = 1e-5
    at, plus, minus = measure(physical), measure(physical + step * direction), measure(physical - step * direction)
    assert at["grad_mean"] @ direction == pytest.approx((plus["load_mean"] - minus["load_mean"]) / (2 * step), rel=1e-5)
    assert at["grad_worst"] @ direction == pytest.approx((plus["ks"] - minus["ks"]) / (2 * step), rel=1e-5)
    assert at["ks"] >= at["load_worst"]


def test_galerkin_element_blocks_equal_the_sparse_triple_product():
    """The reference builds each Galerkin level from element blocks, sum over the 8 children of
    P_c^T B_c P_c (topology_multigrid.py:145-208); the oracle uses P^T A P with the sparse
    prolongation.  They are the same operator, on the first level (children masked on both sides
    by the fine live mask) and on the next (children unmasked): the reference's
    tests/test_topology_multigrid.py:41-53 checks the same identity."""
    from oracle.gmg import MultigridOracle, assemble_blocks, fine_blocks, galerkin_blocks
    shape = (8, 8, 8)
    rng = np.random.default_rng(11)
    moduli = rng.uniform(0.05, 1.0, int(np.prod(shape)))
    moduli[rng.uniform(size=moduli.size) < 0.1] = 0.0                             # some void cells
    nodes = np.indices(tuple(n + 1 for n in shape)).reshape(3, -1)
    fixed = (3 * np.flatnonzero(nodes[0] == 0)[:, None] + np.arange(3)).ravel()
    k0 = hex8.element_matrices((1.0, 1.0, 1.0), 0.3)[0]
    mg = MultigridOracle(shape, k0, moduli, fixed, {"coarsest_dofs": 100})
    assert mg.levels == 3 and mg.padded == shape
    level1 = galerkin_blocks(shape, fine_blocks(shape, k0, moduli, mg.mask[0]))
    level2 = galerkin_blocks((4, 4, 4), level1)
    for level, (grid, blocks) in enumerate((((4, 4, 4), level1), ((2, 2, 2), level2)), start=1):
        difference = assemble_blocks(grid, blocks) - mg.A[level]
        assert abs(difference).max() < 1e-12 * abs(mg.A[level]).max(), level


def test_half_plate_equals_the_full_plate():
    """The mirror-symmetric half model (x >= 0, symmetric and antisymmetric fixture groups, factor 2)
    gives the tr(K^-1 Sigma) and lambda_max of the full plate with mirrored densities, both set up by
    the product's host code and solved directly; the reference checks the same on its cantilever
    (tests/test_topology_problem.py:479-508, relative 1e-8)."""
    import copy
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    shape = (16, 12, 4)
    half, density, cov = problems.plate(shape, 2)
    full = copy.deepcopy(half)
    full.pop("symmetry")
    full["grid"]["shape"] = [2 * shape[0], shape[1], shape[2]]
    full["grid"]["origin_mm"] = [-float(shape[0]), 0.0, 0.0]
    for name in ("allowed", "preserve", "forbidden"):
        full[name] = np.concatenate([half[name][::-1], half[name]], axis=0)
    density_full = np.concatenate([density.reshape(shape)[::-1], density.reshape(shape)], axis=0).ravel()

    def measure(domain, rho):
        grid = tuple(domain["grid"]["shape"])
        system = HexElasticity(domain)
        model = InterfaceCovariance(system, cov, domain["interfaces"])
        moduli, slope = system.moduli(rho, 3.0, 1e-9)
        k = op.assemble(grid, system.ke, moduli).tocsc()
        index = {name: j for j, name in enumerate(model.cases)}
        parts = []
        for members in system.groups.values():
            forces = np.zeros((system.ndof, model.rank))
            for case, part in members:
                forces[:, index[case["name"]]] = part["force"]
            live = op.live_dofs(grid, moduli, members[0][1]["fixed"])
            u = np.zeros_like(forces)
            u[live] = splu(k[live][:, live].tocsc()).solve(forces[live])
            parts.append((forces, u))
        return model, ocov.measure(parts, model.factor, grid, system.ke, slope)

    half_model, half_values = measure(half, density)
    full_model, full_values = measure(full, density_full)
    assert half_model.factor == 2.0 and full_model.factor == 1.0 and len(half_model.system.groups) == 2
    assert half_values["load_mean"] == pytest.approx(full_values["load_mean"], rel=1e-8)
    assert half_values["load_worst"] == pytest.approx(full_values["load_worst"], rel=1e-8)


def test_rank_one_covariance_has_trace_equal_to_lambda_max():
    """With a rank-one Sigma = s s^T there is one load direction, so F is 1 x 1 and
    tr(K^-1 Sigma) = lambda_max (reference tests/test_topology_problem.py:510-516)."""
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    shape = (16, 12, 4)
    domain, density, cov = problems.plate(shape, 1)
    s = np.random.default_rng(4).standard_normal(42)
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, dict(cov, sigma=np.outer(s, s)), domain["interfaces"])
    assert model.rank == 1 and np.allclose(model.directions @ model.directions.T, np.outer(s, s))
    moduli, slope = system.moduli(density, 3.0, 1e-9)
    k = op.assemble(shape, system.ke, moduli).tocsc()
    parts = []
    for members in system.groups.values():
        forces = np.column_stack([part["force"] for _, part in members])
        live = op.live_dofs(shape, moduli, members[0][1]["fixed"])
        u = np.zeros_like(forces)
        u[live] = splu(k[live][:, live].tocsc()).solve(forces[live])
        parts.append((forces, u))
    values = ocov.measure(parts, model.factor, shape, system.ke, slope)
    assert values["load_mean"] == pytest.approx(values["load_worst"], rel=1e-12)
    assert np.allclose(values["grad_mean"], values["grad_worst"], rtol=1e-10, atol=1e-14 * np.abs(values["grad_mean"]).max())


def test_oracle_skips_zero_load_columns_like_the_reference():
    """A zero right-hand side column is not solved (zero solution, 0 iterations, residual 0) and the
    others converge as if alone (reference topology_multigrid.py:350-351 and its
    tests/test_topology_multigrid.py:178-188)."""
    from oracle.gmg import MultigridOracle
    shape = (8, 4, 4)
    k0 = hex8.element_matrices((1.0, 1.0, 1.0), 0.3)[0]
    moduli = np.random.default_rng(2).uniform(0.2, 1.0, int(np.prod(shape)))
    tip, free = clamped_beam(shape)
    fixed = np.setdiff1d(np.arange(3 * int(np.prod(np.asarray(shape) + 1))), free)
    force = np.zeros(3 * int(np.prod(np.asarray(shape) + 1)))
    force[3 * tip + 2] = -1.0 / len(tip)
    mg = MultigridOracle(shape, k0, moduli, fixed, {"tolerance": 1e-10, "coarsest_dofs": 100})
    u, iterations, relative, _ = mg.solve(np.column_stack([force, np.zeros_like(force), 2 * force]))
    alone = mg.solve(force)[0][:, 0]
    assert iterations[1] == 0 and relative[1] == 0 and not u[:, 1].any()
    assert iterations[0] > 0 and relative[0] < 1e-10 and relative[2] < 1e-10
    assert np.allclose(u[:, 0], alone, rtol=0, atol=1e-9 * np.abs(alone).max())
    assert np.allclose(u[:, 2], 2 * alone, rtol=0, atol=1e-9 * np.abs(alone).max())
