"""Every level operator of the device hierarchy against the oracle's Galerkin construction.

The reference checks that its Galerkin coarse operator equals the triple product P^T A P
(tests/test_topology_multigrid.py:40-53).  Here each device level (tf_apply_level: the masked
finest operator, then the assembled 27-point Galerkin stencils) is applied to random vectors and
compared with the oracle's level matrices (oracle/gmg.py: P^T A P over the masked finest
operator, symmetrised, with the dead-dof masks at dead_ratio), to FP64 rounding.  The oracle's
element-block form equals P^T A P on the CPU (tests/test_oracle_known_answers.py); this test pins
the device's assembly, its dead-dof masks and its padding to the same matrices.
"""
import numpy as np
import pytest

from oracle import gmg
from oracle import hex8

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,dead", [((12, 8, 8), False), ((10, 6, 9), True)])
def test_device_levels_equal_oracle_galerkin_operators(cuda, shape, dead):
    import torch
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    rng = np.random.default_rng(7)
    ke = hex8.element_matrices((1.0, 1.0, 1.0), 0.3)[0]
    nelem = int(np.prod(shape))
    density = rng.uniform(0.01, 1.0, nelem)
    moduli = 1e-9 + (1 - 1e-9) * density ** 3
    if dead:
        # a void block (dead cells: modulus 0) leaves nodes without live elements at every level
        cells = np.zeros(shape, bool)
        cells[3:7, 2:5, :4] = True
        moduli[cells.ravel()] = 0.0
    nodes = tuple(n + 1 for n in shape)
    clamp = np.flatnonzero(np.indices(nodes).reshape(3, -1)[0] == 0)
    fixed = (3 * clamp[:, None] + np.arange(3)).ravel()
    settings = {"coarsest_dofs": 150}
    oracle = gmg.MultigridOracle(shape, ke, moduli, fixed, settings)
    mg = GeometricMultigrid(shape, (1.0, 1.0, 1.0), ke, {**settings, "precision": "float64", "device": "cuda"})
    mg.update(moduli)
    assert len(mg.levels) == oracle.levels >= 3 and mg.padded == oracle.padded
    for level in range(oracle.levels):
        n = oracle.A[level].shape[0]
        assert n == 3 * int(np.prod(np.asarray(mg.levels[level].shape) + 1))
        u = rng.standard_normal((n, 3)) * oracle.mask[level][:, None]
        want = oracle._apply(level, u)
        got = mg.apply_level_device("clamped", fixed, level, torch.as_tensor(u.T.copy(), device=cuda)).cpu().numpy().T
        scale = np.abs(want).max()
        assert np.abs(got - want).max() <= 1e-12 * scale, f"level {level}"
        live = oracle.mask[level] > 0
        assert not got[~live].any(), f"level {level}: output on dead dofs"
    assert mg.close() == []


def test_reference_covariance_cantilever_on_the_device(cuda):
    """The reference's own covariance cantilever (domain, covariance settings, density and its
    results in tests/golden/covariance.npz, from its InterfaceCovariance.measure on SuperLU solves)
    measured by the device path: GMG-PCG solves of every direction, F on the device, tr, lambda_max
    and KS within 1e-6 relative and both sensitivity fields within 1e-5 relative (2-norm).  Its
    directions share a fixture group with the domain's static case."""
    import json
    from pathlib import Path
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    g = np.load(Path(__file__).resolve().parent / "golden" / "covariance.npz")
    domain = json.loads(str(g["domain_json"]))
    for name in ("allowed", "preserve", "forbidden"):
        domain[name] = g[f"domain_{name}"]
    system = HexElasticity(domain, multigrid={"tolerance": 1e-10})
    model = InterfaceCovariance(system, json.loads(str(g["covariance_json"])), domain["interfaces"])
    rows = {row["name"]: row for row in model.measure_device(g["density"], float(g["penalization"]), float(g["min_stiffness_ratio"]))}
    assert rows["load_mean"]["value"] == pytest.approx(float(g["load_mean"]), rel=1e-6)
    assert rows["load_worst"]["value"] == pytest.approx(float(g["load_worst"]), rel=1e-6)
    assert rows["load_worst"]["info"]["ks_n_mm"] == pytest.approx(float(g["ks"]), rel=1e-6)
    for name, key in (("load_mean", "grad_mean"), ("load_worst", "grad_worst")):
        got = rows[name]["gradient"].cpu().numpy()
        assert np.linalg.norm(got - g[key]) < 1e-5 * np.linalg.norm(g[key]), name
    expected = json.loads(str(g["info_json"]))
    assert [label for label, _ in rows["load_worst"]["info"]["worst_wrench"]] == [label for label, _ in expected["worst_wrench"]]
    assert system.close() == []
