"""The seeded benchmark workloads are the ones they are named for.  No GPU.

Plate (the covariance-load half model): 96 x 96 x 16 unit voxels, mirror plane x = 0, a clamped
stack patch x in [0, 4], y in [44, 52] through the thickness (8 x 8 x 16 in the full model),
7 interface patches x 6 unit wrenches = 42 load directions, Sigma = X^T X / 60 (Wishart, 60 dof),
densities a Gaussian-smoothed (sigma = 3 voxels) normal field through a sigmoid to [0.001, 1].
Cantilever: 48 x 24 x 24, x = 0 face clamped, one unit -z load at node (48, 12, 0), densities
i.i.d. U[0.01, 1] from default_rng(seed).
"""
import numpy as np
import pytest
from scipy.ndimage import gaussian_filter

from deep_frame_b200 import problems


def test_plate_domain_matches_its_specification():
    domain, density, cov = problems.plate((96, 96, 16), 0)
    assert domain["grid"]["shape"] == [96, 96, 16] and domain["grid"]["spacing_mm"] == [1.0, 1.0, 1.0]
    assert domain["symmetry"] == {"axis": 0, "plane_mm": 0.0}
    stack = domain["load_cases"][0]["fixed_regions"][0]
    assert np.allclose(stack["min_mm"], [-4, 44, 0], atol=1e-5) and np.allclose(stack["max_mm"], [4, 52, 16], atol=1e-5)
    assert list(domain["interfaces"]) == ["motor_front_left", "motor_front_right", "motor_rear_left", "motor_rear_right",
                                          "stack", "battery", "camera"]
    for name in ("motor_front_left", "motor_front_right", "motor_rear_left", "motor_rear_right"):
        lo, hi = (np.asarray(domain["interfaces"][name]["regions"][0][k]) for k in ("min_mm", "max_mm"))
        assert np.allclose(hi[:2] - lo[:2], 4, atol=1e-5) and np.allclose([lo[2], hi[2]], 16, atol=1e-5)   # 4 x 4 pads on the top face
    assert len(cov["labels"]) == 42 and cov["labels"][0] == ["motor_front_left", "Fx"] and cov["labels"][-1] == ["camera", "Mz"]
    x = np.random.default_rng(1000).standard_normal((60, 42))
    assert np.allclose(cov["sigma"], x.T @ x / 60) and np.all(np.linalg.eigvalsh(cov["sigma"]) > 0)
    z = gaussian_filter(np.random.default_rng(0).standard_normal((96, 96, 16)), 3.0)
    assert np.allclose(density, 0.001 + 0.999 / (1 + np.exp(-z / z.std())).ravel())
    assert density.min() >= 0.001 and density.max() <= 1.0 and density.size == 96 * 96 * 16


@pytest.mark.parametrize("seed", [0, 3])
def test_plate_is_seeded(seed):
    a, b = problems.plate((32, 32, 8), seed), problems.plate((32, 32, 8), seed)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2]["sigma"], b[2]["sigma"])
    assert not np.array_equal(a[1], problems.plate((32, 32, 8), seed + 1)[1])


def test_plate_load_model_has_42_directions_and_a_clamped_stack():
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    domain, density, cov = problems.plate((96, 96, 16), 0)
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    assert model.rank == 42 and model.factor == 2.0 and system.ndof == 479859
    assert len(system.groups) == 2 and all(len(members) == 42 for members in system.groups.values())
    nodes = np.indices((97, 97, 17)).reshape(3, -1)
    clamped = np.flatnonzero((nodes[0] <= 4) & (nodes[1] >= 44) & (nodes[1] <= 52))
    for members in system.groups.values():
        fixed = set(members[0][1]["fixed"].tolist())
        assert all(3 * n + c in fixed for n in clamped for c in range(3))


def test_cantilever_matches_its_specification():
    domain, density = problems.cantilever((48, 24, 24), 0)
    assert np.array_equal(density, np.random.default_rng(0).uniform(0.01, 1.0, 48 * 24 * 24))
    case = domain["load_cases"][0]
    fixed, load = case["fixed_regions"][0], case["loads"][0]
    assert np.allclose(fixed["min_mm"], 0, atol=1e-5) and np.allclose(fixed["max_mm"], [0, 24, 24], atol=1e-5)
    assert np.allclose(load["region"]["min_mm"], [48, 12, 0], atol=1e-5) and np.allclose(load["region"]["max_mm"], [48, 12, 0], atol=1e-5)
    assert load["force_n"] == [0.0, 0.0, -1.0]
