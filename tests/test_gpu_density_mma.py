"""Device density filter / projection / pullback and the device MMA step vs the oracle.

Filter: the reference's sparse filter fixtures (tests/golden/filter.npz, from
tests/test_topology_multigrid.py:140-156 semantics), 1e-12.  MMA: the oracle
restatement of Svanberg's method (MMA numerics are not pinned by the
reference, whose mmapy dependency is absent), 1e-9 over several steps.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import density as oden
from oracle import mma as omma

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _domain(g, name):
    shape = tuple(int(s) for s in g[f"{name}_shape"])
    allowed = g[f"{name}_allowed"].reshape(shape).astype(bool)
    return {"grid": {"shape": list(shape), "spacing_mm": g[f"{name}_spacing"].tolist(), "origin_mm": [0.0, 0.0, 0.0]},
            "allowed": allowed, "preserve": g[f"{name}_preserve"].reshape(shape).astype(bool), "forbidden": ~allowed}


@pytest.mark.parametrize("name", ["beam", "unit"])
def test_device_filter_matches_reference_sparse_filter(cuda, name):
    from deep_frame_b200.density import ConeFilter, DensityMap
    g = np.load(GOLDEN / "filter.npz")
    domain = _domain(g, name)
    settings = {"filter_radius_mm": float(g[f"{name}_radius"]), "projection_beta": float(g[f"{name}_beta"]), "projection_eta": 0.5,
                "projection": "single", "beta_schedule": None, "minimum_design_density": 1e-3}
    mapping = DensityMap(domain, settings)
    assert np.max(np.abs(mapping.sums - g[f"{name}_sums"]) / g[f"{name}_sums"]) < 1e-12
    assert np.max(np.abs(mapping.filtered(g[f"{name}_design"]) - g[f"{name}_filtered"])) < 1e-12
    physical, projection = mapping.physical(g[f"{name}_design"])
    assert np.max(np.abs(physical - g[f"{name}_physical"])) < 1e-12
    assert np.max(np.abs(projection - g[f"{name}_projection"])) < 1e-12
    pull = mapping.pullback(g[f"{name}_sensitivity"], projection)
    assert np.max(np.abs(pull - g[f"{name}_pullback"])) < 1e-12 * np.max(np.abs(g[f"{name}_pullback"]))
    conv = ConeFilter(domain["allowed"], domain["allowed"].shape, domain["grid"]["spacing_mm"], float(g[f"{name}_radius"]))
    raw = conv(g[f"{name}_design"])
    assert np.max(np.abs(raw / g[f"{name}_sums"] - g[f"{name}_filtered"])) < 1e-12
    mapping.close()


def test_robust_projection_matches_oracle_formula(cuda):
    from deep_frame_b200.density import DensityMap
    shape = (9, 7, 5)
    allowed = np.random.default_rng(0).uniform(size=shape) > 0.1
    domain = {"grid": {"shape": list(shape), "spacing_mm": [1.0, 1.0, 1.0], "origin_mm": [0.0, 0.0, 0.0]},
              "allowed": allowed, "preserve": np.zeros(shape, dtype=bool), "forbidden": ~allowed}
    settings = {"filter_radius_mm": 1.5, "projection_beta": 8.0, "projection_eta": 0.5, "projection": "robust", "robust_delta": 0.2,
                "beta_schedule": None, "minimum_design_density": 1e-3}
    mapping = DensityMap(domain, settings)
    f = np.random.default_rng(1).uniform(size=allowed.size)
    for eta in (0.3, 0.5, 0.7):
        phys, der = mapping.project(f, eta)
        den = np.tanh(8 * eta) + np.tanh(8 * (1 - eta))
        shifted = 8 * (f - eta)
        decay = np.exp(-2 * np.abs(shifted))
        want = np.clip(np.where(allowed.ravel(), (np.tanh(8 * eta) + np.tanh(shifted)) / den, 0), 0, 1)
        want_d = np.where(allowed.ravel(), 8 * 4 * decay / (1 + decay) ** 2 / den, 0)
        assert np.max(np.abs(phys - want)) < 1e-13 and np.max(np.abs(der - want_d)) < 1e-12
    mapping.close()


@pytest.mark.parametrize("m", [1, 2, 3])
def test_device_mma_matches_oracle(cuda, m):
    from deep_frame_b200.mma import mmasub
    rng = np.random.default_rng(m)
    n = 3000
    w = rng.uniform(0.5, 2.0, n)
    cons = rng.uniform(0.5, 1.5, (m, n))
    x = np.full(n, 0.3)
    xold1, xold2 = x.copy(), x.copy()
    low, upp = np.zeros(n), np.ones(n)
    olow, oupp = low.copy(), upp.copy()
    for it in range(1, 6):
        f0, df0 = np.sum(w / x), -w / x ** 2
        g = cons @ x / (0.3 * n) - 1.0
        dg = cons / (0.3 * n)
        args = (m, n, it, x[:, None], 0.0, 1.0, xold1[:, None], xold2[:, None], 100 * f0, 100 * df0[:, None], 100 * g[:, None],
                100 * dg, None, None, 1.0, np.zeros((m, 1)), np.full((m, 1), 1e4), np.ones((m, 1)))
        got = mmasub(*args[:12], low[:, None], upp[:, None], *args[14:], move=0.2)
        want = omma.mmasub(m, n, it, x, np.zeros(n), np.ones(n), xold1, xold2, 100 * f0, 100 * df0, 100 * g, 100 * dg, olow, oupp,
                           1.0, np.zeros(m), np.full(m, 1e4), np.ones(m), move=0.2)
        xg, lg, ug = got[0].ravel(), got[9].ravel(), got[10].ravel()
        assert np.max(np.abs(lg - want[4])) < 1e-12 and np.max(np.abs(ug - want[5])) < 1e-12
        assert np.max(np.abs(xg - want[0])) < 1e-9, it
        assert np.max(np.abs(got[3].ravel() - want[3])) < 1e-6 * max(1.0, np.max(np.abs(want[3])))
        xold2, xold1 = xold1, x
        x = np.clip(want[0], 0, 1)
        low, upp, olow, oupp = lg, ug, want[4], want[5]
