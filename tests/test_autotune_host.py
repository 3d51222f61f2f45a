"""The autotuner's selection logic with a stand-in solver.  No GPU.

tune_smoother must pick the fastest candidate whose solves all converged, close every solver it
built (one handle at a time), install the winner's settings on the system and fail when no
candidate converges."""
import time
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from deep_frame_b200 import autotune, topology_multigrid


class FakeMultigrid:
    """Costs and convergence keyed by Chebyshev degree: degree 1 fast, 2 slower, 3 does not converge."""
    built = []

    def __init__(self, shape, spacing, ke, settings, me=None):
        self.settings, self.closed = settings, False
        FakeMultigrid.built.append(self)

    def update_device(self, moduli):
        time.sleep({1: 0.002, 2: 0.02, 3: 0.001}[self.settings["chebyshev_degree"]])

    def solve_device(self, key, fixed, forces):
        degree = self.settings["chebyshev_degree"]
        return None, {"converged": degree != 3, "iterations": [10 * degree, 10 * degree + 1]}

    def close(self):
        self.closed = True
        return []


@pytest.fixture
def fake(monkeypatch):
    FakeMultigrid.built = []
    monkeypatch.setattr(topology_multigrid, "GeometricMultigrid", FakeMultigrid)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    previous = FakeMultigrid((1, 1, 1), (1, 1, 1), None, {"chebyshev_degree": 2})
    system = SimpleNamespace(shape=(4, 4, 4), spacing=(1.0, 1.0, 1.0), ke=np.eye(24), me=None,
                             multigrid_settings={"tolerance": 1e-8}, multigrid=previous,
                             groups={"a": [(None, {"fixed": np.arange(3)})], "b": [(None, {"fixed": np.arange(6)})]})
    return system, previous


def test_fastest_converged_candidate_is_installed(fake):
    system, previous = fake
    candidates = [{"smoother": "chebyshev", "chebyshev_degree": d, "growth": 2.0} for d in (2, 3, 1)]
    best, timings = autotune.tune_smoother(system, [("a", None), ("b", None)], None, candidates=candidates, repeats=1)
    assert best == {"tolerance": 1e-8, "smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0}
    assert [t["converged"] for t in timings] == [True, False, True]
    assert timings[2]["iterations"] == [11, 11] and timings[2]["seconds"] < timings[0]["seconds"]
    assert system.multigrid is None and system.multigrid_settings == best
    assert previous.closed and all(m.closed for m in FakeMultigrid.built)


def test_no_converged_candidate_raises(fake):
    system, previous = fake
    with pytest.raises(RuntimeError, match="no smoother candidate converged"):
        autotune.tune_smoother(system, [("a", None)], None, candidates=[{"chebyshev_degree": 3}], repeats=1)
    assert all(m.closed for m in FakeMultigrid.built) and system.multigrid_settings == {"tolerance": 1e-8}


def test_candidates_all_solve_to_the_same_tolerance():
    # candidates change the schedule, depth or apply unit only, never the stopping rule
    for cand in autotune.CANDIDATES:
        assert not {"tolerance", "max_iterations", "precision"} & set(cand)
    assert autotune.CANDIDATES[0] == {"smoother": "chebyshev", "chebyshev_degree": 3, "growth": 2.0}
