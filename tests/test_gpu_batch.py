"""One batched solve over uneven instances (tf_solve_batch) against each instance's own solve.

Instances of different grids, hierarchy depths and load-column counts (one zero column among
them) are solved together; each must give its own tf_solve's answer (1e-7 relative) after the same
PCG iteration counts give or take one (the step-length sums run over differently shaped tiles), and
the first instance is checked against the oracle's direct solve as well.
"""
import numpy as np
import pytest

from test_gpu_solve import cantilever, direct

pytestmark = pytest.mark.gpu

SHAPES = [(16, 8, 8, 3), (24, 12, 6, 5), (32, 16, 8, 2), (20, 20, 12, 6), (12, 10, 4, 4)]


def instances(torch, settings):
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    jobs, host = [], []
    for i, (ex, ey, ez, r) in enumerate(SHAPES):
        shape = (ex, ey, ez)
        k0, _, moduli, fixed, force = cantilever(shape, seed=i)
        rng = np.random.default_rng(100 + i)
        forces = np.column_stack([force] + [rng.normal(size=force.size) for _ in range(r - 1)])
        if i == 1:
            forces[:, 2] = 0.0   # a zero column: skipped by PCG, zero solution
        mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, **settings})
        mg.update(moduli)
        dev = torch.as_tensor(forces.T.copy(), device="cuda")
        jobs.append((mg, "clamped", fixed, dev))
        host.append((shape, k0, moduli, fixed, forces))
    return jobs, host


@pytest.mark.parametrize("settings", [
    {"precision": "float32", "smoother": "chebyshev", "tolerance": 1e-10},
    {"precision": "float64", "smoother": "jacobi", "sweeps": 2, "tolerance": 1e-10},
])
def test_batch_matches_single_solves(cuda, settings):
    import torch
    from deep_frame_b200.topology_multigrid import solve_batch_device
    jobs, host = instances(torch, settings)
    singles = [mg.solve_device(key, fixed, forces) for mg, key, fixed, forces in jobs]
    batched = solve_batch_device(jobs)
    levels = {rep["levels"] for _, rep in batched}
    assert len(levels) > 1, "the instances should have hierarchies of different depths"
    for (u1, r1), (u2, r2), (mg, _, _, forces) in zip(singles, batched, jobs):
        assert r2["converged"] and r2["batches"] <= 1
        assert r2["levels"] == r1["levels"]
        a, b = u1.cpu().numpy(), u2.cpu().numpy()
        for c in range(a.shape[0]):
            scale = max(np.linalg.norm(a[c]), 1e-300)
            assert np.linalg.norm(a[c] - b[c]) <= 1e-7 * scale
        assert r2["zero_rhs_columns"] == r1["zero_rhs_columns"]
        assert all(abs(i1 - i2) <= 1 for i1, i2 in zip(r1["iterations"], r2["iterations"])), (r1["iterations"], r2["iterations"])
        assert max(r2["relative_residual"]) < settings["tolerance"]
        mg.close()
    shape, k0, moduli, fixed, forces = host[0]
    expected = direct(shape, k0, moduli, fixed, forces)
    got = batched[0][0].cpu().numpy().T
    for c in range(forces.shape[1]):
        assert np.linalg.norm(got[:, c] - expected[:, c]) < 1e-6 * np.linalg.norm(expected[:, c])


def test_batch_zero_columns_and_single_instance(cuda):
    import torch
    from deep_frame_b200.topology_multigrid import GeometricMultigrid, solve_batch_device
    shape = (16, 8, 8)
    k0, _, moduli, fixed, force = cantilever(shape)
    mg = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "tolerance": 1e-10})
    mg.update(moduli)
    other = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "tolerance": 1e-10})
    other.update(moduli)
    zero = torch.zeros((2, force.size), dtype=torch.float64, device="cuda")
    live = torch.as_tensor(force[None, :].copy(), device="cuda")
    (u0, r0), (u1, r1) = solve_batch_device([(mg, "clamped", fixed, zero), (other, "clamped", fixed, live)])
    assert r0["zero_rhs_columns"] == 2 and r0["iterations"] == [0, 0] and float(u0.abs().max()) == 0.0
    expected = direct(shape, k0, moduli, fixed, force[:, None])[:, 0]
    assert np.linalg.norm(u1.cpu().numpy()[0] - expected) < 1e-6 * np.linalg.norm(expected)
    mg.close()
    other.close()


def test_batch_rejects_mixed_settings(cuda):
    import torch
    from deep_frame_b200.topology_multigrid import GeometricMultigrid, solve_batch_device
    shape = (12, 8, 4)
    k0, _, moduli, fixed, force = cantilever(shape)
    a = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "smoother": "chebyshev"})
    b = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "smoother": "jacobi"})
    c = GeometricMultigrid(shape, (1, 1, 1), k0, {"coarsest_dofs": 300, "cycle": "W"})
    for mg in (a, b, c):
        mg.update(moduli)
    f = torch.as_tensor(force[None, :].copy(), device="cuda")
    with pytest.raises(ValueError, match="share the V-cycle settings"):
        solve_batch_device([(a, "clamped", fixed, f), (b, "clamped", fixed, f)])
    with pytest.raises(ValueError, match="V-cycles"):
        solve_batch_device([(a, "clamped", fixed, f), (c, "clamped", fixed, f)])
    with pytest.raises(ValueError, match="its own GeometricMultigrid"):
        solve_batch_device([(a, "clamped", fixed, f), (a, "clamped", fixed, f)])
    for mg in (a, b, c):
        mg.close()
