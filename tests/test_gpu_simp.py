"""Device SIMP + MMA loop of the covariance problem vs the same loop on the CPU oracle.

The oracle loop uses direct sparse solves, the oracle cone filter and the oracle MMA
restatement; after a fixed number of iterations the device density must agree to
1e-4 max-abs (the target's bar for the final SIMP density), here checked per iteration.
"""
import numpy as np
import pytest
from scipy.sparse.linalg import spsolve

from oracle import covariance as ocov
from oracle import density as oden
from oracle import hex8, mma as omma, operator as op

pytestmark = pytest.mark.gpu


def oracle_loop(system, model, shape, iterations, vf, radius, p, eps, move):
    mapping = oden.DensityMapOracle(shape, (1, 1, 1), radius, np.ones(int(np.prod(shape)), dtype=bool))
    n = int(np.prod(shape))
    x = np.full(n, vf)
    xold1, xold2, low, upp = x.copy(), x.copy(), np.zeros(n), np.ones(n)
    index = {name: k for k, name in enumerate(model.cases)}
    scale0, out = None, []
    for it in range(1, iterations + 1):
        phys, pder = mapping.physical(x)
        moduli, dE = hex8.simp(phys, p, eps)
        matrix = op.assemble(shape, system.ke, moduli).tocsc()
        parts = []
        for members in system.groups.values():
            forces = np.zeros((system.ndof, model.rank))
            for case, part in members:
                forces[:, index[case["name"]]] = part["force"]
            live = op.live_dofs(shape, moduli, members[0][1]["fixed"])
            u = np.zeros_like(forces)
            u[live] = spsolve(matrix[live][:, live].tocsc(), forces[live])
            parts.append((forces, u))
        res = ocov.measure(parts, model.factor, shape, system.ke, dE)
        scale0 = res["load_mean"] if scale0 is None else scale0
        f0 = res["load_mean"] / scale0
        df0 = mapping.pullback(res["grad_mean"] / scale0, pder)
        g = phys.sum() / (vf * n) - 1
        dg = mapping.pullback(np.full(n, 1 / (vf * n)), pder)
        xn, *_rest, low, upp = omma.mmasub(1, n, it, x, np.zeros(n), np.ones(n), xold1, xold2, 100 * f0, 100 * df0, [100 * g],
                                            100 * dg[None, :], low, upp, 1.0, [0.0], [1e4], [1.0], move=move, asyinit=0.5,
                                            asydecr=0.7, asyincr=1.2, raa0=1e-5)
        xold2, xold1, x = xold1, x, np.clip(xn, 0, 1)
        out.append((x.copy(), res["load_mean"]))
    return out


def test_device_simp_loop_matches_oracle_loop(cuda):
    from deep_frame_b200 import problems
    from deep_frame_b200.optimize import CovarianceSimp
    shape = (16, 12, 4)
    domain, _, cov = problems.plate(shape, 2)
    simp = CovarianceSimp(domain, cov, volume_fraction=0.3, filter_radius=1.5, move=0.2,
                          multigrid={"tolerance": 1e-11, "coarsest_dofs": 300, "precision": "float64"})
    rows = []
    x, history = simp.run(4, callback=rows.append)
    expected = oracle_loop(simp.system, simp.model, shape, 4, 0.3, 1.5, 3.0, 1e-9, 0.2)
    xs = []
    simp2 = CovarianceSimp(domain, cov, volume_fraction=0.3, filter_radius=1.5, move=0.2,
                           multigrid={"tolerance": 1e-11, "coarsest_dofs": 300, "precision": "float64"})
    simp2.run(4, callback=lambda row: None)
    for it, (row, (xo, tr)) in enumerate(zip(history, expected)):
        assert row["tr"] == pytest.approx(tr, rel=1e-6), it
    assert np.max(np.abs(x.cpu().numpy() - expected[-1][0])) < 1e-4
    simp.close()
    simp2.close()


@pytest.mark.parametrize("warm", [True, 2])
def test_warm_started_simp_loop_matches_oracle_loop(cuda, warm):
    """warm_start=True reuses the previous design's displacements, warm_start=2 their energy-optimal
    combination for the new stiffness; the designs still follow the oracle."""
    from deep_frame_b200 import problems
    from deep_frame_b200.optimize import CovarianceSimp
    shape = (16, 12, 4)
    domain, _, cov = problems.plate(shape, 2)
    settings = {"tolerance": 1e-11, "coarsest_dofs": 300, "precision": "float64"}
    loop = CovarianceSimp(domain, cov, volume_fraction=0.3, filter_radius=1.5, move=0.2, multigrid=settings, warm_start=warm)
    cold = CovarianceSimp(domain, cov, volume_fraction=0.3, filter_radius=1.5, move=0.2, multigrid=settings)
    x, history = loop.run(4)
    _, cold_history = cold.run(4)
    expected = oracle_loop(loop.system, loop.model, shape, 4, 0.3, 1.5, 3.0, 1e-9, 0.2)
    for it, (row, (xo, tr)) in enumerate(zip(history, expected)):
        assert row["tr"] == pytest.approx(tr, rel=1e-6), it
    assert np.max(np.abs(x.cpu().numpy() - expected[-1][0])) < 1e-4
    assert sum(max(r["pcg_iterations"]) for r in history[1:]) <= sum(max(r["pcg_iterations"]) for r in cold_history[1:])
    loop.close()
    cold.close()


def test_simp_run_resumes_from_saved_mma_state(cuda, tmp_path):
    """Two iterations, the MMA state written to disk and read back, two more iterations = four in one run."""
    from deep_frame_b200 import problems, results
    from deep_frame_b200.optimize import CovarianceSimp
    shape = (16, 12, 4)
    domain, _, cov = problems.plate(shape, 2)
    settings = {"tolerance": 1e-11, "coarsest_dofs": 300, "precision": "float64"}
    straight = CovarianceSimp(domain, cov, volume_fraction=0.3, filter_radius=1.5, move=0.2, multigrid=settings)
    x4, history4 = straight.run(4)
    first = CovarianceSimp(domain, cov, volume_fraction=0.3, filter_radius=1.5, move=0.2, multigrid=settings)
    saved = []
    x2, _ = first.run(2, checkpoint=lambda x, state, history: results.save_mma_state(tmp_path / "mma.npz", x, state, history) or saved.append(1),
                      checkpoint_interval=2)
    assert saved == [1]
    design, state, history = results.load_mma_state(tmp_path / "mma.npz")
    second = CovarianceSimp(domain, cov, volume_fraction=0.3, filter_radius=1.5, move=0.2, multigrid=settings)
    x, resumed = second.run(2, x=design, state=state)
    assert [row["iteration"] for row in resumed] == [3, 4] and len(history) == 2
    assert np.max(np.abs(x.cpu().numpy() - x4.cpu().numpy())) < 1e-10
    assert resumed[-1]["tr"] == pytest.approx(history4[-1]["tr"], rel=1e-10)
    for loop in (straight, first, second):
        loop.close()
