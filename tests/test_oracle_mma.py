"""The MMA oracle (oracle/mma.py) checked without mmapy.  No GPU.

mmapy, the package the reference calls, is not available, so its numbers cannot pin this
restatement.  What can be checked independently:
* the primal-dual interior-point subsolver returns the minimiser of the convex MMA subproblem it
  is given: SciPy's trust-region constrained solver, a different algorithm, solves the same subproblem (same asymptotes,
  move limits and approximation coefficients) to the same point;
* the step keeps the published rules: the first two iterations place the asymptotes at
  asyinit x (xmax - xmin) from x, later ones widen or narrow them by asyincr / asydecr as the
  last two steps agree or oscillate, and the new design stays within the move limit and the
  box [xmin, xmax];
* the parameters of the reference's call (a0 = 1, a = 0, c = 1e4, d = 1, move 0.2) give a
  feasible decrease on a small compliance-like problem.
"""
import numpy as np
import pytest
from scipy.optimize import Bounds, NonlinearConstraint, minimize

from oracle import mma


def subproblem(seed, n, m):
    rng = np.random.default_rng(seed)
    s = dict(mma.DEFAULTS, move=0.2)
    x = rng.uniform(0.2, 0.8, n)
    xmin, xmax = np.zeros(n), np.ones(n)
    low, upp = mma.asymptotes(1, x, xmin, xmax, x, x, None, None, s)
    df0dx = rng.normal(size=n)
    dfdx = rng.normal(size=(m, n))
    fval = rng.normal(scale=0.1, size=m)
    alfa, beta, p0, q0, P, Q, b = mma.approximation(x, xmin, xmax, low, upp, df0dx, fval, dfdx, s)
    a0, a, c, d = 1.0, np.zeros(m), np.full(m, 1e4), np.ones(m)
    return s, x, low, upp, alfa, beta, p0, q0, P, Q, b, a0, a, c, d


@pytest.mark.parametrize("seed,n,m", [(0, 12, 1), (1, 20, 2), (2, 30, 3), (3, 8, 1)])
def test_subsolver_matches_an_independent_solver(seed, n, m):
    s, x0, low, upp, alfa, beta, p0, q0, P, Q, b, a0, a, c, d = subproblem(seed, n, m)
    x, y, z, lam, *_ = mma.subsolve(m, n, s["epsimin"], low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d)

    def split(v):
        return v[:n], v[n:n + m], v[n + m]

    def objective(v):
        xx, yy, zz = split(v)
        f = np.sum(p0 / (upp - xx) + q0 / (xx - low)) + a0 * zz + np.sum(c * yy + 0.5 * d * yy ** 2)
        g = np.concatenate([p0 / (upp - xx) ** 2 - q0 / (xx - low) ** 2, c + d * yy, [a0]])
        return f, g

    def constraint(v):          # b_i - (f_i(x) - a_i z - y_i) >= 0
        xx, yy, zz = split(v)
        return b - (P @ (1.0 / (upp - xx)) + Q @ (1.0 / (xx - low)) - a * zz - yy)

    def constraint_jac(v):
        xx, _, _ = split(v)
        jx = -(P / (upp - xx)[None, :] ** 2 - Q / (xx - low)[None, :] ** 2)
        return np.hstack([jx, np.eye(m), a[:, None]])

    start = np.concatenate([0.5 * (alfa + beta), np.ones(m), [1.0]])
    bounds = Bounds(np.concatenate([alfa, np.zeros(m + 1)]), np.concatenate([beta, np.full(m + 1, np.inf)]))
    ref = minimize(objective, start, jac=True, method="trust-constr", bounds=bounds,
                   constraints=[NonlinearConstraint(constraint, 0.0, np.inf, jac=constraint_jac)],
                   options={"gtol": 1e-11, "xtol": 1e-13, "barrier_tol": 1e-11, "maxiter": 5000})
    assert ref.status in (1, 2), ref.message
    xr, yr, zr = split(ref.x)
    # the interior-point iterate stops at barrier parameter epsimin = 1e-7: a variable at a move
    # limit sits about epsimin / (its bound multiplier) inside it, up to ~4e-5 here
    assert np.max(np.abs(x - xr)) < 1e-4
    assert np.max(np.abs(y - yr)) < 1e-5 and abs(z - zr) < 1e-5
    assert abs(objective(np.concatenate([x, y, [z]]))[0] - ref.fun) <= 1e-6 * max(1.0, abs(ref.fun))
    assert np.all(constraint(np.concatenate([x, y, [z]])) > -1e-6)


def test_asymptote_rules():
    s = dict(mma.DEFAULTS)
    n = 6
    xmin, xmax = np.zeros(n), np.full(n, 2.0)
    x = np.linspace(0.5, 1.5, n)
    low, upp = mma.asymptotes(2, x, xmin, xmax, x, x, None, None, s)
    assert np.allclose(low, x - 0.5 * 2.0) and np.allclose(upp, x + 0.5 * 2.0)
    xold1 = x - np.array([0.1, -0.1, 0.1, -0.1, 0.0, 0.1])
    xold2 = xold1 - np.array([0.1, 0.1, -0.1, -0.1, 0.1, 0.0])   # agree, oscillate, oscillate, agree, flat, flat
    low1, upp1 = x - 0.3, x + 0.4
    low2, upp2 = mma.asymptotes(3, x, xmin, xmax, xold1, xold2, low1, upp1, s)
    factor = np.array([s["asyincr"], s["asydecr"], s["asydecr"], s["asyincr"], 1.0, 1.0])
    assert np.allclose(low2, x - factor * (xold1 - low1))
    assert np.allclose(upp2, x + factor * (upp1 - xold1))
    # clamped to [asymin, asymax] x span away from x
    low3, upp3 = mma.asymptotes(3, x, xmin, xmax, x - 1e-9, x - 2e-9, x - 1e-6, x + 1e-6, s)
    assert np.allclose(x - low3, s["asymin"] * 2.0) and np.allclose(upp3 - x, s["asymin"] * 2.0)


def test_step_respects_move_limit_box_and_decreases_a_compliance_problem():
    # min sum(w / x) subject to mean(x) <= 0.4 on [0.001, 1]: convex, optimum x ~ sqrt(w)
    rng = np.random.default_rng(5)
    n, m = 40, 1
    w = rng.uniform(0.5, 2.0, n)
    x = np.full(n, 0.4)
    xmin, xmax = np.full(n, 1e-3), np.ones(n)
    xold1, xold2, low, upp = x.copy(), x.copy(), xmin.copy(), xmax.copy()
    history = []
    for it in range(1, 31):
        f0 = np.sum(w / x)
        df0 = -w / x ** 2
        g = np.array([x.mean() - 0.4])
        dg = np.full((1, n), 1.0 / n)
        history.append((f0, g[0]))
        xn, y, z, lam, low, upp = mma.mmasub(m, n, it, x, xmin, xmax, xold1, xold2, 100 * f0, 100 * df0, 100 * g, 100 * dg,
                                            low, upp, 1.0, np.zeros(m), np.full(m, 1e4), np.ones(m), move=0.2)
        assert np.all(xn >= xmin - 1e-12) and np.all(xn <= xmax + 1e-12)
        assert np.all(np.abs(xn - x) <= 0.2 * (xmax - xmin) + 1e-12)
        xold2, xold1, x = xold1, x, xn
    best = np.sqrt(w) * 0.4 * n / np.sqrt(w).sum()
    assert abs(x.mean() - 0.4) < 1e-4
    assert np.sum(w / x) <= np.sum(w / best) * (1 + 1e-4)
    assert history[-1][0] < history[0][0]
