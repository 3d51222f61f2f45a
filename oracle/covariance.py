"""Covariance load model measures (oracle, test only).

Restates deep_frame/topology_problem.py of the reference:
* ``InterfaceCovariance.__init__`` (:584-590): Sigma = D D^T with D = V sqrt(L)
  over the eigenvalues above 1e-10 * max;
* ``InterfaceCovariance.wrenches`` (:624-638): minimum-norm nodal forces
  f = B^T (B B^T)^-1 e_j carrying a unit wrench about the reference point;
* ``InterfaceCovariance.matrix`` (:639-646): F = sym(sum_parts factor * P^T U);
* ``InterfaceCovariance.measure`` (:657-684): tr F, lambda_max F, KS aggregate
  and their sensitivities -factor dE/drho sum u^T K0 u.
"""
import numpy as np

from .operator import element_energy


def directions(sigma):
    values, vectors = np.linalg.eigh((np.asarray(sigma) + np.asarray(sigma).T) / 2)
    values, vectors = values[::-1], vectors[:, ::-1]
    rank = int(np.sum(values > 1e-10 * values[0]))
    return vectors[:, :rank] * np.sqrt(values[:rank])


def unit_wrenches(points, reference):
    """[6, n, 3] nodal forces of the six unit wrenches over the nodes at ``points``."""
    arms = np.asarray(points, dtype=float) - np.asarray(reference, dtype=float)
    n = len(arms)
    b = np.zeros((6, 3 * n))
    for i, (x, y, z) in enumerate(arms):
        b[:3, 3 * i:3 * i + 3] = np.eye(3)
        b[3:, 3 * i:3 * i + 3] = [[0, -z, y], [z, 0, -x], [-y, x, 0]]
    nodal = b.T @ np.linalg.solve(b @ b.T, np.eye(6))
    return nodal.T.reshape(6, n, 3)


def flexibility(parts, factor):
    """parts: list of (forces [ndof, r], solutions [ndof, r]) for the +/- halves."""
    f = sum(factor * p.T @ u for p, u in parts)
    return (f + f.T) / 2


def measure(parts, factor, shape, k0, derivative, ks=50.0, limit_worst=None, cutoff=1e-9):
    """tr F, lambda_max F, KS and the two sensitivity fields (limits of 1)."""
    f = flexibility(parts, factor)
    mean = float(np.trace(f))
    values, vectors = np.linalg.eigh(f)
    values, vectors = values[::-1], vectors[:, ::-1]
    worst = float(values[0])
    scale = limit_worst or worst
    weights = np.exp(ks * (values - worst) / scale)
    ks_value = worst + scale * np.log(weights.sum()) / ks
    weights /= weights.sum()
    grad_mean = np.zeros(int(np.prod(shape)))
    for _, u in parts:
        grad_mean += -factor * derivative * element_energy(shape, k0, u).sum(axis=0)
    grad_worst = np.zeros_like(grad_mean)
    for i, w in enumerate(weights):
        if w > cutoff:
            for _, u in parts:
                grad_worst += w * (-factor * derivative * element_energy(shape, k0, u @ vectors[:, i]))
    return {"load_mean": mean, "load_worst": worst, "ks": float(ks_value), "grad_mean": grad_mean,
            "grad_worst": grad_worst, "eigenvalues": values, "weights": weights, "flexibility": f}
