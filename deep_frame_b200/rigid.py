"""Rigid-body algebra shared by the interface wrenches and the inertia-relief balance.

Both problems are about the map T_i = [I, -[r_i]x] that takes a rigid motion q = (a, w)
(translation and rotation, or linear and angular acceleration) to the motion of a point at arm
r_i, a + w x r_i, and about its transpose, which takes a point force f_i to the wrench
(f_i, r_i x f_i) it exerts.  The 6 x 6 Gram matrix G = sum_i m_i T_i^T T_i of a weighted point set
needs only the set's zeroth, first and second moments:

    G = [[M I,     -[s]x            ],
         [[s]x,    tr(S) I - S      ]]    with M = sum m_i, s = sum m_i r_i, S = sum m_i r_i r_i^T.

* Unit wrenches (deep_frame/topology_problem.py:624-638): the least-norm nodal forces that carry
  the wrench e_j are f_i = T_i (G^-1 e_j) with unit weights, a rigid-motion field evaluated at the
  nodes; no 6 x 3n matrix is formed.
* Inertia relief (deep_frame/topology_optimization.py:539-569): the rigid acceleration q that
  balances applied forces on point masses solves (G + diag(0, J_bodies)) q = sum_i T_i^T F_i with
  arms taken from the mass centre, and the d'Alembert force of mass i is -m_i T_i q.
"""
import numpy as np


def skew(v):
    """[v]x, the matrix with [v]x w = v x w."""
    x, y, z = np.asarray(v, dtype=float)
    return np.array([[0.0, -z, y], [z, 0.0, -x], [-y, x, 0.0]])


def rigid_gram(arms, weights=None):
    """G = sum_i w_i T_i^T T_i for points at ``arms`` [n, 3] (unit weights when ``weights`` is None)."""
    arms = np.asarray(arms, dtype=float)
    w = np.ones(len(arms)) if weights is None else np.asarray(weights, dtype=float)
    first = w @ arms
    second = (arms * w[:, None]).T @ arms
    gram = np.empty((6, 6))
    gram[:3, :3] = w.sum() * np.eye(3)
    gram[:3, 3:] = -skew(first)
    gram[3:, :3] = skew(first)
    gram[3:, 3:] = np.trace(second) * np.eye(3) - second
    return gram


def point_motion(q, arms):
    """Motion a + w x r_i of every point for the rigid motions in the columns of ``q`` [6, k]:
    returns [k, n, 3]."""
    q = np.asarray(q, dtype=float).reshape(6, -1)
    return q[:3].T[:, None, :] + np.cross(q[3:].T[:, None, :], np.asarray(arms, dtype=float)[None, :, :])


def resultant(forces, arms):
    """Wrench (sum f_i, sum r_i x f_i) of point forces [n, 3] at ``arms`` [n, 3]."""
    forces = np.asarray(forces, dtype=float)
    return np.concatenate([forces.sum(axis=0), np.cross(arms, forces).sum(axis=0)])


def unit_wrench_forces(arms):
    """[6, n, 3]: for each unit wrench e_j (Fx, Fy, Fz, Mx, My, Mz about the arms' origin) the nodal
    forces of least 2-norm whose resultant is e_j."""
    return point_motion(np.linalg.inv(rigid_gram(arms)), arms)


def balance(positions, masses, applied, body_inertia=None):
    """Rigid acceleration that balances ``applied`` [n, 3] on point ``masses`` [n] at ``positions``.

    Returns (total mass, mass centre, inertia tensor about it (bodies' own tensors added), linear
    acceleration of the centre, angular acceleration, d'Alembert force of every point [n, 3])."""
    masses = np.asarray(masses, dtype=float)
    total = float(masses.sum())
    centre = (masses / total) @ positions
    arms = positions - centre
    gram = rigid_gram(arms, masses)
    if body_inertia is not None:
        gram[3:, 3:] += body_inertia
    q = np.linalg.solve(gram, resultant(applied, arms))
    inertial = -masses[:, None] * point_motion(q, arms)[0]
    return total, centre, gram[3:, 3:].copy(), q[:3], q[3:], inertial
