"""Assembled hex8 stiffness, matrix-free apply and element energies (oracle, test only).

Restates the reference's
* ``HexElasticity.matrix`` (deep_frame/topology_optimization.py:638-650): COO
  assembly of E_e * K0 over active elements, symmetrised;
* ``GeometricMultigrid.operator`` (deep_frame/topology_multigrid.py:105-109):
  y = mask * sum_e E_e K0 (mask * u)_e;
* ``GeometricMultigrid.mask`` (:138-144): a dof is live when its node touches
  an element with E > 0 and it is not listed as fixed;
* ``GeometricMultigrid.element_energy`` (:458-459) / ``HexElasticity._collect``
  (deep_frame/topology_optimization.py:732): u_e^T K0 u_e per element.
"""
import numpy as np
from scipy.sparse import coo_matrix

from .hex8 import grid_numbering


def assemble(shape, k0, moduli):
    """Global stiffness K = sum_e E_e K0 scattered through the dof table (CSR, symmetrised)."""
    _, dofs = grid_numbering(shape)
    moduli = np.asarray(moduli, dtype=float).ravel()
    ndof = 3 * int(np.prod(np.asarray(shape) + 1))
    live = moduli != 0
    el = dofs[live]
    rows = np.repeat(el, 24, axis=1).ravel()
    cols = np.tile(el, (1, 24)).ravel()
    vals = (moduli[live, None] * np.asarray(k0).ravel()[None, :]).ravel()
    k = coo_matrix((vals, (rows, cols)), shape=(ndof, ndof)).tocsr()
    return ((k + k.T) * 0.5).tocsr()


def live_dofs(shape, moduli, fixed=()):
    """Boolean [ndof] of dofs that touch an element with E > 0 and are not fixed."""
    conn, _ = grid_numbering(shape)
    moduli = np.asarray(moduli, dtype=float).ravel()
    nnode = int(np.prod(np.asarray(shape) + 1))
    node_live = np.zeros(nnode, dtype=bool)
    node_live[np.unique(conn[moduli > 0])] = True
    live = np.repeat(node_live, 3)
    fixed = np.asarray(fixed, dtype=np.int64)
    if fixed.size:
        live[fixed] = False
    return live


def apply(shape, k0, moduli, u, mask=None):
    """Element-by-element y = mask * sum_e E_e K0 (mask * u)_e for u of shape [ndof] or [ndof, R]."""
    _, dofs = grid_numbering(shape)
    moduli = np.asarray(moduli, dtype=float).ravel()
    u = np.asarray(u, dtype=float)
    single = u.ndim == 1
    u = u[:, None] if single else u
    if mask is not None:
        u = u * np.asarray(mask, dtype=float)[:, None]
    ue = u[dofs]                                   # [nelem, 24, R]
    ye = np.einsum("ij,ejr->eir", k0, ue) * moduli[:, None, None]
    y = np.zeros_like(u)
    np.add.at(y, dofs.ravel(), ye.reshape(-1, u.shape[1]))
    if mask is not None:
        y = y * np.asarray(mask, dtype=float)[:, None]
    return y[:, 0] if single else y


def element_energy(shape, k0, u):
    """u_e^T K0 u_e for every element and column: returns [R, nelem] (or [nelem] for one column)."""
    _, dofs = grid_numbering(shape)
    u = np.asarray(u, dtype=float)
    single = u.ndim == 1
    u = u[:, None] if single else u
    ue = u[dofs]                                   # [nelem, 24, R]
    e = np.einsum("eir,ij,ejr->re", ue, k0, ue, optimize=True)
    return e[0] if single else e
