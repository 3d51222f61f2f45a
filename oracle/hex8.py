"""Hex8 element matrices and structured-grid numbering (oracle, test only).

Restates deep_frame/topology_optimization.py:246-319 of the reference:
``_CORNERS`` (:246-249), ``elasticity_matrix`` (:251-258),
``hexahedron_matrices`` (:269-299, 2x2x2 Gauss quadrature of a box element
with trilinear shape functions) and ``regular_grid`` (:301-319, C-order node
and element numbering, dof = 3 * node + component).
"""
import numpy as np

# corner order of the reference element: bottom face counter-clockwise, then top face
CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                    [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int64)


def isotropic_constitutive(nu):
    """6x6 isotropic elasticity matrix for unit Young's modulus (Voigt order xx yy zz xy yz xz)."""
    if not np.isfinite(nu) or not -1.0 < nu < 0.5:
        raise ValueError("Poisson ratio must be between -1 and 0.5")
    lam = nu / ((1 + nu) * (1 - 2 * nu))
    mu = 0.5 / (1 + nu)
    d = np.zeros((6, 6))
    d[:3, :3] = lam
    d[np.arange(3), np.arange(3)] = lam + 2 * mu
    d[np.arange(3, 6), np.arange(3, 6)] = mu
    return d


def element_matrices(spacing, nu, constitutive=None):
    """Return (K0, M0, B) of one box element with edge lengths ``spacing``.

    K0 = sum_g B_g^T D B_g |J|, M0 = sum_g N_g N_g^T (x) I3 |J| over the 8 Gauss
    points at +-1/sqrt(3); B has shape [8, 6, 24].
    """
    h = np.asarray(spacing, dtype=float)
    if h.shape != (3,) or np.any(h <= 0) or not np.all(np.isfinite(h)):
        raise ValueError("Hexahedron spacing must contain three finite positive lengths")
    d = isotropic_constitutive(nu) if constitutive is None else np.asarray(constitutive, dtype=float)
    sign = 2.0 * CORNERS - 1.0                      # [8, 3] natural coordinates of the corners
    jac = np.prod(h) / 8.0
    k0 = np.zeros((24, 24))
    m0 = np.zeros((24, 24))
    bs = []
    g = 1.0 / np.sqrt(3.0)
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                xi = np.array([2 * a - 1, 2 * b - 1, 2 * c - 1]) * g
                f = 1.0 + sign * xi                 # [8, 3] one-dimensional factors
                n = f.prod(axis=1) / 8.0
                grad = np.empty((8, 3))
                for ax in range(3):
                    others = [o for o in range(3) if o != ax]
                    grad[:, ax] = sign[:, ax] * f[:, others[0]] * f[:, others[1]] / (4.0 * h[ax])
                bmat = np.zeros((6, 24))
                for ax in range(3):
                    bmat[ax, ax::3] = grad[:, ax]
                # engineering shear strains: xy, yz, xz
                bmat[3, 0::3], bmat[3, 1::3] = grad[:, 1], grad[:, 0]
                bmat[4, 1::3], bmat[4, 2::3] = grad[:, 2], grad[:, 1]
                bmat[5, 0::3], bmat[5, 2::3] = grad[:, 2], grad[:, 0]
                k0 += bmat.T @ d @ bmat * jac
                m0 += np.kron(np.outer(n, n), np.eye(3)) * jac
                bs.append(bmat)
    return k0, m0, np.asarray(bs)


def grid_numbering(shape):
    """Element -> 24 dof table of a C-ordered structured grid with ``shape`` elements."""
    shape = tuple(int(s) for s in shape)
    nodes = tuple(s + 1 for s in shape)
    ex, ey, ez = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    starts = np.stack([ex.ravel(), ey.ravel(), ez.ravel()], axis=1)      # [nelem, 3]
    corner_nodes = starts[:, None, :] + CORNERS[None, :, :]              # [nelem, 8, 3]
    conn = np.ravel_multi_index(tuple(corner_nodes.transpose(2, 0, 1)), nodes)
    dofs = (3 * conn[:, :, None] + np.arange(3)[None, None, :]).reshape(-1, 24)
    return conn, dofs


def node_points(shape, spacing, origin=(0.0, 0.0, 0.0)):
    nodes = tuple(int(s) + 1 for s in shape)
    idx = np.indices(nodes).reshape(3, -1).T
    return idx * np.asarray(spacing, dtype=float) + np.asarray(origin, dtype=float)


def simp(density, p, eps, e0=1.0, active=None):
    """SIMP modulus and its derivative: E = E0 (eps + (1 - eps) rho^p) (reference :657-661)."""
    rho = np.asarray(density, dtype=float).ravel()
    moduli = e0 * (eps + (1 - eps) * rho ** p)
    deriv = e0 * (1 - eps) * p * rho ** (p - 1)
    if active is not None:
        moduli = np.where(active, moduli, 0.0)
        deriv = np.where(active, deriv, 0.0)
    return moduli, deriv
