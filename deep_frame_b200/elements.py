"""Hex8 element matrices and structured-grid numbering.

Same interface and conventions as the reference's
deep_frame/topology_optimization.py:246-331: ``_CORNERS`` (corner order),
``elasticity_matrix`` / ``orthotropic_matrix`` (6x6 constitutive matrices,
Voigt order xx yy zz xy yz xz with engineering shears), ``hexahedron_matrices``
(K0, M0 and the 8 Gauss-point strain matrices of a box element, 2x2x2
Gauss-Legendre), ``regular_grid`` (C-order nodes, dof = 3 * node + c) and
``select_nodes`` (box selectors with a 1e-7 tolerance).  These run once per
problem on the host; the per-iteration work is in libtfb200.so.
"""
import numpy as np

_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                     [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int32)


def elasticity_matrix(poisson_ratio):
    nu = float(poisson_ratio)
    if not np.isfinite(nu) or not -1 < nu < 0.5:
        raise ValueError("Poisson ratio must be between -1 and 0.5")
    scale = 1.0 / ((1 + nu) * (1 - 2 * nu))
    normal = np.full((3, 3), nu) + np.eye(3) * (1 - 2 * nu)
    shear = np.eye(3) * (0.5 - nu)
    return scale * np.block([[normal, np.zeros((3, 3))], [np.zeros((3, 3)), shear]])


def orthotropic_matrix(constants):
    """Stiffness of a transversely isotropic material (in-plane x-y, axis z) from its engineering
    constants: the inverse of the compliance with 1/E on the normal diagonal, -nu/E off it (nu_xz
    for every coupling with z, taken over E_xy) and 1/G on the shear diagonal (G_xy, G_z, G_z);
    rejected unless that compliance is positive definite (topology_optimization.py:260-267)."""
    e_in, e_z = constants["e_xy_mpa"], constants["e_z_mpa"]
    poisson = np.array([[0.0, constants["nu_xy"], constants["nu_xz"]],
                        [constants["nu_xy"], 0.0, constants["nu_xz"]],
                        [constants["nu_xz"], constants["nu_xz"], 0.0]])
    normal = np.diag([1.0 / e_in, 1.0 / e_in, 1.0 / e_z]) - poisson / e_in
    shear = np.diag(1.0 / np.array([constants["g_xy_mpa"], constants["g_z_mpa"], constants["g_z_mpa"]], dtype=float))
    compliance = np.block([[normal, np.zeros((3, 3))], [np.zeros((3, 3)), shear]])
    if np.linalg.eigvalsh(compliance).min() <= 0:
        raise ValueError("Orthotropic engineering constants are not positive definite")
    return np.linalg.inv(compliance)


def hexahedron_matrices(spacing_mm, poisson_ratio, constitutive=None):
    """Return (K0, M0, strain) of a box element; strain is [8, 6, 24] at the Gauss points."""
    h = np.asarray(spacing_mm, dtype=float)
    if h.shape != (3,) or np.any(h <= 0) or not np.all(np.isfinite(h)):
        raise ValueError("Hexahedron spacing must contain three finite positive lengths")
    d = elasticity_matrix(poisson_ratio) if constitutive is None else np.asarray(constitutive, dtype=float)
    xi = (2.0 * np.array(list(np.ndindex(2, 2, 2))) - 1.0) / np.sqrt(3.0)    # [8 gauss, 3]
    s = 2.0 * _CORNERS - 1.0                                                 # [8 corners, 3]
    lin = 1.0 + xi[:, None, :] * s[None, :, :]                               # [g, c, 3]
    shape = lin.prod(axis=2) / 8.0                                           # [g, c]
    grads = np.empty((8, 8, 3))
    for axis in range(3):
        others = lin[:, :, [o for o in range(3) if o != axis]].prod(axis=2)
        grads[:, :, axis] = s[None, :, axis] * others / (4.0 * h[axis])
    strain = np.zeros((8, 6, 8, 3))
    for axis in range(3):
        strain[:, axis, :, axis] = grads[:, :, axis]
    for row, (a, b) in zip((3, 4, 5), ((0, 1), (1, 2), (0, 2))):
        strain[:, row, :, a] = grads[:, :, b]
        strain[:, row, :, b] = grads[:, :, a]
    strain = strain.reshape(8, 6, 24)
    det = np.prod(h) / 8.0
    stiffness = np.einsum("gia,ij,gjb->ab", strain, d, strain) * det
    mass = np.kron(np.einsum("ga,gb->ab", shape, shape), np.eye(3)) * det
    return stiffness, mass, strain


def regular_grid(grid):
    shape = np.asarray(grid["shape"], dtype=int)
    spacing = np.asarray(grid["spacing_mm"], dtype=float)
    origin = np.asarray(grid["origin_mm"], dtype=float)
    if shape.shape != (3,) or np.any(shape < 1):
        raise ValueError("Grid shape must contain three positive integers")
    if spacing.shape != (3,) or np.any(spacing <= 0) or not np.all(np.isfinite(spacing)):
        raise ValueError("Grid spacing must contain three finite positive lengths")
    if origin.shape != (3,) or not np.all(np.isfinite(origin)):
        raise ValueError("Grid origin must contain three finite coordinates")
    if grid.get("order", "C") != "C" or grid.get("axis_order", "xyz") != "xyz":
        raise ValueError("Only C-order xyz grids are supported")
    nodes = shape + 1
    points = np.stack(np.meshgrid(*[np.arange(n) for n in nodes], indexing="ij"), axis=-1).reshape(-1, 3) * spacing + origin
    strides = np.array([nodes[1] * nodes[2], nodes[2], 1])
    base = (np.stack(np.meshgrid(*[np.arange(n) for n in shape], indexing="ij"), axis=-1).reshape(-1, 3) @ strides)
    connectivity = (base[:, None] + _CORNERS @ strides).astype(np.int32)
    dofs = (3 * connectivity[:, :, None] + np.arange(3)).reshape(-1, 24)
    return points, connectivity, dofs


def select_nodes(points, region):
    """Indices of the nodes inside an axis-aligned box region (bounds included, 1e-7 mm slack);
    an empty box raises "Empty topology node selector" (topology_optimization.py:321-331)."""
    if region.get("kind") != "box":
        raise ValueError("Topology node selectors must be boxes")
    bounds = np.array([region["min_mm"], region["max_mm"]], dtype=float)
    if bounds.shape != (2, 3) or not np.isfinite(bounds).all() or (bounds[0] > bounds[1]).any():
        raise ValueError("Invalid node-selection box")
    outside = np.maximum((bounds[0] - 1e-7) - points, points - (bounds[1] + 1e-7)).max(axis=1)
    inside = np.flatnonzero(outside <= 0)
    if inside.size == 0:
        raise ValueError(f"Empty topology node selector: {region}")
    return inside


def simp(density, penalization, min_stiffness_ratio, young=1.0, active=None):
    """E = E0 (eps + (1 - eps) rho^p) and dE/drho (topology_optimization.py:657-661)."""
    rho = np.asarray(density, dtype=float).ravel()
    moduli = young * (min_stiffness_ratio + (1 - min_stiffness_ratio) * rho ** penalization)
    derivative = young * (1 - min_stiffness_ratio) * penalization * rho ** (penalization - 1)
    if active is not None:
        moduli = np.where(active, moduli, 0.0)
        derivative = np.where(active, derivative, 0.0)
    return moduli, derivative
