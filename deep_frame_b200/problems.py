"""Seeded synthetic benchmark problems (unit voxels, E0 = 1).

* ``cantilever``: the plain-method cantilever: x = 0 face clamped, one unit -z
  point load at the bottom-edge centre of the free end, densities i.i.d.
  U[0.01, 1] (48 x 24 x 24 by default).
* ``plate``: the covariance-load plate half model: mirror symmetry on x = 0, a
  clamped central stack patch through the thickness, 7 interface patches
  (4 motor pads at the corners of the top face, stack, battery deck, camera
  face) x 6 unit wrench components = 42 load directions, Sigma = X^T X / 60
  with X ~ N(0, 1)^{60 x 42} (Wishart, 60 dof), densities from a Gaussian-
  smoothed (sigma = 3 voxels) normal field mapped through a sigmoid to
  [0.001, 1].  Patch boxes scale with the plate; at 96 x 96 x 16 the stack
  patch is x in [0, 4], y in [44, 52] (8 x 8 x 16 in the full model).
All inputs are synthetic; there is no dataset.
"""
import numpy as np

TOL = 1e-6


def box(lo, hi):
    return {"kind": "box", "min_mm": [float(v) for v in lo], "max_mm": [float(v) for v in hi]}


def material(young=1.0, poisson=0.3):
    return {"young_modulus_mpa": float(young), "poisson_ratio": float(poisson), "density_g_cm3": 1.0}


def cantilever(shape=(48, 24, 24), seed=0):
    ex, ey, ez = (int(s) for s in shape)
    allowed = np.ones((ex, ey, ez), dtype=bool)
    domain = {"grid": {"shape": [ex, ey, ez], "spacing_mm": [1.0, 1.0, 1.0], "origin_mm": [0.0, 0.0, 0.0], "order": "C", "axis_order": "xyz"},
              "allowed": allowed, "preserve": np.zeros_like(allowed), "forbidden": ~allowed, "material": material(),
              "load_cases": [{"name": "tip", "analysis": "static", "fixed_regions": [box([-TOL, -TOL, -TOL], [TOL, ey + TOL, ez + TOL])],
                              "loads": [{"region": box([ex - TOL, ey // 2 - TOL, -TOL], [ex + TOL, ey // 2 + TOL, TOL]),
                                         "force_n": [0.0, 0.0, -1.0]}]}]}
    density = np.random.default_rng(seed).uniform(0.01, 1.0, ex * ey * ez)
    return domain, density


def smooth_density(shape, seed, sigma=3.0):
    from scipy.ndimage import gaussian_filter
    field = gaussian_filter(np.random.default_rng(seed).standard_normal(shape), sigma)
    z = field / field.std()
    return (0.001 + 0.999 / (1.0 + np.exp(-z))).ravel()


def wishart_sigma(count=42, dof=60, seed=0):
    x = np.random.default_rng(seed + 1000).standard_normal((dof, count))
    return x.T @ x / dof


def plate(shape=(96, 96, 16), seed=0):
    """Half model x >= 0 of a (2 X) x Y x Z plate; returns (domain, density, covariance settings)."""
    ex, ey, ez = (int(s) for s in shape)
    s = max(ex / 96.0, 0.25)
    pad, stack_x, stack_y = 4 * s, 4 * s, 4 * s
    allowed = np.ones((ex, ey, ez), dtype=bool)
    half_y = ey / 2
    stack = box([-stack_x - TOL, half_y - stack_y - TOL, -TOL], [stack_x + TOL, half_y + stack_y + TOL, ez + TOL])
    top = [ez - TOL, ez + TOL]
    interfaces = {
        "motor_front_left": ([-ex, ey - pad], [-(ex - pad), ey], top, [-(ex - pad / 2), ey - pad / 2, ez]),
        "motor_front_right": ([ex - pad, ey - pad], [ex, ey], top, [ex - pad / 2, ey - pad / 2, ez]),
        "motor_rear_left": ([-ex, 0.0], [-(ex - pad), pad], top, [-(ex - pad / 2), pad / 2, ez]),
        "motor_rear_right": ([ex - pad, 0.0], [ex, pad], top, [ex - pad / 2, pad / 2, ez]),
        "stack": ([-stack_x, half_y - stack_y], [stack_x, half_y + stack_y], top, [0.0, half_y, ez]),
        "battery": ([-8 * s, 0.2 * ey], [8 * s, 0.4 * ey], top, [0.0, 0.3 * ey, ez]),
    }
    regions = {name: {"regions": [box([lo[0] - TOL, lo[1] - TOL, z[0]], [hi[0] + TOL, hi[1] + TOL, z[1]])], "reference_mm": ref}
               for name, (lo, hi, z, ref) in interfaces.items()}
    regions["camera"] = {"regions": [box([-6 * s - TOL, ey - TOL, 0.25 * ez - TOL], [6 * s + TOL, ey + TOL, 0.75 * ez + TOL])],
                         "reference_mm": [0.0, float(ey), 0.5 * ez]}
    names = ["motor_front_left", "motor_front_right", "motor_rear_left", "motor_rear_right", "stack", "battery", "camera"]
    labels = [[name, dof] for name in names for dof in ("Fx", "Fy", "Fz", "Mx", "My", "Mz")]
    domain = {"grid": {"shape": [ex, ey, ez], "spacing_mm": [1.0, 1.0, 1.0], "origin_mm": [0.0, 0.0, 0.0], "order": "C", "axis_order": "xyz"},
              "allowed": allowed, "preserve": np.zeros_like(allowed), "forbidden": ~allowed, "material": material(),
              "symmetry": {"axis": 0, "plane_mm": 0.0}, "interfaces": regions,
              "load_cases": [{"name": "stack", "analysis": "modal", "fixed_regions": [stack]}]}
    covariance = {"support": "stack", "sigma": wishart_sigma(len(labels), 60, seed), "labels": labels}
    return domain, smooth_density((ex, ey, ez), seed), covariance


CONFIGS = {
    "cantilever_48x24x24": {"kind": "cantilever", "shape": (48, 24, 24), "tolerance": 1e-10,
                            "multigrid": {"precision": "float64", "smoother": "jacobi", "sweeps": 2, "coarsest_dofs": 400, "tolerance": 1e-10}},
    "plate_96x96x16": {"kind": "plate", "shape": (96, 96, 16), "tolerance": 1e-8},
    "plate_128x128x24": {"kind": "plate", "shape": (128, 128, 24), "tolerance": 1e-8},
    "plate_192x192x32": {"kind": "plate", "shape": (192, 192, 32), "tolerance": 1e-8},
    "plate_352x352x48": {"kind": "plate", "shape": (352, 352, 48), "tolerance": 1e-8},
}
