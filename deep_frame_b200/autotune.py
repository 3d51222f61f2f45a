"""Measured choice of the V-cycle smoother for a given problem.

The smoother schedule (Chebyshev degree, growth of the sweep count per level,
or damped Jacobi), the cycle (V or W), the depth of the hierarchy and the
finest-level apply (its node-tile height; FP32 CUDA cores or TF32 tensor cores)
change the cost of a V-cycle and the number of PCG iterations, never
the converged answer: every candidate solves to the same
recomputed true relative residual.  ``tune_smoother`` times one full solve of
every fixture group per candidate on the device and returns the fastest.
"""
from time import perf_counter

CANDIDATES = (
    {"smoother": "chebyshev", "chebyshev_degree": 3, "growth": 2.0},   # the reference's MULTIGRID default
    {"smoother": "chebyshev", "chebyshev_degree": 2, "growth": 2.0},
    {"smoother": "chebyshev", "chebyshev_degree": 2, "growth": 1.5},
    {"smoother": "chebyshev", "chebyshev_degree": 3, "growth": 1.0},
    {"smoother": "jacobi", "sweeps": 2, "growth": 2.0},
    # lighter smoothing on the Galerkin levels (fewer sweeps per cycle, possibly more PCG iterations)
    {"smoother": "chebyshev", "chebyshev_degree": 2, "growth": 1.0},
    {"smoother": "chebyshev", "chebyshev_degree": 2, "growth": 1.25},
    {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0},
    {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 1.5},
    {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 3.0},
    # one more level (a coarsest grid of a few hundred dofs: cheaper dense factor, longer V-cycle)
    {"smoother": "chebyshev", "chebyshev_degree": 2, "growth": 1.5, "coarsest_dofs": 1200},
    {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0, "coarsest_dofs": 1200},
    # W-cycles: two coarse corrections per level (more Galerkin-level work, fewer PCG iterations)
    {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0, "cycle": "W"},
    {"smoother": "chebyshev", "chebyshev_degree": 2, "growth": 1.0, "cycle": "W"},
    # the finest operator's node tiles 9 high (fewer padded threads on some grids, register spills)
    {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0, "fine_tz": 9},
    # the finest-level V-cycle apply on the tensor cores (TF32 operands)
    {"smoother": "chebyshev", "chebyshev_degree": 2, "growth": 1.5, "tensor_cores": True},
)


def tune_smoother(system, groups, moduli, base=None, candidates=CANDIDATES, repeats=2):
    """groups: [(key, forces [R, ndof] CUDA tensor)]; moduli: CUDA float64 tensor.

    Times every candidate on its own multigrid handle, closing each one before the next is built
    (on the largest grids two handles do not fit in device memory together), and installs the
    fastest converged settings in ``system`` (its handle is rebuilt on next use).  Returns
    (settings, timings)."""
    import torch
    from .topology_multigrid import GeometricMultigrid
    base = dict(base or system.multigrid_settings or {})
    if system.multigrid is not None:
        system.multigrid.close()
        system.multigrid = None
    timings = []
    best = None
    for cand in candidates:
        settings = {**base, **cand}
        mg = GeometricMultigrid(system.shape, system.spacing, system.ke, settings, system.me)
        seconds, iterations, ok = None, [], True
        try:
            for rep in range(repeats + 1):
                torch.cuda.synchronize()
                t0 = perf_counter()
                mg.update_device(moduli)
                its = []
                for key, forces in groups:
                    part = system.groups[key][0][1]
                    _, report = mg.solve_device(key, part["fixed"], forces)
                    ok &= report["converged"]
                    its.append(max(report["iterations"]))
                torch.cuda.synchronize()
                if rep:   # the first pass builds buffers
                    dt = perf_counter() - t0
                    seconds = dt if seconds is None else min(seconds, dt)
                    iterations = its
        finally:
            mg.close()
        timings.append({"settings": cand, "seconds": seconds, "iterations": iterations, "converged": bool(ok)})
        if ok and (best is None or seconds < best[0]):
            best = (seconds, settings)
    if best is None:
        raise RuntimeError("no smoother candidate converged")
    system.multigrid_settings = best[1]
    return best[1], timings
