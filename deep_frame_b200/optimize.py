"""SIMP + MMA loop of the covariance-load problem, device resident.

One iteration is the reference's ``MMAOptimizer.run`` body
(deep_frame/topology_optimizers.py:99-164) for the covariance objective:
``TopologyProblem.evaluate`` (deep_frame/topology_problem.py:366-379) with the
cone filter and a single projection (beta = 0: identity), the SIMP moduli, the
42-direction covariance solve of both mirror halves, tr(K^-1 Sigma) as the
objective (the ``load_mean`` row used as objective, topology_optimizers.py:48-54),
the volume row ``sum(rho) / (V* n) - 1`` (topology_problem.py:345-346), both
gradients pulled back through the filter, then one MMA step with the
reference's settings (f and g scaled by 100, a0 = 1, a = 0, c = 1e4, d = 1,
asyinit 0.5, asydecr 0.7, asyincr 1.2, raa0 1e-5).  Every field stays on the
device; the host sees scalars and the 42 x 42 flexibility matrix.

``warm_start=True`` starts every design iteration's PCG from the previous
iteration's displacements instead of zero (the reference always starts from
zero); ``warm_start=m`` (an int) starts it from the energy-optimal combination
of the last m iterations' displacements for the new stiffness: per column,
x0 = S c with S^T K S c = S^T f (m extra operator applies per column).  The
converged answer is the same to the solver tolerance; the iteration count
drops as the design settles.
"""
from time import perf_counter

import numpy as np

from . import _lib
from .covariance import InterfaceCovariance
from .density import DensityMap
from .elasticity import HexElasticity
from .mma import MMA

MMA_SETTINGS = {"scale": 100.0, "asyinit": 0.5, "asydecr": 0.7, "asyincr": 1.2, "raa0": 1e-5, "c": 1e4, "d": 1.0}


class CovarianceSimp:
    def __init__(self, domain, covariance, volume_fraction=0.15, filter_radius=1.5, penalization=3.0, min_stiffness_ratio=1e-9,
                 move=0.2, multigrid=None, device="cuda", objective_scale=None, warm_start=False):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.system = HexElasticity(domain, multigrid={**(multigrid or {}), "device": str(self.device)})
        self.model = InterfaceCovariance(self.system, covariance, domain["interfaces"])
        self.map = DensityMap(domain, {"filter_radius_mm": filter_radius, "projection_beta": 0.0, "projection_eta": 0.5,
                                       "projection": "single", "beta_schedule": None, "minimum_design_density": 1e-3}, self.device)
        self.p, self.eps, self.move = float(penalization), float(min_stiffness_ratio), float(move)
        self.volume_max = float(volume_fraction)
        self.allowed = torch.as_tensor(self.map.allowed.astype(np.uint8), device=self.device)
        self.n_allowed = int(self.map.allowed.sum())
        self.free = torch.as_tensor(np.flatnonzero(self.map.free), device=self.device)
        self.mma = MMA(1, len(self.free), self.device)
        self.objective_scale = objective_scale
        self.warm_start = int(warm_start) if not isinstance(warm_start, bool) else (1 if warm_start else 0)
        self.project_guess = not isinstance(warm_start, bool) and self.warm_start > 0
        self.previous = None
        self.basis = {}
        self.lib = _lib.load()
        n = self.system.nelem
        f64 = dict(dtype=torch.float64, device=self.device)
        self.moduli, self.dE = torch.empty(n, **f64), torch.empty(n, **f64)
        self.volume = torch.empty(1, **f64)
        self.dvol = torch.as_tensor(self.map.allowed / (self.volume_max * self.n_allowed), **f64)

    def start(self, value=None):
        x = self.torch.zeros(self.system.nelem, dtype=self.torch.float64, device=self.device)
        x[self.torch.as_tensor(self.map.allowed, device=self.device)] = self.volume_max if value is None else value
        x[self.torch.as_tensor(self.map.preserve, device=self.device)] = 1.0
        return x

    def evaluate(self, x):
        """f0, df0 [n], g, dg [n] for the design x (all device tensors except the scalars)."""
        filtered = self.map.filtered_device(x)
        physical, derivative = self.map.project_device(filtered, 0.5)
        mg = self.system._multigrid()
        status = self.lib.tf_simp(_lib.ptr(physical), physical.numel(), self.p, self.eps, self.system.young, _lib.ptr(self.allowed),
                                  _lib.ptr(self.moduli), _lib.ptr(self.dE), _lib.ptr(self.volume), _lib.stream_of(self.device))
        _lib.check(status, None, "tf_simp")
        mg.update_device(self.moduli)
        guesses = None
        if self.warm_start and self.project_guess and self.basis:
            guesses = {key: self._projected_guess(key, forces) for key, _, forces in self.model.groups() if key in self.basis}
        elif self.warm_start:
            guesses = self.previous
        solved = self.model.solve_all(guesses)
        if self.warm_start:
            self.previous = {key: u for key, _, _, u, _ in solved}
            for key, _, _, u, _ in solved:
                self.basis[key] = ([u.clone()] + self.basis.get(key, []))[:self.warm_start]
        rows = self.model.measure_from(solved, -self.dE, gradients=True, worst_gradient=False)
        tr = rows[0]["value"]
        if self.objective_scale is None:
            self.objective_scale = tr
        f0 = tr / self.objective_scale
        df0 = self.map.pullback_device(rows[0]["gradient"] / self.objective_scale, derivative)
        vol = float(self.volume.item()) / (self.volume_max * self.n_allowed)
        dg = self.map.pullback_device(self.dvol, derivative)
        iterations = [int(np.max(r[4]["iterations"])) for r in solved]
        return {"f0": f0, "df0": df0, "g": vol - 1.0, "dg": dg, "tr": tr, "lambda_max": rows[1]["value"], "volume": vol * self.volume_max,
                "pcg_iterations": iterations, "physical": physical}

    def _projected_guess(self, key, forces):
        """Per column: the combination S c of the kept displacements minimising the energy norm of the error
        for the current stiffness, S^T K S c = S^T f (K applied with the group's live-dof mask)."""
        torch = self.torch
        mg = self.system._multigrid()
        basis = torch.stack(self.basis[key])                       # [m, R, ndof]
        m, r, n = basis.shape
        fixed = self.system.groups[key][0][1]["fixed"]
        applied = mg.apply_device(basis.reshape(m * r, n).contiguous(), key, fixed).reshape(m, r, n)
        gram = torch.einsum("ird,jrd->rij", basis, applied)
        rhs = torch.einsum("ird,rd->ri", basis, forces)
        gram = (gram + gram.transpose(1, 2)) / 2
        ridge = 1e-14 * torch.diagonal(gram, dim1=1, dim2=2).amax(dim=1).clamp_min(1e-300)
        gram = gram + ridge[:, None, None] * torch.eye(m, dtype=gram.dtype, device=gram.device)
        coefficients = torch.linalg.solve(gram, rhs[..., None])[..., 0]      # [R, m]
        return torch.einsum("ri,ird->rd", coefficients, basis).contiguous()

    def run(self, iterations, x=None, callback=None, state=None, checkpoint=None, checkpoint_interval=1):
        """Run ``iterations`` SIMP + MMA iterations from the design ``x`` (default: uniform volume fraction).

        ``state`` resumes an earlier run: the MMA iteration counter, previous iterates and asymptotes
        over the free cells (``old1``, ``old2``, ``low``, ``upp``, as ``results.save_mma_state`` keeps
        them) and the objective normalisation; the resumed run then takes the same steps as an
        uninterrupted one.  ``checkpoint(x, state, history)`` is called every ``checkpoint_interval``
        iterations with the state needed to resume.  The final state is kept in ``self.state``."""
        torch = self.torch
        x = self.start() if x is None else torch.as_tensor(x, dtype=torch.float64, device=self.device).clone()
        free = self.free
        xf = x[free].contiguous()
        dev = lambda v: torch.as_tensor(v, dtype=torch.float64, device=self.device).reshape(-1).clone()
        if state is None:
            first = 1
            xold1, xold2 = xf.clone(), xf.clone()
            low, upp = torch.zeros_like(xf), torch.ones_like(xf)
        else:
            first = int(state["iteration"])
            xold1, xold2, low, upp = (dev(state[key]) for key in ("old1", "old2", "low", "upp"))
            if state.get("objective_scale") is not None:
                self.objective_scale = float(state["objective_scale"])
        zeros, ones = torch.zeros_like(xf), torch.ones_like(xf)
        s = MMA_SETTINGS
        history = []
        for it in range(first, first + iterations):
            t0 = perf_counter()
            res = self.evaluate(x)
            df0 = (s["scale"] * res["df0"][free]).contiguous()
            dg = (s["scale"] * res["dg"][free]).reshape(1, -1).contiguous()
            xnew, y, z, lam = self.mma.step(it, xf, zeros, ones, xold1, xold2, df0, [s["scale"] * res["g"]], dg, low, upp, 1.0,
                                            [0.0], [s["c"]], [s["d"]], move=self.move, asyinit=s["asyinit"], asydecr=s["asydecr"],
                                            asyincr=s["asyincr"], raa0=s["raa0"])
            xnew = xnew.clamp_(0.0, 1.0)
            change = float((xnew - xf).abs().max())
            xold2, xold1, xf = xold1, xf, xnew
            x[free] = xf
            torch.cuda.synchronize(self.device)
            row = {"iteration": it, "f0": res["f0"], "tr": res["tr"], "lambda_max": res["lambda_max"], "volume": res["volume"],
                   "g": res["g"], "change": change, "pcg_iterations": res["pcg_iterations"], "newton": self.mma.newton_iterations,
                   "seconds": perf_counter() - t0}
            history.append(row)
            self.state = {"iteration": it + 1, "old1": xold1, "old2": xold2, "low": low, "upp": upp, "objective_scale": self.objective_scale}
            if callback:
                callback(row)
            if checkpoint and len(history) % checkpoint_interval == 0:
                checkpoint(x, self.state, history)
        return x, history

    def close(self):
        self.mma.close()
        self.map.close()
        return self.system.close()
