"""RHS-column sharding of the covariance measure across ranks.

The 42 load directions of every fixture group are independent solves, so each
rank solves its slice (columns ``rank::world``) with no communication inside
PCG.  One exchange per measure then assembles what the reference's
``InterfaceCovariance.measure`` (deep_frame/topology_problem.py:657-684)
computes on one device:
* the flexibility F = sum_parts factor P^T U: every rank fills its own columns
  of F (P of all directions against its U) and one all-reduce (sum) completes it;
* the tr(K^-1 Sigma) sensitivity: per-rank partial energy sums, one all-reduce;
* the lambda_max / KS sensitivity: for every KS-weighted eigenvector v_i the
  rank forms its partial U_local v_i, one all-reduce of those dof vectors, then
  every rank evaluates the energies of the complete vectors.
F's eigen-decomposition is computed identically on every rank.  The solver,
the P^T U product and the energy kernel are passed in (``ops``), so the same
exchange runs on NCCL with the device kernels and on gloo with CPU test
doubles.  Every rank takes the same collective steps in the same order.
"""
import numpy as np

from .covariance import Spectrum


class ShardedMeasure:
    def __init__(self, groups, rank_count, factor, ops, group=None, ks=50.0, ks_cutoff=1e-9):
        """groups: [(key, ks [m] direction indices, forces [m, ndof] tensor)] of all directions."""
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.rank_count, self.factor, self.ops = int(rank_count), float(factor), ops
        self.ks, self.ks_cutoff = float(ks), float(ks_cutoff)
        self.groups = []
        for key, ks_all, forces in groups:
            local = np.arange(len(ks_all))[self.rank::self.world]
            self.groups.append({"key": key, "ks": np.asarray(ks_all), "forces": forces, "local": local,
                                "local_ks": np.asarray(ks_all)[local], "local_forces": forces[local]})

    def _all_reduce(self, tensor):
        if self.world > 1:
            self.dist.all_reduce(tensor, group=self.group)
        return tensor

    def measure(self, scale):
        """scale: per-element -dE/drho (tensor).  Returns (rows, flexibility)."""
        import torch
        device = scale.device
        flex = torch.zeros((self.rank_count, self.rank_count), dtype=torch.float64, device=device)
        solved = []
        for g in self.groups:
            u = self.ops.solve(g["key"], g["local_forces"]) if len(g["local"]) else None
            solved.append(u)
            if u is not None:
                block = self.ops.gram(g["forces"], u)            # [m_all, m_local] = P_all U_local^T
                idx = torch.as_tensor(g["ks"], device=device)
                loc = torch.as_tensor(g["local_ks"], device=device)
                flex[idx[:, None], loc[None, :]] += self.factor * block
        self._all_reduce(flex)
        spectrum = Spectrum(flex.cpu().numpy(), self.ks)
        nelem = scale.numel()
        grad_mean = torch.zeros(nelem, dtype=torch.float64, device=device)
        for g, u in zip(self.groups, solved):
            if u is not None:
                grad_mean += self.ops.energy(u, np.full(len(g["local"]), self.factor), scale)
        self._all_reduce(grad_mean)
        kept = spectrum.kept(self.ks_cutoff)
        coefficients = spectrum.weights[kept] * self.factor
        grad_worst = torch.zeros(nelem, dtype=torch.float64, device=device)
        for g, u in zip(self.groups, solved):
            # this rank's partial combinations U_local v_i, completed by one all-reduce of [kept, ndof]
            mixing = spectrum.vectors[np.ix_(g["local_ks"], kept)]
            partial = (self.ops.combine(u, mixing) if u is not None else
                       torch.zeros((len(kept), g["forces"].shape[1]), dtype=torch.float64, device=device))
            self._all_reduce(partial)
            grad_worst += self.ops.energy(partial, coefficients, scale)
        rows = [{"name": "load_mean", "value": spectrum.trace, "gradient": grad_mean},
                {"name": "load_worst", "value": spectrum.top, "gradient": grad_worst,
                 "info": {"ks_n_mm": spectrum.ks, "eigenvalues_n_mm": spectrum.values[:6].tolist()}}]
        return rows, spectrum.matrix


class DeviceOps:
    """The device kernels behind ShardedMeasure: GMG-PCG solve, tf_gram, tf_element_energy."""

    def __init__(self, system):
        self.system = system

    def solve(self, key, forces):
        return self.system.solve_group_device(key, forces.contiguous())[0]

    def gram(self, p_all, u_local):
        import torch
        from . import _lib
        lib = _lib.load()
        mg = self.system._multigrid()
        m, k = p_all.shape[0], u_local.shape[0]
        out = torch.empty((m, k), dtype=torch.float64, device=u_local.device)
        scratch = torch.empty(int(lib.tf_gram_scratch_size(m, k)), dtype=torch.float64, device=u_local.device)
        _lib.check(lib.tf_gram(_lib.ptr(p_all), m, _lib.ptr(u_local), k, u_local.shape[1], _lib.ptr(out), _lib.ptr(scratch),
                               mg._stream()), None, "tf_gram")
        return out

    def energy(self, columns, coefficients, scale):
        return self.system._multigrid().energy_device(columns, coefficients=coefficients, scale=scale)

    def combine(self, columns, mixing):
        """[k, ndof] = mixing^T columns, on the device (tf_combine)."""
        return self.system._multigrid().combine_device(columns, mixing)
