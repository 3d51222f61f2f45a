"""Covariance load model on the device: 42-direction RHS, tr(K^-1 Sigma), lambda_max, KS.

Host-side mirror of the reference's ``InterfaceCovariance``
(deep_frame/topology_problem.py:572-684):
* Sigma = D D^T from its eigenpairs, rank = eigenvalues above 1e-10 * max (:584-590);
* unit-wrench minimum-norm nodal forces f = B^T (B B^T)^-1 e_j per interface,
  mirrored on half models (:624-638);
* one static case per direction, RHS_k = sum_j D_jk f_j, registered on the
  support case and split into +/- parts by ``HexElasticity`` (:599-611);
* ``measure``: F = sym(sum_parts factor P^T U), tr F, lambda_max and the KS
  aggregate, and the sensitivities of tr and of the KS-weighted eigenvalues
  (:657-684).
Solves, F = P^T U, and the sensitivity sums run on the GPU (libtfb200.so);
only the rank x rank eigen-decomposition of F runs on the host.
"""
import ctypes

import numpy as np

from . import _lib

DOFS = ["Fx", "Fy", "Fz", "Mx", "My", "Mz"]
SETTINGS = {"prefix": "sigma_", "ks": 50.0, "ks_cutoff": 1e-9, "limits": {"mean_n_mm": None, "worst_n_mm": None}}


class InterfaceCovariance:
    def __init__(self, system, settings, interfaces):
        self.system = system
        self.settings = {**SETTINGS, **settings}
        sigma = np.asarray(self.settings["sigma"], dtype=float)
        labels = [tuple(label) for label in self.settings["labels"]]
        missing = sorted({name for name, _ in labels} - set(interfaces))
        if missing:
            raise ValueError("Covariance interfaces missing from the domain: " + ", ".join(missing))
        values, vectors = np.linalg.eigh((sigma + sigma.T) / 2)
        values, vectors = values[::-1], vectors[:, ::-1]
        if values[-1] < -1e-9 * values[0]:
            raise ValueError("Load covariance is not positive semidefinite")
        self.sigma, self.labels = sigma, labels
        self.rank = int(np.sum(values > 1e-10 * values[0]))
        self.directions = vectors[:, :self.rank] * np.sqrt(values[:self.rank])
        self.factor = 1.0 if system.symmetry is None else 2.0
        units = {name: self.wrenches(interfaces[name]) for name in dict.fromkeys(name for name, _ in labels)}
        columns = [units[name][DOFS.index(dof)] for name, dof in labels]
        self.cases, self.forces = [], []
        for k in range(self.rank):
            force, mirrored = np.zeros(system.ndof), np.zeros(system.ndof)
            for weight, (direct, direct_values, mirror, mirror_values) in zip(self.directions[:, k], columns):
                np.add.at(force, direct, weight * direct_values)
                np.add.at(mirrored, mirror, weight * mirror_values)
            case = system.add_case(self.settings["prefix"] + str(k), self.settings["support"], force, mirrored)
            self.cases.append(case["name"])
            self.forces.append({part["sign"]: part["force"] for part in case["parts"]})
        self._groups = None

    def wrenches(self, interface):
        """Per unit wrench component (Fx, Fy, Fz, Mx, My, Mz about the interface's reference point):
        (direct dofs, direct values, mirror dofs, mirror values) of the least-norm nodal forces over the
        interface nodes that carry exactly that wrench, f = B^T (B B^T)^-1 e_j with B_i = [I; [r_i]x]
        (topology_problem.py:624-638).  Mirror-side nodes enter with their reflected positions and get
        their forces reflected back."""
        system = self.system
        sides = [system._select_both(region, "covariance", "load") for region in interface["regions"]]
        direct = np.unique(np.concatenate([here for here, _ in sides]))
        mirror = np.unique(np.concatenate([there for _, there in sides]))
        reflect = np.ones(3) if system.symmetry is None else system._flip()
        r = np.vstack([system.points[direct], system.points[mirror] * reflect]) - np.asarray(interface["reference_mm"], dtype=float)
        if np.linalg.matrix_rank(r - r[0], tol=1e-8) < 2:
            raise ValueError("An interface wrench needs at least three non-collinear nodes")
        count = len(r)
        # B as [6, node, 3]: a force f_i at r_i contributes f_i to the resultant and r_i x f_i to the moment
        b = np.zeros((6, count, 3))
        b[0, :, 0] = b[1, :, 1] = b[2, :, 2] = 1.0
        x, y, z = r.T
        b[3, :, 1], b[3, :, 2] = -z, y
        b[4, :, 0], b[4, :, 2] = z, -x
        b[5, :, 0], b[5, :, 1] = -y, x
        flat = b.reshape(6, 3 * count)
        nodal = np.linalg.solve(flat @ flat.T, flat).reshape(6, count, 3)            # row j: the forces for e_j
        dof = lambda nodes: (3 * nodes[:, None] + np.arange(3)).ravel()
        k = len(direct)
        return [(dof(direct), nodal[j, :k].ravel(), dof(mirror), (nodal[j, k:] * reflect).ravel()) for j in range(6)]

    def _worst_wrench(self, vector):
        """The six interface wrench components of largest magnitude in Sigma^1/2's image of F's top
        eigenvector: [["interface/dof", value], ...] (the reference's info row)."""
        wrench = self.directions @ vector
        return [["/".join(self.labels[i]), float(wrench[i])] for i in np.argsort(np.abs(wrench))[::-1][:6]]

    def _limits(self):
        """Constraint limits scaled by the calibration factor (one number, or a dict with a per-support
        entry; without interface bodies the "rails" entry applies)."""
        limits = self.settings["limits"]
        calibration = limits.get("calibration", 1.0)
        if isinstance(calibration, dict):
            calibration = calibration.get("rails", calibration)
        out = {}
        for key in ("mean_n_mm", "worst_n_mm"):
            scale = calibration[key] if isinstance(calibration, dict) else calibration
            out[key] = limits.get(key) and limits[key] * scale
        return out

    # --------------------------------------------------------------- host --
    def matrix(self, solutions):
        """F = factor * sum over mirror signs of P_s^T U_s, symmetrised, from the host solutions that
        HexElasticity.solve returns (``solutions[case]["fields"][sign]``), and the stacked U_s
        (the reference's matrix, topology_problem.py:639-646)."""
        zero = np.zeros(self.system.ndof)
        signs = sorted({sign for name in self.cases for sign in solutions[name]["fields"]})
        stacked = {sign: np.stack([solutions[name]["fields"].get(sign, zero) for name in self.cases], axis=1) for sign in signs}
        loads = {sign: np.stack([parts.get(sign, zero) for parts in self.forces], axis=1) for sign in signs}
        flexibility = self.factor * sum(loads[sign].T @ stacked[sign] for sign in signs)
        return (flexibility + flexibility.T) / 2, stacked

    def energy(self, stacked, vector, derivative):
        """Sensitivity of v^T F v to the element densities: -factor * dE/drho times the strain energy
        density of the combined displacement U_s v, summed over mirror signs
        (topology_problem.py:647-652)."""
        combined = [field @ vector for field in stacked.values()]
        per_element = sum(np.einsum("ea,ab,eb->e", u[self.system.dofs], self.system.ke, u[self.system.dofs], optimize=True) for u in combined)
        return -self.factor * np.asarray(derivative) * per_element

    def measure(self, solutions):
        """The load_mean / load_worst rows from host solutions (the reference's measure,
        topology_problem.py:657-684, without interface bodies): tr F, lambda_max F, the KS aggregate
        over F's eigenvalues and, where a limit is set, the constraint values and gradients."""
        limits, s = self._limits(), self.settings["ks"]
        flexibility, stacked = self.matrix(solutions)
        mean = float(np.trace(flexibility))
        values, vectors = np.linalg.eigh(flexibility)
        values, vectors = values[::-1], vectors[:, ::-1]
        worst = float(values[0])
        scale = limits["worst_n_mm"] or worst
        weights = np.exp(s * (values - worst) / scale)
        ks_value = worst + scale * np.log(weights.sum()) / s
        weights /= weights.sum()
        info = {"eigenvalues_n_mm": values[:6].tolist(), "ks_n_mm": float(ks_value), "ks": s, "rank": self.rank,
                "worst_wrench": self._worst_wrench(vectors[:, 0])}
        rows = [{"name": "load_mean", "value": mean, "limit": limits["mean_n_mm"], "unit": "N mm", "sense": "<=", "g": None, "gradient": None},
                {"name": "load_worst", "value": worst, "limit": limits["worst_n_mm"], "unit": "N mm", "sense": "<=", "g": None, "gradient": None,
                 "info": info}]
        if limits["mean_n_mm"]:
            gradient = sum(solutions[name]["derivative"] for name in self.cases)
            rows[0].update(g=mean / limits["mean_n_mm"] - 1, gradient=gradient / limits["mean_n_mm"])
        if limits["worst_n_mm"]:
            derivative = solutions[self.cases[0]]["modulus_derivative"]
            keep = np.flatnonzero(weights > self.settings["ks_cutoff"])
            gradient = sum(weights[i] * self.energy(stacked, vectors[:, i], derivative) for i in keep)
            rows[1].update(g=float(ks_value / limits["worst_n_mm"] - 1), gradient=gradient / limits["worst_n_mm"])
        return rows

    # ------------------------------------------------------------- device --
    def group_members(self):
        """Per fixture group holding covariance directions: (key, direction indices k, their parts).

        A group can also hold other static load cases of the domain (the reference registers the
        directions on the support case's fixture, topology_problem.py:599-611); only the covariance
        directions enter F, so only their parts are kept, in registration order."""
        index = {name: k for k, name in enumerate(self.cases)}
        out = []
        for key, members in self.system.groups.items():
            mine = [(index[case["name"]], part) for case, part in members if case["name"] in index]
            if mine:
                out.append((key, np.asarray([k for k, _ in mine]), [part for _, part in mine]))
        return out

    def groups(self):
        """Per fixture group: (key, case indices k, device force block [m, ndof])."""
        if self._groups is None:
            mg = self.system._multigrid()
            torch = mg.torch
            self._groups = [(key, ks, torch.as_tensor(np.stack([part["force"] for part in parts]), dtype=torch.float64, device=mg.device))
                            for key, ks, parts in self.group_members()]
        return self._groups

    def measure_device(self, physical_density, penalization=3.0, min_stiffness_ratio=1e-6, gradients=True):
        """Solve every direction on the GPU and return the load_mean / load_worst rows."""
        system = self.system
        mg = system._multigrid()
        torch = mg.torch
        lib = _lib.load()
        moduli, derivative = system.moduli(physical_density, penalization, min_stiffness_ratio)
        mg.update(moduli)
        scale = torch.as_tensor(-derivative, dtype=torch.float64, device=mg.device)
        return self.measure_from(self.solve_all(), scale, gradients)

    def solve_all(self, initial=None):
        """Solve every fixture group; ``initial`` maps a group key to a warm-start guess."""
        system = self.system
        solved = []
        for key, ks, forces in self.groups():
            guess = None if initial is None else initial.get(key)
            u, report = system.solve_group_device(key, forces, initial=guess)
            solved.append((key, ks, forces, u, report))
        return solved

    def measure_from(self, solved, scale, gradients=True, worst_gradient=True):
        """Rows of the reference's measure (topology_problem.py:657-684) from device solutions."""
        mg = self.system._multigrid()
        torch = mg.torch
        lib = _lib.load()
        flex = np.zeros((self.rank, self.rank))
        for key, ks, forces, u, _ in solved:
            m = len(ks)
            out = torch.empty((m, m), dtype=torch.float64, device=mg.device)
            scratch = torch.empty(int(lib.tf_gram_scratch_size(m, m)), dtype=torch.float64, device=mg.device)
            _lib.check(lib.tf_gram(_lib.ptr(forces), m, _lib.ptr(u), m, forces.shape[1], _lib.ptr(out), _lib.ptr(scratch),
                                   mg._stream()), None, "tf_gram")
            flex[np.ix_(ks, ks)] += self.factor * out.cpu().numpy()
        flex = (flex + flex.T) / 2
        s = self.settings["ks"]
        limits = self._limits()
        mean = float(np.trace(flex))
        values, vectors = np.linalg.eigh(flex)
        values, vectors = values[::-1], vectors[:, ::-1]
        worst = float(values[0])
        ks_scale = limits.get("worst_n_mm") or worst
        weights = np.exp(s * (values - worst) / ks_scale)
        ks_value = worst + ks_scale * np.log(weights.sum()) / s
        weights /= weights.sum()
        rows = [{"name": "load_mean", "value": mean, "limit": limits.get("mean_n_mm"), "unit": "N mm", "sense": "<=", "g": None, "gradient": None},
                {"name": "load_worst", "value": worst, "limit": limits.get("worst_n_mm"), "unit": "N mm", "sense": "<=", "g": None, "gradient": None,
                 "info": {"eigenvalues_n_mm": values[:6].tolist(), "ks_n_mm": float(ks_value), "ks": s, "rank": self.rank,
                          "worst_wrench": self._worst_wrench(vectors[:, 0])}}]
        if gradients:
            grad_mean = torch.zeros(self.system.nelem, dtype=torch.float64, device=mg.device)
            grad_worst = torch.zeros_like(grad_mean)
            keep = np.flatnonzero(weights > self.settings["ks_cutoff"])
            for key, ks, forces, u, _ in solved:
                m = len(ks)
                mg.energy_device(u, coefficients=np.full(m, self.factor), scale=scale, out=grad_mean, accumulate=True)
                if worst_gradient:
                    comb = vectors[np.ix_(ks, keep)]
                    mg.energy_device(u, combination=comb, coefficients=weights[keep] * self.factor, scale=scale, out=grad_worst, accumulate=True)
            limit_mean = limits.get("mean_n_mm") or 1.0
            limit_worst = limits.get("worst_n_mm") or 1.0
            rows[0].update(g=mean / limit_mean - 1, gradient=grad_mean / limit_mean)
            rows[1].update(g=float(ks_value / limit_worst - 1), gradient=grad_worst / limit_worst if worst_gradient else None)
        self.flexibility = flex
        return rows
