"""Covariance load model on the device: 42-direction RHS, tr(K^-1 Sigma), lambda_max, KS.

Host-side mirror of the reference's ``InterfaceCovariance``
(deep_frame/topology_problem.py:572-684):
* Sigma = D D^T from its eigenpairs, rank = eigenvalues above 1e-10 * max (:584-590);
* unit-wrench least-norm nodal forces per interface (:624-638), here the rigid-motion fields of
  ``rigid.unit_wrench_forces`` (no 6 x 3n matrix), mirrored on half models;
* one static case per direction, RHS_k = sum_j D_jk f_j, registered on the
  support case and split into +/- parts by ``HexElasticity`` (:599-611);
* ``measure``: F = sym(sum_parts factor P^T U), tr F, lambda_max and the KS
  aggregate, and the sensitivities of tr and of the KS-weighted eigenvalues
  (:657-684).  Every measure path (host solutions, device solutions, the
  column-sharded multi-GPU measure) reads F through one ``Spectrum`` record.
Solves, F = P^T U, and the sensitivity sums run on the GPU (libtfb200.so);
only the rank x rank eigen-decomposition of F runs on the host.
"""
import numpy as np

from . import _lib
from .rigid import unit_wrench_forces

DOFS = ["Fx", "Fy", "Fz", "Mx", "My", "Mz"]
SETTINGS = {"prefix": "sigma_", "ks": 50.0, "ks_cutoff": 1e-9, "limits": {"mean_n_mm": None, "worst_n_mm": None}}


class Spectrum:
    """What the covariance constraints read from a flexibility matrix F (rank x rank).

    ``trace`` = tr F; ``values`` / ``vectors`` = F's eigenpairs in descending order; ``ks`` = the
    Kreisselmeier-Steinhauser aggregate (scale / s) log sum exp(s lambda_i / scale) of the
    eigenvalues, with ``scale`` the worst-case limit when one is set and lambda_max otherwise;
    ``weights`` = d ks / d lambda_i, the softmax of s lambda / scale.  Computed through one
    log-sum-exp, so exp never overflows whatever the scale."""

    def __init__(self, flexibility, s, scale=None):
        f = np.asarray(flexibility, dtype=float)
        self.matrix = 0.5 * (f + f.T)
        ascending, basis = np.linalg.eigh(self.matrix)
        self.values, self.vectors = np.flip(ascending), np.flip(basis, axis=1)
        self.trace = float(np.trace(self.matrix))
        self.top = float(self.values[0])
        self.scale = scale or self.top
        exponents = s * self.values / self.scale
        peak = exponents[0]
        log_sum = peak + np.log(np.sum(np.exp(exponents - peak)))
        self.ks = float(self.scale * log_sum / s)
        self.weights = np.exp(exponents - log_sum)

    def kept(self, cutoff):
        """Indices of the eigenvalues whose KS weight exceeds ``cutoff``."""
        return np.flatnonzero(self.weights > cutoff)


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
        self.cases, self.forces = [], []
        here, there = self._label_basis(interfaces)
        for k in range(self.rank):
            case = system.add_case(self.settings["prefix"] + str(k), self.settings["support"], here @ self.directions[:, k],
                                   there @ self.directions[:, k])
            self.cases.append(case["name"])
            self.forces.append({part["sign"]: part["force"] for part in case["parts"]})
        self._groups = None

    def _label_basis(self, interfaces):
        """The unit-wrench nodal forces of every covariance label as sparse [ndof, labels] matrices,
        this side and mirror side; a direction's loads are these times its column of D."""
        from scipy.sparse import csc_matrix
        fields, entries = {}, (([], [], []), ([], [], []))
        for column, (name, dof) in enumerate(self.labels):
            if name not in fields:
                fields[name] = self.wrenches(interfaces[name])
            here_dofs, here_values, there_dofs, there_values = fields[name][DOFS.index(dof)]
            for side, dofs, values in ((0, here_dofs, here_values), (1, there_dofs, there_values)):
                entries[side][0].append(dofs)
                entries[side][1].append(np.full(len(dofs), column))
                entries[side][2].append(values)
        shape = (self.system.ndof, len(self.labels))
        return [csc_matrix((np.concatenate(v), (np.concatenate(r), np.concatenate(c))), shape=shape) for r, c, v in entries]

    def wrenches(self, interface):
        """Per unit wrench component (Fx, Fy, Fz, Mx, My, Mz about the interface's reference point):
        (direct dofs, direct values, mirror dofs, mirror values) of the least-norm nodal forces over
        the interface nodes that carry exactly that wrench (topology_problem.py:624-638).  Mirror
        side nodes enter with their reflected positions and get their forces reflected back."""
        system = self.system
        picked = [system._select_both(region, "covariance", "load") for region in interface["regions"]]
        direct = np.unique(np.concatenate([pair[0] for pair in picked]))
        mirror = np.unique(np.concatenate([pair[1] for pair in picked]))
        reflect = np.ones(3) if system.symmetry is None else system._flip()
        arms = np.vstack([system.points[direct], reflect * system.points[mirror]]) - np.asarray(interface["reference_mm"], dtype=float)
        spread = arms - arms[0]
        singular = np.sqrt(np.clip(np.linalg.eigvalsh(spread.T @ spread), 0.0, None))
        if np.count_nonzero(singular > 1e-8) < 2:
            raise ValueError("An interface wrench needs at least three non-collinear nodes")
        forces = unit_wrench_forces(arms)                       # [6, nodes, 3]
        split = len(direct)
        here = (3 * direct[:, None] + np.arange(3)).ravel()
        there = (3 * mirror[:, None] + np.arange(3)).ravel()
        return [(here, forces[j, :split].ravel(), there, (forces[j, split:] * reflect).ravel()) for j in range(6)]

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

    def _rows(self, spectrum, limits):
        """The load_mean / load_worst constraint rows (values, limits, info; no gradients yet)."""
        info = {"eigenvalues_n_mm": spectrum.values[:6].tolist(), "ks_n_mm": spectrum.ks, "ks": self.settings["ks"],
                "rank": self.rank, "worst_wrench": self._worst_wrench(spectrum.vectors[:, 0])}
        common = {"unit": "N mm", "sense": "<=", "g": None, "gradient": None}
        return [{"name": "load_mean", "value": spectrum.trace, "limit": limits["mean_n_mm"], **common},
                {"name": "load_worst", "value": spectrum.top, "limit": limits["worst_n_mm"], **common, "info": info}]

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
        """Sensitivity of v^T F v to the element densities (``vector`` [rank] or [rank, k] for k
        combinations at once): -factor * dE/drho times the strain energy of U_s v, summed over mirror
        signs (topology_problem.py:647-652).  Returns [nelem] or [nelem, k]."""
        ke, dofs = self.system.ke, self.system.dofs
        v = np.asarray(vector, dtype=float)
        columns = v.reshape(self.rank, -1)
        total = 0.0
        for field in stacked.values():
            element = (field @ columns)[dofs]                              # [nelem, 24, k]
            total = total + np.einsum("eak,ab,ebk->ek", element, ke, element, optimize=True)
        out = -self.factor * np.asarray(derivative)[:, None] * total
        return out[:, 0] if v.ndim == 1 else out

    def measure(self, solutions):
        """The load_mean / load_worst rows from host solutions (the reference's measure,
        topology_problem.py:657-684, without interface bodies): tr F, lambda_max F, the KS aggregate
        over F's eigenvalues and, where a limit is set, the constraint values and gradients."""
        limits = self._limits()
        flexibility, stacked = self.matrix(solutions)
        spectrum = Spectrum(flexibility, self.settings["ks"], limits["worst_n_mm"])
        rows = self._rows(spectrum, limits)
        if limits["mean_n_mm"]:
            gradient = np.sum([solutions[name]["derivative"] for name in self.cases], axis=0)
            rows[0].update(g=spectrum.trace / limits["mean_n_mm"] - 1, gradient=gradient / limits["mean_n_mm"])
        if limits["worst_n_mm"]:
            kept = spectrum.kept(self.settings["ks_cutoff"])
            slope = solutions[self.cases[0]]["modulus_derivative"]
            gradient = self.energy(stacked, spectrum.vectors[:, kept], slope) @ spectrum.weights[kept]
            rows[1].update(g=float(spectrum.ks / limits["worst_n_mm"] - 1), gradient=gradient / limits["worst_n_mm"])
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

    def flexibility_device(self, solved):
        """F from device solutions: one tf_gram (P^T U on the device) per fixture group, placed at the
        group's direction indices; symmetrised on the host."""
        mg = self.system._multigrid()
        torch = mg.torch
        lib = _lib.load()
        flex = np.zeros((self.rank, self.rank))
        for _, ks, forces, u, _ in solved:
            m = len(ks)
            out = torch.empty((m, m), dtype=torch.float64, device=mg.device)
            scratch = torch.empty(int(lib.tf_gram_scratch_size(m, m)), dtype=torch.float64, device=mg.device)
            _lib.check(lib.tf_gram(_lib.ptr(forces), m, _lib.ptr(u), m, forces.shape[1], _lib.ptr(out), _lib.ptr(scratch),
                                   mg._stream()), None, "tf_gram")
            flex[np.ix_(ks, ks)] += self.factor * out.cpu().numpy()
        return 0.5 * (flex + flex.T)

    def measure_from(self, solved, scale, gradients=True, worst_gradient=True):
        """Rows of the reference's measure (topology_problem.py:657-684) from device solutions; the
        sensitivities are sums of element energies formed on the device (``tf_combine`` for the
        eigenvector combinations, ``tf_element_energy`` for the energies)."""
        mg = self.system._multigrid()
        torch = mg.torch
        limits = self._limits()
        spectrum = Spectrum(self.flexibility_device(solved), self.settings["ks"], limits["worst_n_mm"])
        rows = self._rows(spectrum, limits)
        if gradients:
            grad_mean = torch.zeros(self.system.nelem, dtype=torch.float64, device=mg.device)
            grad_worst = torch.zeros_like(grad_mean)
            kept = spectrum.kept(self.settings["ks_cutoff"])
            for _, ks, _, u, _ in solved:
                mg.energy_device(u, coefficients=np.full(len(ks), self.factor), scale=scale, out=grad_mean, accumulate=True)
                if worst_gradient:
                    # the KS-weighted eigenvector combinations U v_i formed once (tf_combine), then their energies
                    combined = mg.combine_device(u, spectrum.vectors[np.ix_(ks, kept)])
                    mg.energy_device(combined, coefficients=spectrum.weights[kept] * self.factor, scale=scale, out=grad_worst,
                                     accumulate=True)
            mean_limit, worst_limit = limits["mean_n_mm"] or 1.0, limits["worst_n_mm"] or 1.0
            rows[0].update(g=spectrum.trace / mean_limit - 1, gradient=grad_mean / mean_limit)
            rows[1].update(g=float(spectrum.ks / worst_limit - 1), gradient=grad_worst / worst_limit if worst_gradient else None)
        self.flexibility = spectrum.matrix
        return rows
