"""Geometric multigrid-preconditioned CG on the CPU (oracle and CPU baseline, test only).

Restates deep_frame/topology_multigrid.py of the reference with SciPy sparse
matrices instead of convolutions:
* level count and padding (:58-63);
* live mask of the finest level (:138-144) and Jacobi diagonals (:118-124);
* Galerkin coarse operators (:145-208): summing P_c^T K_c P_c over the children
  of every coarse element equals the sparse triple product P^T A P, with the
  finest operator masked on both sides (children gated by the fine mask) and
  the deeper levels unmasked; coarse dofs whose diagonal is <= dead_ratio *
  max are dropped;
* trilinear prolongation P, the transpose of the full-weighting restriction
  conv3d((x)[1/2, 1, 1/2], stride 2, padding 1) (:314-316);
* lambda_max(D^-1 A) by power iteration (:214-223), Jacobi / Chebyshev
  smoothing (:284-305), V/W cycle (:306-317), the max|r| scaling of the
  preconditioner (:318-324);
* the coarsest solve as a sparse LU of the live dofs (the reference uses cuDSS);
* batched flexible PCG with the true-residual recheck and the active-set
  shrink (:407-454).
"""
import numpy as np
from scipy.sparse import coo_matrix, csr_matrix, diags, kron, identity
from scipy.sparse.linalg import splu

from .hex8 import CORNERS, grid_numbering
from .operator import assemble, live_dofs

DEFAULTS = {"coarsest_dofs": 8000, "max_levels": 8, "smoother": "chebyshev", "sweeps": 2, "damping": 1.0,
            "chebyshev_degree": 3, "chebyshev_ratio": 20.0, "growth": 2.0, "cycle": "V", "power_iterations": 20,
            "tolerance": 1e-8, "max_iterations": 2000, "dead_ratio": 1e-12, "zero_rhs": 1e-12}


def level_count(shape, settings):
    count = 2
    while count < settings["max_levels"] and np.prod(np.ceil(np.asarray(shape) / 2 ** (count - 1)) + 1) * 3 > settings["coarsest_dofs"]:
        count += 1
    return count


def prolongation_1d(n_coarse_elems):
    """(2e+1) x (e+1) linear interpolation between node lines."""
    nf, nc = 2 * n_coarse_elems + 1, n_coarse_elems + 1
    rows, cols, vals = [], [], []
    for i in range(nf):
        if i % 2 == 0:
            rows.append(i); cols.append(i // 2); vals.append(1.0)
        else:
            rows += [i, i]; cols += [(i - 1) // 2, (i + 1) // 2]; vals += [0.5, 0.5]
    return coo_matrix((vals, (rows, cols)), shape=(nf, nc)).tocsr()


def prolongation(coarse_shape):
    """Dof prolongation for node-major, component-minor vectors of a grid of coarse_shape elements."""
    px, py, pz = (prolongation_1d(n) for n in coarse_shape)
    return kron(kron(kron(px, py), pz), identity(3)).tocsr()


def local_interpolation():
    """[8 children, 24 fine dofs, 24 coarse dofs]: the trilinear weight of every coarse-element corner
    at every corner of each of its 8 children (children in C order of their offsets), per component
    (the reference's ``_interpolation``, topology_multigrid.py:19-27)."""
    offsets = np.array(list(np.ndindex(2, 2, 2)), dtype=float)
    at = (offsets[:, None, :] + CORNERS[None, :, :]) / 2.0                        # [child, fine corner, xyz]
    weight = np.prod(np.where(CORNERS[None, None, :, :] == 1, at[:, :, None, :], 1.0 - at[:, :, None, :]), axis=3)
    return np.einsum("cfk,ij->cfikj", weight, np.eye(3)).reshape(8, 24, 24)


def fine_blocks(shape, k0, moduli, mask):
    """[nelem, 24, 24] element matrices E_e K0 gated on both sides by the fine live mask (the children
    of the first Galerkin level, topology_multigrid.py:131-135)."""
    _, dofs = grid_numbering(shape)
    m = np.asarray(mask, dtype=float)[dofs]                                       # [nelem, 24]
    return np.asarray(moduli, dtype=float).ravel()[:, None, None] * m[:, :, None] * m[:, None, :] * np.asarray(k0)[None]


def galerkin_blocks(shape, children):
    """Coarse element blocks sum_c P_c^T B_c P_c over the 8 children of every coarse element,
    symmetrised (topology_multigrid.py:173-178); ``shape`` is the children's grid, even in every axis."""
    cx, cy, cz = (n // 2 for n in shape)
    index = np.arange(int(np.prod(shape))).reshape(cx, 2, cy, 2, cz, 2).transpose(0, 2, 4, 1, 3, 5).reshape(-1, 8)
    local = local_interpolation()
    blocks = np.einsum("cia,ecij,cjb->eab", local, children[index], local, optimize=True)
    return (blocks + blocks.transpose(0, 2, 1)) / 2


def assemble_blocks(shape, blocks):
    """Sparse matrix of per-element [24, 24] blocks on a grid of ``shape`` elements."""
    _, dofs = grid_numbering(shape)
    ndof = 3 * int(np.prod(np.asarray(shape) + 1))
    rows = np.repeat(dofs, 24, axis=1).ravel()
    cols = np.tile(dofs, (1, 24)).ravel()
    return coo_matrix((blocks.reshape(-1), (rows, cols)), shape=(ndof, ndof)).tocsr()


class MultigridOracle:
    def __init__(self, shape, k0, moduli, fixed, settings=None):
        self.s = {**DEFAULTS, **(settings or {})}
        self.shape = tuple(int(n) for n in shape)
        count = level_count(self.shape, self.s)
        factor = 2 ** (count - 1)
        self.padded = tuple(int(np.ceil(n / factor) * factor) for n in self.shape)
        moduli = np.asarray(moduli, dtype=float).reshape(self.shape)
        padded_moduli = np.zeros(self.padded)
        padded_moduli[:self.shape[0], :self.shape[1], :self.shape[2]] = moduli
        # padded fine operator and mask
        self.nodes = tuple(n + 1 for n in self.shape)
        pnodes = tuple(n + 1 for n in self.padded)
        self.embed = self._embedding(self.nodes, pnodes)
        fixed_p = self.embed[np.asarray(fixed, dtype=np.int64)] if len(fixed) else np.zeros(0, dtype=np.int64)
        k = assemble(self.padded, k0, padded_moduli.ravel())
        mask0 = live_dofs(self.padded, padded_moduli.ravel(), fixed_p).astype(float)
        m0 = diags(mask0)
        self.A = [(m0 @ k @ m0).tocsr()]
        self.mask = [mask0]
        diag0 = k.diagonal() * mask0
        self.inv = [np.where(mask0 > 0, 1.0 / np.where(diag0 > 0, diag0, 1.0), 0.0)]
        self.P = []
        unmasked = self.A[0]
        for level in range(1, count):
            cshape = tuple(n // 2 ** level for n in self.padded)
            p = prolongation(cshape)
            self.P.append(p)
            coarse = (p.T @ unmasked @ p).tocsr()
            coarse = ((coarse + coarse.T) * 0.5).tocsr()
            d = coarse.diagonal()
            mask = (d > self.s["dead_ratio"] * d.max()).astype(float)
            self.mask.append(mask)
            self.inv.append(np.where(mask > 0, 1.0 / np.where(d > 0, d, 1.0), 0.0))
            self.A.append(coarse)
            unmasked = coarse
        self.levels = count
        self.lam = [self._spectrum(l) for l in range(count - 1)]
        live = np.flatnonzero(self.mask[-1] > 0)
        self.coarse_live = live
        self.coarse_lu = splu(self.A[-1][live][:, live].tocsc()) if len(live) else None

    @staticmethod
    def _embedding(nodes, pnodes):
        idx = np.indices(nodes).reshape(3, -1).T
        pnode = np.ravel_multi_index(tuple(idx.T), pnodes)
        return (3 * pnode[:, None] + np.arange(3)).ravel()

    def _apply(self, level, x):
        y = self.A[level] @ x
        return y * self.mask[level][:, None] if y.ndim == 2 else y * self.mask[level]

    def _spectrum(self, level):
        rng = np.random.default_rng(0)
        v = (rng.uniform(size=self.A[level].shape[0]) - 0.5) * self.mask[level]
        est = 1.0
        for _ in range(self.s["power_iterations"]):
            v = self.inv[level] * self._apply(level, v)
            est = float(np.linalg.norm(v))
            v = v / est
        return est

    def _smooth(self, level, b, x):
        s = self.s
        inv = self.inv[level][:, None]
        if s["smoother"] == "jacobi":
            count = max(1, int(round(s["sweeps"] * s["growth"] ** level)))
            step = s["damping"] / self.lam[level]
            for _ in range(count):
                x = step * inv * b if x is None else x + step * inv * (b - self._apply(level, x))
            return x
        count = max(1, int(round(s["chebyshev_degree"] * s["growth"] ** level)))
        upper = 1.1 * self.lam[level]
        lower = upper / s["chebyshev_ratio"]
        theta, delta = (upper + lower) / 2, (upper - lower) / 2
        sigma = theta / delta
        rho = 1 / sigma
        r = b if x is None else b - self._apply(level, x)
        d = inv * r / theta
        x = d if x is None else x + d
        for _ in range(count - 1):
            r = r - self._apply(level, d)
            rn = 1 / (2 * sigma - rho)
            d = rn * rho * d + 2 * rn / delta * inv * r
            rho = rn
            x = x + d
        return x

    def _cycle(self, level, b):
        if level == self.levels - 1:
            x = np.zeros_like(b)
            if self.coarse_lu is not None:
                x[self.coarse_live] = self.coarse_lu.solve(b[self.coarse_live])
            return x
        x = self._smooth(level, b, None)
        reps = 2 if self.s["cycle"] == "W" and level + 2 < self.levels else 1
        for _ in range(reps):
            r = (b - self._apply(level, x)) * self.mask[level][:, None]
            bc = (self.P[level].T @ r) * self.mask[level + 1][:, None]
            x = x + (self.P[level] @ self._cycle(level + 1, bc)) * self.mask[level][:, None]
        return self._smooth(level, b, x)

    def precondition(self, r):
        scale = np.maximum(np.abs(r).max(axis=0, keepdims=True), 1e-300)
        return self._cycle(0, r / scale) * scale

    def solve(self, forces, max_iterations=None):
        """Flexible PCG per column; forces [ndof_unpadded, R] -> (u, iterations, relative, history).

        Columns whose norm is at most zero_rhs times the largest are not solved: zero solution, 0
        iterations, relative residual 0 (the reference's solve, topology_multigrid.py:350-351)."""
        forces = np.asarray(forces, dtype=float)
        forces = forces[:, None] if forces.ndim == 1 else forces
        norms = np.linalg.norm(forces, axis=0)
        live = np.flatnonzero(norms > self.s["zero_rhs"] * max(norms.max(initial=0.0), 1e-300))
        u = np.zeros_like(forces)
        iterations, relative = np.zeros(forces.shape[1], dtype=int), np.zeros(forces.shape[1])
        history = []
        if len(live):
            u[:, live], iterations[live], relative[live], history = self._pcg(forces[:, live], max_iterations)
        return u, iterations, relative, history

    def _pcg(self, forces, max_iterations=None):
        """Batched flexible PCG of the live columns (topology_multigrid.py:407-454)."""
        limit = self.s["max_iterations"] if max_iterations is None else max_iterations
        tol = self.s["tolerance"]
        n_p = self.A[0].shape[0]
        b = np.zeros((n_p, forces.shape[1]))
        b[self.embed] = forces
        b *= self.mask[0][:, None]
        count = b.shape[1]
        norm = np.linalg.norm(b, axis=0)
        x = np.zeros_like(b)
        iterations, relative = np.zeros(count, dtype=int), np.ones(count)
        active = np.arange(count)
        r = b.copy()
        z = self.precondition(r)
        p = z.copy()
        rz = (r * z).sum(axis=0)
        step, history = 0, []
        while len(active) and step < limit:
            q = self._apply(0, p)
            alpha = rz / (p * q).sum(axis=0)
            x[:, active] += alpha * p
            r = r - alpha * q
            step += 1
            current = np.linalg.norm(r, axis=0) / norm[active]
            history.append(float(current.max()))
            conv = current < tol
            if conv.any():
                true = b[:, active] - self._apply(0, x[:, active])
                current = np.linalg.norm(true, axis=0) / norm[active]
                conv = current < tol
                r = np.where(conv[None, :], r, true)
            iterations[active[conv]] = step
            relative[active[conv]] = current[conv]
            keep = ~conv
            if not keep.any():
                active = active[keep]
                break
            active, r, p, z, rz = active[keep], r[:, keep], p[:, keep], z[:, keep], rz[keep]
            zn = self.precondition(r)
            beta = (r * (zn - z)).sum(axis=0) / rz
            rz = (r * zn).sum(axis=0)
            p = zn + beta * p
            z = zn
        if len(active):
            final = b[:, active] - self._apply(0, x[:, active])
            relative[active] = np.linalg.norm(final, axis=0) / norm[active]
            iterations[active] = step
        return x[self.embed], iterations, relative, history
