"""Drop-in ``GeometricMultigrid`` backed by the sm_100a library.

Same constructor, methods, settings keys and report keys as the reference's
deep_frame/topology_multigrid.py:46-548, so ``HexElasticity(...,
linear_solver="multigrid")`` style callers can swap it in.  All numerical
work (operator, hierarchy, V-cycle, PCG, energies) runs in libtfb200.so; the
torch tensors here only hold device memory and carry the current stream.
There is no CPU path: without CUDA or without the built library every call
raises.

Host-facing calls (``solve``, ``product``) take and return NumPy arrays like
the reference; ``solve_device`` / ``update_device`` keep everything in HBM.
"""
import ctypes
from time import perf_counter

import numpy as np

from . import _lib

# The reference's MULTIGRID defaults (topology_multigrid.py:8-10) with two
# differences: the coarsest grid is factored densely on the device, so it is
# kept at <= 8000 dofs, and all live RHS columns share one PCG launch (batch 0).
MULTIGRID = {"coarse": "galerkin", "coarsest_dofs": 8000, "max_levels": 8, "smoother": "chebyshev", "sweeps": 2,
             "damping": 1.0, "chebyshev_degree": 3, "chebyshev_ratio": 20.0, "growth": 2.0, "cycle": "V",
             "power_iterations": 20, "precision": "float32", "tolerance": 1e-8, "max_iterations": 2000, "batch": 0,
             "projection": True, "coarsest_projection": True, "dead_ratio": 1e-12, "zero_rhs": 1e-12, "retries": 2,
             "device": "cuda", "eigen_tolerance": 1e-8, "eigen_iterations": 300, "eigen_guard": 2, "eigen_refresh": 10,
             "eigen_drop": 1e-12, "eigen_seed": 0, "tensor_cores": False, "pcg_precision": "float64", "reliable": 0.01, "fine_tz": 0}
PRECISIONS = ("float64", "float32", "bfloat16", "float16")


def _torch():
    import torch
    return torch


class Level:
    """Shape bookkeeping of one multigrid level (reference topology_multigrid.py:40-44)."""

    def __init__(self, shape, spacing):
        self.shape, self.spacing = tuple(int(n) for n in shape), np.asarray(spacing, dtype=float)
        self.nodes = tuple(n + 1 for n in self.shape)
        self.lambda_max = None


def _native_settings(settings):
    s = _lib.default_settings()
    if settings["precision"] not in PRECISIONS or settings["coarse"] not in ("galerkin", "rediscretize") \
            or settings["smoother"] not in ("jacobi", "chebyshev") or settings["cycle"] not in ("V", "W"):
        raise ValueError("Invalid multigrid settings")
    s.precision = _lib.PRECISION[settings["precision"]]
    s.smoother = _lib.SMOOTHER[settings["smoother"]]
    s.cycle = _lib.CYCLE[settings["cycle"]]
    s.coarse = _lib.COARSE[settings["coarse"]]
    for name in ("sweeps", "chebyshev_degree", "max_levels", "power_iterations", "max_iterations", "retries", "batch",
                 "coarsest_dofs"):
        setattr(s, name, int(settings[name]))
    for name in ("damping", "chebyshev_ratio", "growth", "tolerance", "dead_ratio", "zero_rhs"):
        setattr(s, name, float(settings[name]))
    s.tensor_cores = 1 if settings.get("tensor_cores") else 0
    if settings["pcg_precision"] not in ("float64", "float32"):
        raise ValueError("Invalid multigrid settings")
    s.pcg_precision = _lib.PRECISION[settings["pcg_precision"]]
    s.reliable = float(settings["reliable"])
    s.fine_tz = int(settings["fine_tz"])
    return s


class GeometricMultigrid:
    def __init__(self, shape, spacing, ke, settings=None, me=None):
        torch = _torch()
        self.torch = torch
        self.settings = {**MULTIGRID, **(settings or {})}
        native = _native_settings(self.settings)
        self.device = torch.device(self.settings["device"])
        if self.device.type != "cuda" or not torch.cuda.is_available():
            raise RuntimeError("GeometricMultigrid runs on the CUDA device only (no CPU fallback)")
        self.lib = _lib.load()
        self.shape = tuple(int(n) for n in shape)
        self.spacing = np.asarray(spacing, dtype=float)
        self.ke64 = np.ascontiguousarray(np.asarray(ke, dtype=float))
        if self.ke64.shape != (24, 24):
            raise ValueError("ke must be a 24x24 element stiffness")
        self.me64 = None if me is None else np.ascontiguousarray(np.asarray(me, dtype=float))
        grid = _lib.TfGrid()
        for d in range(3):
            grid.shape[d] = self.shape[d]
            grid.spacing[d] = float(self.spacing[d])
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.tf_create(ctypes.byref(grid), self.ke64.ctypes.data_as(ctypes.c_void_p),
                                          None if self.me64 is None else self.me64.ctypes.data_as(ctypes.c_void_p),
                                          ctypes.byref(native), ctypes.byref(handle)), None, "tf_create")
        self.handle = handle
        levels, padded = ctypes.c_int32(), (ctypes.c_int64 * 3)()
        _lib.check(self.lib.tf_levels(self.handle, ctypes.byref(levels), padded), self.handle, "tf_levels")
        self.padded = tuple(int(p) for p in padded)
        self.levels = [Level(np.asarray(self.padded) // 2 ** level, self.spacing * 2 ** level) for level in range(levels.value)]
        self.center = np.asarray(self.shape) * self.spacing / 2
        self.nodes = tuple(n + 1 for n in self.shape)
        self.ndof = 3 * int(np.prod(self.nodes))
        self.nelem = int(np.prod(self.shape))
        self.moduli = None
        self._moduli_host = None
        self._keys, self._fixed = {}, {}
        self.hierarchies, self.statistics = {}, []

    # ------------------------------------------------------------ helpers --
    def _stream(self):
        return _lib.stream_of(self.device)

    def _key(self, key, fixed):
        fixed = np.ascontiguousarray(np.asarray(fixed, dtype=np.int64).ravel())
        if key not in self._keys:
            self._keys[key] = len(self._keys) + 1
        ident = self._keys[key]
        known = self._fixed.get(ident)
        if known is None or not np.array_equal(known, fixed):
            _lib.check(self.lib.tf_set_bc(self.handle, ident, fixed.ctypes.data_as(ctypes.c_void_p), len(fixed)),
                       self.handle, "tf_set_bc")
            self._fixed[ident] = fixed
            self.hierarchies.pop(key, None)
        return ident

    def _columns(self, flat):
        """NumPy or torch [ndof] / [ndof, R] -> contiguous device FP64 [R, ndof]."""
        torch = self.torch
        data = torch.as_tensor(flat, dtype=torch.float64, device=self.device)
        data = data[:, None] if data.ndim == 1 else data
        if data.shape[0] != self.ndof:
            raise ValueError(f"expected {self.ndof} dofs, got {data.shape[0]}")
        return data.T.contiguous()

    def grid(self, flat, dtype=None):
        """Flat [ndof, R] (dof = 3 node + component, C-order nodes) -> the reference's grid layout
        [R, 3, padded nodes] with zeros in the padding (topology_multigrid.py:80-88)."""
        torch = self.torch
        values = torch.as_tensor(flat, device=self.device, dtype=dtype or torch.float64)
        if values.ndim == 1:
            values = values.unsqueeze(1)
        columns = values.shape[1]
        nx, ny, nz = self.nodes
        planes = values.T.reshape(columns, nx, ny, nz, 3).movedim(-1, 1)          # component planes [R, 3, nx, ny, nz]
        out = values.new_zeros((columns, 3) + tuple(self.levels[0].nodes))
        out[..., :nx, :ny, :nz] = planes
        return out

    def flat(self, grid):
        """Inverse of ``grid``: [R, 3, padded nodes] -> [ndof, R] without the padding."""
        nx, ny, nz = self.nodes
        return grid[..., :nx, :ny, :nz].movedim(1, -1).reshape(grid.shape[0], -1).T

    def element_field(self, values, dtype=None):
        torch = self.torch
        field = torch.zeros(self.padded, dtype=dtype or torch.float64, device=self.device)
        field[:self.shape[0], :self.shape[1], :self.shape[2]] = torch.as_tensor(
            np.asarray(values, dtype=float).reshape(self.shape), dtype=field.dtype, device=self.device)
        return field

    # -------------------------------------------------------------- state --
    def update(self, moduli):
        """Set element moduli [nelem] (host or device) and drop every hierarchy (topology_multigrid.py:97-100)."""
        torch = self.torch
        values = torch.as_tensor(moduli, dtype=torch.float64, device=self.device).reshape(-1).contiguous()
        if values.numel() != self.nelem:
            raise ValueError(f"expected {self.nelem} moduli, got {values.numel()}")
        self.update_device(values)

    def update_device(self, moduli):
        if moduli.dtype != self.torch.float64 or not moduli.is_cuda or not moduli.is_contiguous() or moduli.numel() != self.nelem:
            raise ValueError("moduli must be a contiguous CUDA float64 tensor with one value per element")
        _lib.check(self.lib.tf_update(self.handle, _lib.ptr(moduli), self._stream()), self.handle, "tf_update")
        self.moduli = moduli
        self._moduli_host = None
        self.hierarchies.clear()

    def mask(self, fixed):
        """(live mask, constrained) grids [3, padded nodes] (topology_multigrid.py:138-144)."""
        torch = self.torch
        if self.moduli is None:
            raise ValueError("update(moduli) must be called first")
        if self._moduli_host is None:
            self._moduli_host = self.moduli.cpu().numpy().reshape(self.shape)
        touched = np.zeros(tuple(p + 1 for p in self.padded), dtype=bool)
        live = self._moduli_host > 0
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    touched[dx:dx + self.shape[0], dy:dy + self.shape[1], dz:dz + self.shape[2]] |= live
        active = torch.as_tensor(np.broadcast_to(touched, (3,) + touched.shape).astype(float), device=self.device)
        constrained = torch.zeros_like(active)
        fixed = np.asarray(fixed, dtype=np.int64)
        if len(fixed):
            flags = np.zeros(self.ndof)
            flags[fixed] = 1.0
            constrained = self.grid(flags)[0] * active
        return active * (1 - constrained), constrained

    def hierarchy(self, key, fixed):
        """Build (or reuse) the hierarchy of `key` and return its summary (topology_multigrid.py:145-208)."""
        if key in self.hierarchies:
            return self.hierarchies[key]
        ident = self._key(key, fixed)
        report = _lib.TfReport()
        _lib.check(self.lib.tf_prepare(self.handle, ident, ctypes.byref(report), self._stream()), self.handle, "tf_prepare")
        levels = [Level(level.shape, level.spacing) for level in self.levels]
        for index, level in enumerate(levels[:-1]):
            level.lambda_max = float(report.lambda_max[index])
        hierarchy = {"key": key, "id": ident, "levels": levels, "fixed": np.asarray(fixed, dtype=np.int64),
                     "coarsest": {"dofs": int(report.coarsest_dofs), "pins": 0}, "setup_s": float(report.setup_s),
                     "kernel_check": [], "coefficients": np.zeros((6, 0))}
        self.hierarchies[key] = hierarchy
        return hierarchy

    # ------------------------------------------------------------ solving --
    def solve(self, key, fixed, forces, support=None):
        """Reference-compatible solve: NumPy forces [ndof, R] in, (NumPy [ndof, R], report) out."""
        torch = self.torch
        started = perf_counter()
        forces = np.asarray(forces, dtype=float)
        columns = self._columns(forces.reshape(len(forces), -1))
        out, report = self.solve_device(key, fixed, columns, support=support)
        flat = out.T.cpu().numpy()
        report["seconds"] = perf_counter() - started
        return flat, report

    def _report_arrays(self, count):
        iterations = np.zeros(count, dtype=np.int32)
        relative = np.zeros(count, dtype=np.float64)
        history = np.zeros(self.settings["max_iterations"] * (1 + self.settings["retries"]) + 8, dtype=np.float64)
        report = _lib.TfReport()
        report.iterations = iterations.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        report.relative_residual = relative.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        report.history = history.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        report.history_capacity = len(history)
        return report, (iterations, relative, history)

    def _result(self, report, arrays, started):
        iterations, relative, history = arrays
        levels = int(report.levels)
        result = {"iterations": iterations.tolist(), "relative_residual": relative.tolist(),
                  "converged": bool(report.converged), "history": [history[:report.history_len].tolist()],
                  "batches": int(report.batches), "retried_columns": int(report.retried_columns),
                  "zero_rhs_columns": int(report.zero_rhs_columns), "seconds": perf_counter() - started,
                  "setup_s": float(report.setup_s), "floating": False, "levels": levels,
                  "coarsest_dofs": int(report.coarsest_dofs), "kernel": 0, "rhs_kernel_component": None,
                  "kernel_check": [], "lambda_max": [float(report.lambda_max[i]) for i in range(levels - 1)],
                  "steps": int(report.steps)}
        self.statistics.append(result)
        return result

    def _check_forces(self, forces):
        torch = self.torch
        if self.moduli is None:
            raise ValueError("update(moduli) must be called before solve")
        if forces.dtype != torch.float64 or not forces.is_cuda or not forces.is_contiguous() or forces.shape[-1] != self.ndof:
            raise ValueError("forces must be a contiguous CUDA float64 [R, ndof] tensor")

    def solve_device(self, key, fixed, forces, out=None, support=None, initial=None):
        """Device-resident solve: forces [R, ndof] contiguous CUDA float64; returns (u [R, ndof], report).

        ``initial`` ([R, ndof] CUDA float64) starts PCG from that guess instead of zero, as the
        reference's ``_pcg(hierarchy, rhs, initial)`` does for its retries.

        ``support`` (the statically determinate support dofs of an inertia-relief part, contained in
        ``fixed``) is accepted for the reference's signature: the reference then solves the floating
        structure with the rigid modes projected out and shifts the result to zero at the support
        (topology_multigrid.py:340-349,368-370); for balanced loads that is the solution with every
        dof of ``fixed`` held, which is what this solve computes."""
        torch = self.torch
        if support is not None and not np.isin(np.asarray(support, dtype=np.int64), np.asarray(fixed, dtype=np.int64)).all():
            raise ValueError("support dofs must be part of fixed")
        started = perf_counter()
        self._check_forces(forces)
        count = forces.shape[0]
        ident = self._key((key, False), fixed)
        out = torch.empty_like(forces) if out is None else out
        if initial is not None:
            if initial.shape != forces.shape or initial.dtype != torch.float64 or not initial.is_cuda:
                raise ValueError("initial must be a CUDA float64 tensor shaped like forces")
            if initial.data_ptr() != out.data_ptr():
                out.copy_(initial)
        report, arrays = self._report_arrays(count)
        entry = self.lib.tf_solve if initial is None else self.lib.tf_solve_guess
        _lib.check(entry(self.handle, ident, _lib.ptr(forces), count, _lib.ptr(out), ctypes.byref(report), self._stream()),
                   self.handle, "tf_solve" if initial is None else "tf_solve_guess")
        return out, self._result(report, arrays, started)

    def precondition(self, hierarchy, residual):
        """One V-cycle z = M^-1 r of `hierarchy` on a residual grid [R, 3, padded nodes]."""
        columns = self.flat(residual).T.contiguous().to(self.torch.float64)
        out = self.torch.empty_like(columns)
        _lib.check(self.lib.tf_precondition(self.handle, hierarchy["id"], _lib.ptr(columns), columns.shape[0], _lib.ptr(out),
                                            self._stream()), self.handle, "tf_precondition")
        return self.grid(out.T)

    # ----------------------------------------------------------- operators --
    def apply_device(self, columns, key=None, fixed=None, out=None):
        """y = K u on [R, ndof] device columns; with key/fixed the live mask of that hierarchy is applied."""
        out = self.torch.empty_like(columns) if out is None else out
        ident = 0 if key is None else self._key((key, False), fixed)
        _lib.check(self.lib.tf_apply(self.handle, ident, 0 if key is None else 1, _lib.ptr(columns), columns.shape[0],
                                     _lib.ptr(out), self._stream()), self.handle, "tf_apply")
        return out

    def apply_level_device(self, key, fixed, level, columns, out=None):
        """y = mask_l * A_l (mask_l * u) on [R, 3 * nodes_l] device columns of the padded level-l grid:
        the level operators of the hierarchy of ``key`` in FP64 (level 0 the masked finest operator,
        deeper levels the Galerkin operators; topology_multigrid.py:110-117)."""
        ident = self._key((key, False), fixed)
        out = self.torch.empty_like(columns) if out is None else out
        _lib.check(self.lib.tf_apply_level(self.handle, ident, int(level), _lib.ptr(columns), columns.shape[0], _lib.ptr(out),
                                           self._stream()), self.handle, "tf_apply_level")
        return out

    def combine_device(self, columns, mixing, out=None):
        """[k, ndof] = mixing^T columns for device columns [m, ndof] and a host mixing matrix [m, k]
        (tf_combine): the combinations U v whose energies the lambda_max sensitivity sums."""
        torch = self.torch
        mixing = np.ascontiguousarray(np.asarray(mixing, dtype=float))
        m, n = columns.shape
        coef = torch.as_tensor(mixing, device=columns.device)
        out = torch.empty((mixing.shape[1], n), dtype=torch.float64, device=columns.device) if out is None else out
        _lib.check(self.lib.tf_combine(_lib.ptr(columns), m, n, _lib.ptr(coef), mixing.shape[1], _lib.ptr(out), self._stream()),
                   None, "tf_combine")
        return out

    def operator(self, grid, moduli=None, mask=None):
        """y = mask * K (mask * u) on a grid [R, 3, padded nodes] (topology_multigrid.py:105-109)."""
        if moduli is not None:
            raise NotImplementedError("operator(moduli=...) is not supported; call update() instead")
        grid = grid if mask is None else grid * mask
        columns = self.flat(grid).T.contiguous().to(self.torch.float64)
        result = self.grid(self.apply_device(columns).T, dtype=grid.dtype)
        return result if mask is None else result * mask

    def product(self, flat):
        """K u for host columns (topology_multigrid.py:455-457)."""
        flat = np.asarray(flat, dtype=float)
        columns = self._columns(flat.reshape(len(flat), -1))
        return self.apply_device(columns).T.cpu().numpy()

    def element_energy(self, grid):
        """u_e^T K0 u_e per column and element, padded element grid [R, *padded] (topology_multigrid.py:458-459)."""
        torch = self.torch
        columns = self.flat(grid).T.contiguous().to(torch.float64)
        energy = self.energy_device(columns)
        out = torch.zeros((columns.shape[0],) + self.padded, dtype=torch.float64, device=self.device)
        out[:, :self.shape[0], :self.shape[1], :self.shape[2]] = energy.reshape((-1,) + self.shape)
        return out

    def energy_device(self, columns, combination=None, coefficients=None, scale=None, out=None, accumulate=False):
        """Element energies on device columns [R, ndof].

        Without ``coefficients`` returns per-column energies [R, nelem].  With
        ``coefficients`` returns the weighted sum  scale * sum_j c_j w_j^T K0 w_j
        with w_j = columns[j] (``combination`` None) or w_j = sum_r combination[r, j] columns[r].
        """
        torch = self.torch
        count = columns.shape[0]
        per_column = coefficients is None
        if per_column:
            out = torch.empty((count, self.nelem), dtype=torch.float64, device=self.device) if out is None else out
        else:
            out = torch.zeros(self.nelem, dtype=torch.float64, device=self.device) if out is None else out
        comb = None if combination is None else torch.as_tensor(combination, dtype=torch.float64, device=self.device).contiguous()
        coef = None if coefficients is None else torch.as_tensor(coefficients, dtype=torch.float64, device=self.device).contiguous()
        ncomb = 0 if comb is None else comb.shape[1]
        _lib.check(self.lib.tf_element_energy(self.handle, _lib.ptr(columns), count, _lib.ptr(comb), ncomb, _lib.ptr(coef),
                                              _lib.ptr(scale), _lib.ptr(out), 1 if accumulate else 0,
                                              1 if per_column else 0, self._stream()), self.handle, "tf_element_energy")
        return out

    # ----------------------------------------------------------- lifecycle --
    # -------------------------------------------------------------- modes --
    def mass_device(self, columns, key, fixed, mass, lumped=None, out=None):
        """y = mask (sum_e mass_e M0 u_e + lumped u) on [R, ndof] device columns (tf_mass_apply)."""
        if self.me64 is None:
            raise ValueError("mass operator needs the element mass matrix (me) at construction")
        out = self.torch.empty_like(columns) if out is None else out
        ident = self._key((key, False), fixed)
        _lib.check(self.lib.tf_mass_apply(self.handle, ident, _lib.ptr(mass), _lib.ptr(lumped), _lib.ptr(columns), columns.shape[0],
                                          _lib.ptr(out), self._stream()), self.handle, "tf_mass_apply")
        return out

    def eigenpairs(self, key, fixed, mass, lumped, count, initial=None):
        """Lowest ``count`` eigenpairs of K v = lambda M v by LOBPCG preconditioned with the V-cycle.

        The reference's GeometricMultigrid.eigenpairs (topology_multigrid.py:488-534): a block of
        count + eigen_guard vectors, SVQB M-orthonormalisation, Rayleigh-Ritz on [X, W, P], search
        directions only for the columns above eigen_tolerance, explicit re-application of K and M every
        eigen_refresh steps and before convergence is accepted.  ``mass`` are element masses [nelem],
        ``lumped`` nodal masses [ndof] (or None); ``initial`` a [count + eigen_guard, ndof] block to
        start from (e.g. the previous design's vectors).  Returns (values[:count] as NumPy, the device
        vectors [count + eigen_guard, ndof] M-orthonormal, report).  The small dense Gram and Ritz
        problems are solved on the host in FP64; K, M, the V-cycle and the block products run on the
        device."""
        torch = self.torch
        torch.cuda.synchronize(self.device)
        started = perf_counter()
        settings, tolerance, drop = self.settings, float(self.settings["eigen_tolerance"]), float(self.settings["eigen_drop"])
        if self.moduli is None:
            raise ValueError("update(moduli) must be called before eigenpairs")
        hierarchy = self.hierarchy((key, False), fixed)
        ident = hierarchy["id"]
        dev = lambda v: torch.as_tensor(np.ascontiguousarray(np.asarray(v, dtype=float).ravel()), device=self.device)
        mass = dev(mass)
        if mass.numel() != self.nelem:
            raise ValueError(f"expected {self.nelem} element masses")
        lumped = None if lumped is None else dev(lumped)
        if lumped is not None and lumped.numel() != self.ndof:
            raise ValueError(f"expected {self.ndof} lumped nodal masses")
        ones = torch.ones((1, self.ndof), dtype=torch.float64, device=self.device)
        zero_mass = torch.zeros_like(mass)
        mask = self.mass_device(ones, key, fixed, zero_mass, ones[0])[0]        # the hierarchy's live-dof mask (0 / 1)

        def apply(v):
            v = (v * mask).contiguous()
            return [v, self.apply_device(v, key, fixed), self.mass_device(v, key, fixed, mass, lumped)]

        def gram(a, b):
            return (a @ b.T).cpu().numpy()

        def combine(blocks, coefficients):
            c = torch.as_tensor(coefficients, device=self.device)
            return [c.T @ block for block in blocks]

        def norms(blocks):
            return (blocks[0] * blocks[2]).sum(1).cpu().numpy()

        def svqb(blocks, reference=None):
            g = gram(blocks[0], blocks[2])
            g = (g + g.T) / 2
            diagonal = np.diag(g).copy()
            limit = drop * (diagonal.max() if reference is None else reference)
            live = diagonal > limit
            coefficients = np.zeros((len(diagonal), 0))
            if live.any():
                scale = 1 / np.sqrt(diagonal[live])
                values, rotation = np.linalg.eigh(scale[:, None] * g[np.ix_(live, live)] * scale[None, :])
                keep = values > drop * values.max()
                coefficients = np.zeros((len(diagonal), int(keep.sum())))
                coefficients[live] = scale[:, None] * rotation[:, keep] / np.sqrt(values[keep])
            return combine(blocks, coefficients)

        def project(blocks, basis):
            c = basis[2] @ blocks[0].T
            return [block - c.T @ base for block, base in zip(blocks, basis)]

        def rayleigh(blocks, size):
            stiffness, g = gram(blocks[0], blocks[1]), gram(blocks[0], blocks[2])
            values, rotation = np.linalg.eigh((g + g.T) / 2)
            basis = rotation[:, values > drop * values.max()]
            basis = basis / np.sqrt(np.diag(basis.T @ g @ basis))
            reduced = basis.T @ stiffness @ basis
            values, inner = np.linalg.eigh((reduced + reduced.T) / 2)
            return values[:size], basis @ inner[:, :size]

        def residual(blocks, values):
            v = torch.as_tensor(values, device=self.device)
            r = blocks[1] - v[:, None] * blocks[2]
            return r, (torch.linalg.vector_norm(r, dim=1) / torch.linalg.vector_norm(blocks[1], dim=1)).cpu().numpy()

        size = int(count) + int(settings["eigen_guard"])
        if initial is None or tuple(initial.shape) != (size, self.ndof):
            generator = torch.Generator(device=self.device).manual_seed(int(settings["eigen_seed"]))
            initial = torch.rand((size, self.ndof), generator=generator, device=self.device, dtype=torch.float64) - 0.5
        blocks = svqb(apply(torch.as_tensor(initial, dtype=torch.float64, device=self.device)))
        values, rotation = rayleigh(blocks, size)
        current, previous, step, history = combine(blocks, rotation), None, 0, []
        while True:
            res, relative = residual(current, values)
            if step % settings["eigen_refresh"] == 0 or bool((relative[:count] < tolerance).all()):
                current = apply(current[0])
                res, relative = residual(current, values)
            history.append(float(relative[:count].max()))
            if bool((relative[:count] < tolerance).all()) or step >= settings["eigen_iterations"]:
                break
            active = torch.as_tensor(np.flatnonzero(relative >= tolerance), device=self.device)
            z = torch.empty_like(res)
            _lib.check(self.lib.tf_precondition(self.handle, ident, _lib.ptr(res.contiguous()), res.shape[0], _lib.ptr(z), self._stream()),
                       self.handle, "tf_precondition")
            search = apply(z[active])
            search = svqb(project(project(search, current), current), norms(search))
            parts = [current, search]
            if previous is not None:
                reference = norms(previous)
                previous = svqb(project(project(project(previous, current), search), search), reference)
                if previous[0].shape[0]:
                    parts.append(previous)
            blocks = [torch.cat(group) for group in zip(*parts)]
            values, rotation = rayleigh(blocks, size)
            current = combine(blocks, rotation)
            rotation[:size] = 0
            previous = combine(blocks, rotation)
            step += 1
        blocks = svqb(apply(current[0]))
        values, rotation = rayleigh(blocks, size)
        current = combine(blocks, rotation)
        relative = residual(current, values)[1]
        torch.cuda.synchronize(self.device)
        report = {"iterations": step, "relative_residual": relative[:count].tolist(), "converged": bool((relative[:count] < tolerance).all()),
                  "history": history, "seconds": perf_counter() - started, "setup_s": hierarchy.pop("setup_s", 0.0),
                  "levels": len(hierarchy["levels"]), "coarsest_dofs": hierarchy["coarsest"]["dofs"], "kernel": None,
                  "lambda_max": [level.lambda_max for level in hierarchy["levels"][:-1]]}
        self.statistics.append(report)
        return values[:count].copy(), current[0], report

    def diagnostics(self):
        return {"settings": self.settings, "levels": [{"shape": list(level.shape), "spacing_mm": level.spacing.tolist()} for level in self.levels],
                "padded_shape": list(self.padded), "solves": self.statistics[-64:]}

    def close(self):
        """Release the native handle; returns the list of cleanup errors (always empty or one entry)."""
        errors = []
        if getattr(self, "handle", None):
            try:
                status = self.lib.tf_destroy(self.handle)
                if status:
                    message = (self.lib.tf_last_error(None) or b"").decode(errors="replace")
                    errors.append(f"tf_destroy failed ({_lib.STATUS.get(status, status)}): {message}")
            except Exception as error:  # pragma: no cover - defensive
                errors.append(str(error))
            self.handle = None
        return errors

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_batch_device(jobs):
    """Several independent solves at once (tf_solve_batch): every PCG and V-cycle stage runs as one
    launch over all of them.  ``jobs`` = [(multigrid, key, fixed, forces)], one GeometricMultigrid
    (its own handle) per job, forces a contiguous CUDA float64 [R, ndof] tensor; returns
    [(u [R, ndof], report)] in job order, each what that job's solve_device would return.  The
    instances share the element stiffness and the V-cycle settings and run the FP64 PCG."""
    if not jobs:
        return []
    torch = jobs[0][0].torch
    started = perf_counter()
    count = len(jobs)
    handles = (ctypes.c_void_p * count)()
    keys = (ctypes.c_uint64 * count)()
    forces_p = (ctypes.c_void_p * count)()
    outs_p = (ctypes.c_void_p * count)()
    nrhs = (ctypes.c_int32 * count)()
    reports = (_lib.TfReport * count)()
    outs, arrays = [], []
    seen = set()
    for i, (mg, key, fixed, forces) in enumerate(jobs):
        if id(mg) in seen:
            raise ValueError("each job needs its own GeometricMultigrid")
        seen.add(id(mg))
        mg._check_forces(forces)
        keys[i] = mg._key((key, False), fixed)
        handles[i] = mg.handle
        out = torch.empty_like(forces)
        outs.append(out)
        forces_p[i] = _lib.ptr(forces)
        outs_p[i] = _lib.ptr(out)
        nrhs[i] = forces.shape[0]
        report, held = mg._report_arrays(forces.shape[0])
        reports[i] = report
        arrays.append(held)
    lib = jobs[0][0].lib
    _lib.check(lib.tf_solve_batch(handles, keys, count, forces_p, nrhs, outs_p, reports, jobs[0][0]._stream()), None,
               "tf_solve_batch")
    return [(outs[i], jobs[i][0]._result(reports[i], arrays[i], started)) for i in range(count)]


def solve_elasticity(system, multigrid, physical_density, penalization=3.0, min_stiffness_ratio=1e-6):
    """Compliance, sensitivity and displacement fields of every static case of ``system`` with the
    device multigrid (the reference's module-level solve_elasticity, topology_multigrid.py:553-581):
    one batched solve per fixture group, the parts of a case summed with the half-model factor."""
    moduli, slope = system.moduli(physical_density, penalization, min_stiffness_ratio)
    multigrid.update(moduli)
    factor = 2.0 if system.symmetry is not None else 1.0
    results = {}
    for members in system.groups.values():
        held = members[0][1]["fixed"]
        u, report = multigrid.solve_device(held.tobytes(), held, multigrid._columns(np.column_stack([part["force"] for _, part in members])))
        energies = multigrid.energy_device(u).cpu().numpy()
        host = u.cpu().numpy()
        for column, (case, part) in enumerate(members):
            entry = results.get(case["name"])
            if entry is None:
                entry = results[case["name"]] = {"compliance_n_mm": 0.0, "energy": np.zeros(system.nelem), "relative_residual": 0.0,
                                                 "iterations": [], "fields": {}}
            entry["compliance_n_mm"] += factor * float(host[column] @ part["force"])
            entry["energy"] += factor * energies[column]
            entry["relative_residual"] = max(entry["relative_residual"], report["relative_residual"][column])
            entry["iterations"].append(report["iterations"][column])
            entry["fields"][part["sign"]] = host[column]
    for entry in results.values():
        entry["derivative"] = -slope * entry.pop("energy")
    return results
