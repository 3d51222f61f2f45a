"""Drop-in ``CudaDirectSolver`` (FP64 Cholesky on the device).

Same constructor, methods and attributes as the reference's cuDSS wrapper
(deep_frame/topology_optimization.py:80-244): ``CudaDirectSolver(matrix,
rhs)`` runs the structure analysis, ``solve(matrix, rhs)`` refactors the
values and solves, ``substitute(rhs)`` reuses the factor, ``same_structure``,
``diagnostics`` and ``close() -> list of cleanup errors``; device buffers are
exposed as ``rhs_device`` / ``solution_device``.  The factorisation runs in
libtfb200.so on the (symmetrised) matrix: banded when its band is much smaller
than the dense matrix (a voxel grid's reduced stiffness in its natural order,
bandwidth about 3 (ny + 1)(nz + 1); the band may take up to 96 GB), dense with
an explicit inverse factor otherwise (at most 32768 unknowns).  Invalid input
raises ValueError like the reference; a non-positive-definite matrix raises
RuntimeError.
"""
import ctypes
from time import perf_counter

import numpy as np

from . import _lib


class CudaDirectSolver:
    def __init__(self, matrix, rhs):
        import torch
        self.torch = torch
        self.closed = True
        self.cleanup_errors = []
        self.timings = []
        self.handle = None
        started = perf_counter()
        matrix = matrix.tocsr()
        matrix.sort_indices()
        if matrix.shape[0] != matrix.shape[1] or matrix.nnz > np.iinfo(np.int32).max:
            raise ValueError("direct solver requires a square matrix with 32-bit CSR indices")
        rhs = np.asarray(rhs)
        if rhs.ndim != 2 or rhs.shape[0] != matrix.shape[0] or rhs.shape[1] < 1:
            raise ValueError("direct solver requires a nonempty two-dimensional RHS matching the matrix")
        if not np.all(np.isfinite(matrix.data)) or not np.all(np.isfinite(rhs)):
            raise ValueError("direct solver matrix and RHS must be finite")
        self.lib = _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.shape = matrix.shape
        self.indptr = matrix.indptr.astype(np.int32, copy=True)
        self.indices = matrix.indices.astype(np.int32, copy=True)
        self.row_device = torch.as_tensor(self.indptr, device=self.device)
        self.column_device = torch.as_tensor(self.indices, device=self.device)
        self.values_device = torch.as_tensor(matrix.data.astype(np.float64), device=self.device)
        self.rhs_device = torch.zeros((rhs.shape[1], rhs.shape[0]), dtype=torch.float64, device=self.device)
        self.solution_device = torch.zeros_like(self.rhs_device)
        handle = ctypes.c_void_p()
        _lib.check(self.lib.tf_chol_create(self.shape[0], ctypes.byref(handle)), None, "tf_chol_create")
        self.handle = handle
        self.closed = False
        self.analysis_s = perf_counter() - started

    def _check(self, status, what):
        if status:
            message = (self.lib.tf_chol_last_error(self.handle) or b"").decode()
            raise (ValueError if status == 1 else RuntimeError)(f"{what} failed: {message}")

    def _stream(self):
        return _lib.stream_of(self.device)

    def solve(self, matrix, rhs):
        if self.closed:
            raise RuntimeError("direct solver is closed")
        started = perf_counter()
        matrix = matrix.tocsr()
        matrix.sort_indices()
        if matrix.shape != self.shape or not np.array_equal(matrix.indptr, self.indptr) or not np.array_equal(matrix.indices, self.indices):
            raise ValueError("symbolic reuse requires unchanged sparse structure")
        rhs = np.asarray(rhs)
        if rhs.shape != (self.shape[0], self.rhs_device.shape[0]) or not np.all(np.isfinite(matrix.data)) or not np.all(np.isfinite(rhs)):
            raise ValueError("direct solver requires finite values and an unchanged RHS shape")
        self.values_device.copy_(self.torch.as_tensor(matrix.data.astype(np.float64)))
        t0 = perf_counter()
        self._check(self.lib.tf_chol_factor_csr(self.handle, _lib.ptr(self.row_device), _lib.ptr(self.column_device),
                                                _lib.ptr(self.values_device), self._stream()), "tf_chol_factor_csr")
        self.torch.cuda.synchronize(self.device)
        factor_s = perf_counter() - t0
        t0 = perf_counter()
        solution = self._substitute(rhs)
        self.timings.append({"factor_s": factor_s, "solve_s": perf_counter() - t0, "transfer_factor_solve_s": perf_counter() - started})
        return solution

    def _substitute(self, rhs):
        self.rhs_device.copy_(self.torch.as_tensor(np.ascontiguousarray(np.asarray(rhs, dtype=np.float64).T)))
        self._check(self.lib.tf_chol_solve(self.handle, _lib.ptr(self.rhs_device), self.rhs_device.shape[0],
                                           _lib.ptr(self.solution_device), self._stream()), "tf_chol_solve")
        return self.solution_device.T.cpu().numpy()

    def substitute(self, rhs):
        rhs = np.asarray(rhs)
        if self.closed or rhs.shape != (self.shape[0], self.rhs_device.shape[0]) or not np.all(np.isfinite(rhs)):
            raise ValueError("substitution requires an open solver and a finite RHS of unchanged shape")
        return self._substitute(rhs)

    def same_structure(self, matrix):
        matrix = matrix.tocsr()
        matrix.sort_indices()
        return matrix.shape == self.shape and np.array_equal(matrix.indptr, self.indptr) and np.array_equal(matrix.indices, self.indices)

    def diagnostics(self):
        props = self.torch.cuda.get_device_properties(self.device)
        return {"precision": "float64", "numeric_factorization": "banded or dense blocked Cholesky (sm_100a), chosen by the bandwidth",
                "device_name": props.name, "analysis_s": self.analysis_s, "shape": list(self.shape), "nnz": len(self.indices),
                "device_total_bytes": props.total_memory, "solves": self.timings}

    def close(self):
        if self.closed:
            return self.cleanup_errors.copy()
        try:
            self.torch.cuda.synchronize(self.device)
        except Exception as error:
            self.cleanup_errors.append("CUDA cleanup synchronization: " + str(error))
        try:
            status = self.lib.tf_chol_destroy(self.handle)
            if status:
                message = (self.lib.tf_chol_last_error(None) or b"").decode(errors="replace")
                self.cleanup_errors.append(f"tf_chol_destroy failed ({_lib.STATUS.get(status, status)}): {message}")
        except Exception as error:
            self.cleanup_errors.append(str(error))
        self.handle = None
        self.closed = True
        for name in ("row_device", "column_device", "values_device", "rhs_device", "solution_device"):
            setattr(self, name, None)
        return self.cleanup_errors.copy()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
