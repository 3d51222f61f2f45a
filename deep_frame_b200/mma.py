"""Method of moving asymptotes on the device.

``mmasub`` has the signature and return tuple of ``mmapy.mmasub`` as the
reference calls it (deep_frame/topology_optimizers.py:40,61-63): column
vectors of shape (n, 1) / (m, 1) in, ``(xmma, ymma, zmma, lam, xsi, eta, mu,
zet, s, low, upp)`` out (the dual slacks xsi .. s are not returned by the
device solver and come back as None; the reference uses indices 0, 9, 10).
``MMA`` keeps the n-sized work arrays on the device between steps for callers
that hold x, the gradients and the asymptotes in HBM.
"""
import ctypes

import numpy as np

from . import _lib

DEFAULTS = {"move": 0.5, "asyinit": 0.5, "asydecr": 0.7, "asyincr": 1.2, "asymin": 0.01, "asymax": 10.0,
            "raa0": 1e-5, "albefa": 0.1, "epsimin": 1e-7}


class MMA:
    """Device MMA subproblem solver for n variables and m <= 8 constraints."""

    def __init__(self, m, n, device="cuda"):
        import torch
        self.torch, self.device = torch, torch.device(device)
        self.lib = _lib.load()
        self.m, self.n = int(m), int(n)
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            status = self.lib.tf_mma_create(self.m, self.n, ctypes.byref(handle))
        _lib.check(status, None, "tf_mma_create")
        self.handle = handle
        self.newton_iterations = 0

    def step(self, iteration, x, xmin, xmax, xold1, xold2, df0dx, fval, dfdx, low, upp, a0, a, c, d, **settings):
        """Device tensors x..xold2, df0dx [n], dfdx [m, n], low / upp [n] (updated in place); returns (xnew, y, z, lam)."""
        s = _lib.TfMmaSettings(**{**DEFAULTS, **settings})
        m = self.m
        host = lambda v: np.ascontiguousarray(np.asarray(v, dtype=float).ravel())
        fval, a, c, d = host(fval), host(a), host(c), host(d)
        if not (len(fval) == len(a) == len(c) == len(d) == m):
            raise ValueError("fval, a, c and d must have m entries")
        xnew = self.torch.empty_like(x)
        y, lam = np.zeros(m), np.zeros(m)
        z, newton = ctypes.c_double(), ctypes.c_int32()
        ptr = lambda arr: arr.ctypes.data_as(ctypes.c_void_p)
        status = self.lib.tf_mma_step(self.handle, int(iteration), _lib.ptr(x), _lib.ptr(xmin), _lib.ptr(xmax), _lib.ptr(xold1),
                                      _lib.ptr(xold2), _lib.ptr(df0dx), ptr(fval), _lib.ptr(dfdx), _lib.ptr(low), _lib.ptr(upp),
                                      float(a0), ptr(a), ptr(c), ptr(d), ctypes.byref(s), _lib.ptr(xnew), ptr(y), ctypes.byref(z),
                                      ptr(lam), ctypes.byref(newton), _lib.stream_of(self.device))
        if status:
            message = (self.lib.tf_mma_last_error(self.handle) or b"").decode()
            if status == 1:
                raise ValueError(f"tf_mma_step failed: {message}")
            raise _lib.TfError(status, f"tf_mma_step failed: {message}")
        self.newton_iterations = int(newton.value)
        return xnew, y, float(z.value), lam

    def close(self):
        if getattr(self, "handle", None):
            self.lib.tf_mma_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_solvers = {}


def mmasub(m, n, iter, xval, xmin, xmax, xold1, xold2, f0val, df0dx, fval, dfdx, low, upp, a0, a, c, d, move=0.5, asyinit=0.5,
           asydecr=0.7, asyincr=1.2, asymin=0.01, asymax=10.0, raa0=1e-5, albefa=0.1):
    """Drop-in for mmapy.mmasub on host arrays (the solve runs on the device)."""
    import torch
    device = torch.device("cuda", torch.cuda.current_device())
    key = (int(m), int(n), device.index)
    solver = _solvers.get(key)
    if solver is None:
        solver = _solvers[key] = MMA(m, n, device)
    dev = lambda v: torch.as_tensor(np.array(np.broadcast_to(np.asarray(v, dtype=float).ravel(), (n,))), device=device)
    lo, up = dev(low), dev(upp)
    xnew, y, z, lam = solver.step(iter, dev(xval), dev(xmin), dev(xmax), dev(xold1), dev(xold2), dev(df0dx), fval,
                                  torch.as_tensor(np.ascontiguousarray(np.asarray(dfdx, dtype=float).reshape(m, n)), device=device),
                                  lo, up, a0, a, c, d, move=move, asyinit=asyinit, asydecr=asydecr, asyincr=asyincr, asymin=asymin,
                                  asymax=asymax, raa0=raa0, albefa=albefa)
    col = lambda t: t.cpu().numpy().reshape(-1, 1)
    return (col(xnew), y.reshape(-1, 1), z, lam.reshape(-1, 1), None, None, None, None, None, col(lo), col(up))
