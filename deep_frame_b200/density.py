"""Cone density filter, threshold projection and pullback on the device.

Mirrors the reference's ``ConeFilter`` / ``cone_filter`` / ``DensityMap``
(deep_frame/topology_optimization.py:1071-1195): the same weights
max(r - |offset * h|, 0) between allowed cells, row sums with 1 on forbidden
cells, ``filtered``, ``project`` (single and robust tanh projections),
``physical``, ``fields``, ``volume``, ``pullback`` and the bisection
``initial`` design, and the optimality-criteria update ``_oc_update``
(:1197-1233).  The convolution, its adjoint, the projection, the fused volume
and the whole OC multiplier search run in libtfb200.so; host-array methods keep
the reference's NumPy signatures and the ``*_device`` methods take and return
CUDA tensors.  Corridor blends and prop-disc volume weights of the reference
are not part of this library.
"""
import ctypes

import numpy as np

from . import _lib


class ConeFilter:
    """The reference's convolution filter: x -> allowed * (W (allowed * x)) (no normalisation)."""

    def __init__(self, allowed, shape, spacing, radius, device="cuda"):
        import torch
        self.torch, self.shape = torch, tuple(int(s) for s in shape)
        self.device = torch.device(device)
        self.map = _Filter(np.asarray(allowed, dtype=bool).reshape(self.shape), None, spacing, radius, self.device)
        self.sums = self.map.sums.cpu().numpy()

    def __call__(self, vector):
        torch = self.torch
        x = torch.as_tensor(np.asarray(vector, dtype=float).ravel(), device=self.device)
        # filtered = (W (m x)) m / sums  ->  multiply back by sums
        return (self.map.apply(x) * self.map.sums).cpu().numpy()


class _Filter:
    def __init__(self, allowed, preserve, spacing, radius, device):
        import torch
        self.torch, self.device = torch, device
        self.lib = _lib.load()
        shape = (ctypes.c_int64 * 3)(*allowed.shape)
        spacing = (ctypes.c_double * 3)(*[float(h) for h in spacing])
        allowed_u8 = np.ascontiguousarray(allowed.ravel().astype(np.uint8))
        preserve_u8 = None if preserve is None else np.ascontiguousarray(preserve.ravel().astype(np.uint8))
        handle = ctypes.c_void_p()
        with torch.cuda.device(device):
            status = self.lib.tf_filter_create(shape, spacing, float(radius), allowed_u8.ctypes.data_as(ctypes.c_void_p),
                                               None if preserve_u8 is None else preserve_u8.ctypes.data_as(ctypes.c_void_p),
                                               ctypes.byref(handle))
        _lib.check(status, None, "tf_filter_create")
        self.handle = handle
        self.n = int(allowed.size)
        self.sums = torch.empty(self.n, dtype=torch.float64, device=device)
        self._check(self.lib.tf_filter_sums(self.handle, _lib.ptr(self.sums), _lib.stream_of(device)), "tf_filter_sums")

    def _check(self, status, what):
        if status:
            message = (self.lib.tf_filter_last_error(self.handle) or b"").decode()
            if status == 1:
                raise ValueError(f"{what} failed: {message}")
            raise _lib.TfError(status, f"{what} failed: {message}")

    def apply(self, x, multiplier=None, adjoint=False, out=None):
        out = self.torch.empty_like(x) if out is None else out
        self._check(self.lib.tf_filter_apply(self.handle, _lib.ptr(x), _lib.ptr(multiplier), _lib.ptr(out), 1 if adjoint else 0,
                                             _lib.stream_of(self.device)), "tf_filter_apply")
        return out

    def volume(self, design, beta, eta, robust=False, weights=None, out=None):
        out = self.torch.empty(1, dtype=self.torch.float64, device=self.device) if out is None else out
        self._check(self.lib.tf_filter_volume(self.handle, _lib.ptr(design), _lib.ptr(weights), float(beta), float(eta),
                                              1 if robust else 0, _lib.ptr(out), _lib.stream_of(self.device)), "tf_filter_volume")
        return out

    def oc_update(self, design, objective_derivative, volume_derivative, target, minimum, move, beta, eta, robust, weights=None):
        candidate = self.torch.empty_like(design)
        report = _lib.TfOcReport()
        self._check(self.lib.tf_oc_update(self.handle, _lib.ptr(design), _lib.ptr(objective_derivative), _lib.ptr(volume_derivative),
                                          _lib.ptr(weights), float(target), float(minimum), float(move), float(beta), float(eta),
                                          1 if robust else 0, _lib.ptr(candidate), ctypes.byref(report), _lib.stream_of(self.device)),
                    "tf_oc_update")
        return candidate, {"multiplier": report.multiplier, "lower": report.lower, "volume": report.volume,
                           "evaluations": int(report.evaluations), "lowest": bool(report.lowest)}

    def project(self, filtered, beta, eta, robust=False, derivative=True):
        physical = self.torch.empty_like(filtered)
        deriv = self.torch.empty_like(filtered) if derivative else None
        self._check(self.lib.tf_filter_project(self.handle, _lib.ptr(filtered), float(beta), float(eta), 1 if robust else 0,
                                               _lib.ptr(physical), _lib.ptr(deriv), _lib.stream_of(self.device)), "tf_filter_project")
        return physical, deriv

    def close(self):
        if getattr(self, "handle", None):
            self.lib.tf_filter_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DensityMap:
    """Density mapping x -> filtered -> projected on the device (reference DensityMap, :1110-1195)."""

    def __init__(self, domain, settings, device="cuda"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.settings = settings
        if settings.get("corridor") is not None or settings.get("prop_discs") is not None:
            raise NotImplementedError("corridor blends and prop-disc volume weights are not part of this library")
        self.beta = settings["beta_schedule"][0] if settings.get("beta_schedule") else settings["projection_beta"]
        self.robust = settings.get("projection", "single") == "robust"
        eta, delta = settings["projection_eta"], settings.get("robust_delta", 0.25)
        self.thresholds = {"eroded": eta + delta, "intermediate": eta, "dilated": eta - delta} if self.robust else {"intermediate": eta}
        shape = tuple(domain["grid"]["shape"])
        self.allowed = np.asarray(domain["allowed"], dtype=bool).reshape(shape)
        self.preserve = np.asarray(domain["preserve"], dtype=bool).reshape(shape)
        forbidden = np.asarray(domain["forbidden"], dtype=bool).reshape(shape)
        if not np.array_equal(forbidden, ~self.allowed) or np.any(self.preserve & forbidden):
            raise ValueError("Forbidden must complement allowed; preserve must be allowed")
        self.allowed, self.preserve = self.allowed.ravel(), self.preserve.ravel()
        self.free = self.allowed & ~self.preserve
        self.forbidden = ~self.allowed
        self.n = self.allowed.size
        self.filter = _Filter(self.allowed.reshape(shape), self.preserve.reshape(shape), domain["grid"]["spacing_mm"],
                              settings["filter_radius_mm"], self.device)
        self.sums = self.filter.sums.cpu().numpy()
        self.weights = np.ones(self.n)

    # ------------------------------------------------------------- device --
    def filtered_device(self, design):
        return self.filter.apply(design)

    def project_device(self, filtered, eta):
        return self.filter.project(filtered, self.beta, eta, self.robust)

    def pullback_device(self, sensitivity, projection_derivative):
        return self.filter.apply(sensitivity, projection_derivative, adjoint=True)

    def fields_device(self, design):
        filtered = self.filtered_device(design)
        return {name: self.project_device(filtered, eta) for name, eta in self.thresholds.items()}, filtered

    def volume_eta(self):
        """Threshold of the volume field: dilated for the robust projection, else intermediate."""
        return self.thresholds["dilated"] if self.robust else self.settings["projection_eta"]

    def volume_device(self, design):
        return float(self.filter.volume(design, self.beta, self.volume_eta(), self.robust).item())

    def oc_update_device(self, design, objective_derivative, volume_derivative, target, move_limit):
        """Device ``_oc_update``: (candidate tensor, search report)."""
        for name, value in (("design", design), ("objective_derivative", objective_derivative), ("volume_derivative", volume_derivative)):
            if value.dtype != self.torch.float64 or value.numel() != self.n or not value.is_contiguous() or value.device != self.device:
                raise ValueError(f"{name} must be a contiguous float64 tensor of {self.n} cells on {self.device}")
        return self.filter.oc_update(design, objective_derivative, volume_derivative, target,
                                     self.settings["minimum_design_density"], move_limit, self.beta, self.volume_eta(), self.robust)

    # --------------------------------------------------------------- host --
    def _host(self, tensor):
        return tensor.cpu().numpy()

    def _dev(self, array):
        return self.torch.as_tensor(np.ascontiguousarray(np.asarray(array, dtype=float).ravel()), device=self.device)

    def filtered(self, design):
        design = np.asarray(design, dtype=float).ravel()
        if design.size != self.n or not np.all(np.isfinite(design)) or np.any(design < 0) or np.any(design > 1):
            raise ValueError("Design densities must be finite and within [0, 1]")
        return self._host(self.filtered_device(self._dev(design)))

    def project(self, filtered, eta):
        physical, derivative = self.project_device(self._dev(filtered), eta)
        return self._host(physical), self._host(derivative)

    def physical(self, design):
        return self.project(self.filtered(design), self.settings["projection_eta"])

    def fields(self, design):
        filtered = self.filtered(design)
        return {name: self.project(filtered, eta) for name, eta in self.thresholds.items()}, filtered

    def volume(self, design):
        design = np.asarray(design, dtype=float).ravel()
        if design.size != self.n or not np.all(np.isfinite(design)) or np.any(design < 0) or np.any(design > 1):
            raise ValueError("Design densities must be finite and within [0, 1]")
        return self.volume_device(self._dev(design))

    def pullback(self, sensitivity, projection_derivative):
        return self._host(self.pullback_device(self._dev(sensitivity), self._dev(projection_derivative)))

    def initial(self, target):
        """Uniform free density whose physical volume meets ``target`` (preserves at 1), found by 70
        bisection steps from the minimum design density up (topology_optimization.py:1179-1195)."""
        design = np.where(self.preserve, 1.0, 0.0)
        low, high = self.settings["minimum_design_density"], 1.0
        design[self.free] = low
        if self.volume(design) > target + 1e-8:
            raise ValueError("Volume budget cannot contain preserves and their filtered transition")
        for _ in range(70):
            design[self.free] = mid = 0.5 * (low + high)
            low, high = (low, mid) if self.volume(design) > target else (mid, high)
        design[self.free] = low
        return design

    def close(self):
        self.filter.close()


def _oc_update(design, objective_derivative, volume_derivative, mapping, target, settings, move_limit):
    """The reference's ``_oc_update`` (topology_optimization.py:1197-1233) with NumPy arrays, run on the device.

    ``settings["minimum_design_density"]`` must match the mapping's settings; errors raise RuntimeError
    ("Invalid OC sensitivities" / "OC could not bracket the volume multiplier") as in the reference."""
    if settings["minimum_design_density"] != mapping.settings["minimum_design_density"]:
        mapping = _with_minimum(mapping, settings["minimum_design_density"])
    candidate, _ = mapping.oc_update_device(mapping._dev(design), mapping._dev(objective_derivative), mapping._dev(volume_derivative),
                                            target, move_limit)
    return candidate.cpu().numpy()


def _with_minimum(mapping, minimum):
    import copy
    clone = copy.copy(mapping)
    clone.settings = {**mapping.settings, "minimum_design_density": minimum}
    return clone
