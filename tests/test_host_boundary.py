"""Host side of the drop-in boundary on a machine without a CUDA device.  No GPU.

The reference pins "no CPU fallback" (tests/test_topology_optimization.py:406-416): when the GPU
solver cannot run, the OC driver reports status "failed" with the error and an empty history
instead of solving on the CPU, and unknown solver names are "invalid" (:400-404).  The same
holds here, and every device entry point fails loudly before any work.
"""
import numpy as np
import pytest
import torch

from deep_frame_b200 import _lib

no_cuda = pytest.mark.skipif(torch.cuda.is_available(), reason="checks the path of a host without a CUDA device")


def beam_domain(shape=(5, 3, 3), spacing=2.0):
    extent = np.array(shape) * spacing
    return {"grid": {"shape": list(shape), "spacing_mm": [spacing] * 3, "origin_mm": [0.0] * 3, "order": "C", "axis_order": "xyz"},
            "allowed": np.ones(shape, bool), "preserve": np.zeros(shape, bool), "forbidden": np.zeros(shape, bool),
            "material": {"young_modulus_mpa": 4430.0, "poisson_ratio": 0.3, "density_g_cm3": 1.09}, "point_masses": [],
            "load_cases": [{"name": "tip", "analysis": "static",
                            "fixed_regions": [{"kind": "box", "min_mm": [-0.01] * 3, "max_mm": [0.01, extent[1] + 0.01, extent[2] + 0.01]}],
                            "loads": [{"region": {"kind": "box", "min_mm": [extent[0] - 0.01, -0.01, -0.01], "max_mm": (extent + 0.01).tolist()},
                                       "force_n": [0.0, 0.0, -1.0]}]}]}


@no_cuda
def test_oc_driver_fails_without_cpu_fallback():
    from deep_frame_b200.topology_optimization import optimize_topology
    result = optimize_topology(beam_domain(), {"volume_fraction": 0.65, "filter_radius_mm": 3.1})
    assert result["status"] == "failed"
    assert result["history"] == [] and len(result["diagnostics"]) == 1 and result["diagnostics"][0]


def test_unknown_linear_solver_is_invalid():
    from deep_frame_b200.topology_optimization import _settings, optimize_topology
    with pytest.raises(ValueError, match="linear_solver"):
        _settings({"linear_solver": "fake_gpu"})
    result = optimize_topology(beam_domain(), {"linear_solver": "fake_gpu"})
    assert result["status"] == "invalid" and "linear_solver" in result["diagnostics"][0]


@no_cuda
def test_multigrid_refuses_to_run_on_the_cpu():
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    from deep_frame_b200.elements import hexahedron_matrices
    ke = hexahedron_matrices((1.0, 1.0, 1.0), 0.3)[0]
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        GeometricMultigrid((4, 4, 4), (1.0, 1.0, 1.0), ke, {"device": "cpu"})
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        GeometricMultigrid((4, 4, 4), (1.0, 1.0, 1.0), ke)


def test_multigrid_settings_are_validated_and_translated():
    from deep_frame_b200.topology_multigrid import MULTIGRID, _native_settings
    native = _native_settings(dict(MULTIGRID, smoother="jacobi", cycle="W", sweeps=3, tolerance=1e-9, batch=12, tensor_cores=True))
    assert native.smoother == _lib.SMOOTHER["jacobi"] and native.cycle == _lib.CYCLE["W"]
    assert native.sweeps == 3 and native.tolerance == 1e-9 and native.batch == 12 and native.tensor_cores == 1
    assert native.coarsest_dofs == MULTIGRID["coarsest_dofs"] and native.chebyshev_degree == MULTIGRID["chebyshev_degree"]
    for bad in ({"precision": "int8"}, {"smoother": "gauss_seidel"}, {"cycle": "F"}, {"coarse": "algebraic"}):
        with pytest.raises(ValueError, match="Invalid multigrid settings"):
            _native_settings(dict(MULTIGRID, **bad))


def test_missing_library_raises_instead_of_falling_back(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIBRARY", tmp_path / "libtfb200.so")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()


def test_oc_driver_needs_a_static_case():
    """A domain with only a modal case is invalid for the OC driver, as in the reference
    (topology_optimization.py:440-441), and is reported before any device work."""
    from deep_frame_b200.topology_optimization import optimize_topology
    domain = beam_domain()
    domain["load_cases"] = [{"name": "modes", "analysis": "modal", "fixed_regions": domain["load_cases"][0]["fixed_regions"]}]
    result = optimize_topology(domain, {"volume_fraction": 0.65, "filter_radius_mm": 3.1})
    assert result["status"] == "invalid" and result["diagnostics"] == ["Topology optimization requires at least one static case"]
    assert result["history"] == []


def test_close_hands_back_device_errors_instead_of_raising():
    """GeometricMultigrid.close and CudaDirectSolver.close return the errors met while releasing
    their handles (the reference's close returns its collected error strings,
    topology_multigrid.py:543-548 and topology_optimization.py:205-239); a stand-in library whose
    destroy reports a CUDA error plays the device here."""
    from types import SimpleNamespace
    from deep_frame_b200.direct import CudaDirectSolver
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    destroyed = []
    lib = SimpleNamespace(tf_destroy=lambda h: destroyed.append(h) or 2, tf_last_error=lambda h: b"tf_destroy: an illegal memory access was encountered",
                          tf_chol_destroy=lambda h: destroyed.append(h) or 2, tf_chol_last_error=lambda h: b"tf_chol_destroy: unspecified launch failure")
    mg = object.__new__(GeometricMultigrid)
    mg.lib, mg.handle = lib, "multigrid-handle"
    assert mg.close() == ["tf_destroy failed (cuda): tf_destroy: an illegal memory access was encountered"]
    assert mg.handle is None and mg.close() == [] and destroyed == ["multigrid-handle"]

    def failing_sync(device):
        raise RuntimeError("CUDA error: unspecified launch failure")

    solver = object.__new__(CudaDirectSolver)
    solver.lib, solver.handle, solver.closed, solver.cleanup_errors, solver.device = lib, "chol-handle", False, [], None
    solver.torch = SimpleNamespace(cuda=SimpleNamespace(synchronize=failing_sync))
    errors = solver.close()
    assert errors == ["CUDA cleanup synchronization: CUDA error: unspecified launch failure",
                      "tf_chol_destroy failed (cuda): tf_chol_destroy: unspecified launch failure"]
    assert solver.closed and solver.handle is None and solver.close() == errors and destroyed[-1] == "chol-handle"


def test_cleanup_errors_follow_the_primary_error(monkeypatch):
    """When an iteration fails and closing the solver fails too, the outcome is "failed" with the
    original error first and the cleanup error after it (reference
    tests/test_topology_optimization.py:418-427).  Stand-ins replace the device density map and
    elasticity system."""
    import torch
    from deep_frame_b200 import topology_optimization as topo
    closed = []

    class Mapping:
        def __init__(self, domain, settings, device):
            shape = tuple(domain["grid"]["shape"])
            self.allowed, self.preserve = np.ones(shape, bool), np.zeros(shape, bool)
            self.n, self.device, self.beta, self.robust = int(np.prod(shape)), torch.device("cpu"), 1.0, False

        def initial(self, target):
            return np.full(self.n, target / self.n)

        def _dev(self, values):
            return torch.as_tensor(values)

        def fields_device(self, design):
            raise RuntimeError("CUDA solve unavailable in controlled test")

        def close(self):
            closed.append("mapping")

    class System:
        def __init__(self, domain, **kwargs):
            pass

        def close(self):
            closed.append("system")
            return ["cleanup failed in controlled test"]

    monkeypatch.setattr(topo, "DensityMap", Mapping)
    monkeypatch.setattr(topo, "HexElasticity", System)
    result = topo.optimize_topology(beam_domain(), {"volume_fraction": 0.65, "filter_radius_mm": 3.1})
    assert result["status"] == "failed" and result["history"] == []
    assert result["diagnostics"] == ["CUDA solve unavailable in controlled test", "cleanup failed in controlled test"]
    assert closed == ["system", "mapping"]


def test_grid_layout_round_trip():
    """GeometricMultigrid.grid / .flat (the reference's layout helpers, topology_multigrid.py:80-96) on
    the CPU: dof 3 n + c of node n = (i, j, k) lands at [column, c, i, j, k], padding stays zero and
    flat undoes grid."""
    from types import SimpleNamespace
    from deep_frame_b200.topology_multigrid import GeometricMultigrid
    mg = object.__new__(GeometricMultigrid)
    mg.torch, mg.device, mg.nodes = torch, torch.device("cpu"), (3, 2, 4)
    mg.levels = [SimpleNamespace(nodes=(5, 3, 5))]
    flat = np.random.default_rng(0).standard_normal((3 * 3 * 2 * 4, 2))
    grid = mg.grid(flat)
    assert tuple(grid.shape) == (2, 3, 5, 3, 5)
    i, j, k, c, col = 2, 1, 3, 2, 1
    assert grid[col, c, i, j, k].item() == flat[3 * ((i * 2 + j) * 4 + k) + c, col]
    assert not grid[:, :, 3:].any() and not grid[:, :, :, 2:].any() and not grid[..., 4:].any()
    assert np.array_equal(mg.flat(grid).numpy(), flat)
    assert tuple(mg.grid(flat[:, 0]).shape) == (1, 3, 5, 3, 5)
