"""Parity on the benchmark's largest workloads (too large for a CPU oracle solve).

* The 352 x 352 x 48 plate (18.3 M dofs, 2 x 42 columns to 1e-8): the fast path (FP32
  V-cycle) against the plain FP64 GMG-PCG (FP64 V-cycle) on the same device: tr, lambda_max and
  KS within 1e-6 relative, both sensitivity fields within 1e-5 relative (2-norm).  Each path
  converges on its own FP64 true residual; these are the agreement bars asked of the fast path.
* The 128 x 128 x 24 plate (volume fraction 0.15, cone filter 1.5, move 0.2):
  a fixed number of SIMP + MMA iterations with the FP32 V-cycle and with the FP64 V-cycle give
  final physical densities within 1e-4 max-abs and the same tr history to 1e-6.
The 96 x 96 x 16 plate is held to the FP64 oracle fixture in test_gpu_covariance.py.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(precision):
    import torch
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    domain, density, cov = problems.plate((352, 352, 48), 0)
    system = HexElasticity(domain, multigrid={"precision": precision, "tolerance": 1e-8, "smoother": "chebyshev",
                                              "chebyshev_degree": 1, "growth": 2.0})
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    rows = {row["name"]: row for row in model.measure_device(density, 3.0, 1e-9)}
    out = {"tr": rows["load_mean"]["value"], "lambda_max": rows["load_worst"]["value"], "ks": rows["load_worst"]["info"]["ks_n_mm"],
           "grad_mean": rows["load_mean"]["gradient"].cpu().numpy(), "grad_worst": rows["load_worst"]["gradient"].cpu().numpy()}
    assert system.close() == []
    del rows, model, system
    torch.cuda.empty_cache()
    return out


def test_plate_352_fast_path_agrees_with_plain_fp64(cuda):
    fast = _rows("float32")
    plain = _rows("float64")
    for key in ("tr", "lambda_max", "ks"):
        assert fast[key] == pytest.approx(plain[key], rel=1e-6), key
    for key in ("grad_mean", "grad_worst"):
        assert np.linalg.norm(fast[key] - plain[key]) < 1e-5 * np.linalg.norm(plain[key]), key


def test_plate_128_simp_designs_agree_across_vcycle_precisions(cuda):
    import torch
    from deep_frame_b200 import problems
    from deep_frame_b200.optimize import CovarianceSimp
    domain, _, cov = problems.plate((128, 128, 24), 0)
    designs, histories = {}, {}
    for precision in ("float32", "float64"):
        loop = CovarianceSimp(domain, cov, volume_fraction=0.15, filter_radius=1.5, move=0.2,
                              multigrid={"precision": precision, "tolerance": 1e-8, "smoother": "chebyshev", "chebyshev_degree": 1,
                                         "growth": 2.0})
        x, history = loop.run(8)
        designs[precision] = loop.map.filtered_device(x).cpu().numpy()
        histories[precision] = np.asarray([row["tr"] for row in history])
        loop.close()
        torch.cuda.empty_cache()
    assert np.max(np.abs(designs["float32"] - designs["float64"])) < 1e-4
    assert np.max(np.abs(histories["float32"] / histories["float64"] - 1)) < 1e-6
