"""Covariance load model on the GPU vs the oracle's direct solves (tr, lambda_max, KS, gradients).

Tolerances follow the target: tr(K^-1 Sigma) and lambda_max within 1e-6 relative,
sensitivities within 1e-5 relative (PCG tolerance 1e-10 here).
"""
import numpy as np
import pytest
from scipy.sparse.linalg import spsolve

from oracle import covariance as ocov
from oracle import operator as op

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_plate_covariance_matches_direct_oracle(cuda, precision):
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    shape = (16, 12, 4)
    domain, density, cov = problems.plate(shape, 3)
    system = HexElasticity(domain, multigrid={"precision": precision, "tolerance": 1e-10, "coarsest_dofs": 300})
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    rows = model.measure_device(density, 3.0, 1e-9)
    moduli, derivative = system.moduli(density, 3.0, 1e-9)
    matrix = op.assemble(shape, system.ke, moduli).tocsc()
    parts = []
    for key, members in system.groups.items():
        forces = np.zeros((system.ndof, model.rank))
        index = {name: k for k, name in enumerate(model.cases)}
        for case, part in members:
            forces[:, index[case["name"]]] = part["force"]
        live = op.live_dofs(shape, moduli, members[0][1]["fixed"])
        u = np.zeros_like(forces)
        u[live] = spsolve(matrix[live][:, live].tocsc(), forces[live])
        parts.append((forces, u))
    ref = ocov.measure(parts, model.factor, shape, system.ke, derivative, ks=50.0)
    got = {row["name"]: row for row in rows}
    assert got["load_mean"]["value"] == pytest.approx(ref["load_mean"], rel=1e-6)
    assert got["load_worst"]["value"] == pytest.approx(ref["load_worst"], rel=1e-6)
    assert got["load_worst"]["info"]["ks_n_mm"] == pytest.approx(ref["ks"], rel=1e-6)
    gm = got["load_mean"]["gradient"].cpu().numpy()
    gw = got["load_worst"]["gradient"].cpu().numpy()
    assert np.linalg.norm(gm - ref["grad_mean"]) < 1e-5 * np.linalg.norm(ref["grad_mean"])
    assert np.linalg.norm(gw - ref["grad_worst"]) < 1e-5 * np.linalg.norm(ref["grad_worst"])
    system.close()


def test_gram_is_reproducible_and_exact(cuda):
    import torch
    from deep_frame_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(0)
    a = torch.as_tensor(rng.normal(size=(42, 100003)), device=cuda)
    b = torch.as_tensor(rng.normal(size=(37, 100003)), device=cuda)
    out = torch.empty((42, 37), dtype=torch.float64, device=cuda)
    scratch = torch.empty(int(lib.tf_gram_scratch_size(42, 37)), dtype=torch.float64, device=cuda)
    results = []
    for _ in range(2):
        _lib.check(lib.tf_gram(_lib.ptr(a), 42, _lib.ptr(b), 37, 100003, _lib.ptr(out), _lib.ptr(scratch), None))
        torch.cuda.synchronize()
        results.append(out.cpu().numpy().copy())
    assert np.array_equal(results[0], results[1])
    expected = a.cpu().numpy() @ b.cpu().numpy().T
    assert np.max(np.abs(results[0] - expected)) < 1e-9 * np.max(np.abs(expected))


def test_combine_matches_host_product(cuda):
    """tf_combine (the per-rank partial U v of the sharded lambda_max gradient) equals the host
    product mixing^T U to FP64 rounding, for more combinations than one 16-wide group."""
    import torch
    from deep_frame_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(1)
    u = rng.normal(size=(21, 50021))
    mixing = rng.normal(size=(21, 19))
    out = torch.empty((19, 50021), dtype=torch.float64, device=cuda)
    u_dev, mixing_dev = torch.as_tensor(u, device=cuda), torch.as_tensor(mixing, device=cuda)
    _lib.check(lib.tf_combine(_lib.ptr(u_dev), 21, 50021, _lib.ptr(mixing_dev), 19, _lib.ptr(out), None))
    expected = mixing.T @ u
    assert np.max(np.abs(out.cpu().numpy() - expected)) < 1e-12 * np.max(np.abs(expected))


@pytest.mark.parametrize("precision,pcg", [("float32", "float64"), ("float64", "float64"), ("float32", "float32")])
def test_benchmark_plate_matches_fp64_oracle(cuda, precision, pcg):
    """The benchmark workload itself (96 x 96 x 16 plate, seed 0, 2 x 42 columns solved to the
    benchmark's 1e-8) against the FP64 oracle of tests/golden/plate_96x96x16.npz (the oracle's
    GMG-PCG to 1e-10; made by tests/golden/make_plate_oracle.py): tr and lambda_max within 1e-6
    relative, both sensitivity fields within 1e-5 relative (2-norm)."""
    from pathlib import Path
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    ref = np.load(Path(__file__).resolve().parent / "golden" / "plate_96x96x16.npz")
    domain, density, cov = problems.plate((96, 96, 16), 0)
    system = HexElasticity(domain, multigrid={"precision": precision, "pcg_precision": pcg, "tolerance": 1e-8})
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    rows = {row["name"]: row for row in model.measure_device(density, 3.0, 1e-9)}
    assert rows["load_mean"]["value"] == pytest.approx(float(ref["tr"]), rel=1e-6)
    assert rows["load_worst"]["value"] == pytest.approx(float(ref["lambda_max"]), rel=1e-6)
    assert rows["load_worst"]["info"]["ks_n_mm"] == pytest.approx(float(ref["ks"]), rel=1e-6)
    for name, key in (("load_mean", "grad_mean"), ("load_worst", "grad_worst")):
        got = rows[name]["gradient"].cpu().numpy()
        assert np.linalg.norm(got - ref[key]) < 1e-5 * np.linalg.norm(ref[key]), name
    system.close()
