"""The CPU oracle (and the product's host-side element code) against golden vectors
produced by the reference's own code (tests/golden/make_golden.py).  No GPU needed."""
from pathlib import Path

import numpy as np
import pytest
from scipy.sparse.linalg import splu, spsolve

from oracle import covariance as ocov
from oracle import density as oden
from oracle import hex8, operator as op

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden(name):
    path = GOLDEN / f"{name}.npz"
    if not path.exists():
        pytest.fail(f"missing golden fixture {path}")
    return np.load(path)


@pytest.mark.parametrize("name", ["unit", "aniso", "beam"])
def test_hex8_matrices_match_reference(name):
    from deep_frame_b200.elements import hexahedron_matrices
    g = golden("hex8")
    k, m, b = hex8.element_matrices(g[f"{name}_spacing"], 0.3)
    assert np.allclose(k, g[f"{name}_k0"], rtol=0, atol=1e-13 * np.abs(k).max())
    assert np.allclose(m, g[f"{name}_m0"], rtol=0, atol=1e-13 * np.abs(m).max())
    assert np.allclose(b, g[f"{name}_b"], rtol=0, atol=1e-13 * np.abs(b).max())
    k2, m2, b2 = hexahedron_matrices(g[f"{name}_spacing"], 0.3)
    assert np.allclose(k2, g[f"{name}_k0"], rtol=0, atol=1e-13 * np.abs(k).max())
    assert np.allclose(m2, g[f"{name}_m0"], rtol=0, atol=1e-13 * np.abs(m).max())
    assert np.allclose(b2, g[f"{name}_b"], rtol=0, atol=1e-13 * np.abs(b).max())


def test_hex8_known_answers():
    """Six rigid modes and the patch test (reference tests/test_topology_optimization.py:37-54)."""
    from deep_frame_b200.elements import hexahedron_matrices, regular_grid
    k, m, _ = hexahedron_matrices((2.0, 3.0, 4.0), 0.3)
    values = np.linalg.eigvalsh(k)
    assert np.max(np.abs(values[:6])) < 1e-12 and values[6] > 0.01
    points, connectivity, _ = regular_grid({"shape": [1, 1, 1], "spacing_mm": [2.0, 3.0, 4.0], "origin_mm": [0, 0, 0]})
    transform = np.array([[0.01, 0.02, -0.01], [0.03, -0.02, 0.01], [0.04, 0.02, 0.03]])
    u = (points[connectivity[0]] @ transform.T).ravel()
    strain = np.array([transform[0, 0], transform[1, 1], transform[2, 2], transform[0, 1] + transform[1, 0],
                       transform[1, 2] + transform[2, 1], transform[0, 2] + transform[2, 0]])
    from deep_frame_b200.elements import elasticity_matrix
    assert u @ k @ u == pytest.approx(strain @ elasticity_matrix(0.3) @ strain * 24.0, rel=1e-12)
    assert m.sum() == pytest.approx(3 * 24.0, rel=1e-12)


def test_grid_numbering_matches_reference_convention():
    from deep_frame_b200.elements import regular_grid
    points, connectivity, dofs = regular_grid({"shape": [3, 2, 4], "spacing_mm": [1, 1, 1], "origin_mm": [0, 0, 0]})
    conn, odofs = hex8.grid_numbering((3, 2, 4))
    assert np.array_equal(connectivity, conn) and np.array_equal(dofs, odofs)
    assert np.array_equal(points[connectivity[0]], hex8.CORNERS)


@pytest.mark.parametrize("name", ["cantilever", "tiny"])
def test_oracle_operator_matches_reference_operator(name):
    g = golden("operator")
    shape, ke, moduli, vectors = tuple(g[f"{name}_shape"]), g[f"{name}_ke"], g[f"{name}_moduli"], g[f"{name}_vectors"]
    matrix = op.assemble(shape, ke, moduli)
    assembled = matrix @ vectors
    assert np.linalg.norm(assembled - g[f"{name}_assembled"]) < 1e-12 * np.linalg.norm(g[f"{name}_assembled"])
    ebe = op.apply(shape, ke, moduli, vectors)
    assert np.linalg.norm(ebe - g[f"{name}_operator"]) < 1e-12 * np.linalg.norm(g[f"{name}_operator"])
    live = op.live_dofs(shape, moduli, g[f"{name}_fixed"])
    masked = np.zeros_like(vectors)
    masked[live] = vectors[live]
    reduced = op.apply(shape, ke, moduli, masked, mask=live)
    free = g[f"{name}_free"]
    assert np.array_equal(np.flatnonzero(live), free)
    assert np.linalg.norm(reduced[free] - g[f"{name}_reduced"][free]) < 1e-12 * np.linalg.norm(g[f"{name}_reduced_expected"])
    energy = op.element_energy(shape, ke, vectors)
    assert np.max(np.abs(energy - g[f"{name}_energy"])) < 1e-12 * np.max(np.abs(g[f"{name}_energy"]))


def test_oracle_direct_solve_matches_reference_superlu():
    g = golden("cantilever_small")
    shape = tuple(g["shape"])
    k0, _, _ = hex8.element_matrices((1, 1, 1), 0.3)
    moduli, derivative = hex8.simp(g["density"], 3.0, 1e-9)
    live = op.live_dofs(shape, moduli, g["fixed"])
    matrix = op.assemble(shape, k0, moduli).tocsc()
    u = np.zeros(matrix.shape[0])
    u[live] = spsolve(matrix[live][:, live].tocsc(), g["force"][live])
    assert np.linalg.norm(u - g["displacement"]) < 1e-9 * np.linalg.norm(g["displacement"])
    assert g["force"] @ u == pytest.approx(float(g["compliance"]), rel=1e-10)
    sens = -derivative * op.element_energy(shape, k0, u)
    assert np.linalg.norm(sens - g["derivative"]) < 1e-9 * np.linalg.norm(g["derivative"])


@pytest.mark.parametrize("name", ["beam", "unit"])
def test_oracle_filter_matches_reference_sparse_filter(name):
    g = golden("filter")
    mapping = oden.DensityMapOracle(g[f"{name}_shape"], g[f"{name}_spacing"], float(g[f"{name}_radius"]), g[f"{name}_allowed"],
                                    g[f"{name}_preserve"], beta=float(g[f"{name}_beta"]))
    assert np.max(np.abs(mapping.sums.ravel() - g[f"{name}_sums"]) / g[f"{name}_sums"]) < 1e-12
    assert np.max(np.abs(mapping.filtered(g[f"{name}_design"]) - g[f"{name}_filtered"])) < 1e-12
    physical, projection = mapping.physical(g[f"{name}_design"])
    assert np.max(np.abs(physical - g[f"{name}_physical"])) < 1e-12
    assert np.max(np.abs(projection - g[f"{name}_projection"])) < 1e-12
    pull = mapping.pullback(g[f"{name}_sensitivity"], projection)
    assert np.max(np.abs(pull - g[f"{name}_pullback"])) < 1e-12 * np.max(np.abs(g[f"{name}_pullback"]))


def test_oracle_covariance_matches_reference_measure():
    g = golden("covariance")
    shape = tuple(g["shape"])
    moduli, derivative = hex8.simp(g["density"], float(g["penalization"]), float(g["min_stiffness_ratio"]), float(g["young"]))
    k0 = g["ke"]
    matrix = op.assemble(shape, k0, moduli).tocsc()
    rank = int(g["rank"])
    parts = []
    for sign in ("p", "m"):
        ndof = matrix.shape[0]
        # a case whose half has no resolvable force is not registered for that half (topology_optimization.py:453)
        forces = np.column_stack([g[f"force_{k}_{sign}"] if f"force_{k}_{sign}" in g.files else np.zeros(ndof) for k in range(rank)])
        live = op.live_dofs(shape, moduli, g[f"fixed_{sign}"])
        u = np.zeros_like(forces)
        u[live] = spsolve(matrix[live][:, live].tocsc(), forces[live]).reshape(u[live].shape)
        parts.append((forces, u))
    res = ocov.measure(parts, float(g["factor"]), shape, k0, derivative, ks=50.0, limit_worst=1.0)
    assert res["load_mean"] == pytest.approx(float(g["load_mean"]), rel=1e-9)
    assert res["load_worst"] == pytest.approx(float(g["load_worst"]), rel=1e-9)
    assert res["ks"] == pytest.approx(float(g["ks"]), rel=1e-9)
    assert np.linalg.norm(res["grad_mean"] - g["grad_mean"]) < 1e-8 * np.linalg.norm(g["grad_mean"])
    assert np.linalg.norm(res["grad_worst"] - g["grad_worst"]) < 1e-8 * np.linalg.norm(g["grad_worst"])
    assert np.allclose(ocov.directions(g["sigma"]), g["directions"], atol=1e-12 * np.abs(g["directions"]).max())


def test_benchmark_plate_fixture_is_converged():
    """tests/golden/plate_96x96x16.npz (tests/golden/make_plate_oracle.py): every one of the 84
    columns reached the fixture's FP64 tolerance, and the measures are consistent (tr >= lambda_max,
    KS >= lambda_max, sensitivities of energies with a positive SIMP slope are <= 0)."""
    g = golden("plate_96x96x16")
    assert g["relative"].shape == (84,) and np.all(g["relative"] < g["tolerance"]) and g["tolerance"] <= 1e-10
    assert float(g["tr"]) > float(g["lambda_max"]) > 0 and float(g["ks"]) >= float(g["lambda_max"])
    for key in ("grad_mean", "grad_worst"):
        assert g[key].shape == (96 * 96 * 16,) and np.all(np.isfinite(g[key])) and np.all(g[key] <= 0)


def test_product_covariance_setup_matches_reference():
    """The product's host set-up of the covariance model, rebuilt from the reference's own domain and
    settings (stored in the fixture): the same unit-wrench load directions split into the same
    mirror parts with the same fixed dofs (topology_problem.py:584-638 of the reference)."""
    import json
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    g = golden("covariance")
    domain = json.loads(str(g["domain_json"]))
    for name in ("allowed", "preserve", "forbidden"):
        domain[name] = g[f"domain_{name}"]
    settings = json.loads(str(g["covariance_json"]))
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, settings, domain["interfaces"])
    assert model.rank == int(g["rank"]) and model.factor == float(g["factor"])
    assert np.allclose(model.directions, g["directions"], rtol=0, atol=1e-12 * np.abs(g["directions"]).max())
    scale = max(np.abs(g[key]).max() for key in g.files if key.startswith("force_"))
    for k, parts in enumerate(model.forces):
        for sign, force in parts.items():
            key = f"force_{k}_{'p' if sign > 0 else 'm'}"
            assert key in g.files, key
            assert np.allclose(force, g[key], rtol=0, atol=1e-12 * scale), key
    assert sum(len(p) for p in model.forces) == sum(key.startswith("force_") for key in g.files)
    fixed = {members[0][1]["sign"]: members[0][1]["fixed"] for members in system.groups.values()}
    for sign, label in ((1, "p"), (-1, "m")):
        assert np.array_equal(np.sort(fixed[sign]), np.sort(g[f"fixed_{label}"]))


def test_covariance_groups_skip_other_load_cases_of_the_fixture():
    """In the reference's covariance cantilever the static "tip" case shares the support fixture
    with the covariance directions; the device force blocks take the directions' parts only."""
    import json
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    g = golden("covariance")
    domain = json.loads(str(g["domain_json"]))
    for name in ("allowed", "preserve", "forbidden"):
        domain[name] = g[f"domain_{name}"]
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, json.loads(str(g["covariance_json"])), domain["interfaces"])
    assert any(case["name"] == "tip" for members in system.groups.values() for case, _ in members)
    chosen = model.group_members()
    seen = set()
    for key, ks, parts in chosen:
        assert len(ks) == len(parts) >= 1
        for k, part in zip(ks, parts):
            expected = g[f"force_{k}_{'p' if part['sign'] > 0 else 'm'}"]
            assert np.allclose(part["force"], expected, rtol=0, atol=1e-12 * np.abs(expected).max())
            seen.add((int(k), part["sign"]))
    assert len(seen) == sum(key.startswith("force_") for key in g.files)


def test_benchmark_plate_setup_matches_reference():
    """The benchmark plate's 42 load directions and their mirror parts as the product sets them up
    equal the reference's own InterfaceCovariance on the same seeded domain (tests/golden/plate_setup.npz,
    fingerprints per direction and sign: 2-norm, sum, dot with a seeded random vector; fixed sets)."""
    import importlib.util
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    make_golden = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(make_golden)
    g = golden("plate_setup")
    domain, _, cov = problems.plate((96, 96, 16), 0)
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    assert system.ndof == int(g["ndof"]) and model.rank == int(g["rank"]) and model.factor == float(g["factor"])
    assert np.allclose(model.directions, g["directions"], rtol=0, atol=1e-12 * np.abs(g["directions"]).max())
    fixed = {members[0][1]["sign"]: members[0][1]["fixed"] for members in system.groups.values()}
    mine = make_golden.setup_checksums(model.forces, fixed, system.ndof)
    assert set(mine) == {key for key in g.files if key.startswith(("force_", "fixed_"))}
    for key, value in mine.items():
        assert np.allclose(value, g[key], rtol=1e-12, atol=1e-12 * max(1.0, np.abs(g[key]).max())), key


def test_system_diagnostics_match_reference():
    """HexElasticity.diagnostics() on the reference's own diagnostic domains (tests/golden/diagnostics.npz,
    built by make_golden.py) has the reference's keys and values, selector expansions and
    interface-policy filtering included; only the solver records differ by design (the device
    multigrid / Cholesky instead of SuperLU / cuDSS)."""
    import importlib.util
    import json
    from deep_frame_b200.elasticity import HexElasticity
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    make_golden = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(make_golden)
    g = golden("diagnostics")
    solver_keys = {"linear_solver", "requested_linear_solver", "gpu_symbolic_reanalyses", "gpu_solver_residency",
                   "gpu_transient_releases", "gpu_solver_details"}
    cases = dict(make_golden.diagnostic_domains(), **{name: (d, "allowed_adjacent") for name, d in make_golden.relief_domains().items()})
    assert set(cases) == set(g.files)
    for name, (domain, policy) in cases.items():
        expected = json.loads(str(g[name]))
        got = json.loads(json.dumps(HexElasticity(domain, interface_node_policy=policy).diagnostics(), default=lambda v: v.tolist()))
        assert set(got) == set(expected), (name, set(got) ^ set(expected))
        for key in set(expected) - solver_keys:
            assert _same_record(got[key], expected[key]), (name, key)


def _same_record(a, b):
    """Structure, strings and integers equal; floats within 1e-9 relative or 1e-12 absolute."""
    if isinstance(a, dict) and isinstance(b, dict):
        return a.keys() == b.keys() and all(_same_record(a[k], b[k]) for k in a)
    if isinstance(a, list) and isinstance(b, list):
        return len(a) == len(b) and all(_same_record(x, y) for x, y in zip(a, b))
    if isinstance(a, float) or isinstance(b, float):
        return isinstance(a, (int, float)) and isinstance(b, (int, float)) and bool(np.isclose(a, b, rtol=1e-9, atol=1e-12))
    return a == b


def test_host_measure_matches_reference_rows():
    """InterfaceCovariance.matrix / energy / measure on host solutions in HexElasticity.solve's format
    (fields per mirror sign, per-case derivative, modulus derivative) reproduce the reference's own
    rows on its covariance cantilever: tr, lambda_max, KS, both gradients and the info record."""
    import json
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    g = golden("covariance")
    domain = json.loads(str(g["domain_json"]))
    for name in ("allowed", "preserve", "forbidden"):
        domain[name] = g[f"domain_{name}"]
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, json.loads(str(g["covariance_json"])), domain["interfaces"])
    shape = tuple(g["shape"])
    moduli, slope = hex8.simp(g["density"], float(g["penalization"]), float(g["min_stiffness_ratio"]), float(g["young"]))
    matrix = op.assemble(shape, g["ke"], moduli).tocsc()
    solutions = {}
    for members in system.groups.values():
        live = op.live_dofs(shape, moduli, members[0][1]["fixed"])
        lu = splu(matrix[live][:, live].tocsc())
        for case, part in members:
            u = np.zeros(system.ndof)
            u[live] = lu.solve(part["force"][live])
            entry = solutions.setdefault(case["name"], {"fields": {}, "energy": np.zeros(system.nelem)})
            entry["fields"][part["sign"]] = u
            entry["energy"] += model.factor * op.element_energy(shape, g["ke"], u)
    for entry in solutions.values():
        entry.update(derivative=-slope * entry.pop("energy"), modulus_derivative=slope)
    rows = {row["name"]: row for row in model.measure(solutions)}
    assert rows["load_mean"]["value"] == pytest.approx(float(g["load_mean"]), rel=1e-9)
    assert rows["load_worst"]["value"] == pytest.approx(float(g["load_worst"]), rel=1e-9)
    assert rows["load_worst"]["info"]["ks_n_mm"] == pytest.approx(float(g["ks"]), rel=1e-9)
    assert np.linalg.norm(rows["load_mean"]["gradient"] - g["grad_mean"]) < 1e-8 * np.linalg.norm(g["grad_mean"])
    assert np.linalg.norm(rows["load_worst"]["gradient"] - g["grad_worst"]) < 1e-8 * np.linalg.norm(g["grad_worst"])
    info, expected = rows["load_worst"]["info"], json.loads(str(g["info_json"]))
    assert set(info) == set(expected) and info["rank"] == expected["rank"] and info["ks"] == expected["ks"]
    assert np.allclose(info["eigenvalues_n_mm"], expected["eigenvalues_n_mm"], rtol=1e-9)
    assert [label for label, _ in info["worst_wrench"]] == [label for label, _ in expected["worst_wrench"]]
    assert np.allclose([v for _, v in info["worst_wrench"]], [v for _, v in expected["worst_wrench"]], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("name", ["plain", "relief_half"])
def test_solve_metrics_match_reference(name):
    """The metrics record of HexElasticity.solve(..., metrics=True) (per-load mean and directional
    displacement, load stiffness, peak displacement, peak von Mises stress) from the product's host
    code, fed displacements of the oracle's direct solves, equals the reference's own record
    (tests/golden/metrics.npz, SuperLU) on a full beam and on a mirrored half relief domain."""
    import importlib.util
    import json
    from deep_frame_b200.elasticity import HexElasticity
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    make_golden = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(make_golden)
    domain = {"plain": make_golden.diagnostic_domains()["plain"][0], "relief_half": make_golden.relief_domains()["relief_half"]}[name]
    g = golden("metrics")
    expected = json.loads(str(g[f"{name}_metrics"]))
    system = HexElasticity(domain)
    shape = tuple(domain["grid"]["shape"])
    moduli, _ = system.moduli(g[f"{name}_density"], 3.0, 1e-6)
    matrix = op.assemble(shape, system.ke, moduli).tocsc()
    for case in system.cases:
        if case["name"] not in expected:
            continue
        direct, mirror = np.zeros(system.ndof), np.zeros(system.ndof)
        for part in case["parts"]:
            live = op.live_dofs(shape, moduli, part["fixed"])
            u = np.zeros(system.ndof)
            u[live] = spsolve(matrix[live][:, live].tocsc(), part["force"][live])
            direct += u
            mirror += part["sign"] * u
        got = system._metrics([direct] if system.symmetry is None else [direct, mirror], moduli, case)
        want = expected[case["name"]]
        assert got["max_displacement_mm"] == pytest.approx(want["max_displacement_mm"], rel=1e-8)
        assert got["max_von_mises_mpa"] == pytest.approx(want["max_von_mises_mpa"], rel=1e-8)
        assert (got["stiffness_n_per_mm"] is None) == (want["stiffness_n_per_mm"] is None)
        assert len(got["loads"]) == len(want["loads"])
        for a, b in zip(got["loads"], want["loads"]):
            assert a["node_count"] == b["node_count"] and np.allclose(a["force_n"], b["force_n"], rtol=1e-12)
            assert np.allclose(a["mean_displacement_mm"], b["mean_displacement_mm"], rtol=1e-8, atol=1e-12)
            assert a["directional_displacement_mm"] == pytest.approx(b["directional_displacement_mm"], rel=1e-8, abs=1e-14)
