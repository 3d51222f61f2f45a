"""Generate the golden fixtures of tests/golden/ from the reference's own Python code.

Run where the reference source tree is available, passing its path (required):

    python tests/golden/make_golden.py PATH_TO_REFERENCE [--only=NAME,...] [--skip-config1]

The reference tree is copied to a scratch directory (its mount is read-only and
pytest/pycache write files), imported, and run on the CPU: SciPy SuperLU for the
direct solves, CPU torch for the reference's matrix-free operator and its
density filter, and the reference's InterfaceCovariance for tr / lambda_max.
Nothing under tests/ reads the reference at test time; only these .npz files.
"""
import json
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def load_reference(source):
    scratch = Path(tempfile.mkdtemp(prefix="refcopy_"))
    for name in ("deep_frame", "tests", "tools"):
        shutil.copytree(Path(source) / name, scratch / name, ignore=shutil.ignore_patterns("__pycache__"))
    sys.path.insert(0, str(scratch))
    import deep_frame.topology_optimization as topt
    import deep_frame.topology_multigrid as tmg
    import deep_frame.topology_problem as tprob
    return topt, tmg, tprob


def box(lo, hi):
    return {"kind": "box", "min_mm": list(map(float, lo)), "max_mm": list(map(float, hi))}


def cantilever_domain(shape):
    """The unit-voxel cantilever of the benchmark: x = 0 face clamped, unit -z load at node (Ex, Ey/2, 0)."""
    ex, ey, ez = shape
    t = 1e-6
    allowed = np.ones(shape, dtype=bool)
    return {"grid": {"shape": list(shape), "spacing_mm": [1.0, 1.0, 1.0], "origin_mm": [0.0, 0.0, 0.0], "order": "C", "axis_order": "xyz"},
            "allowed": allowed, "preserve": np.zeros(shape, dtype=bool), "forbidden": ~allowed,
            "material": {"young_modulus_mpa": 1.0, "poisson_ratio": 0.3, "density_g_cm3": 1.0},
            "point_masses": [],
            "load_cases": [{"name": "tip", "analysis": "static", "fixed_regions": [box([-t, -t, -t], [t, ey + t, ez + t])],
                            "loads": [{"region": box([ex - t, ey // 2 - t, -t], [ex + t, ey // 2 + t, t]), "force_n": [0.0, 0.0, -1.0]}]}]}


def hex8(topt):
    out = {}
    for name, spacing in (("unit", (1.0, 1.0, 1.0)), ("aniso", (2.0, 3.0, 4.0)), ("beam", (0.747, 0.753, 0.667))):
        k, m, b = topt.hexahedron_matrices(spacing, 0.3)
        out[f"{name}_spacing"] = np.asarray(spacing)
        out[f"{name}_k0"], out[f"{name}_m0"], out[f"{name}_b"] = k, m, b
    np.savez_compressed(OUT / "hex8.npz", **out)


def operator(topt, tmg, tprob):
    """Reference matrix-free operator (CPU torch) and assembled matrix products on the reference test domains."""
    import torch
    out = {}
    from tests.test_topology_problem import tiny_domain
    for name, domain in (("cantilever", tprob.cantilever_domain((8, 3, 5), 1.0)), ("tiny", tiny_domain())):
        system = topt.HexElasticity(domain, linear_solver="cpu_superlu")
        rng = np.random.default_rng(0)
        density = np.clip(rng.uniform(0.3, 1.2, system.nelem), 0, 1)
        moduli = system.young * (1e-6 + (1 - 1e-6) * density ** 3)
        active = np.where(system.active_elements, moduli, 0)
        mg = tmg.GeometricMultigrid(domain["grid"]["shape"], system.spacing, system.ke, {"device": "cpu", "coarsest_dofs": 200})
        mg.update(active)
        vectors = np.random.default_rng(1).normal(size=(system.ndof, 2))
        vectors[np.setdiff1d(np.arange(system.ndof), system.active_dofs)] = 0
        matrix = system.matrix(moduli).tocsr()
        part = next(iter(system.groups.values()))[0][1]
        masked = np.zeros_like(vectors)
        masked[part["free"]] = vectors[part["free"]]
        with torch.no_grad():
            full = mg.flat(mg.operator(mg.grid(vectors))).cpu().numpy()
            reduced = mg.flat(mg.operator(mg.grid(masked), mask=mg.mask(part["fixed"])[0])).cpu().numpy()
        shape = tuple(domain["grid"]["shape"])
        energy = mg.element_energy(mg.grid(vectors))[:, :shape[0], :shape[1], :shape[2]].reshape(2, -1).cpu().numpy()
        out.update({f"{name}_shape": np.asarray(shape), f"{name}_spacing": system.spacing, f"{name}_ke": system.ke,
                    f"{name}_moduli": active, f"{name}_vectors": vectors, f"{name}_assembled": matrix @ vectors,
                    f"{name}_operator": full, f"{name}_fixed": part["fixed"], f"{name}_free": part["free"],
                    f"{name}_reduced": reduced, f"{name}_reduced_expected": matrix[part["free"]][:, part["free"]] @ vectors[part["free"]],
                    f"{name}_energy": energy})
    np.savez_compressed(OUT / "operator.npz", **out)


def direct(topt, shape, seed, name):
    """Reference SuperLU compliance / sensitivities / displacement of the unit-voxel cantilever."""
    domain = cantilever_domain(shape)
    system = topt.HexElasticity(domain, linear_solver="cpu_superlu")
    rho = np.random.default_rng(seed).uniform(0.01, 1.0, system.nelem)
    result = system.solve(rho, 3.0, 1e-9, metrics=True)["tip"]
    part = system.groups[next(iter(system.groups))][0][1]
    fields = result.get("fields")
    out = {"shape": np.asarray(shape), "seed": seed, "density": rho, "compliance": result["compliance_n_mm"],
           "derivative": result["derivative"], "relative_residual": result["relative_residual"],
           "max_displacement": result["max_displacement_mm"], "fixed": part["fixed"], "force": part["force"]}
    if fields is None:
        system2 = topt.HexElasticity(domain, linear_solver="cpu_superlu")
        moduli = 1e-9 + (1 - 1e-9) * rho ** 3
        matrix = system2.matrix(moduli).tocsc()
        free = part["free"]
        from scipy.sparse.linalg import splu
        u = np.zeros(system2.ndof)
        u[free] = splu(matrix[free][:, free].tocsc(), permc_spec="MMD_AT_PLUS_A", options={"SymmetricMode": True}).solve(part["force"][free])
        fields = {1.0: u}
    if int(np.prod(shape)) <= 4096:
        out["displacement"] = next(iter(fields.values()))
    np.savez_compressed(OUT / f"{name}.npz", **out)


def density_filter(topt):
    """Reference sparse cone filter: sums, filtered field and pullback (topology_optimization.py:1094-1178)."""
    from tests.test_topology_optimization import beam_domain
    out = {}
    cases = {"beam": ((14, 11, 9), (0.747, 0.753, 0.667), 2.84, 4.0, 0.2), "unit": ((12, 10, 6), (1.0, 1.0, 1.0), 1.5, 0.0, 0.0)}
    for name, (shape, spacing, radius, beta, forbid) in cases.items():
        domain = beam_domain(shape, spacing)
        allowed = np.random.default_rng(3).uniform(size=shape) >= forbid
        allowed[0] = allowed[-1] = True
        preserve = np.zeros(shape, dtype=bool)
        preserve[0] = True
        domain.update(allowed=allowed, forbidden=~allowed, preserve=preserve & allowed)
        mapping = topt.DensityMap(domain, topt._settings({"filter_radius_mm": radius, "projection_beta": beta, "density_filter": "sparse"}))
        rng = np.random.default_rng(5)
        design, sensitivity = rng.uniform(size=allowed.size), rng.normal(size=allowed.size)
        physical, projection = mapping.physical(design)
        out.update({f"{name}_shape": np.asarray(shape), f"{name}_spacing": np.asarray(spacing), f"{name}_radius": radius,
                    f"{name}_beta": beta, f"{name}_allowed": allowed.ravel(), f"{name}_preserve": (preserve & allowed).ravel(),
                    f"{name}_design": design, f"{name}_sensitivity": sensitivity, f"{name}_sums": mapping.sums,
                    f"{name}_filtered": mapping.filtered(design), f"{name}_physical": physical, f"{name}_projection": projection,
                    f"{name}_pullback": mapping.pullback(sensitivity, projection)})
    np.savez_compressed(OUT / "filter.npz", **out)


def covariance(topt, tprob):
    """Reference InterfaceCovariance on the covariance cantilever half model: tr, lambda_max and their gradients."""
    shape = (16, 3, 6)
    domain, problem = tprob.covariance_cantilever(shape, limits={"mean_n_mm": 1.0, "worst_n_mm": 1.0})
    problem["covariance"]["ks"] = 50.0
    tp = tprob.TopologyProblem(domain, problem)
    density = np.random.default_rng(3).uniform(0.3, 1.0, int(np.prod(shape)))
    rows = {row["name"]: row for part in tp.physics(density)[:2] for row in part}
    cov = tp.covariance
    system = tp.system
    # the per-case force pairs and the registered parts (sign, fixed) the reference solves
    forces = {f"force_{k}_{'p' if sign > 0 else 'm'}": v for k, f in enumerate(cov.forces) for sign, v in f.items()}
    parts = {}
    for key, members in system.groups.items():
        sign = members[0][1]["sign"]
        parts[f"fixed_{'p' if sign > 0 else 'm'}"] = members[0][1]["fixed"]
    out = {"shape": np.asarray(shape), "density": density, "sigma": np.asarray(cov.sigma), "directions": cov.directions,
           "factor": cov.factor, "rank": cov.rank, "load_mean": rows["load_mean"]["value"], "load_worst": rows["load_worst"]["value"],
           "ks": rows["load_worst"]["info"]["ks_n_mm"], "grad_mean": rows["load_mean"]["gradient"],
           "grad_worst": rows["load_worst"]["gradient"], "ke": system.ke, "penalization": 3.0, "min_stiffness_ratio": 1e-6,
           "young": system.young, **forces, **parts}
    # the inputs themselves, so the product's own set-up (wrench forces, mirror parts, fixed sets) can be
    # rebuilt from them and compared with the reference's
    keep = ("grid", "symmetry", "material", "load_cases", "interfaces", "point_masses")
    out["domain_json"] = json.dumps({k: domain[k] for k in keep})
    for name in ("allowed", "preserve", "forbidden"):
        out[f"domain_{name}"] = np.asarray(domain[name])
    out["info_json"] = json.dumps(rows["load_worst"]["info"])
    settings = problem["covariance"]
    out["covariance_json"] = json.dumps({"support": settings["support"], "sigma": np.asarray(settings["sigma"]).tolist(),
                                         "labels": settings["labels"], "prefix": settings["prefix"], "ks": settings["ks"],
                                         "ks_cutoff": settings["ks_cutoff"],
                                         "limits": {k: settings["limits"][k] for k in ("mean_n_mm", "worst_n_mm")}})
    np.savez_compressed(OUT / "covariance.npz", **out)
    tp.close()


def optimality_criteria(topt):
    """Reference OC driver runs and standalone _oc_update calls on the reference's beam test domains
    (tests/test_topology_optimization.py:16-35, :139-147, :231-245, :491-535)."""
    import json
    from copy import deepcopy
    from tests.test_topology_optimization import ROBUST_RUN, beam_domain
    out = {}
    runs = {
        "single": ((5, 3, 3), (2.0, 2.0, 2.0), {"volume_fraction": 0.65, "filter_radius_mm": 3.1, "max_iterations": 3, "change_tolerance": 1e-12}),
        "robust": ((8, 4, 4), (1.0, 1.0, 1.0), {**ROBUST_RUN, "volume_fraction": 0.5, "beta_schedule": [1, 4], "beta_interval": 2,
                                                 "beta_minimum_iterations": 2, "max_iterations": 4, "change_tolerance": 1e-12,
                                                 "move_limit_late_beta": 4}),
    }
    for name, (shape, spacing, settings) in runs.items():
        domain = beam_domain(shape, spacing)
        result = topt.optimize_topology(deepcopy(domain), settings)
        assert result["status"] == "ok", result["diagnostics"]
        system = topt.HexElasticity(domain)
        cases = [(case["name"], case["fixed"], case["parts"][0]["force"]) for case in system.cases if case["analysis"] == "static"]
        out.update({f"{name}_shape": np.asarray(shape), f"{name}_spacing": np.asarray(spacing), f"{name}_settings": json.dumps(settings),
                    f"{name}_ke": system.ke, f"{name}_young": system.young, f"{name}_allowed": domain["allowed"].ravel(),
                    f"{name}_preserve": domain["preserve"].ravel(), f"{name}_case_names": json.dumps([c[0] for c in cases]),
                    f"{name}_density": result["density"].ravel(), f"{name}_design": result["design_density"].ravel(),
                    f"{name}_objective": np.asarray([e["objective"] for e in result["history"]]),
                    f"{name}_compliance": np.asarray([[e["compliances_n_mm"][c[0]] for c in cases] for e in result["history"]]),
                    f"{name}_change": np.asarray([np.nan if e["maximum_design_change"] is None else e["maximum_design_change"] for e in result["history"]])})
        for k, (_, fixed, force) in enumerate(cases):
            out[f"{name}_fixed_{k}"], out[f"{name}_force_{k}"] = fixed, force
        if name == "robust":
            out.update(robust_eroded=result["eroded_density"].ravel(), robust_dilated=result["dilated_density"].ravel(),
                       robust_beta=np.asarray([e["projection_beta"] for e in result["history"]]),
                       robust_move=np.asarray([np.nan if e["move_limit"] is None else e["move_limit"] for e in result["history"]]),
                       robust_volume_target=np.asarray([e["dilated_volume_target"] for e in result["history"]]))
    # standalone updates on the robust map (beta 4) of the 6x4x4 beam
    domain = beam_domain((6, 4, 4), (1.0, 1.0, 1.0))
    mapping = topt.DensityMap(domain, topt._settings({"projection": "robust", "filter_radius_mm": 2.6}))
    mapping.beta = 4.0
    design = np.random.default_rng(5).uniform(0.2, 0.8, mapping.n)
    design[mapping.preserve] = 1
    fields, _ = mapping.fields(design)
    objective = -np.random.default_rng(2).uniform(0.5, 1.5, mapping.n)
    volume = mapping.pullback(np.ones(mapping.n), fields["dilated"][1])
    target = 0.97 * mapping.volume(design)
    out.update(update_design=design, update_objective=objective, update_volume_derivative=volume, update_target=target,
               update_candidate=topt._oc_update(design, objective, volume, mapping, target, mapping.settings, 0.2),
               update_lowest_target=0.5 * mapping.volume(design),
               update_lowest=topt._oc_update(design, objective, volume, mapping, 0.5 * mapping.volume(design), mapping.settings, 0.05),
               update_allowed=domain["allowed"].ravel(), update_preserve=domain["preserve"].ravel())
    np.savez_compressed(OUT / "oc.npz", **out)


def _domain_json(domain):
    """A domain dict as JSON text (boolean masks as nested lists)."""
    import json
    return json.dumps(domain, default=lambda value: value.tolist() if hasattr(value, "tolist") else float(value))


def inertia_relief(topt):
    """Reference inertia-relief cases (free-flying frame, determinate support, d'Alembert loads) solved by
    SuperLU: the tiny half-model domain of tests/test_topology_problem.py:156-172 and the full / half
    relief domain of tests/test_topology_optimization.py:585-612."""
    from tests.test_topology_problem import tiny_domain
    out = {}

    def halves(domain, axis=0):
        """Full (mirror-symmetrised masks) and half (cells on the positive side, symmetry plane at 0) domains."""
        allowed = domain["allowed"] & np.flip(domain["allowed"], axis)
        preserve = (domain["preserve"] | np.flip(domain["preserve"], axis)) & allowed
        full = {**domain, "allowed": allowed, "preserve": preserve, "forbidden": ~allowed}
        n = domain["grid"]["shape"][axis]
        grid = {**domain["grid"], "shape": list(domain["grid"]["shape"]), "origin_mm": list(domain["grid"]["origin_mm"])}
        grid["shape"][axis], grid["origin_mm"][axis] = n // 2, 0.0
        cut = tuple(slice(n // 2, None) if d == axis else slice(None) for d in range(3))
        half = {**full, "grid": grid, "symmetry": {"axis": axis, "plane_mm": 0.0},
                **{key: full[key][cut].copy() for key in ("allowed", "preserve", "forbidden")}}
        return full, half
    shape = (8, 4, 4)
    box = lambda low, high: {"kind": "box", "min_mm": low, "max_mm": high}
    preserve = np.zeros(shape, dtype=bool)
    preserve[[0, -1]] = True
    relief = {"point_masses": [{"region": box([-8.01, -0.01, -0.01], [-5.99, 8.01, 0.01]), "mass_g": 3.0},
                               {"region": box([3.99, 1.99, 7.99], [8.01, 6.01, 8.01]), "mass_g": 5.0}], "preserve_mass_g": 2.0}
    loads = {"thrust": [{"region": box([5.99, -0.01, 7.99], [8.01, 8.01, 8.01]), "force_n": [0.0, 0.0, 2.0]},
                        {"region": box([-8.01, -0.01, 7.99], [-5.99, 8.01, 8.01]), "force_n": [0.0, 0.0, 2.0]}],
             "crash": [{"region": box([1.99, 7.99, 3.99], [6.01, 8.01, 8.01]), "force_n": [0.4, -3.0, 0.5]}]}
    relief_domain = {"grid": {"shape": list(shape), "spacing_mm": [2.0, 2.0, 2.0], "origin_mm": [-8.0, 0.0, 0.0], "order": "C", "axis_order": "xyz"},
                     "allowed": np.ones(shape, dtype=bool), "preserve": preserve, "forbidden": np.zeros(shape, dtype=bool),
                     "material": {"young_modulus_mpa": 4430.0, "poisson_ratio": 0.3, "density_g_cm3": 1.09}, "point_masses": [],
                     "load_cases": [{"name": name, "analysis": "static", "fixed_regions": [], "loads": load, "inertia_relief": relief} for name, load in loads.items()]}
    full, half = halves(relief_domain)
    domains = {"tiny": tiny_domain(), "relief_full": full, "relief_half": half}
    for name, domain in domains.items():
        system = topt.HexElasticity(domain, linear_solver="cpu_superlu")
        density = np.random.default_rng(3).uniform(0.2, 1.0, system.nelem)
        result = system.solve(density, metrics=True)
        out[f"{name}_domain"] = _domain_json(domain)
        out[f"{name}_density"] = density
        out[f"{name}_support"] = system.support[1] if system.support is not None else np.zeros(0, dtype=np.int64)
        names = sorted(result)
        out[f"{name}_cases"] = np.asarray(names)
        for case_name in names:
            entry = result[case_name]
            out[f"{name}_{case_name}_compliance"] = entry["compliance_n_mm"]
            out[f"{name}_{case_name}_derivative"] = entry["derivative"]
            out[f"{name}_{case_name}_max_displacement"] = entry["max_displacement_mm"]
            case = next(c for c in system.cases if c["name"] == case_name)
            if "inertia_relief" in case:
                ir = case["inertia_relief"]
                out[f"{name}_{case_name}_mass_g"] = ir["mass_g"]
                out[f"{name}_{case_name}_center"] = np.asarray(ir["center_of_mass_mm"])
                out[f"{name}_{case_name}_acceleration"] = np.asarray(ir["acceleration_n_per_g"])
            for k, part in enumerate(case["parts"]):
                out[f"{name}_{case_name}_part{k}_fixed"] = part["fixed"]
                out[f"{name}_{case_name}_part{k}_force"] = part["force"]
                out[f"{name}_{case_name}_part{k}_support"] = part["support"]
        system.close()
    np.savez_compressed(OUT / "inertia_relief.npz", **out)


def setup_checksums(forces, fixed, ndof):
    """Compact fingerprints of a covariance set-up: per (direction, sign) force the 2-norm, the sum and
    the dot product with a seeded random vector; per sign the sorted fixed dofs' count, sum and
    weighted sum.  Shared by the fixture writer and the test that rebuilds the set-up."""
    probe = np.random.default_rng(7).standard_normal(ndof)
    out = {}
    for k, parts in enumerate(forces):
        for sign, f in parts.items():
            tag = f"{k}_{'p' if sign > 0 else 'm'}"
            out[f"force_{tag}"] = np.array([np.linalg.norm(f), f.sum(), f @ probe])
    for sign, dofs in fixed.items():
        d = np.sort(np.asarray(dofs, dtype=np.int64))
        out[f"fixed_{'p' if sign > 0 else 'm'}"] = np.array([len(d), d.sum(), (d.astype(float) * probe[d]).sum()])
    return out


def plate_setup(topt, tprob):
    """The reference's host set-up of the benchmark plate (96 x 96 x 16, seed 0): its InterfaceCovariance
    directions and every direction's mirror parts, fingerprinted (the full 84 force vectors would be
    320 MB)."""
    sys.path.insert(0, str(OUT.parents[1]))
    from deep_frame_b200 import problems
    domain, _, cov = problems.plate((96, 96, 16), 0)
    # the reference's HexElasticity wants a static case at construction; one on the same stack fixture
    # (loaded on the battery deck) joins the covariance directions' fixture group without changing them
    stack = domain["load_cases"][0]["fixed_regions"]
    battery = domain["interfaces"]["battery"]["regions"][0]
    domain = dict(domain, load_cases=domain["load_cases"] + [{"name": "probe", "analysis": "static", "fixed_regions": stack,
                                                              "loads": [{"region": battery, "force_n": [0.0, 0.0, -1.0]}]}])
    system = topt.HexElasticity(domain)
    settings = {"support": cov["support"], "sigma": cov["sigma"], "labels": cov["labels"], "prefix": "sigma_"}
    model = tprob.InterfaceCovariance(system, settings, domain["interfaces"])
    fixed = {members[0][1]["sign"]: members[0][1]["fixed"] for members in system.groups.values()}
    out = setup_checksums(model.forces, fixed, system.ndof)
    out.update(rank=model.rank, factor=model.factor, directions=model.directions, ndof=system.ndof)
    np.savez_compressed(OUT / "plate_setup.npz", **out)


def diagnostic_domains():
    """Two beams for the system summary: the OC test beam (fixture, tip and side loads, modes) and a
    beam whose load selectors lose nodes to forbidden cells and to the preserve-adjacent interface
    policy, plus a point selector between nodes that needs the half-voxel expansion."""
    def beam(shape):
        extent = np.array(shape, dtype=float)
        fixture = box([-0.01, -0.01, -0.01], [0.01, extent[1] + 0.01, extent[2] + 0.01])
        preserve = np.zeros(shape, dtype=bool)
        preserve[0] = preserve[-1] = True
        return extent, fixture, {"grid": {"shape": list(shape), "spacing_mm": [1.0, 1.0, 1.0], "origin_mm": [0.0, 0.0, 0.0],
                                          "order": "C", "axis_order": "xyz"},
                                 "allowed": np.ones(shape, dtype=bool), "preserve": preserve, "forbidden": np.zeros(shape, dtype=bool),
                                 "material": {"young_modulus_mpa": 4430.0, "poisson_ratio": 0.3, "density_g_cm3": 1.09}, "point_masses": []}
    extent, fixture, plain = beam((6, 4, 4))
    tip = box([extent[0] - 0.01, -0.01, -0.01], (extent + 0.01).tolist())
    plain["load_cases"] = [{"name": "tip", "analysis": "static", "fixed_regions": [fixture], "loads": [{"region": tip, "force_n": [0.0, 0.0, -1.0]}]},
                           {"name": "side", "analysis": "static", "fixed_regions": [fixture], "loads": [{"region": tip, "force_n": [0.0, 0.6, 0.0]}]},
                           {"name": "modes", "analysis": "modal", "fixed_regions": [fixture]}]
    extent, fixture, filtered = beam((8, 4, 4))
    filtered["allowed"][3:5, :, 3] = False
    filtered["forbidden"] = ~filtered["allowed"]
    top = box([3.99, -0.01, 3.99], [8.01, 4.01, 4.01])
    point = box([7.49, 1.99, 3.99], [7.51, 2.01, 4.01])
    filtered["load_cases"] = [{"name": "deck", "analysis": "static", "fixed_regions": [fixture], "loads": [{"region": top, "force_n": [0.0, 0.0, -1.0]}]},
                              {"name": "point", "analysis": "static", "fixed_regions": [fixture], "loads": [{"region": point, "force_n": [0.0, 1.0, 0.0]}]}]
    return {"plain": (plain, "allowed_adjacent"), "filtered": (filtered, "preserve_adjacent")}


def system_diagnostics(topt):
    """The reference's HexElasticity.diagnostics() on the diagnostic domains, as JSON."""
    out = {}
    for name, (domain, policy) in diagnostic_domains().items():
        system = topt.HexElasticity(domain, interface_node_policy=policy)
        out[name] = json.dumps(system.diagnostics())
    # and the inertia-relief domains of inertia_relief.npz (their cases carry a relief summary)
    for name, domain in relief_domains().items():
        out[name] = json.dumps(topt.HexElasticity(domain).diagnostics())
    np.savez_compressed(OUT / "diagnostics.npz", **out)


def solve_metrics(topt):
    """The reference's metrics records (HexElasticity.solve(..., metrics=True), SuperLU) on the plain
    diagnostic beam and on the mirrored half relief domain, with the seeded densities used."""
    out = {}
    domains = {"plain": diagnostic_domains()["plain"][0], "relief_half": relief_domains()["relief_half"]}
    for name, domain in domains.items():
        system = topt.HexElasticity(domain, linear_solver="cpu_superlu")
        density = np.random.default_rng(5).uniform(0.2, 1.0, system.nelem)
        result = system.solve(density, metrics=True)
        keep = ("max_displacement_mm", "max_von_mises_mpa", "loads", "stiffness_n_per_mm")
        out[f"{name}_density"] = density
        out[f"{name}_metrics"] = json.dumps({case: {key: entry[key] for key in keep} for case, entry in result.items()})
        system.close()
    np.savez_compressed(OUT / "metrics.npz", **out)


def relief_domains():
    """The domains stored in inertia_relief.npz, rebuilt from their JSON text."""
    relief = np.load(OUT / "inertia_relief.npz")
    out = {}
    for name in ("tiny", "relief_full", "relief_half"):
        domain = json.loads(str(relief[f"{name}_domain"]))
        for key in ("allowed", "preserve", "forbidden"):
            domain[key] = np.asarray(domain[key], dtype=bool)
        out[name] = domain
    return out


def main(source):
    """Regenerate every fixture; ``--only NAME[,NAME]`` limits it to the named generators."""
    topt, tmg, tprob = load_reference(source)
    steps = {"hex8": lambda: hex8(topt), "operator": lambda: operator(topt, tmg, tprob),
             "cantilever_small": lambda: direct(topt, (16, 8, 8), 0, "cantilever_small"), "filter": lambda: density_filter(topt),
             "covariance": lambda: covariance(topt, tprob), "oc": lambda: optimality_criteria(topt),
             "inertia_relief": lambda: inertia_relief(topt), "plate_setup": lambda: plate_setup(topt, tprob),
             "diagnostics": lambda: system_diagnostics(topt), "metrics": lambda: solve_metrics(topt),
             "cantilever_48x24x24": lambda: direct(topt, (48, 24, 24), 0, "cantilever_48x24x24")}
    only = next((arg.split("=", 1)[1] for arg in sys.argv if arg.startswith("--only=")), None)
    for name, step in steps.items():
        if only is not None and name not in only.split(","):
            continue
        if name == "cantilever_48x24x24" and "--skip-config1" in sys.argv:
            continue
        step()


if __name__ == "__main__":
    if len(sys.argv) < 2 or sys.argv[1].startswith("--"):
        sys.exit("usage: python tests/golden/make_golden.py PATH_TO_REFERENCE [--only=NAME,...] [--skip-config1]")
    main(sys.argv[1])
