"""FP64 oracle values of the benchmark workload: the 96 x 96 x 16 covariance plate, seed 0.

    python tests/golden/make_plate_oracle.py [workers]

Writes tests/golden/plate_96x96x16.npz: tr(K^-1 Sigma), lambda_max, the KS aggregate and both
sensitivity fields of the plate that ``bench.py`` evaluates, from the oracle's FP64 GMG-PCG
(oracle/gmg.py, the restatement of the reference's topology_multigrid.py that
tests/test_oracle_golden.py pins against the reference's own SuperLU results) solved to a true
relative residual of 1e-10 with the reference's default smoother (in FP64 the true residual of
this plate, whose moduli span 1e-9 to 1, floors at 2e-12 to 6e-12 per column, and a column held
below its floor restarts until the flexible PCG diverges, so the target keeps a margin above it),
and the covariance measures
of oracle/covariance.py (topology_problem.py:639-684 of the reference).  A direct solve is out of
reach at 480 k dofs x 84 columns on the CPU, so this tight iterative solve stands in for it.

The columns are solved by a spawn-started pool of single-threaded workers, each with its own
hierarchy of its mirror half.  No GPU is used.
"""
import sys
import time
from concurrent.futures import ProcessPoolExecutor
import multiprocessing as mp
import os
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
ROOT = OUT.parents[1]
SHAPE = (96, 96, 16)
SEED = 0
TOLERANCE = 1e-10


def _solve(task):
    from oracle.gmg import MultigridOracle
    shape, ke, moduli, fixed, forces, settings = task
    mg = MultigridOracle(shape, ke, moduli, fixed, settings)
    u, iterations, relative, _ = mg.solve(forces)
    return u, iterations, relative


def main(workers):
    sys.path.insert(0, str(ROOT))
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    from oracle import covariance as ocov
    domain, density, cov = problems.plate(SHAPE, SEED)
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    moduli, derivative = system.moduli(density, 3.0, 1e-9)
    settings = {"tolerance": TOLERANCE, "max_iterations": 60}
    index = {name: k for k, name in enumerate(model.cases)}
    halves, tasks, owner = [], [], []
    per_half = max(1, workers // len(system.groups))
    for h, members in enumerate(system.groups.values()):
        forces = np.zeros((system.ndof, model.rank))
        for case, part in members:
            forces[:, index[case["name"]]] = part["force"]
        halves.append(forces)
        live_columns = np.flatnonzero(np.abs(forces).max(axis=0) > 0)
        for chunk in np.array_split(live_columns, min(per_half, len(live_columns))):
            tasks.append((SHAPE, system.ke, moduli, members[0][1]["fixed"], np.ascontiguousarray(forces[:, chunk]), settings))
            owner.append((h, chunk))
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    t0 = time.perf_counter()
    with ProcessPoolExecutor(max_workers=len(tasks), mp_context=mp.get_context("spawn")) as pool:
        results = list(pool.map(_solve, tasks))
    print(f"{len(tasks)} workers, {time.perf_counter() - t0:.1f} s", flush=True)
    solutions = [np.zeros_like(f) for f in halves]
    iterations, relative = [], []
    for (h, chunk), (u, it, rel) in zip(owner, results):
        solutions[h][:, chunk] = u
        iterations += [int(i) for i in it]
        relative += [float(r) for r in rel]
    assert max(relative) < TOLERANCE, max(relative)
    parts = list(zip(halves, solutions))
    ref = ocov.measure(parts, model.factor, SHAPE, system.ke, derivative, ks=50.0)
    np.savez_compressed(OUT / "plate_96x96x16.npz", tr=ref["load_mean"], lambda_max=ref["load_worst"], ks=ref["ks"],
                        grad_mean=ref["grad_mean"], grad_worst=ref["grad_worst"], tolerance=TOLERANCE,
                        iterations=np.asarray(iterations), relative=np.asarray(relative))
    print(f"tr {ref['load_mean']!r} lambda_max {ref['load_worst']!r} ks {ref['ks']!r}; PCG iterations "
          f"{min(iterations)}-{max(iterations)}, relative residual <= {max(relative):.2e}")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else len(os.sched_getaffinity(0)))
