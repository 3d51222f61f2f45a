"""Benchmark: seconds per 42-RHS covariance hex8 solve to 1e-8 relative residual, fast path vs plain FP64.

One step = one design evaluation of the covariance-load plate half model (default 352 x 352 x 48
voxels, 18 317 523 dofs, mirror symmetry on x = 0): new element moduli, both multigrid hierarchies
rebuilt (symmetric and antisymmetric fixture groups), the 42 load directions of each half solved by
batched GMG-PCG to a recomputed FP64 true relative residual below 1e-8 (84 column solves), then
F = P^T U, tr(K^-1 Sigma), lambda_max and both sensitivity fields.

* ``value``: the fastest path (FP32 V-cycle; with ``--pcg float32`` FP32 inner PCG iterations under
  FP64 reliable residual updates; with ``--tensor-cores`` the finest-level applies on tcgen05), every
  input resident in HBM.
* ``results.plain_fp64``: the same step with the plain FP64 GMG-PCG (FP64 V-cycle, FP64 PCG) on the
  same GPU, its time, the ratio to ``value`` and the agreement of tr, lambda_max and the
  sensitivities between the two paths.
* ``e2e``: the reference-facing ``InterfaceCovariance.measure_device`` call with a host density in
  and both sensitivity fields read back to the host.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--config NAME]
For N > 1 (torchrun, one rank per GPU) the 42 directions of each half are sharded across ranks;
the flexibility columns are gathered with one NCCL all-reduce per solve.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "42-RHS hex8 solve s @1e-8 resid; SIMP iter/s: learned+mixed vs plain FP64"
CONFIG = "plate_352x352x48"
PLATES = ("plate_96x96x16", "plate_128x128x24", "plate_192x192x32", "plate_352x352x48")
#: the smoother schedule the autotuner picks on the 96 x 96 x 16 plate (Chebyshev degree 1, growth 2)
SCHEDULE = "1,2"
#: largest problem the oracle's CPU GMG-PCG is timed on in full (one evaluation = all columns solved)
CPU_MAX_DOFS = 2_000_000


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default=CONFIG, choices=PLATES,
                    help="covariance plate workload (the 48 x 24 x 24 cantilever is a parity case of the tests, not a bench line)")
    ap.add_argument("--precision", default="float32", help="work precision of the fast path's V-cycle")
    ap.add_argument("--pcg", default="float64", choices=["float64", "float32"],
                    help="fast path's PCG iterations: FP64, or FP32 with FP64 reliable residual updates")
    ap.add_argument("--tensor-cores", action="store_true", help="fast path's finest-level V-cycle applies on tcgen05")
    ap.add_argument("--fine-tz", type=int, default=0, choices=[0, 7, 8, 9],
                    help="node-tile height of the finest-level operator in both arms (0: the library's choice)")
    ap.add_argument("--plain-steps", type=int, default=None, help="timed steps of the plain FP64 arm (default min(steps, 3))")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 arm")
    ap.add_argument("--storage-trial", default="", metavar="P1,P2",
                    help="also time the fast path with these V-cycle storage precisions (bfloat16, float16: vectors rounded "
                         "to 16 bits when stored) and report their PCG iterations")
    ap.add_argument("--e2e-steps", type=int, default=None, help="timed steps of the end-to-end leg (default min(steps, 3))")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--autotune", action="store_true", help="pick the smoother schedule with the autotuner instead of --schedule")
    ap.add_argument("--schedule", default=SCHEDULE, metavar="DEGREE,GROWTH", help="Chebyshev smoother schedule of both arms")
    ap.add_argument("--coarsest-dofs", type=int, default=0,
                    help="coarsest-grid size of both arms (default: the library's 8000; the reference's default is 80000, "
                         "factored banded above 24000)")
    ap.add_argument("--instances", type=int, default=0,
                    help="solve N independent seeded plates of uneven size and RHS count concurrently and report solves/s")
    ap.add_argument("--instance-sizes", choices=("plate", "small"), default="plate",
                    help="grids of --instances: 64 x 64 x 12 ... 160 x 160 x 24 with 6-42 columns per half (plate), "
                         "or 16 x 16 x 4 ... 48 x 48 x 8 with 3-12 columns (small)")
    ap.add_argument("--learned", action="store_true", help="train the learned initial guess and report PCG with / without it")
    ap.add_argument("--learned-epochs", type=int, default=4, help="training epochs of --learned")
    ap.add_argument("--simp", type=int, default=0, help="run N SIMP + MMA iterations (default plate 128 x 128 x 24) instead")
    ap.add_argument("--simp-compare", action="store_true", help="also run the plain FP64 V-cycle and compare the designs")
    ap.add_argument("--warm-start", type=int, default=0, nargs="?", const=-1,
                    help="SIMP: start every PCG from the previous design's solution (no value), or from the energy-optimal "
                         "combination of the last M designs' solutions (--warm-start M)")
    return ap.parse_args(argv)


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one 42-column finest-level FP32 residual
# apply of the 96 x 96 x 16 plate (159 953 nodes), from an ncu capture of that launch; other grids are
# scaled by their node count (the kernel's traffic is proportional to nodes x columns)
FINE_TRAFFIC = {"cheb": 434e6, "resid": 220.5e6}
FINE_TRAFFIC_NODES = 159953


def peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), float(data["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


# CUDA-core lanes per SM of sm_100 (FP32 FMA and FP64 FMA) and its SM count: the nominal non-tensor
# peaks are lanes x 2 flop x SMs x SM clock.  No measured figure exists for these pipes.
FMA_LANES = {"fp32": 128, "fp64": 64}
SMS = 148


def fma_roof(precision, flops_per_launch, per_launch_ms, sm_mhz=None, sm_max_mhz=1965.0):
    """Compute side of the dominant kernel's roofline: its algorithmic flops per launch over the
    launch time, against the nominal CUDA-core FMA peak at the maximum SM clock and, when clocks
    were sampled, at the median SM clock seen under load."""
    achieved = flops_per_launch / (per_launch_ms * 1e-3) / 1e12
    lanes = FMA_LANES[precision]
    peak_max = lanes * 2 * SMS * sm_max_mhz * 1e6 / 1e12
    out = {"bound": "fma", "pipe": precision, "achieved": round(achieved, 2), "unit": "TFLOP/s",
           "peak": round(peak_max, 1), "frac": round(achieved / peak_max, 4), "peak_source": "nominal at the maximum SM clock",
           "flops_per_launch": int(flops_per_launch)}
    if sm_mhz:
        peak_seen = lanes * 2 * SMS * sm_mhz * 1e6 / 1e12
        out["peak_at_sampled_clock"] = round(peak_seen, 1)
        out["frac_at_sampled_clock"] = round(achieved / peak_seen, 4)
    return out


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def schedule_settings(text, coarsest_dofs=None):
    degree, growth = text.split(",")
    out = {"smoother": "chebyshev", "chebyshev_degree": int(degree), "growth": float(growth)}
    if coarsest_dofs:
        out["coarsest_dofs"] = int(coarsest_dofs)
    return out


def fast_settings(args):
    return {"precision": args.precision, "pcg_precision": args.pcg, "tensor_cores": bool(args.tensor_cores), "fine_tz": args.fine_tz}


PLAIN = {"precision": "float64", "pcg_precision": "float64", "tensor_cores": False}


def build_problem(config, device, multigrid):
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    spec = problems.CONFIGS[config]
    domain, density, cov = problems.plate(spec["shape"], 0)
    system = HexElasticity(domain, multigrid={"tolerance": spec["tolerance"], "device": str(device), **multigrid})
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    return spec, system, model, density


def rebuild_multigrid(system, multigrid):
    """Close the system's multigrid handle and let the next use build one with ``multigrid`` settings
    (the same grid, element stiffness and fixture groups)."""
    if system.multigrid is not None:
        system.multigrid.close()
        system.multigrid = None
    system.multigrid_settings = {**(system.multigrid_settings or {}), "max_iterations": 2000, "retries": 2, **multigrid}
    system.multigrid_settings.pop("_tuned", None)


def timed_steps(step, steps, warmup, world, dist, device, clocks_index=None):
    """W untimed steps, then K steps bracketed by a barrier and a synchronize on both sides, timed
    with CUDA events on the current stream; the max over ranks in ms per step, the last step's
    output and the clock record (when ``clocks_index`` is given)."""
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(clocks_index) if clocks_index is not None else None
    if clocks:
        clocks.__enter__()
    try:
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")   # lets a profiler select the timed steps' launches
        start.record()
        for _ in range(steps):
            out = step()
        stop.record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    finally:
        if clocks:
            clocks.__exit__(None, None, None)
    if world > 1:
        dist.barrier()
    t = torch.tensor([start.elapsed_time(stop) / steps], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item()), out, (clocks.summary() if clocks else None)


def ours(args):
    import ctypes
    import datetime
    import torch
    import torch.distributed as dist
    from deep_frame_b200 import _lib
    from deep_frame_b200.distributed import DeviceOps, ShardedMeasure
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    smoother = schedule_settings(args.schedule, args.coarsest_dofs)
    spec, system, model, density = build_problem(args.config, device, {**fast_settings(args), **smoother})
    moduli_host, derivative = system.moduli(density, 3.0, 1e-9)
    moduli = torch.as_tensor(moduli_host, device=device)
    scale = torch.as_tensor(-derivative, device=device)
    groups = model.groups()
    tuning = None
    if args.autotune:
        # measured smoother choice (outside the timed region); every candidate solves to the same tolerance
        from deep_frame_b200.autotune import tune_smoother
        choice = [None]
        if rank == 0:
            tuned, tuning = tune_smoother(system, [(key, forces) for key, _, forces in groups], moduli)
            choice = [tuned]
        if world > 1:
            dist.broadcast_object_list(choice, src=0)
            if rank != 0:
                tune_smoother(system, [(key, forces) for key, _, forces in groups], moduli,
                              candidates=[{k: v for k, v in choice[0].items() if k in ("smoother", "chebyshev_degree", "growth", "sweeps",
                                                                                        "tensor_cores", "coarsest_dofs", "cycle", "fine_tz")}], repeats=1)

    def arm():
        mg = system._multigrid()
        measure = ShardedMeasure(groups, model.rank, model.factor, DeviceOps(system))

        def step():
            mg.update_device(moduli)
            return measure.measure(scale)
        return mg, step, measure

    mg, step, measure = arm()
    reports = mg.statistics
    first_report = len(reports) + args.warmup * len(groups)
    launches0 = int(_lib.load().tf_launch_count())
    ms, (rows, flex), clocks = timed_steps(step, args.steps, args.warmup, world, dist, device, clocks_index=local)
    launches = int(_lib.load().tf_launch_count()) - launches0
    timed = reports[first_report:]
    # per-kernel-class breakdown of one more step (CUDA events on the launching stream)
    lib = _lib.load()
    lib.tf_timers(mg.handle, 1, None, None, 0)
    torch.cuda.synchronize()
    step()
    torch.cuda.synchronize()
    n = len(_lib.TIMER_CLASSES)
    tms, tcnt = (ctypes.c_double * n)(), (ctypes.c_int64 * n)()
    _lib.check(lib.tf_timers(mg.handle, 0, tms, tcnt, n), mg.handle, "tf_timers")
    lib.tf_timers(mg.handle, 0, None, None, 0)
    breakdown = {name: {"ms": round(tms[i], 3), "launches": int(tcnt[i])} for i, name in enumerate(_lib.TIMER_CLASSES)}
    result = {"ms": ms, "launches_per_step": launches / (args.warmup + args.steps), "breakdown": breakdown,
              "iterations_max": [int(np.max(r["iterations"])) for r in timed[-len(groups):]], "clocks": clocks,
              "world": world, "rank": rank, "columns": [len(g["local"]) for g in measure.groups],
              "ndof": system.ndof, "levels": timed[-1]["levels"], "coarsest_dofs": timed[-1]["coarsest_dofs"],
              "converged": all(r["converged"] for r in timed),
              "smoother": {k: v for k, v in mg.settings.items() if k in ("smoother", "chebyshev_degree", "growth", "sweeps", "tensor_cores",
                                                                          "coarsest_dofs", "precision", "pcg_precision", "cycle",
                                                                          "fine_tz")},
              "tuning": tuning, "rows": rows}
    # the kernel the roofline reports: the finest-level V-cycle apply (class fine_work), the largest
    # class of the step; the FP64 PCG class is not used because half of its launches are the gated
    # true-residual applies that exit at once, which would halve its per-launch time
    dominant = "fine_work"
    result["dominant"] = dominant
    if breakdown[dominant]["launches"]:
        result["dominant_per_launch_ms"] = breakdown[dominant]["ms"] / breakdown[dominant]["launches"]
    result["nodes"] = int(np.prod(np.asarray(mg.padded) + 1))
    result["cols"] = sum(result["columns"])
    if world == 1 and not args.no_e2e:
        # the reference-facing measure call: InterfaceCovariance.measure_device with a host density,
        # both sensitivity fields read back to the host
        host_density = np.ascontiguousarray(density)

        def e2e_step():
            r = model.measure_device(host_density, 3.0, 1e-9)
            return r[0]["gradient"].cpu().numpy(), r[1]["gradient"].cpu().numpy()

        e2e_steps = args.e2e_steps or min(args.steps, 3)
        e_ms, grads, _ = timed_steps(e2e_step, e2e_steps, 1, 1, dist, device)
        result["e2e"] = {"ms": e_ms, "steps": e2e_steps, "h2d_bytes_per_step": int(moduli_host.nbytes),
                         "d2h_bytes_per_step": int(grads[0].nbytes + grads[1].nbytes + model.rank * model.rank * 8)}
    if world == 1 and args.storage_trial:
        # the same step with 16-bit V-cycle storage (the same schedule, tolerance and outer PCG)
        result["storage_trial"] = {}
        for precision in [p for p in args.storage_trial.split(",") if p]:
            # capped: a storage precision that stalls the PCG is reported unconverged instead of running 2000 iterations
            rebuild_multigrid(system, {**fast_settings(args), "precision": precision, "tensor_cores": False, "max_iterations": 300,
                                       "retries": 0})
            torch.cuda.empty_cache()
            trial_mg, trial_step, _ = arm()
            first = len(trial_mg.statistics) + len(groups)
            try:
                t_ms, (t_rows, _), _ = timed_steps(trial_step, min(args.steps, 2), 1, 1, dist, device)
                stats = trial_mg.statistics[first:]
                result["storage_trial"][precision] = {"s": round(t_ms / 1e3, 6), "pcg_iterations": [int(np.max(r["iterations"])) for r in stats[-len(groups):]],
                                                      "converged": all(r["converged"] for r in stats),
                                                      "tr": t_rows[0]["value"], "lambda_max": t_rows[1]["value"]}
            except (RuntimeError, ValueError) as exc:
                result["storage_trial"][precision] = {"error": f"{type(exc).__name__}: {exc}"}
    if world == 1 and not args.no_plain:
        # the plain FP64 GMG-PCG drop-in on the same GPU: FP64 V-cycle and FP64 PCG, the same smoother
        # schedule, hierarchy depth and tolerance
        rebuild_multigrid(system, PLAIN)
        torch.cuda.empty_cache()
        plain_mg, plain_step, _ = arm()
        plain_first = len(plain_mg.statistics) + len(groups)
        plain_steps = args.plain_steps or min(args.steps, 3)
        p_ms, (p_rows, _), p_clocks = timed_steps(plain_step, plain_steps, 1, 1, dist, device, clocks_index=local)
        p_timed = plain_mg.statistics[plain_first:]
        result["plain"] = {"ms": p_ms, "steps": plain_steps, "rows": p_rows, "clocks": p_clocks,
                           "iterations_max": [int(np.max(r["iterations"])) for r in p_timed[-len(groups):]],
                           "converged": all(r["converged"] for r in p_timed)}
    if world > 1:
        dist.destroy_process_group()
    return result, system, model, density
def cpu_samples(system, density, count=1, cores=None):
    """The oracle's GMG-PCG on the host cores: ``count`` measured evaluations (``oracle/baseline.py``).

    One single-threaded spawn-started worker per usable core (at most one per column, and no more
    than host memory holds at ~10 KB per dof each); in every evaluation each worker rebuilds its
    half's hierarchy from the moduli and solves its whole share of the columns to 1e-8 with the
    reference's default smoother, so every column of both halves is solved and nothing is scaled.
    Returns ``[(evaluation seconds, record), ...]``."""
    from oracle.baseline import ParallelBaseline, sample_text, worker_count
    moduli, _ = system.moduli(density, 3.0, 1e-9)
    groups = [(members[0][1]["fixed"], np.stack([part["force"] for _, part in members], axis=1))
              for members in system.groups.values()]
    settings = {"tolerance": 1e-8}
    workers = worker_count([f.shape[1] for _, f in groups], cores=cores, bytes_per_worker=10_000 * system.ndof)
    out = []
    with ParallelBaseline(workers) as pool:
        for _ in range(count):
            value, record = pool.sample(system.shape, system.ke, moduli, groups, settings, block=None)
            record["text"] = sample_text(record, settings)
            out.append((value, record))
    return out


def cpu_unavailable(ndof):
    """Why the oracle's CPU GMG-PCG is not timed on a problem of ``ndof`` dofs, or None when it is."""
    if ndof <= CPU_MAX_DOFS:
        return None
    return (f"oracle CPU GMG-PCG not run on {ndof} dofs: budget (about 10 KB of host memory per dof and worker, "
            f"{ndof * 10e3 / 1e9:.0f} GB for one worker, and an estimated hour or more per evaluation on the host cores); "
            f"the GPU line's cpu_baseline carries a full measured evaluation of the 96 x 96 x 16 plate")


def reference(args):
    """--impl reference: the oracle's CPU restatement of the reference GMG-PCG path on all of this box's host cores.

    Rank 0 alone runs (other ranks return at once).  Every step is one full measured evaluation
    (all columns of both halves solved to 1e-8, nothing scaled); a problem beyond the host's budget
    prints an ``unavailable`` line instead.  The CPU arm runs at most one warm-up and three timed
    steps, and its line says how many ran."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    from deep_frame_b200 import problems
    from deep_frame_b200.elasticity import HexElasticity
    from deep_frame_b200.covariance import InterfaceCovariance
    spec = problems.CONFIGS[args.config]
    shape = spec["shape"]
    ndof = 3 * int(np.prod(np.asarray(shape) + 1))
    reason = cpu_unavailable(ndof)
    if reason:
        line = {"impl": "reference", "unavailable": reason, "config": {"workload": args.config, "ndof": ndof}}
        print(json.dumps(line))
        return line
    domain, density, cov = problems.plate(shape, 0)
    system = HexElasticity(domain)
    InterfaceCovariance(system, cov, domain["interfaces"])
    warmup, steps = min(args.warmup, 1), min(args.steps, 3)
    samples, cores = None, None
    while samples is None:
        try:
            samples = cpu_samples(system, density, count=warmup + steps, cores=cores)[warmup:]
        except (OSError, MemoryError, RuntimeError) as exc:   # BrokenProcessPool is a RuntimeError
            from oracle.baseline import host_cores
            cores = (cores or host_cores()) // 2
            if cores < 2:
                print(json.dumps({"impl": "reference", "unavailable": f"oracle CPU baseline failed: {type(exc).__name__}: {exc}"}))
                return None
    v = float(np.mean([value for value, _ in samples]))
    record = samples[-1][1]
    line = {"metric": METRIC, "value": round(v, 3), "unit": "s", "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
            "steps_requested": args.steps, "warmup_requested": args.warmup,
            "ms_per_step": round(v * 1e3, 1), "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": args.config, "rhs_per_half": 42, "halves": 2, "ndof": system.ndof, "tolerance": 1e-8,
                       "smoother": "reference default (Chebyshev degree 3, growth 2)",
                       "pcg_iterations_mean": round(record["iterations_mean"], 2)},
            "cpu_baseline": {"value": round(v, 3), "unit": "s", "cores": record["workers"], "kind": "port", "sample": record["text"]},
            "e2e": {"value": round(v, 3), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return line


def simp(args):
    """--simp N: iterations/s of the covariance SIMP + MMA loop (the mixed-precision loop of the 128 x 128 x 24 plate).

    Every iteration: filter, SIMP moduli, both hierarchies, 2 x 42 solves to the tolerance, F, tr, the tr
    sensitivity, pullbacks and one device MMA step.  Timed with CUDA events on the current stream around
    the whole loop (host work between launches included).  With --simp-compare the plain FP64 V-cycle runs
    the same loop and the final physical densities, tr histories and times are compared."""
    import torch
    from deep_frame_b200 import _lib, problems
    from deep_frame_b200.optimize import CovarianceSimp
    config = args.config if args.config != CONFIG else "plate_128x128x24"
    spec = problems.CONFIGS[config]
    domain, _, cov = problems.plate(spec["shape"], 0)
    smoother = {"smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0}   # the plate's autotuned schedule
    if args.schedule:
        degree, growth = args.schedule.split(",")
        smoother = {"smoother": "chebyshev", "chebyshev_degree": int(degree), "growth": float(growth)}
    precisions = [args.precision] + (["float64"] if args.simp_compare and args.precision != "float64" else [])
    runs, physical = {}, {}
    for precision in precisions:
        warm = True if args.warm_start == -1 else int(args.warm_start)
        loop = CovarianceSimp(domain, cov, volume_fraction=0.15, filter_radius=1.5, move=0.2, warm_start=warm,
                              multigrid={"precision": precision, "tolerance": spec["tolerance"], **smoother})
        loop.run(1)                                   # buffers, constant slots and MMA workspace (not timed)
        loop.objective_scale, loop.previous, loop.basis = None, None, {}
        torch.cuda.synchronize()
        launches0 = int(_lib.load().tf_launch_count())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(0) as clocks:
            e0.record()
            x, history = loop.run(args.simp)
            e1.record()
            torch.cuda.synchronize()
        seconds = e0.elapsed_time(e1) / 1e3
        physical[precision] = loop.map.filtered_device(x).cpu().numpy()     # physical density (beta = 0)
        runs[precision] = {"iter_per_s": args.simp / seconds, "seconds": seconds, "tr_history": [r["tr"] for r in history],
                           "final_tr": history[-1]["tr"], "final_volume": history[-1]["volume"],
                           "pcg_iterations_mean": float(np.mean([max(r["pcg_iterations"]) for r in history])),
                           "gpu_launches": int(_lib.load().tf_launch_count()) - launches0, "clocks": clocks.summary()}
        loop.close()
    main_run = runs[args.precision]
    line = {"metric": "SIMP iter/s (covariance tr objective, MMA)", "value": round(main_run["iter_per_s"], 4), "unit": "iter/s",
            "n_gpus": 1, "steps": args.simp, "warmup": 1, "higher_is_better": True, "dtype": "f64 outer / " + args.precision + " V-cycle",
            "data": "synthetic",
            "config": {"workload": config, "iterations": args.simp, "volume_fraction": 0.15, "filter_radius": 1.5, "penalization": 3.0,
                       "move": 0.2, "rhs_per_half": 42, "tolerance": spec["tolerance"], "smoother": smoother, "warm_start": args.warm_start},
            "clocks": main_run["clocks"], "gpu_launches": main_run["gpu_launches"],
            "runs": {p: {k: v for k, v in r.items() if k not in ("tr_history", "clocks")} for p, r in runs.items()}}
    if "float64" in runs and args.precision != "float64":
        a, b = runs[args.precision]["tr_history"], runs["float64"]["tr_history"]
        line["vs_fp64"] = {"final_density_max_abs": float(np.max(np.abs(physical[args.precision] - physical["float64"]))),
                           "tr_history_max_rel": float(np.max(np.abs(np.asarray(a) / np.asarray(b) - 1))),
                           "speedup": runs[args.precision]["iter_per_s"] / runs["float64"]["iter_per_s"]}
    print(json.dumps(line))


def instances(args):
    """--instances N: N independent seeded plate instances (grids from 64 x 64 x 12 to 160 x 160 x 24,
    6 to 42 load columns per half; with --instance-sizes small from 16 x 16 x 4 to 48 x 48 x 8, 3 to 12
    columns), each with its own solver handle, solved to 1e-8 three ways: as one
    batch (tf_solve_batch: every PCG and V-cycle stage one launch over all instances; one batch per
    mirror half), one after another on one stream, and concurrently on one host thread and CUDA
    stream per instance.  After one untimed round of each (buffers, hierarchies, constant slots) the
    time of one round gives solves/s (one solve = all columns of both halves of one instance)."""
    import threading
    import torch
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    from deep_frame_b200.topology_multigrid import solve_batch_device
    rng = np.random.default_rng(2026)
    if args.instance_sizes == "small":
        sizes, columns = [(16, 16, 4), (24, 24, 4), (24, 24, 6), (32, 32, 6), (32, 32, 8), (40, 40, 8), (48, 48, 8)], (3, 13)
    else:
        sizes, columns = [(64, 64, 12), (80, 80, 12), (96, 96, 16), (112, 112, 16), (128, 128, 16), (128, 128, 24), (144, 144, 24),
                          (160, 160, 24)], (6, 43)
    specs = []
    for i in range(args.instances):
        shape = sizes[int(rng.integers(len(sizes)))]
        specs.append((shape, int(rng.integers(*columns)), i))
    settings = {"tolerance": 1e-8, "smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0}
    work = []
    for shape, rhs, seed in specs:
        domain, density, cov = problems.plate(shape, seed)
        system = HexElasticity(domain, multigrid=dict(settings))
        model = InterfaceCovariance(system, cov, domain["interfaces"])
        moduli = torch.as_tensor(system.moduli(density, 3.0, 1e-9)[0], device="cuda")
        groups = [(key, forces[:rhs].contiguous()) for key, _, forces in model.groups()]
        work.append({"system": system, "moduli": moduli, "groups": groups, "stream": torch.cuda.Stream(), "shape": shape, "rhs": rhs})
    for item in work:
        item["system"]._multigrid().update_device(item["moduli"])
    torch.cuda.synchronize()
    errors = []

    def solve(item):
        try:
            with torch.cuda.stream(item["stream"]):
                its = []
                for key, forces in item["groups"]:
                    _, report = item["system"].solve_group_device(key, forces)
                    its.append(max(report["iterations"]))
                item["iterations"] = its
                item["stream"].synchronize()
        except Exception as error:          # surfaced after the join
            errors.append(repr(error))

    def threaded():
        threads = [threading.Thread(target=solve, args=(item,)) for item in work]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        torch.cuda.synchronize()
        if errors:
            raise RuntimeError("; ".join(errors))
        return time.perf_counter() - t0

    def serial():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for item in work:
            solve(item)
        torch.cuda.synchronize()
        if errors:
            raise RuntimeError("; ".join(errors))
        return time.perf_counter() - t0

    def batched():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        results = []
        for half in range(max(len(item["groups"]) for item in work)):
            jobs = []
            for item in work:
                if half < len(item["groups"]):
                    key, forces = item["groups"][half]
                    mg = item["system"]._multigrid()
                    jobs.append((mg, key, item["system"].groups[key][0][1]["fixed"], forces))
            results.append(solve_batch_device(jobs))
        torch.cuda.synchronize()
        seconds = time.perf_counter() - t0
        for half in results:
            for (_, report) in half:
                if not report["converged"]:
                    raise RuntimeError(f"batched solve did not converge: {max(report['relative_residual'])}")
        return seconds, results

    batched()                                 # untimed: allocations, hierarchies, constant slots
    batch_seconds, results = batched()
    serial()
    serial_seconds = serial()
    # the batch against the instances' own solves (the serial round just ran them)
    worst = 0.0
    for half, outcome in enumerate(results):
        for item, (u, report) in zip([w for w in work if half < len(w["groups"])], outcome):
            key, forces = item["groups"][half]
            single, _ = item["system"].solve_group_device(key, forces)
            worst = max(worst, float(((u - single).norm(dim=1) / single.norm(dim=1).clamp_min(1e-300)).max()))
    threaded()
    threaded_seconds = threaded()
    columns = sum(2 * item["rhs"] for item in work)
    line = {"metric": "independent uneven instances: solves/s", "value": round(len(work) / batch_seconds, 4), "unit": "solves/s", "n_gpus": 1,
            "higher_is_better": True, "data": "synthetic",
            "config": {"instances": [{"shape": list(item["shape"]), "rhs_per_half": item["rhs"], "pcg_iterations": item.get("iterations")}
                                     for item in work], "sizes": args.instance_sizes, "tolerance": 1e-8,
                       "batched": "tf_solve_batch: one launch per PCG / V-cycle stage over all instances, one batch per mirror half"},
            "seconds": round(batch_seconds, 4), "column_solves_per_s": round(columns / batch_seconds, 2),
            "serial_seconds": round(serial_seconds, 4), "speedup_vs_serial": round(serial_seconds / batch_seconds, 3),
            "threaded_seconds": round(threaded_seconds, 4), "threaded_speedup_vs_serial": round(serial_seconds / threaded_seconds, 3),
            "batch_vs_own_solves_max_rel": worst}
    for item in work:
        item["system"].close()
    print(json.dumps(line))


def learned_guess(args):
    """--learned: train the four-level convolutional initial guess (channels 16, 32, 48, 64) on about
    2,000 load-column snapshots of seeded 96 x 96 x 16 covariance-plate SIMP trajectories (seeds 0-2,
    16 designs each, every second column of both halves), then time one covariance solve (2 x 42
    columns to 1e-8) from zero and from the network's guess (tensor-core FP16 inference included) on
    held-out designs: the 12th design of a seed-7 trajectory at 96 x 96 x 16 and the seeded
    192 x 192 x 32 plate density."""
    import torch
    from deep_frame_b200 import learned, problems
    from deep_frame_b200.elasticity import HexElasticity
    settings = {"tolerance": 1e-8, "smoother": "chebyshev", "chebyshev_degree": 1, "growth": 2.0}
    train_shape = (96, 96, 16)
    channels = (16, 32, 48, 64)
    t0 = time.perf_counter()
    snapshots, live, grid = [], None, None
    for seed in (0, 1, 2):
        domain, _, cov = problems.plate(train_shape, seed)
        part, live_part, grid = learned.record_trajectory(domain, cov, 16, multigrid=settings, stride=2)
        snapshots += part
        live = live_part
    record_s = time.perf_counter() - t0
    count = int(sum(1 for _ in learned.samples(snapshots, live, grid)))
    net = learned.GuessNet(channels=channels, seed=0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = learned.train(net, snapshots, live, grid, epochs=args.learned_epochs, batch=8, lr=2e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del snapshots
    net.pack()
    cases = {}
    held_domain, _, held_cov = problems.plate(train_shape, 7)
    held, _, _ = learned.record_trajectory(held_domain, held_cov, 12, multigrid=settings, stride=1000)
    cases["plate_96x96x16_seed7_design12"] = learned.compare(net, held_domain, held_cov, held[-1][0], multigrid=settings)
    dom, density, cv = problems.plate((192, 192, 32), 0)
    moduli = HexElasticity(dom, multigrid=settings).moduli(density, 3.0, 1e-9)[0]
    cases["plate_192x192x32"] = learned.compare(net, dom, cv, moduli, multigrid=settings)
    policy = learned.GuessPolicy(net)
    for row in cases.values():
        policy.assess(row["network"]["mean_iterations"], row["zero"]["mean_iterations"], row["network"]["seconds"], row["zero"]["seconds"])
    line = {"metric": "PCG iterations / seconds to 1e-8 with and without the learned initial guess", "unit": "iterations",
            "n_gpus": 1, "data": "synthetic (SIMP trajectory snapshots of seeded plates)",
            "config": {"network": f"{len(channels)}-level conv encoder/decoder, channels {channels}, {len(net.specs)} conv layers; "
                                  "training in FP32 (im2col + own SGEMM), inference on the tensor cores (tcgen05 kind::f16, "
                                  "FP16 weights and activations, FP32 accumulation)",
                       "training": {"shape": list(train_shape), "seeds": [0, 1, 2], "designs": 48, "samples": count,
                                    "epochs": args.learned_epochs, "losses": [round(v, 5) for v in losses],
                                    "record_s": round(record_s, 2), "train_s": round(train_s, 2)},
                       "solver": settings},
            "cases": {name: {label: {k: (round(v, 4) if isinstance(v, float) else v) for k, v in row[label].items() if k != "iterations"}
                             for label in row} for name, row in cases.items()},
            "network_kept": policy.enabled}
    print(json.dumps(line))


def row_values(rows):
    """tr, lambda_max, KS and both sensitivity fields (host arrays) of a measure's rows."""
    return {"tr": rows[0]["value"], "lambda_max": rows[1]["value"], "ks": rows[1]["info"]["ks_n_mm"],
            "grad_mean": rows[0]["gradient"].cpu().numpy(), "grad_worst": rows[1]["gradient"].cpu().numpy()}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


def agreement(got, want):
    """Relative differences of tr, lambda_max, KS and the two sensitivity fields (2-norm)."""
    return {"tr_rel": rel(got["tr"], want["tr"]), "lambda_max_rel": rel(got["lambda_max"], want["lambda_max"]),
            "ks_rel": rel(got["ks"], want["ks"]), "grad_mean_rel": rel(got["grad_mean"], want["grad_mean"]),
            "grad_worst_rel": rel(got["grad_worst"], want["grad_worst"]),
            "bars": {"tr": 1e-6, "lambda_max": 1e-6, "sensitivities": 1e-5}}


def oracle_errors(config, values):
    """Errors of the step's values against the FP64 oracle of the same workload
    (tests/golden/<workload>.npz, from tests/golden/make_plate_oracle.py: the oracle's GMG-PCG to a
    1e-10 true relative residual); None when no such file exists."""
    path = ROOT / "tests" / "golden" / f"{config}.npz"
    if not path.exists():
        return None
    ref = np.load(path)
    out = agreement(values, {"tr": float(ref["tr"]), "lambda_max": float(ref["lambda_max"]), "ks": float(ref["ks"]),
                             "grad_mean": ref["grad_mean"], "grad_worst": ref["grad_worst"]})
    out["oracle"] = f"FP64 GMG-PCG to {float(ref['tolerance']):g} (tests/golden/{path.name})"
    return out


def roofline(args, result):
    """Roofline of the step's dominant kernel class: algorithmic bytes of one launch over its
    CUDA-event duration against the measured HBM copy bandwidth, with the compute side beside it."""
    if "dominant_per_launch_ms" not in result:
        return None
    hbm, _, source = peaks()
    # algorithmic bytes of one launch, per node and column: the words its mode must read and write
    # (+ the element moduli, once per launch).  PCG operator: u read, y written (6).  Work-precision
    # finest level with Chebyshev degree d: per V-cycle 2 residual applies (u, b read, y written: 9)
    # and 2 (d - 1) Chebyshev steps (u, res, x read; y, res, x written: 18).
    dominant = result["dominant"]
    word = 8 if dominant == "fine_fp64" or args.precision == "float64" else 4
    nodes, cols = result["nodes"], result["cols"]
    per_launch_cols = cols / max(1, len(result["columns"]))
    words = 6.0
    sm = result["smoother"]
    degree = int(sm.get("chebyshev_degree", 3))
    if dominant == "fine_work" and sm.get("smoother", "chebyshev") == "chebyshev":
        words = (2 * 9 + 2 * (degree - 1) * 18) / (2 * degree)
    traffic_alg = nodes * per_launch_cols * (words * word) + nodes * word
    traffic = None
    if args.precision == "float32" and dominant == "fine_work" and sm.get("smoother", "chebyshev") == "chebyshev" \
            and not sm.get("tensor_cores"):
        # ncu capture of the 96 x 96 x 16 plate's launch, scaled by nodes x columns
        traffic = FINE_TRAFFIC["resid" if degree == 1 else "cheb"] * nodes * per_launch_cols / (FINE_TRAFFIC_NODES * 42)
    achieved = traffic_alg / (result["dominant_per_launch_ms"] * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
            "traffic": traffic, "kernel": dominant, "peak_source": source,
            "per_launch_ms": round(result["dominant_per_launch_ms"], 4), "algorithmic_bytes_per_launch": int(traffic_alg)}
    clk = result["clocks"] or {}
    roof["compute"] = fma_roof("fp64" if word == 8 else "fp32", 1152.0 * nodes * per_launch_cols, result["dominant_per_launch_ms"],
                               clk.get("sm_mhz"), clk.get("sm_max_mhz") or 1965.0)
    return roof


def main():
    args = parse()
    if args.learned:
        learned_guess(args)
        return
    if args.instances:
        instances(args)
        return
    if args.impl == "reference":
        reference(args)
        return
    if args.simp:
        simp(args)
        return
    result, system, model, density = ours(args)
    if result["rank"] != 0:
        return
    ms = result["ms"]
    cpu = None
    if not args.no_cpu and result["world"] == 1:
        # a full measured evaluation of the 96 x 96 x 16 plate when this workload is beyond the host
        sample_config = args.config
        try:
            if cpu_unavailable(system.ndof):
                sample_config = "plate_96x96x16"
                _, system, _, density = cpu_problem(sample_config)
            value, sample = cpu_samples(system, density)[0]
            cpu = {"value": round(value, 2), "unit": "s", "cores": sample["workers"], "kind": "port", "workload": sample_config,
                   "sample": sample["text"] + ("" if sample_config == args.config else f"; workload {sample_config}, not {args.config}")}
        except (OSError, MemoryError, RuntimeError) as exc:   # the GPU line is kept whatever the CPU leg does
            cpu = {"value": None, "unit": "s", "cores": None, "kind": "port", "error": f"{type(exc).__name__}: {exc}"}
    sm = result["smoother"]
    fast = row_values(result["rows"])
    line = {"metric": METRIC, "value": round(ms / 1e3, 6), "unit": "s", "n_gpus": result["world"], "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.config, "rhs_per_half": 42, "halves": 2, "ndof": result["ndof"], "tolerance": 1e-8,
                       "outer": "fp64 PCG" if sm.get("pcg_precision", "float64") == "float64" else "fp32 PCG, fp64 reliable residual updates",
                       "vcycle": args.precision + (" (finest apply: tcgen05)" if sm.get("tensor_cores") else ""),
                       "levels": result["levels"], "coarsest_dofs": result["coarsest_dofs"], "pcg_iterations": result["iterations_max"],
                       "smoother": sm,
                       "smoother_choice": (f"autotuned (fastest of {len(result['tuning'])} schedules / depths / finest-apply units)"
                                           if result["tuning"] else "fixed: the autotuner's pick on the 96 x 96 x 16 plate"),
                       "l2": "working set > L2 (FP64 vector blocks of %.0f MB per half)" % (result["ndof"] * 42 * 8 / 1e6),
                       "learned_guess": "off: dropped by its policy (no iteration gain measured)",
                       "parallelism": f"rhs-sharded x{result['world']}"},
            "clocks": result["clocks"], "gpu_launches": int(result["launches_per_step"] * args.steps),
            "roofline": roofline(args, result), "cpu_baseline": cpu, "breakdown_ms": result["breakdown"], "converged": result["converged"]}
    if "e2e" in result:
        e = result["e2e"]
        line["e2e"] = {"value": round(e["ms"] / 1e3, 6), "unit": "s", "h2d_bytes_per_step": e["h2d_bytes_per_step"],
                       "d2h_bytes_per_step": e["d2h_bytes_per_step"], "steps": e["steps"],
                       "call": "InterfaceCovariance.measure_device(host density): SIMP moduli, update, both halves solved, "
                               "F, tr, lambda_max, both sensitivity fields to the host"}
    line["results"] = {"tr_K_inv_sigma": fast["tr"], "lambda_max": fast["lambda_max"], "ks": fast["ks"]}
    if "plain" in result:
        plain = result["plain"]
        line["results"]["plain_fp64"] = {
            "s": round(plain["ms"] / 1e3, 6), "steps": plain["steps"], "speedup_of_value": round(plain["ms"] / ms, 3),
            "pcg_iterations": plain["iterations_max"], "converged": plain["converged"], "clocks": plain["clocks"],
            "path": "FP64 V-cycle, FP64 PCG, CUDA-core operators, same schedule and tolerance",
            "fast_vs_plain": agreement(fast, row_values(plain["rows"]))}
    if "storage_trial" in result:
        line["results"]["storage_trial"] = {
            "what": "V-cycle vectors rounded to 16 bits when stored (FP32 buffers and arithmetic), FP64 outer PCG; same schedule",
            **{p: ({**r, "tr_rel_to_value": abs(r["tr"] / fast["tr"] - 1)} if "tr" in r else r) for p, r in result["storage_trial"].items()}}
    parity = oracle_errors(args.config, fast)
    if parity:
        line["results"]["vs_fp64_oracle"] = parity
    print(json.dumps(line))


def cpu_problem(config):
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    spec = problems.CONFIGS[config]
    domain, density, cov = problems.plate(spec["shape"], 0)
    system = HexElasticity(domain)
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    return spec, system, model, density


if __name__ == "__main__":
    main()
