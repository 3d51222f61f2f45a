"""Multi-core timing of the oracle GMG-PCG: the CPU baseline of the covariance-evaluation benchmark.

Test and benchmark infrastructure like the rest of this package: only the CPU-baseline legs of
``bench.py`` use it, as the timed CPU restatement of the reference's solve.

What one design evaluation costs on the host cores.  Every fixture group (a mirror half) rebuilds
its multigrid hierarchy from the new element moduli (``topology_multigrid.py:145-223`` of the
reference: Galerkin levels, diagonals, lambda_max, coarsest factor) and solves its load columns by
batched flexible PCG to the true relative residual tolerance (``:407-454``).  With W cores, each of
the G groups gets W / G single-threaded workers; a worker builds its group's hierarchy once and
solves its share of that group's columns as one batched block.

The sample.  A spawn-started pool of W workers runs concurrently, so the cores contend for memory
bandwidth as they would in a full evaluation.  Each worker does one hierarchy set-up and solves
its whole share of the columns to convergence (the benchmark's default, a complete measured
evaluation), or a block of at most ``block`` of them.  The step time is, per group, the slowest
worker's set-up plus its solve time (scaled by share / block when a block is smaller than the
share), and the maximum over groups.
"""
import multiprocessing as mp
import os
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np

#: thread-count variables set to 1 in the workers: every core runs one single-threaded worker
_THREAD_VARS = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS", "NUMEXPR_NUM_THREADS")


def _read(path):
    try:
        with open(path) as f:
            return f.read().strip()
    except OSError:
        return None


def host_cores():
    """Cores this process may use: its CPU affinity, capped by a cgroup CPU quota if one is set
    (``cpu.max`` of cgroup v2, else ``cpu.cfs_quota_us`` / ``cpu.cfs_period_us`` of cgroup v1)."""
    cores = len(os.sched_getaffinity(0))
    try:
        v2 = _read("/sys/fs/cgroup/cpu.max")
        if v2 is not None:
            quota, period = v2.split()[:2]
            if quota != "max":
                cores = min(cores, max(1, int(quota) // int(period)))
        else:
            quota, period = _read("/sys/fs/cgroup/cpu/cpu.cfs_quota_us"), _read("/sys/fs/cgroup/cpu/cpu.cfs_period_us")
            if quota is not None and period is not None and int(quota) > 0:
                cores = min(cores, max(1, int(quota) // int(period)))
    except ValueError:
        pass
    return cores


def available_bytes():
    """Host memory this process may still use, in bytes: MemAvailable of /proc/meminfo, capped by
    the room left under a cgroup memory limit if one is set (v2 ``memory.max`` - ``memory.current``,
    else v1 ``memory.limit_in_bytes`` - ``memory.usage_in_bytes``); None where nothing is readable."""
    avail = None
    info = _read("/proc/meminfo")
    if info:
        for line in info.splitlines():
            if line.startswith("MemAvailable:"):
                avail = int(line.split()[1]) * 1024
                break
    for limit_path, used_path in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                                  ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        limit, used = _read(limit_path), _read(used_path)
        if limit is None or used is None:
            continue
        try:
            room = int(limit) - int(used)
        except ValueError:          # "max": no limit
            break
        if int(limit) < (1 << 60):  # v1 reports "no limit" as a huge number
            avail = room if avail is None else min(avail, room)
        break
    return avail


def worker_count(columns_per_group, cores=None, bytes_per_worker=None):
    """Workers for one sample: all usable cores, at most one per column, at least one per group,
    and no more than the available memory holds (``bytes_per_worker`` each, with 25 % headroom)."""
    groups = len(columns_per_group)
    count = min(host_cores() if cores is None else int(cores), int(sum(columns_per_group)))
    if bytes_per_worker:
        avail = available_bytes()
        if avail is not None:
            count = min(count, int(0.8 * avail // bytes_per_worker))
    return max(groups, count)


def assignment(columns_per_group, workers):
    """Split ``workers`` over the groups in proportion to their column counts (at least one each).

    Returns, per group, its worker count and each worker's share of the group's columns (shares
    differ by at most one and sum to the group's column count)."""
    groups = len(columns_per_group)
    total = float(sum(columns_per_group))
    per = [max(1, int(workers * c / total)) for c in columns_per_group]
    # hand out what rounding left over, largest remaining load first
    while sum(per) < workers:
        g = max(range(groups), key=lambda i: columns_per_group[i] / per[i] if per[i] < columns_per_group[i] else -1.0)
        if per[g] >= columns_per_group[g]:
            break
        per[g] += 1
    out = []
    for c, w in zip(columns_per_group, per):
        w = min(w, c)
        base, extra = divmod(c, w)
        out.append((w, [base + (1 if i < extra else 0) for i in range(w)]))
    return out


def _solve_block(task):
    """One worker: the group's hierarchy from the moduli, then its block of columns to convergence."""
    from .gmg import MultigridOracle
    shape, ke, moduli, fixed, forces, settings = task
    t0 = time.perf_counter()
    mg = MultigridOracle(shape, ke, moduli, fixed, settings)
    t1 = time.perf_counter()
    _, iterations, relative, _ = mg.solve(forces)
    t2 = time.perf_counter()
    rss = 0
    try:
        import resource
        rss = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss * 1024
    except (ImportError, OSError):
        pass
    return {"setup_s": t1 - t0, "solve_s": t2 - t1, "iterations": [int(i) for i in iterations],
            "relative": [float(r) for r in relative], "columns": int(forces.shape[1]), "rss_bytes": int(rss)}


class ParallelBaseline:
    """Spawn-started pool of single-threaded oracle workers, reused across samples.

    ``spawn`` keeps the workers independent of any CUDA context the parent holds.  A worker that
    dies (killed for memory, say) breaks the pool: the sample raises ``BrokenProcessPool`` instead
    of waiting for a task that will never finish."""

    def __init__(self, workers):
        self.workers = int(workers)
        # the thread caps must be in the environment when the workers start (they start on the first
        # submit), so they stay set while the pool lives and are restored by close()
        self._saved = {k: os.environ.get(k) for k in _THREAD_VARS}
        for k in _THREAD_VARS:
            os.environ[k] = "1"
        self.pool = ProcessPoolExecutor(max_workers=self.workers, mp_context=mp.get_context("spawn"))

    def close(self):
        if self.pool is not None:
            self.pool.shutdown(wait=True, cancel_futures=True)
            self.pool = None
            for k, v in self._saved.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def sample(self, shape, ke, moduli, groups, settings, block=None):
        """Time one parallel evaluation sample.

        ``groups``: per fixture group ``(fixed dofs, forces [ndof, R])``; ``block`` caps the columns a
        worker solves (None: its whole share, so the sample is a complete evaluation).  Returns the
        step time in seconds (an estimate when a block is smaller than its share) and a record of
        what was measured."""
        plan = assignment([f.shape[1] for _, f in groups], self.workers)
        tasks, owner = [], []
        for g, ((fixed, forces), (count, shares)) in enumerate(zip(groups, plan)):
            start = 0
            for share in shares:
                width = share if block is None else min(share, block)
                tasks.append((tuple(shape), ke, moduli, fixed, np.ascontiguousarray(forces[:, start:start + width]), settings))
                owner.append((g, share))
                start += share
        t0 = time.perf_counter()
        results = list(self.pool.map(_solve_block, tasks))
        wall = time.perf_counter() - t0
        estimate = 0.0
        per_group = []
        for g in range(len(groups)):
            mine = [(r, share) for r, (gg, share) in zip(results, owner) if gg == g]
            t = max(r["setup_s"] + r["solve_s"] * share / r["columns"] for r, share in mine)
            per_group.append(t)
            estimate = max(estimate, t)
        iterations = [i for r in results for i in r["iterations"]]
        return estimate, {"workers": len(tasks), "wall_s": wall, "group_s": per_group,
                          "setup_s": float(np.mean([r["setup_s"] for r in results])),
                          "column_s": float(np.mean([r["solve_s"] / r["columns"] for r in results])),
                          "sampled_columns": int(sum(r["columns"] for r in results)),
                          "columns": int(sum(f.shape[1] for _, f in groups)),
                          "max_share": int(max(s for _, s in owner)), "block": int(block) if block is not None else None,
                          "iterations_mean": float(np.mean(iterations)), "iterations_max": int(max(iterations)),
                          "relative_max": float(max(x for r in results for x in r["relative"])),
                          "rss_bytes_max": int(max(r["rss_bytes"] for r in results))}


def sample_text(record, settings):
    """One-line description of a sample for the benchmark's ``cpu_baseline.sample``."""
    block = record["block"]
    scaled = (f"each worker's block of {block} columns scaled to its share of {record['max_share']}"
              if block is not None and record["max_share"] > block else "nothing scaled (every worker solved its whole share)")
    return (f"oracle GMG-PCG (NumPy/SciPy, one single-threaded process per core, {record['workers']} processes run "
            f"concurrently): per worker one hierarchy set-up of its mirror half plus a batched block of its columns "
            f"solved to {settings.get('tolerance', 1e-8):g} ({record['sampled_columns']} of {record['columns']} columns, "
            f"{record['iterations_mean']:.1f} PCG iterations on average); {scaled}; step = slowest half")
