"""The multi-core CPU baseline of the benchmark (oracle/baseline.py): worker plan and one tiny sample.  No GPU."""
import numpy as np

from oracle import hex8
from oracle.baseline import ParallelBaseline, assignment, sample_text, worker_count


def test_assignment_splits_workers_by_columns():
    for columns, workers in (([42, 42], 8), ([42, 42], 84), ([42, 42], 200), ([5, 1], 8), ([7, 3, 2], 5), ([42, 42], 2)):
        plan = assignment(columns, workers)
        assert len(plan) == len(columns)
        for c, (w, shares) in zip(columns, plan):
            assert 1 <= w <= c and len(shares) == w
            assert sum(shares) == c and max(shares) - min(shares) <= 1
        assert sum(w for w, _ in plan) <= max(workers, len(columns))
    assert [w for w, _ in assignment([42, 42], 8)] == [4, 4]
    assert [w for w, _ in assignment([42, 42], 200)] == [42, 42]


def test_worker_count_bounds():
    assert worker_count([42, 42], cores=8) == 8
    assert worker_count([42, 42], cores=500) == 84
    assert worker_count([3, 2], cores=1) == 2          # at least one worker per group
    assert worker_count([42, 42], cores=64, bytes_per_worker=1 << 62) == 2


def test_parallel_sample_converges():
    shape = (8, 4, 4)
    k0 = hex8.element_matrices((1.0, 1.0, 1.0), 0.3)[0]
    nodes = tuple(n + 1 for n in shape)
    rng = np.random.default_rng(0)
    moduli = rng.uniform(0.1, 1.0, int(np.prod(shape)))
    clamp = np.flatnonzero(np.indices(nodes).reshape(3, -1)[0] == 0)
    fixed = (3 * clamp[:, None] + np.arange(3)).ravel()
    ndof = 3 * int(np.prod(nodes))
    forces_a = rng.standard_normal((ndof, 3))
    forces_b = rng.standard_normal((ndof, 2))
    forces_a[fixed] = 0.0
    forces_b[fixed] = 0.0
    settings = {"tolerance": 1e-8}
    with ParallelBaseline(2) as pool:
        value, record = pool.sample(shape, k0, moduli, [(fixed, forces_a), (fixed, forces_b)], settings, block=1)
    assert record["workers"] == 2 and record["columns"] == 5 and record["sampled_columns"] == 2
    assert record["max_share"] == 3 and record["relative_max"] < 1e-8
    assert value >= max(record["group_s"]) - 1e-12 and value > 0
    assert "scaled to its share of 3" in sample_text(record, settings)


def test_full_share_sample_scales_nothing():
    shape = (6, 4, 4)
    k0 = hex8.element_matrices((1.0, 1.0, 1.0), 0.3)[0]
    nodes = tuple(n + 1 for n in shape)
    rng = np.random.default_rng(1)
    moduli = rng.uniform(0.1, 1.0, int(np.prod(shape)))
    clamp = np.flatnonzero(np.indices(nodes).reshape(3, -1)[0] == 0)
    fixed = (3 * clamp[:, None] + np.arange(3)).ravel()
    forces = rng.standard_normal((3 * int(np.prod(nodes)), 3))
    forces[fixed] = 0.0
    settings = {"tolerance": 1e-8}
    with ParallelBaseline(2) as pool:
        value, record = pool.sample(shape, k0, moduli, [(fixed, forces)], settings)
    assert record["sampled_columns"] == record["columns"] == 3 and record["block"] is None
    assert "nothing scaled" in sample_text(record, settings) and value == max(record["group_s"])
