"""CPU oracle for the hex8 SIMP / GMG-PCG / covariance / filter / MMA path.

This package is TEST INFRASTRUCTURE. It restates the reference algorithm in
plain NumPy/SciPy so that the CUDA product path can be checked against it.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` may import it, and only as the checker or the timed CPU
baseline.  Nothing in ``deep_frame_b200`` imports it, and the product path
never falls back to it.

Each module cites the reference file:line it follows.  Parity is pinned by
``tests/golden/*.npz`` (generated from the reference's own Python code by
``tests/golden/make_golden.py``); the MMA restatement has no reference
numbers to pin against (mmapy is not vendored), so MMA parity is unpinned.
"""
