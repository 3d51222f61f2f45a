"""tf_gram_static: the flexibility product F = A B^T for callers that cannot allocate device
memory (a host that owns every allocation through a fixed budget, or code inside its
callbacks).  It must agree with tf_gram, which takes a caller-allocated scratch buffer,
on consecutive calls that reuse the library's one static scratch array.

This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_scratch_gram_matches_gram_on_consecutive_calls(cuda):
    import torch
    from deep_frame_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(11)
    # (ra, rb, n): a 42 x 42 covariance-sized product, then a smaller one that leaves
    # stale partials from the first call in the shared array
    for ra, rb, n in ((42, 42, 100003), (5, 7, 4099)):
        a = torch.as_tensor(rng.normal(size=(ra, n)), device=cuda)
        b = torch.as_tensor(rng.normal(size=(rb, n)), device=cuda)
        want = torch.empty((ra, rb), dtype=torch.float64, device=cuda)
        scratch = torch.empty(int(lib.tf_gram_scratch_size(ra, rb)), dtype=torch.float64, device=cuda)
        _lib.check(lib.tf_gram(_lib.ptr(a), ra, _lib.ptr(b), rb, n, _lib.ptr(want), _lib.ptr(scratch), None))
        for _ in range(2):
            got = torch.full((ra, rb), float("nan"), dtype=torch.float64, device=cuda)
            status = lib.tf_gram_static(_lib.ptr(a), ra, _lib.ptr(b), rb, n, _lib.ptr(got), None)
            assert status == 0, lib.tf_last_error(None)
            torch.cuda.synchronize()
            w, g = want.cpu().numpy(), got.cpu().numpy()
            assert np.max(np.abs(g - w)) <= 1e-12 * np.max(np.abs(w))
        exact = a.cpu().numpy() @ b.cpu().numpy().T
        assert np.max(np.abs(g - exact)) < 1e-9 * np.max(np.abs(exact))


def test_static_scratch_gram_rejects_oversized_requests(cuda):
    import torch
    from deep_frame_b200 import _lib
    lib = _lib.load()
    a = torch.zeros((64, 8), dtype=torch.float64, device=cuda)
    out = torch.zeros((64, 64), dtype=torch.float64, device=cuda)
    assert lib.tf_gram_static(_lib.ptr(a), 64, _lib.ptr(a), 64, 8, _lib.ptr(out), None) == 1
    assert b"exceeds the static scratch limit" in lib.tf_last_error(None)


def test_static_scratch_gram_allocates_no_device_memory(cuda):
    """After its first call on the device (which resolves the static array's address), further calls
    leave the device's free memory unchanged: the entry point allocates nothing."""
    import torch
    from deep_frame_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(3)
    a = torch.as_tensor(rng.normal(size=(42, 65537)), device=cuda)
    out = torch.empty((42, 42), dtype=torch.float64, device=cuda)
    assert lib.tf_gram_static(_lib.ptr(a), 42, _lib.ptr(a), 42, 65537, _lib.ptr(out), None) == 0
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert lib.tf_gram_static(_lib.ptr(a), 42, _lib.ptr(a), 42, 65537, _lib.ptr(out), None) == 0
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
