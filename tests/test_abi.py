"""The C-ABI library loads and exports every symbol include/tf_b200.h declares (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    symbols = set()
    for header in sorted((ROOT / "include").glob("*.h")):
        text = header.read_text()
        symbols |= set(re.findall(r"TF_API\s+[\w\s\*]*?\b(tf_\w+)\s*\(", text))
    return symbols


@pytest.fixture(scope="module")
def library():
    from deep_frame_b200 import build
    path = build.build()
    return ctypes.CDLL(str(path))


def test_header_declares_entry_points():
    symbols = declared_symbols()
    assert {"tf_create", "tf_solve", "tf_apply", "tf_element_energy", "tf_destroy", "tf_last_error"} <= symbols


def test_library_exports_every_declared_symbol(library):
    for name in declared_symbols():
        assert hasattr(library, name), name


def test_binding_covers_every_declared_symbol():
    from deep_frame_b200 import _lib
    header = declared_symbols()
    bound = {name for name in header if name.startswith("tf_")}
    assert set(_lib.SYMBOLS) <= header
    missing = {name for name in bound if name not in _lib.SYMBOLS and not name.startswith(("tf_filter", "tf_mma", "tf_cov"))}
    assert not missing, missing


def test_host_only_entry_points(library):
    from deep_frame_b200 import _lib
    lib = _lib.load()
    settings = _lib.default_settings()
    assert settings.tolerance == 1e-8 and settings.max_iterations == 2000 and settings.chebyshev_degree == 3
    # invalid arguments are rejected before any device work, with a message
    handle = ctypes.c_void_p()
    assert lib.tf_create(None, None, None, None, ctypes.byref(handle)) == 1
    assert b"must not be NULL" in lib.tf_last_error(None)
    assert lib.tf_destroy(None) == 0


def test_handleless_failures_carry_a_message(library):
    """Entry points without a handle (and the create calls, whose handle stays NULL on failure)
    return TF_STATUS_INVALID with a message that every *_last_error(NULL) getter returns."""
    import numpy as np
    from deep_frame_b200 import _lib
    lib = _lib.load()
    P = ctypes.c_void_p
    out = P()
    assert lib.tf_mma_create(0, 10, ctypes.byref(out)) == 1 and out.value is None
    assert b"constraints" in lib.tf_mma_last_error(None) and lib.tf_last_error(None) == lib.tf_mma_last_error(None)
    assert lib.tf_chol_create(0, ctypes.byref(out)) == 1 and b"unknowns" in lib.tf_chol_last_error(None)
    shape, spacing = (ctypes.c_int64 * 3)(4, 4, 4), (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    allowed = np.ones(64, np.uint8)
    assert lib.tf_filter_create(shape, spacing, -1.0, allowed.ctypes.data_as(P), None, ctypes.byref(out)) == 1
    assert b"radius" in lib.tf_filter_last_error(None)
    assert lib.tf_gram(None, -1, None, 2, 10, None, None, None) == 1 and lib.tf_last_error(None).startswith(b"tf_gram:")
    assert lib.tf_simp(None, 10, 3.0, 1e-9, 1.0, None, None, None, None, None) == 1
    assert lib.tf_last_error(None).startswith(b"tf_simp:")
    assert lib.tf_combine(None, 3, 10, None, 65, None, None) == 1 and lib.tf_last_error(None).startswith(b"tf_combine:")
    assert lib.tf_solve_batch(None, None, 0, None, None, None, None, None) == 1
    assert lib.tf_last_error(None).startswith(b"tf_solve_batch: count")
    handles = (P * 2)()
    keys, counts, ptrs = (ctypes.c_uint64 * 2)(), (ctypes.c_int32 * 2)(1, 1), (P * 2)()
    assert lib.tf_solve_batch(handles, keys, 2, ptrs, counts, ptrs, None, None) == 1
    assert b"handle 0 is NULL" in lib.tf_last_error(None)


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the path of a host without a CUDA device")
def test_create_without_a_device_reports_a_cuda_error(library):
    """On a host without a usable GPU the create calls fail with TF_STATUS_CUDA, a message and a
    NULL handle: no crash and no CPU fallback."""
    import numpy as np
    from deep_frame_b200 import _lib
    from deep_frame_b200.elements import hexahedron_matrices
    lib = _lib.load()
    grid = _lib.TfGrid()
    for d in range(3):
        grid.shape[d], grid.spacing[d] = 4, 1.0
    ke = np.ascontiguousarray(hexahedron_matrices((1.0, 1.0, 1.0), 0.3)[0])
    settings = _lib.default_settings()
    handle = ctypes.c_void_p()
    assert lib.tf_create(ctypes.byref(grid), ke.ctypes.data_as(ctypes.c_void_p), None, ctypes.byref(settings), ctypes.byref(handle)) == 2
    assert handle.value is None and lib.tf_last_error(None)
    assert lib.tf_mma_create(1, 10, ctypes.byref(handle)) == 2 and handle.value is None and lib.tf_mma_last_error(None)
    assert lib.tf_chol_create(10, ctypes.byref(handle)) == 2 and handle.value is None and lib.tf_chol_last_error(None)
