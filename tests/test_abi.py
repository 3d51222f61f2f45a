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
