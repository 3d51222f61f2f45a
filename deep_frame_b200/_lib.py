"""ctypes binding of ``libtfb200.so`` (the C ABI declared in include/tf_b200.h).

The library is loaded from the package directory.  There is no fallback: if
the shared library is missing or fails to load, every entry point raises.
"""
import ctypes
import threading
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "libtfb200.so"

STATUS = {0: "ok", 1: "invalid", 2: "cuda", 3: "not_converged", 4: "numeric", 5: "internal"}
PRECISION = {"float64": 0, "float32": 1, "bfloat16": 2, "float16": 3}
SMOOTHER = {"jacobi": 0, "chebyshev": 1}
CYCLE = {"V": 0, "W": 1}
COARSE = {"galerkin": 0, "rediscretize": 1}

# every symbol include/tf_b200.h declares (checked by the CPU test suite)
SYMBOLS = ("tf_default_settings", "tf_create", "tf_levels", "tf_update", "tf_set_bc", "tf_prepare", "tf_precondition",
           "tf_solve", "tf_solve_guess", "tf_solve_batch", "tf_apply", "tf_apply_level", "tf_mass_apply", "tf_element_energy", "tf_gram", "tf_gram_scratch_size", "tf_gram_static", "tf_combine", "tf_timers", "tf_launch_count",
           "tf_destroy", "tf_last_error")
SYMBOLS += ("tf_filter_create", "tf_filter_apply", "tf_filter_sums", "tf_filter_project", "tf_filter_volume", "tf_oc_update",
            "tf_filter_destroy",
            "tf_filter_last_error", "tf_mma_create", "tf_mma_step", "tf_mma_destroy", "tf_mma_last_error", "tf_simp",
            "tf_chol_create", "tf_chol_factor_csr", "tf_chol_solve", "tf_chol_destroy", "tf_chol_last_error")
SYMBOLS += ("tf_nn_last_error", "tf_nn_gemm", "tf_nn_pack16", "tf_nn_conv16", "tf_nn_im2col", "tf_nn_col2im", "tf_nn_bias_act", "tf_nn_act_back", "tf_nn_pool",
            "tf_nn_resample", "tf_nn_mse", "tf_nn_mse_scratch_doubles", "tf_nn_adam")
TIMER_CLASSES = ("fine_fp64", "fine_work", "coarse", "transfer", "vector", "coarsest", "setup", "energy", "fine_pcg32")


class TfSettings(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("smoother", ctypes.c_int32), ("cycle", ctypes.c_int32),
                ("coarse", ctypes.c_int32), ("sweeps", ctypes.c_int32), ("chebyshev_degree", ctypes.c_int32),
                ("max_levels", ctypes.c_int32), ("power_iterations", ctypes.c_int32), ("max_iterations", ctypes.c_int32),
                ("retries", ctypes.c_int32), ("batch", ctypes.c_int32), ("tensor_cores", ctypes.c_int32),
                ("coarsest_dofs", ctypes.c_int64), ("damping", ctypes.c_double), ("chebyshev_ratio", ctypes.c_double),
                ("growth", ctypes.c_double), ("tolerance", ctypes.c_double), ("dead_ratio", ctypes.c_double),
                ("zero_rhs", ctypes.c_double), ("reliable", ctypes.c_double), ("pcg_precision", ctypes.c_int32),
                ("fine_tz", ctypes.c_int32)]


class TfGrid(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int64 * 3), ("spacing", ctypes.c_double * 3)]


class TfReport(ctypes.Structure):
    _fields_ = [("iterations", ctypes.POINTER(ctypes.c_int32)), ("relative_residual", ctypes.POINTER(ctypes.c_double)),
                ("history", ctypes.POINTER(ctypes.c_double)), ("history_capacity", ctypes.c_int32),
                ("history_len", ctypes.c_int32), ("converged", ctypes.c_int32), ("batches", ctypes.c_int32),
                ("retried_columns", ctypes.c_int32), ("zero_rhs_columns", ctypes.c_int32), ("levels", ctypes.c_int32),
                ("steps", ctypes.c_int32), ("coarsest_dofs", ctypes.c_int64), ("seconds", ctypes.c_double),
                ("setup_s", ctypes.c_double), ("lambda_max", ctypes.c_double * 16)]


class TfMmaSettings(ctypes.Structure):
    _fields_ = [(name, ctypes.c_double) for name in ("move", "asyinit", "asydecr", "asyincr", "asymin", "asymax", "raa0", "albefa", "epsimin")]


class TfOcReport(ctypes.Structure):
    _fields_ = [("multiplier", ctypes.c_double), ("lower", ctypes.c_double), ("volume", ctypes.c_double),
                ("evaluations", ctypes.c_int32), ("lowest", ctypes.c_int32)]


class TfError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


_lock = threading.Lock()
_lib = None


def load():
    """Load the library once; raises RuntimeError when it is missing (no CPU fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIBRARY.exists():
            raise RuntimeError(f"{LIBRARY.name} is not built; run `python -m deep_frame_b200.build` "
                               "(the CUDA path has no CPU fallback)")
        lib = ctypes.CDLL(str(LIBRARY))
        P, I32, I64, U64, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
        sig = {
            "tf_default_settings": [ctypes.POINTER(TfSettings)],
            "tf_create": [ctypes.POINTER(TfGrid), P, P, ctypes.POINTER(TfSettings), ctypes.POINTER(P)],
            "tf_levels": [P, ctypes.POINTER(I32), ctypes.POINTER(I64)],
            "tf_update": [P, P, P],
            "tf_set_bc": [P, U64, P, I64],
            "tf_prepare": [P, U64, ctypes.POINTER(TfReport), P],
            "tf_precondition": [P, U64, P, I32, P, P],
            "tf_solve": [P, U64, P, I32, P, ctypes.POINTER(TfReport), P],
            "tf_solve_guess": [P, U64, P, I32, P, ctypes.POINTER(TfReport), P],
            "tf_solve_batch": [P, P, I32, P, P, P, ctypes.POINTER(TfReport), P],
            "tf_mass_apply": [P, U64, P, P, P, I32, P, P],
            "tf_apply": [P, U64, I32, P, I32, P, P],
            "tf_apply_level": [P, U64, I32, P, I32, P, P],
            "tf_element_energy": [P, P, I32, P, I32, P, P, P, I32, I32, P],
            "tf_gram": [P, I32, P, I32, I64, P, P, P],
            "tf_gram_scratch_size": [I32, I32],
            "tf_gram_static": [P, I32, P, I32, I64, P, P],
            "tf_timers": [P, I32, ctypes.POINTER(D), ctypes.POINTER(I64), I32],
            "tf_launch_count": [],
            "tf_destroy": [P],
            "tf_last_error": [P],
            "tf_filter_create": [ctypes.POINTER(I64), ctypes.POINTER(D), D, P, P, ctypes.POINTER(P)],
            "tf_filter_apply": [P, P, P, P, I32, P],
            "tf_filter_sums": [P, P, P],
            "tf_filter_project": [P, P, D, D, I32, P, P, P],
            "tf_filter_volume": [P, P, P, D, D, I32, P, P],
            "tf_oc_update": [P, P, P, P, P, D, D, D, D, D, I32, P, ctypes.POINTER(TfOcReport), P],
            "tf_filter_destroy": [P],
            "tf_filter_last_error": [P],
            "tf_mma_create": [I32, I64, ctypes.POINTER(P)],
            "tf_mma_step": [P, I32, P, P, P, P, P, P, P, P, P, P, D, P, P, P, ctypes.POINTER(TfMmaSettings), P, P, P, P,
                            ctypes.POINTER(I32), P],
            "tf_mma_destroy": [P],
            "tf_mma_last_error": [P],
            "tf_simp": [P, I64, D, D, D, P, P, P, P, P],
            "tf_combine": [P, I32, I64, P, I32, P, P],
            "tf_chol_create": [I64, ctypes.POINTER(P)],
            "tf_chol_factor_csr": [P, P, P, P, P],
            "tf_chol_solve": [P, P, I32, P, P],
            "tf_chol_destroy": [P],
            "tf_chol_last_error": [P],
            "tf_nn_last_error": [],
            "tf_nn_gemm": [I32, I32, I32, I32, I32, ctypes.c_float, P, I32, P, I32, ctypes.c_float, P, I32, P, I64, P],
            "tf_nn_pack16": [P, I32, I32, P, I32, I32, P],
            "tf_nn_conv16": [P, I32, P, P, I32, I32, I32, P, I32, P, P, P],
            "tf_nn_im2col": [P, I32, P, P, P],
            "tf_nn_col2im": [P, I32, P, P, P],
            "tf_nn_bias_act": [P, P, I32, I64, I32, P],
            "tf_nn_act_back": [P, P, I32, I64, I32, P, I32, P],
            "tf_nn_pool": [P, I32, P, P, P, P],
            "tf_nn_resample": [P, I32, P, P, I32, P, P],
            "tf_nn_mse": [P, P, P, I64, D, P, P, P, P],
            "tf_nn_mse_scratch_doubles": [],
            "tf_nn_adam": [P, P, P, P, I64, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, I32, P],
        }
        for name, args in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = {"tf_last_error": ctypes.c_char_p, "tf_filter_last_error": ctypes.c_char_p, "tf_mma_last_error": ctypes.c_char_p, "tf_chol_last_error": ctypes.c_char_p,
                          "tf_nn_last_error": ctypes.c_char_p, "tf_nn_mse_scratch_doubles": ctypes.c_int64,
                          "tf_gram_scratch_size": ctypes.c_int64, "tf_launch_count": ctypes.c_int64}.get(name, ctypes.c_int)
        _lib = lib
        return lib


def check(status, handle=None, what="call"):
    """Raise ValueError for invalid arguments and TfError for device/numeric failures."""
    if status == 0:
        return
    lib = load()
    message = (lib.tf_last_error(handle) or b"").decode(errors="replace")
    text = f"{what} failed ({STATUS.get(status, status)}): {message}"
    if status == 1:
        raise ValueError(text)
    raise TfError(status, text)


def default_settings():
    s = TfSettings()
    check(load().tf_default_settings(ctypes.byref(s)))
    return s


def ptr(tensor):
    """Raw device pointer of a tensor (None for None)."""
    return None if tensor is None else ctypes.c_void_p(tensor.data_ptr())


def stream_of(device):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
