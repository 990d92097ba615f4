"""ctypes binding of the in-tree CUDA library ``libfemk.so`` (the C ABI of ``include/femk.h``).

There is no CPU fallback: if the library is missing or no CUDA device is present, every entry
point raises. Status codes map to exceptions with the library's own message.
"""

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfemk.so")

FEMK_OK = 0
FEMK_EINVAL = 1
FEMK_ECUDA = 2
FEMK_ENOMEM = 3
FEMK_NOT_CONVERGED = 4
FEMK_NONFINITE = 5
FEMK_TIMEOUT = 6
FEMK_EBOUNDS = 7
FEMK_BREAKDOWN = 8

COEF_EXP, COEF_LINEAR, COEF_CONST = 0, 1, 2
COEF_NODAL_EXP, COEF_NODAL_LINEAR = 3, 4  # nodal P1 parameters (one value per P1 vertex)
MIXED_RELIABLE, MIXED_RESTART = 0, 1
DIRICHLET_SYMMETRIC, DIRICHLET_ROWS = 0, 1  # transient A': symmetric elimination / row replacement

_STATUS_NAMES = {
    1: "EINVAL",
    2: "ECUDA",
    3: "ENOMEM",
    4: "NOT_CONVERGED",
    5: "NONFINITE",
    6: "TIMEOUT",
    7: "EBOUNDS",
    8: "BREAKDOWN",
}


class FemkError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"femk error {_STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("order", ctypes.c_int32),
        ("ndof_local", ctypes.c_int32),
        ("ntet", ctypes.c_int64),
        ("nvert", ctypes.c_int64),
        ("n", ctypes.c_int64),
        ("nnz", ctypes.c_int64),
        ("n_dirichlet", ctypes.c_int64),
        ("cols16", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("sell_nnz", ctypes.c_int64),
        ("batch_graph", ctypes.c_int32),
        ("sell_col_units", ctypes.c_int64),
        ("dim", ctypes.c_int32),
    ]


class PlanOptions(ctypes.Structure):
    """``femk_plan_options`` (include/femk.h): per-plan layout and tuning options."""

    _fields_ = [
        ("size", ctypes.c_int32),
        ("solver_layout", ctypes.c_int32),
        ("column_tables", ctypes.c_int32),
        ("cols16", ctypes.c_int32),
        ("graph_replay", ctypes.c_int32),
        ("l2_hints", ctypes.c_int32),
        ("ring64", ctypes.c_int32),
        ("ring32", ctypes.c_int32),
        ("csr_lanes", ctypes.c_int32),
        ("csr_rows", ctypes.c_int32),
        ("sell_batch", ctypes.c_int32),
        ("vec_blocks", ctypes.c_int32),
        ("split_updates", ctypes.c_int32),
        ("test_skip_arrival", ctypes.c_int32),
        ("mixed_delta2", ctypes.c_double),
        ("barrier_limit_ms", ctypes.c_double),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

#: name -> argtypes of every entry point declared in include/femk.h
SIGNATURES = {
    "femk_version": [],
    "femk_bounds_checked": [],
    "femk_kernel_launches": [],
    "femk_last_error_string": [],
    "femk_plan_create": [_P, _I64, _P, _I64, _I, _P, _P, ctypes.POINTER(_P)],
    "femk_plan_create_simplex": [_P, _I, _I64, _P, _I64, _I, _P, _P, ctypes.POINTER(_P)],
    "femk_plan_options_default": [_P],
    "femk_plan_create_ex": [_P, _I, _I64, _P, _I64, _I, _P, _P, _P, ctypes.POINTER(_P)],
    "femk_plan_destroy": [_P],
    "femk_plan_get_info": [_P, ctypes.POINTER(PlanInfo)],
    "femk_plan_export": [_P, _P, _P, _P, _P, _P, _P, _P, _P],
    "femk_assemble": [_P, _P, _I, _D, _D, _P, _P, _P, _P],
    "femk_assemble_vjp": [_P, _P, _I, _D, _P, _P, _P, _P, _P],
    "femk_compact": [_P, _P, _P, _P, _P, _I64, ctypes.POINTER(_I64), _P],
    "femk_element_matrices": [_P, _P, _P, _P],
    "femk_jacobi": [_P, _P, _P, _P],
    "femk_jacobi_matfree": [_P, _P, _I, _D, _P, _P],
    "femk_spmv": [_P, _P, _P, _P, _P],
    "femk_prepare_operator": [_P, _P, _P],
    "femk_spmv_prepared": [_P, _P, _P, _P],
    "femk_set_profiling": [_P, _I],
    "femk_get_profile": [_P, _P, _P, _P, _P],
    "femk_spmv_matfree": [_P, _P, _I, _D, _P, _P, _P],
    "femk_pcg": [_P, _P, _P, _P, _P, _D, _D, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_D), _P],
    "femk_pcg_noalloc": [_P, _P, _P, _P, _P, _D, _D, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_D), _P],
    "femk_bicgstab": [_P, _P, _P, _P, _P, _D, _D, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_D), _P],
    "femk_gmres": [_P, _P, _P, _P, _P, _D, _D, _I32, ctypes.c_int64, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                   ctypes.POINTER(_D), _P],
    "femk_pcg_matfree": [_P, _P, _I, _D, _P, _P, _P, _D, _D, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_D), _P],
    "femk_pcg_mixed": [_P, _P, _P, _P, _P, _D, _D, _I32, _I, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                       ctypes.POINTER(_D), _P],
    "femk_pcg_batched": [_P, _I32, _P, _P, _P, _P, _P, _D, _D, _I32, _I32, _I32, _P, _P, _P, _P],
    "femk_pcg_batched_mixed": [_P, _I32, _P, _P, _P, _P, _P, _D, _D, _I32, _I32, _I32, _P, _P, _P, _P, _P],
    "femk_adjoint_grad": [_P, _P, _I, _D, _P, _P, _P, _P],
    "femk_lumped_mass": [_P, _P, _P],
    "femk_mass_matrix": [_P, _I, _P, _P],
    "femk_assemble_theta": [_P, _P, _I, _D, _D, _P, _D, _D, _I, _P, _P, _P, _P],
    "femk_theta_march": [_P, _P, _P, _P, _P, _I32, _D, _I32, _D, _P, _P, _P, ctypes.POINTER(_D), _P],
}

_lib = None
_lock = threading.Lock()


def load():
    """Load and type the library (once). Raises ImportError if it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build the sm_100a kernels with `python -m jno_b200._build` "
                "(there is no CPU fallback)"
            )
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = {"femk_last_error_string": ctypes.c_char_p, "femk_kernel_launches": ctypes.c_int64,
                          "femk_plan_options_default": None}.get(name, ctypes.c_int)
        _lib = lib
        return lib


def check(status, allow=()):
    if status == FEMK_OK or status in allow:
        return status
    msg = load().femk_last_error_string().decode(errors="replace")
    raise FemkError(status, msg)


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_handle(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
