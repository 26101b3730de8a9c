"""ctypes mirrors of include/gsb.h and the loader of libgsb.so.

The structs are the C-ABI of the library; ``SOLVER_STATUS_DTYPE`` is the numpy view of
``GsbStatus64``, which has the byte layout of the reference's ``SolverStatus{Float64}``
(src/base/status.jl:101-117: offsets 0, 2, 4, 8, 16, 24, 28, 29, 30, 32, 40, 48, 56, 64, 65;
size 72).
"""

from __future__ import annotations

import ctypes
import os
from enum import IntEnum

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgsb.so")


class ReturnCode(IntEnum):
    """ReturnCode, src/base/returncodes.jl:14."""

    SUCCESS = 0
    STALLED = 1
    MAXITERS = 2
    SINGULAR = 3
    NONFINITE = 4
    LINESEARCH_FAILED = 5


class Family(IntEnum):
    CUBIC_AFFINE = 1
    EXPSUM3_LSQ = 2
    IRK3_HENON_HEILES = 3
    HETERO6 = 100
    COUPLED2 = 101
    WOOD = 102
    CUBIC_AFFINE_DUAL = 103


class GsbStatus64(ctypes.Structure):
    _fields_ = [
        ("code", ctypes.c_uint8),
        ("pad0_", ctypes.c_uint8),
        ("f_calls", ctypes.c_int16),
        ("iterations", ctypes.c_int32),
        ("fnorm", ctypes.c_double),
        ("stepnorm", ctypes.c_double),
        ("step_failures", ctypes.c_int32),
        ("promoted", ctypes.c_uint8),
        ("stationary", ctypes.c_uint8),
        ("jvp_calls", ctypes.c_int16),
        ("rank", ctypes.c_int32),
        ("pad1_", ctypes.c_uint32),
        ("nullnorm", ctypes.c_double),
        ("gradratio", ctypes.c_double),
        ("rate", ctypes.c_double),
        ("contracted", ctypes.c_uint8),
        ("reused", ctypes.c_uint8),
        ("pad2_", ctypes.c_uint8 * 6),
    ]


SOLVER_STATUS_DTYPE = np.dtype(
    {
        "names": [
            "code", "f_calls", "iterations", "fnorm", "stepnorm", "step_failures", "promoted",
            "stationary", "jvp_calls", "rank", "nullnorm", "gradratio", "rate", "contracted",
            "reused",
        ],
        "formats": [
            np.uint8, np.int16, np.int32, np.float64, np.float64, np.int32, np.bool_, np.bool_,
            np.int16, np.int32, np.float64, np.float64, np.float64, np.bool_, np.bool_,
        ],
        "offsets": [0, 2, 4, 8, 16, 24, 28, 29, 30, 32, 40, 48, 56, 64, 65],
        "itemsize": 72,
    }
)
assert ctypes.sizeof(GsbStatus64) == 72


class GsbOptions(ctypes.Structure):
    _fields_ = [
        ("f_abstol", ctypes.c_double),
        ("f_reltol", ctypes.c_double),
        ("x_abstol", ctypes.c_double),
        ("x_reltol", ctypes.c_double),
        ("min_iterations", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32),
        ("max_stalls", ctypes.c_int32),
        ("norm", ctypes.c_int32),
        ("g_tol", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("roundoff", ctypes.c_uint8),
        ("rate_test", ctypes.c_uint8),
        ("pad_", ctypes.c_uint8 * 6),
    ]


class GsbProblem(ctypes.Structure):
    _fields_ = [
        ("family", ctypes.c_int32),
        ("n", ctypes.c_int32),
        ("m", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("shared", ctypes.c_void_p),
        ("shared_len", ctypes.c_int64),
    ]


class GsbMethod(ctypes.Structure):
    _fields_ = [
        ("linsolve", ctypes.c_int32),
        ("factor_precision", ctypes.c_int32),
        ("refinement", ctypes.c_int32),
        ("refine_maxiter", ctypes.c_int32),
        ("refine_eta", ctypes.c_double),
        ("globalization", ctypes.c_int32),
        ("bt_maxiter", ctypes.c_int32),
        ("static_alpha", ctypes.c_double),
        ("bt_c1", ctypes.c_double),
        ("bt_p", ctypes.c_double),
        ("lm_mu0", ctypes.c_double),
        ("lm_mu_min", ctypes.c_double),
        ("lm_mu_max", ctypes.c_double),
        ("lm_mu_decrease", ctypes.c_double),
        ("lm_mu_increase", ctypes.c_double),
        ("lm_rho_accept", ctypes.c_double),
        ("regularization", ctypes.c_double),
        ("arithmetic", ctypes.c_int32),
        ("threads_per_system", ctypes.c_int32),
        ("reuse", ctypes.c_int32),
        ("trial_precision", ctypes.c_int32),
        ("dogleg_radius", ctypes.c_double),
    ]


class GsbTally(ctypes.Structure):
    _fields_ = [("counts", ctypes.c_int64 * 6)]


class GsbBucketConfig(ctypes.Structure):
    _fields_ = [("threads_per_system", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                ("systems_per_cta", ctypes.c_int32), ("pad_", ctypes.c_int32)]


GSB_UNEVEN_BUCKETS = 9
UNEVEN_SIZES = (2, 3, 4, 6, 8, 12, 16, 24, 32)


class GsbSummary(ctypes.Structure):
    """BatchSummary{Float64}'s layout (src/nonlinear/batched.jl:63-69): offsets 0, 8, 16, 24, 32;
    size 40."""

    _fields_ = [
        ("fnorm", ctypes.c_double),
        ("all_converged", ctypes.c_uint8),
        ("pad0_", ctypes.c_uint8 * 7),
        ("failure_count", ctypes.c_int64),
        ("max_iterations", ctypes.c_int32),
        ("pad1_", ctypes.c_int32),
        ("total_iterations", ctypes.c_int64),
    ]


assert ctypes.sizeof(GsbSummary) == 40


GSB_AOS, GSB_SOA = 0, 1
GSB_STATUS64, GSB_CODES = 0, 1
GSB_LU, GSB_QR = 0, 1
GSB_F64, GSB_F32 = 0, 1
GSB_NO_REFINEMENT, GSB_REFINEMENT = 0, 1
GSB_STATIC, GSB_BACKTRACKING, GSB_LEVENBERG_MARQUARDT, GSB_DOGLEG = 0, 1, 2, 3
GSB_FUSED, GSB_UNFUSED = 0, 1

# The symbols include/gsb.h declares (checked by the CPU tests against the built library).
EXPORTED_SYMBOLS = (
    "gsb_abi_version",
    "gsb_last_error",
    "gsb_param_count",
    "gsb_default_options",
    "gsb_default_method",
    "gsb_solve_batch",
    "gsb_batch_summary",
    "gsb_solve_batch_summary",
    "gsb_synchronize",
    "gsb_solve_batch_counts_noalloc",
    "gsb_uneven_sizes",
    "gsb_solve_batch_uneven",
    "gsb_solve_batch_host",
    "gsb_umma_selftest",
    "gsb_mlp_sizes",
    "gsb_mlp_pack",
    "gsb_mlp_predict",
    "gsb_mlp_grad",
    "gsb_mlp_adam",
    "gsb_warm_start_select",
)

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libgsb.so (built by ``build.py``); raise if it is missing. There is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"libgsb.so not found at {path}: build it with `python -c 'import __graft_entry__ as g; "
            "g.build()'` (the batch solver has no CPU fallback)"
        )
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    lib.gsb_abi_version.restype = ctypes.c_int
    lib.gsb_last_error.restype = ctypes.c_char_p
    lib.gsb_param_count.argtypes = [P(GsbProblem)]
    lib.gsb_param_count.restype = ctypes.c_int64
    lib.gsb_default_options.argtypes = [P(GsbOptions)]
    lib.gsb_default_options.restype = None
    lib.gsb_default_method.argtypes = [P(GsbMethod)]
    lib.gsb_default_method.restype = None
    lib.gsb_solve_batch.argtypes = [
        P(GsbProblem), P(GsbMethod), P(GsbOptions),
        ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
        ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
        ctypes.c_int64, ctypes.c_void_p, P(GsbTally),
    ]
    lib.gsb_solve_batch.restype = ctypes.c_int
    lib.gsb_batch_summary.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, P(GsbSummary)]
    lib.gsb_batch_summary.restype = ctypes.c_int
    lib.gsb_solve_batch_summary.argtypes = [
        P(GsbProblem), P(GsbMethod), P(GsbOptions),
        ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
        ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p, P(GsbSummary),
    ]
    lib.gsb_solve_batch_summary.restype = ctypes.c_int
    lib.gsb_synchronize.argtypes = [ctypes.c_void_p]
    lib.gsb_synchronize.restype = ctypes.c_int
    lib.gsb_solve_batch_counts_noalloc.argtypes = [
        P(GsbProblem), P(GsbMethod), P(GsbOptions),
        ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
        ctypes.c_int64, ctypes.c_void_p, P(GsbTally),
    ]
    lib.gsb_solve_batch_counts_noalloc.restype = ctypes.c_int
    lib.gsb_uneven_sizes.argtypes = [ctypes.POINTER(ctypes.c_int32)]
    lib.gsb_uneven_sizes.restype = ctypes.c_int
    lib.gsb_solve_batch_uneven.argtypes = [
        P(GsbMethod), P(GsbOptions), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
    ]
    lib.gsb_solve_batch_uneven.restype = ctypes.c_int
    lib.gsb_solve_batch_host.argtypes = [
        P(GsbProblem), P(GsbMethod), P(GsbOptions), ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
    ]
    lib.gsb_solve_batch_host.restype = ctypes.c_int
    lib.gsb_umma_selftest.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
    lib.gsb_umma_selftest.restype = ctypes.c_int
    V = ctypes.c_void_p
    lib.gsb_mlp_sizes.argtypes = [ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    lib.gsb_mlp_pack.argtypes = [V, V, V]
    lib.gsb_mlp_predict.argtypes = [V, V, V, V, V, V, ctypes.c_int64, V, V]
    lib.gsb_mlp_grad.argtypes = [V, V, V, V, V, ctypes.c_int64, V, V, V, V]
    lib.gsb_mlp_adam.argtypes = [V, V, V, V, V, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                 ctypes.c_float, ctypes.c_int32, V]
    lib.gsb_warm_start_select.argtypes = [V, V, V, V, V, V, ctypes.c_int64, V]
    for f in ("gsb_mlp_sizes", "gsb_mlp_pack", "gsb_mlp_predict", "gsb_mlp_grad", "gsb_mlp_adam",
              "gsb_warm_start_select"):
        getattr(lib, f).restype = ctypes.c_int
    _lib = lib
    return lib
