"""ctypes binding of liblu_b200.so (the C ABI in include/lu_b200.h).

The product path has no fallback: if the in-tree library is missing or fails
to load, every call raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblu_b200.so")

LU_OK = 0
LU_ERR_ARG, LU_ERR_CUDA, LU_ERR_TIMEOUT, LU_ERR_NONFINITE = -1, -2, -3, -4
LU_ERR_NOCONV, LU_ERR_ALIGN, LU_ERR_NOMEM, LU_ERR_UNSUPPORTED = -5, -6, -7, -8
LU_PREC_FP64, LU_PREC_BF16, LU_PREC_FP16S, LU_PREC_FP16X3, LU_PREC_FP32 = 0, 1, 2, 3, 4
LU_IR_CLASSIC, LU_IR_GMRES = 0, 1
LU_LAYOUT_ROW, LU_LAYOUT_COL = 0, 1

# every symbol the header declares (checked by the CPU test suite)
EXPORTS = [
    "lu_config_default", "lu_create", "lu_destroy", "lu_workspace_bytes", "lu_status", "lu_factor",
    "lu_solve", "lu_factor_solve", "lu_residual", "lu_refine_solve", "lu_refine_solve_host", "lu_adjoint",
    "lu_batched_factor_solve", "lu_generate_uniform", "lu_matgen_host", "lu_status_string",
    "lu_profile", "lu_phase_times", "lu_launch_count", "lu_solve_noalloc",
    "lu_batched_work_bytes", "lu_batched_set_tuning", "lu_refine_factor", "lu_refine_apply",
    "lu_refine_adjoint", "lu_panel_factor", "lu_apply_pivots", "lu_trsm_lower_unit", "lu_gemm_update",
    "lu_trsv_block", "lu_gemv_update", "lu_copy_2d", "lu_transpose_square", "lu_status_clear",
    "lu_refine_precond_norm", "lu_batched_refine_histogram",
]
PHASES = ["panel", "laswp", "trsm", "gemm", "gemm_inner", "solve", "other"]


class LuConfig(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64), ("block_size", ctypes.c_int32), ("pivot_batch", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("lookahead", ctypes.c_int32), ("use_graph", ctypes.c_int32),
        ("ir_mode", ctypes.c_int32), ("ir_max_iter", ctypes.c_int32), ("layout", ctypes.c_int32),
        ("sing_threshold", ctypes.c_double), ("ir_target", ctypes.c_double), ("spin_limit", ctypes.c_int64),
        ("gmres_restart", ctypes.c_int32), ("ir_stall", ctypes.c_int32), ("gmres_tol", ctypes.c_double),
    ]


class LuResidualInfo(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("amax", "anorm", "bnorm", "xnorm", "rnorm", "r_ref", "r_hpl")]


class LuRefineInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("gmres_iterations", ctypes.c_int32),
                ("used_gmres", ctypes.c_int32), ("status", ctypes.c_int32),
                ("r_hpl", ctypes.c_double), ("r_hpl_initial", ctypes.c_double), ("host_bytes", ctypes.c_int64),
                ("rejected", ctypes.c_int32), ("reserved", ctypes.c_int32)]


_lib = None


def load():
    """Load the in-tree library (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"liblu_b200.so not built at {LIB_PATH}; run charmlu_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    P, i64, i32, u64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64
    H = ctypes.c_void_p
    sig = {
        "lu_config_default": ([ctypes.POINTER(LuConfig), i64, i32], ctypes.c_int),
        "lu_create": ([ctypes.POINTER(LuConfig), ctypes.POINTER(H)], ctypes.c_int),
        "lu_destroy": ([H], ctypes.c_int),
        "lu_workspace_bytes": ([ctypes.POINTER(LuConfig)], ctypes.c_size_t),
        "lu_status": ([H, P], ctypes.c_int),
        "lu_factor": ([H, P, i64, P, P, P], ctypes.c_int),
        "lu_solve": ([H, P, i64, P, P, i64, i64, ctypes.c_int, P], ctypes.c_int),
        "lu_factor_solve": ([H, P, i64, P, P, P], ctypes.c_int),
        "lu_residual": ([H, P, i64, P, P, ctypes.POINTER(LuResidualInfo), P], ctypes.c_int),
        "lu_refine_solve": ([H, P, i64, P, P, ctypes.POINTER(LuRefineInfo), P], ctypes.c_int),
        "lu_refine_solve_host": ([H, P, i64, P, P, ctypes.POINTER(LuRefineInfo), P], ctypes.c_int),
        "lu_panel_factor": ([H, P, i64, i64, i32, P, i64, P], ctypes.c_int),
        "lu_apply_pivots": ([H, P, i64, i64, i32, P, i64, i32, i32, i32, P, P], ctypes.c_int),
        "lu_trsm_lower_unit": ([H, P, i64, i32, P, i64, i64, P], ctypes.c_int),
        "lu_gemm_update": ([H, P, i64, P, i64, P, i64, i64, i64, i64, P], ctypes.c_int),
        "lu_trsv_block": ([H, P, i64, i32, i32, P, P], ctypes.c_int),
        "lu_gemv_update": ([H, P, i64, i64, i32, P, P, P], ctypes.c_int),
        "lu_copy_2d": ([P, i64, P, i64, i64, i64, P], ctypes.c_int),
        "lu_transpose_square": ([P, i64, i64, P], ctypes.c_int),
        "lu_status_clear": ([H, P], ctypes.c_int),
        "lu_adjoint": ([H, P, i64, P, P, i64, P, i64, i64, P, i64, P, i64, P], ctypes.c_int),
        "lu_refine_factor": ([H, P, i64, P], ctypes.c_int),
        "lu_refine_apply": ([H, P, i64, i32, P, i64, P, i64, i64, ctypes.POINTER(LuRefineInfo), P], ctypes.c_int),
        "lu_refine_adjoint": ([H, P, i64, P, i64, P, i64, i64, P, i64, P, i64, ctypes.POINTER(LuRefineInfo), P],
                              ctypes.c_int),
        "lu_refine_precond_norm": ([H, P, i64, i32, ctypes.POINTER(ctypes.c_double), P], ctypes.c_int),
        "lu_batched_factor_solve": ([i32, P, P, P, P, P, P, i32, P, ctypes.c_size_t, P], ctypes.c_int),
        "lu_generate_uniform": ([P, i64, i64, i64, u64, u64, P], ctypes.c_int),
        "lu_matgen_host": ([P, i64, i32, i64], ctypes.c_int),
        "lu_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "lu_profile": ([H, ctypes.c_int], ctypes.c_int),
        "lu_phase_times": ([H, P, P, P], ctypes.c_int),
        "lu_launch_count": ([], ctypes.c_int64),
        "lu_solve_noalloc": ([P, i64, i64, P, P, P, P], ctypes.c_int),
        "lu_batched_work_bytes": ([i32, P, i32], ctypes.c_size_t),
        "lu_batched_set_tuning": ([i32, P], ctypes.c_int),
        "lu_batched_refine_histogram": ([P, P, P], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L
