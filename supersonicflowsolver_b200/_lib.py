"""ctypes binding of libpsst_b200.so (C ABI declared in include/psst_b200.h).

The shared library is built in-tree by ``__graft_entry__.build()`` (or
``make -C supersonicflowsolver_b200/csrc``). There is no CPU fallback: if the
library is missing, importing the solver API fails loudly.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# PSST_B200_LIB selects another build of the library (e.g. one compiled with
# other register budgets); default: the in-tree build.
LIB_PATH = os.environ.get("PSST_B200_LIB") or os.path.join(HERE, "_build", "libpsst_b200.so")

PSST_OK = 0
STATUS_NAMES = {1: "PSST_ERR_ARG", 2: "PSST_ERR_IO", 3: "PSST_ERR_FORMAT", 4: "PSST_ERR_CUDA",
                5: "PSST_ERR_NONFINITE", 6: "PSST_ERR_FLUX", 7: "PSST_ERR_TIMEOUT",
                8: "PSST_ERR_UNSUPPORTED", 9: "PSST_ERR_STATE"}

# every symbol include/psst_b200.h declares (checked by tests/test_abi.py)
EXPORTED = [
    "psst_last_error", "psst_abi_version", "psst_grid_read_fluent", "psst_grid_from_fluent",
    "psst_grid_get_info", "psst_grid_get_array", "psst_grid_free", "psst_case_read",
    "psst_grid_set_boundary", "psst_solver_create", "psst_solver_set_state", "psst_solver_get_state",
    "psst_gradient_calculate", "psst_convective_calculate", "psst_stage_update", "psst_explicit_solve",
    "psst_solver_get_array", "psst_solver_set_stream", "psst_solver_last_stats", "psst_solver_profile",
    "psst_solver_autotune", "psst_solver_launch_shape", "psst_solver_iter",
    "psst_solver_destroy", "psst_convective_residual_static",
    "psst_grid_merge", "psst_grid_case_count", "psst_grid_initial_state", "psst_write_fluent",
    "psst_solver_use_graphs", "psst_solver_set_active", "psst_solver_case_residuals",
    "psst_solver_use_wavefront", "psst_solver_set_wait_limit", "psst_solver_schedule_info",
    "psst_solver_set_stop_rule", "psst_solver_case_status", "psst_solver_save_checkpoint",
    "psst_solver_load_checkpoint", "psst_solver_run_to_stop",
    "psst_mlp_create", "psst_mlp_param_count", "psst_mlp_get_params", "psst_mlp_set_params", "psst_mlp_forward",
    "psst_mlp_gradients", "psst_mlp_train_step", "psst_mlp_set_stream", "psst_mlp_destroy", "psst_tc_gemm_bf16",
    "psst_tc_gemm_bf16_wait", "psst_tc_gemm_bf16_time",
]


class PsstError(RuntimeError):
    """A failing libpsst_b200 call; ``status`` is the psst_status code."""

    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status
        self.message = message


class GridInfo(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int32), ("nvol", ctypes.c_int64), ("ninterior", ctypes.c_int64),
                ("nghost", ctypes.c_int64), ("nface", ctypes.c_int64), ("max_faces_per_cell", ctypes.c_int32),
                ("min_vol", ctypes.c_double)]


class Scheme(ctypes.Structure):
    """psst_scheme: the settings psstGridFV::solver_parameters selects."""
    _fields_ = [("flux", ctypes.c_int32), ("order", ctypes.c_int32), ("grad", ctypes.c_int32),
                ("limiter", ctypes.c_int32), ("lc", ctypes.c_int32), ("lc1_mode", ctypes.c_int32),
                ("rk_level", ctypes.c_int32), ("rk", ctypes.c_double * 16), ("cfl", ctypes.c_double),
                ("rm", ctypes.c_double), ("cp", ctypes.c_double), ("cv", ctypes.c_double),
                ("gamma", ctypes.c_double), ("ref_vel", ctypes.c_double), ("venkat_k", ctypes.c_double),
                ("precision", ctypes.c_int32), ("renumber", ctypes.c_int32), ("iter", ctypes.c_int64),
                ("max_iter", ctypes.c_int64), ("iter_step", ctypes.c_int64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "rk"}
        d["rk"] = list(self.rk)[: self.rk_level]
        return d


class ZoneDesc(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("bc_type", ctypes.c_int64), ("first", ctypes.c_int64),
                ("last", ctypes.c_int64), ("name", ctypes.c_char_p)]


class FluentDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int32), ("nvert", ctypes.c_int64), ("verts", ctypes.c_void_p),
                ("nface", ctypes.c_int64), ("face_ptr", ctypes.c_void_p), ("face_nodes", ctypes.c_void_p),
                ("face_c0", ctypes.c_void_p), ("face_c1", ctypes.c_void_p), ("ncell", ctypes.c_int64),
                ("nzone", ctypes.c_int32), ("zones", ctypes.POINTER(ZoneDesc))]


_lib = None


def load():
    """Loads libpsst_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libpsst_b200.so is not built (%s); run __graft_entry__.build()" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    P, I, I64, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_char_p
    sig = {
        "psst_last_error": (S, []),
        "psst_abi_version": (I, []),
        "psst_grid_read_fluent": (I, [S, ctypes.POINTER(P)]),
        "psst_grid_from_fluent": (I, [ctypes.POINTER(FluentDesc), ctypes.POINTER(P)]),
        "psst_grid_get_info": (I, [P, ctypes.POINTER(GridInfo)]),
        "psst_grid_get_array": (I, [P, S, P, I64]),
        "psst_grid_free": (None, [P]),
        "psst_case_read": (I, [P, S, S, ctypes.POINTER(Scheme), P]),
        "psst_grid_set_boundary": (I, [P, S, I, P, D, I, D]),
        "psst_solver_create": (I, [P, ctypes.POINTER(Scheme), I, ctypes.POINTER(P)]),
        "psst_solver_set_state": (I, [P, P]),
        "psst_solver_get_state": (I, [P, P, P]),
        "psst_gradient_calculate": (I, [P]),
        "psst_convective_calculate": (I, [P]),
        "psst_stage_update": (I, [P, I, P]),
        "psst_explicit_solve": (I, [P, I, P, P]),
        "psst_solver_get_array": (I, [P, S, P, I64]),
        "psst_solver_set_stream": (I, [P, P]),
        "psst_solver_last_stats": (I, [P, ctypes.POINTER(I64), ctypes.POINTER(D)]),
        "psst_solver_profile": (I, [P, I, P, P]),
        "psst_solver_autotune": (I, [P, I, P]),
        "psst_solver_launch_shape": (I, [P, P, P]),
        "psst_solver_iter": (I64, [P]),
        "psst_solver_destroy": (None, [P]),
        "psst_convective_residual_static": (I, [ctypes.c_int32] * 5 + [P] * 7 + [D] * 4 + [P, P]),
        "psst_grid_merge": (I, [P, ctypes.c_int32, ctypes.POINTER(P)]),
        "psst_write_fluent": (I, [P, P, P, S]),
        "psst_grid_case_count": (I, [P, P, P]),
        "psst_grid_initial_state": (I, [P, P, I64]),
        "psst_solver_use_graphs": (I, [P, I]),
        "psst_solver_set_active": (I, [P, P]),
        "psst_solver_case_residuals": (I, [P, I, P]),
        "psst_solver_use_wavefront": (I, [P, I]),
        "psst_solver_set_wait_limit": (I, [P, I64]),
        "psst_solver_schedule_info": (I, [P, P]),
        "psst_solver_set_stop_rule": (I, [P, D, ctypes.c_int32, P, P]),
        "psst_solver_case_status": (I, [P, P, P, P, P]),
        "psst_solver_run_to_stop": (I, [P, I64, I, P, P, P]),
        "psst_solver_save_checkpoint": (I, [P, S]),
        "psst_solver_load_checkpoint": (I, [P, S]),
        "psst_mlp_create": (I, [I, ctypes.c_uint64, ctypes.POINTER(P)]),
        "psst_mlp_param_count": (I64, [P]),
        "psst_mlp_get_params": (I, [P, P, I64]),
        "psst_mlp_set_params": (I, [P, P, I64]),
        "psst_mlp_forward": (I, [P, P, I, P]),
        "psst_mlp_gradients": (I, [P, P, P, I, P, ctypes.POINTER(ctypes.c_float)]),
        "psst_mlp_train_step": (I, [P, P, P, I, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]),
        "psst_mlp_set_stream": (I, [P, P]),
        "psst_mlp_destroy": (None, [P]),
        "psst_tc_gemm_bf16": (I, [P, I64, I64, P, I64, I64, I, I, I, I, P, I64, P]),
        "psst_tc_gemm_bf16_wait": (I, [P, I64, I64, P, I64, I64, I, I, I, I, P, I64, P, I64]),
        "psst_tc_gemm_bf16_time": (I, [P, I64, I64, P, I64, I64, I, I, I, I, P, I64, P, I, ctypes.POINTER(D)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status):
    if status != PSST_OK:
        raise PsstError(status, load().psst_last_error().decode(errors="replace"))
