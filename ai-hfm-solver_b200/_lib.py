"""ctypes binding of ``libhfm.so`` (the C ABI declared in ``include/hfm.h``).

The library is loaded from this package directory.  There is no fallback: if the shared
library is missing or a CUDA call fails, the operation raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhfm.so")

# hfm_status
(OK, ERR_BAD_ARG, ERR_OOM, ERR_NOT_CONVERGED, ERR_NAN, ERR_TIMEOUT, ERR_CUDA, ERR_UNSUPPORTED,
 ERR_CANCELLED) = range(9)
# hfm_dtype
F32, BF16, F16, F64 = range(4)
# hfm_op_kind
OP_CONST7, OP_SIGMA7, OP_DIR7, OP_K27, OP_FACE7 = range(5)
# flags
FLAG_ZERO_XEND, FLAG_TOP_COPY, FLAG_ZERO_GUESS, FLAG_PERIODIC, FLAG_SAME_LEVEL_CORR = 1, 2, 4, 8, 16
FLAG_TWO_SWEEPS = 32
# hfm_cycle / hfm_accel
CYCLE_SAWTOOTH, CYCLE_V, CYCLE_F = range(3)
ACCEL_NONE, ACCEL_CG, ACCEL_IR = range(3)
(OPT_NO_FUSED_COARSE, OPT_NO_FUSED_PRE, OPT_SAWTOOTH_COARSE_SWEEPS, OPT_NO_FACES,
 OPT_PERSISTENT, OPT_TEMPORAL) = 1, 2, 4, 8, 16, 32


class HfmOperator(C.Structure):
    _fields_ = [("kind", C.c_int), ("coef_dtype", C.c_int), ("k", C.c_float * 27),
                ("c", C.c_float * 3), ("scale", C.c_float), ("coef", C.c_void_p * 7)]


class HfmMgConfig(C.Structure):
    _fields_ = [("op_kind", C.c_int), ("cycle", C.c_int), ("accel", C.c_int),
                ("n_levels", C.c_int), ("min_coarse_edge", C.c_int), ("nu_pre", C.c_int),
                ("nu_post", C.c_int), ("coarse_sweeps", C.c_int), ("omega", C.c_float),
                ("coarse_omega", C.c_float), ("coarse_scale", C.c_float),
                ("sawtooth_fine_smooth", C.c_int), ("flags", C.c_uint), ("storage", C.c_int),
                ("tol", C.c_double), ("max_cycles", C.c_int), ("cycles_per_launch", C.c_int),
                ("inner_tol", C.c_double), ("inner_max_cycles", C.c_int), ("options", C.c_int)]


class HfmSlotStats(C.Structure):
    _fields_ = [("active", C.c_int), ("status", C.c_int), ("cycles", C.c_int),
                ("outer", C.c_int), ("norm_b", C.c_double), ("rel_resid", C.c_double)]


SERVE_MAX_EDGES = 16


class HfmServeConfig(C.Structure):
    _fields_ = [("n_edges", C.c_int), ("edges", C.c_int * SERVE_MAX_EDGES), ("slots", C.c_int),
                ("budget_bytes", C.c_double), ("cycles_per_tick", C.c_int),
                ("solver", HfmMgConfig)]


class HfmServeResult(C.Structure):
    _fields_ = [("ticket", C.c_int64), ("status", C.c_int), ("cycles", C.c_int),
                ("outer", C.c_int), ("rel_resid", C.c_double)]


class HfmError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status


STATUS_NAMES = {OK: "HFM_OK", ERR_BAD_ARG: "HFM_ERR_BAD_ARG", ERR_OOM: "HFM_ERR_OOM",
                ERR_NOT_CONVERGED: "HFM_ERR_NOT_CONVERGED", ERR_NAN: "HFM_ERR_NAN",
                ERR_TIMEOUT: "HFM_ERR_TIMEOUT", ERR_CUDA: "HFM_ERR_CUDA",
                ERR_UNSUPPORTED: "HFM_ERR_UNSUPPORTED", ERR_CANCELLED: "HFM_ERR_CANCELLED"}

P = C.c_void_p
I = C.c_int
F = C.c_float
U = C.c_uint
I64 = C.c_int64

# name -> (restype, argtypes)
SIGNATURES = {
    "hfm_abi_version": (I, []),
    "hfm_status_string": (C.c_char_p, [I]),
    "hfm_last_error": (C.c_char_p, []),
    "hfm_device_sm_count": (I, [C.POINTER(I)]),
    "hfm_kernel_launch_count": (I64, []),
    "hfm_set_wait_budget": (I, [I]),
    "hfm_device_timeouts": (I, [C.POINTER(I), I]),
    "hfm_device_drain_timeouts": (I, [C.POINTER(I), I]),
    "hfm_conv3d_k3": (I, [P, P, I, I, I, I, P, P]),
    "hfm_restrict_avg": (I, [P, P, I, I, I, I, P]),
    "hfm_prolong_nearest": (I, [P, P, I, I, I, I, P]),
    "hfm_op_apply": (I, [P, P, P, I, I, I, I, P]),
    "hfm_op_residual": (I, [P, P, P, P, I, I, I, I, U, P]),
    "hfm_op_jacobi": (I, [P, P, P, P, P, I, I, I, I, F, I, U, P]),
    "hfm_op_jacobi_typed": (I, [P, I, P, P, P, I, I, I, I, F, U, P]),
    "hfm_op_residual_typed": (I, [P, I, P, P, P, I, I, I, I, U, P]),
    "hfm_residual_restrict_typed": (I, [P, I, P, P, P, P, I, I, I, I, U, P]),
    "hfm_prolong_correct_smooth_typed": (I, [P, I, P, P, P, P, I, I, I, I, F, U, P]),
    "hfm_face7_smooth2_typed": (I, [P, I, P, P, P, P, I, I, I, I, F, P]),
    "hfm_sigma7_faces": (I, [I, P, P, P, F, F, F, P, P, P, I, I, I, I, P]),
    "hfm_face7_elems": (I, [I, I, I, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]),
    "hfm_residual_restrict": (I, [P, P, P, P, P, I, I, I, I, U, P]),
    "hfm_serve_config_default": (None, [P]),
    "hfm_serve_create": (I, [P, P]),
    "hfm_serve_bucket_slots": (I, [P, I, C.POINTER(I)]),
    "hfm_serve_submit": (I, [P, I, P, P, P, P, P, C.POINTER(I64)]),
    "hfm_serve_poll": (I, [P, P, I, C.POINTER(I)]),
    "hfm_serve_cancel": (I, [P, I64]),
    "hfm_serve_pending": (I, [P, C.POINTER(I), C.POINTER(I)]),
    "hfm_serve_destroy": (I, [P]),
    "hfm_prolong_correct_smooth": (I, [P, P, P, P, P, I, I, I, I, F, U, P]),
    "hfm_stencil7_const_apply": (I, [P, P, I, I, I, I, F, F, F, P]),
    "hfm_stencil7_const_residual": (I, [P, P, P, I, I, I, I, F, F, F, U, P]),
    "hfm_stencil7_const_jacobi": (I, [P, P, P, P, I, I, I, I, F, F, F, F, I, U, P]),
    "hfm_stencil7_var_apply": (I, [P, P, P, P, P, I, I, I, I, F, F, F, P]),
    "hfm_stencil7_var_residual": (I, [P, P, P, P, P, P, I, I, I, I, F, F, F, U, P]),
    "hfm_stencil7_var_jacobi": (I, [P, P, P, P, P, P, P, I, I, I, I, F, F, F, F, I, U, P]),
    "hfm_stencil27_apply": (I, [P, P, I, I, I, I, P, P]),
    "hfm_stencil27_residual": (I, [P, P, P, I, I, I, I, P, U, P]),
    "hfm_stencil27_jacobi": (I, [P, P, P, P, I, I, I, I, P, F, I, U, P]),
    "hfm_reduce_scratch_bytes": (C.c_size_t, [I64, I]),
    "hfm_norm2_f64": (I, [P, I64, I, P, P, P]),
    "hfm_max_abs": (I, [P, I64, I, P, P, P]),
    "hfm_norm2_f64_noalloc": (I, [P, I64, I, P, P]),
    "hfm_dot_f64": (I, [P, P, I64, I, I64, P, P, P]),
    "hfm_cg_update_xr": (I, [P, P, P, P, P, P, I64, I, I64, P]),
    "hfm_cg_update_p": (I, [P, P, P, P, I64, I, I64, P]),
    "hfm_ns_momentum": (I, [P, P, P, P, P, P, P, P, P, I, I, I, P, P, P, P, F, P]),
    "hfm_ns_pressure_gradient": (I, [P, P, P, P, I, I, I, P, P, P, P]),
    "hfm_ns_divergence": (I, [P, P, P, P, I, I, I, P, P, P, I, P]),
    "hfm_ns_immersed_body": (I, [P, P, P, P, I, I, I, F, P]),
    "hfm_ns_bc_scratch_bytes": (C.c_size_t, [I, I, I]),
    "hfm_ns_bc_velocity": (I, [P, P, P, I, I, I, F, P, P]),
    "hfm_ns_bc_pressure": (I, [P, I, I, I, P, P]),
    "hfm_sigma7_grad_logsigma": (I, [P, P, P, P, P, I, I, I, I, F, F, F, P, P, P, I, P]),
    "hfm_ns_momentum_pg": (I, [P, P, P, P, P, P, P, P, P, P, P, P, I, I, I, P, P, P, F, P]),
    "hfm_ns_pg_scratch_bytes": (C.c_size_t, [I, I, I]),
    "hfm_ns_pg_dissipation": (I, [P, P, P, P, P, P, P, I, I, I, P, P, P, P, F, F, P, P]),
    # 2D operators and the Kolmogorov-flow stepper
    "hfm_conv2d_k3": (I, [P, P, I, I, I, P, U, P]),
    "hfm_restrict_avg2d": (I, [I, P, P, I, I, I, P]),
    "hfm_prolong_nearest2d": (I, [I, P, P, I, I, I, P]),
    "hfm_jacobi2d": (I, [I, P, P, P, F, P, P, I, I, I, F, U, P]),
    "hfm_residual2d": (I, [I, P, P, P, P, I, I, I, U, P]),
    "hfm_residual_restrict2d": (I, [I, P, P, P, P, I, I, I, U, P]),
    "hfm_pre2_restrict2d": (I, [I, P, P, P, P, I, I, I, F, U, P]),
    "hfm_outer_residual2d": (I, [P, P, P, I, P, I, I, I, U, P, P, P]),
    "hfm_update2d": (I, [P, I, P, F, I64, P]),
    "hfm_coarse_jacobi2d": (I, [I, P, P, P, I, I, I, F, I, U, P]),
    "hfm_subcycle2d": (I, [I, P, P, P, I, I, I, I, F, I, I, I, U, P]),
    "hfm_mean_subtract2d": (I, [P, I, I64, P]),
    "hfm_kolmogorov_stage": (I, [P, P, P, P, P, P, I, I, F, F, F, F, F, F, P]),
    "hfm_kolmogorov_divergence": (I, [P, P, P, I, I, F, F, P]),
    "hfm_kolmogorov_project": (I, [P, P, P, I, I, F, F, P]),
    "hfm_mg_config_default": (None, [C.POINTER(HfmMgConfig)]),
    "hfm_mg_footprint_bytes": (C.c_size_t, [C.POINTER(HfmMgConfig), I, I, I, I]),
    "hfm_mg_create": (I, [C.POINTER(HfmMgConfig), I, I, I, I, C.POINTER(P)]),
    "hfm_mg_destroy": (I, [P]),
    "hfm_mg_num_levels": (I, [P]),
    "hfm_mg_level_shape": (I, [P, I, C.POINTER(I), C.POINTER(I), C.POINTER(I)]),
    "hfm_mg_set_operator": (I, [P, I, C.POINTER(HfmOperator), P]),
    "hfm_mg_load": (I, [P, I, P, P, P]),
    "hfm_mg_run": (I, [P, I, P]),
    "hfm_mg_query": (I, [P, C.POINTER(HfmSlotStats), P]),
    "hfm_mg_query_async": (I, [P, P, P]),
    "hfm_mg_fetch": (I, [P, I, P, P]),
    "hfm_mg_cancel": (I, [P, I, P]),
    "hfm_mg_solve": (I, [P, P, P, C.POINTER(HfmSlotStats), P]),
    "hfm_mg_read_level": (I, [P, I, I, I, P, P]),
    "hfm_mg_load_f64": (I, [P, I, P, P, P]),
    "hfm_mg_fetch_f64": (I, [P, I, P, P]),
}

_lib = None


def lib():
    """Load libhfm.so (once).  Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libhfm.so not built: run `python ai-hfm-solver_b200/build.py` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, what=""):
    if status != OK:
        msg = lib().hfm_last_error().decode(errors="replace")
        raise HfmError(status, (what + ": " if what else "") + msg)
    return status


def call(name, *args):
    return check(getattr(lib(), name)(*args), name)
