"""ctypes binding of librigidfibers.so (the CUDA kernels behind include/rigidfibers.h).

The library is built in-tree (``rigidfibers_kth_b200/_lib/librigidfibers.so``)
by ``build()``.  Loading fails loudly when it is missing: there is no CPU
fallback for any computation.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RIGIDFIBERS_LIB") or os.path.join(_HERE, "_lib", "librigidfibers.so")
CSRC = os.path.join(_HERE, "csrc")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "rigidfibers.h")

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_h = ctypes.c_void_p

RF_OK = 0
STATUS = {
    0: "RF_OK",
    1: "RF_ERR_INVALID_ARG",
    2: "RF_ERR_OOM",
    3: "RF_ERR_CUDA",
    4: "RF_ERR_NOT_CONVERGED",
    5: "RF_ERR_DEVICE_TIMEOUT",
    6: "RF_ERR_NAN",
    7: "RF_ERR_NO_DEVICE",
}
RF_ERR_NOT_CONVERGED = 4

PREC_FP64, PREC_FP32, PREC_MIXED_BF16, PREC_MIXED_FP32 = 0, 1, 2, 3
PC_NONE, PC_CLUSTER, PC_LEARNED = 0, 1, 2
VEL_RECOMPUTE, VEL_REUSE = 0, 1


class RfParams(ctypes.Structure):
    """Mirror of ``rf_params`` (include/rigidfibers.h)."""

    _fields_ = [
        ("slenderness", ctypes.c_double),
        ("timestep", ctypes.c_double),
        ("num_fibers", ctypes.c_int32),
        ("num_timesteps", ctypes.c_int32),
        ("num_terms_in_force_expansion", ctypes.c_int32),
        ("num_quadrature_intervals", ctypes.c_int32),
        ("use_analytical_integration", ctypes.c_int32),
        ("use_direct_solver", ctypes.c_int32),
        ("gmres_restart", ctypes.c_int32),
        ("gmres_max_iters", ctypes.c_int32),
        ("gmres_tol", ctypes.c_double),
        ("external_force", ctypes.c_double * 3),
        ("precision", ctypes.c_int32),
        ("preconditioner", ctypes.c_int32),
        ("velocity_mode", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("max_refinements", ctypes.c_int32),
        ("cluster_size", ctypes.c_int32),
        ("inner_tol", ctypes.c_double),
        ("near_field_c", ctypes.c_double),
        ("shard_index", ctypes.c_int32),
        ("shard_count", ctypes.c_int32),
        ("pc_damping", ctypes.c_double),
        ("reserved", ctypes.c_int32 * 4),
    ]


class RfSolveStats(ctypes.Structure):
    _fields_ = [
        ("converged", ctypes.c_int32),
        ("iterations", ctypes.c_int32),
        ("matvecs", ctypes.c_int32),
        ("refinements", ctypes.c_int32),
        ("residual", ctypes.c_double),
        ("seconds", ctypes.c_double),
        ("pc_fallback", ctypes.c_int32),
        ("precision_fallback", ctypes.c_int32),
        ("preconditioned", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class RfError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def build(verbose=False):
    """Compile the CUDA library for sm_100a with nvcc (make in csrc/)."""
    out = subprocess.run(["make", "-s", "-j8", "-C", CSRC], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("librigidfibers build failed:\n" + out.stdout + out.stderr)
    if verbose:
        print(out.stdout)


_lib = None


def lib():
    """Load librigidfibers.so; raises if the CUDA library has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"CUDA library {LIB_PATH} is missing; build it with rigidfibers_kth_b200.build() "
            "(there is no CPU fallback)"
        )
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER(RfParams)
    sig = {
        "rf_params_default": (None, [P]),
        "rf_create": (ctypes.c_int, [P, _dp, _dp, ctypes.POINTER(_h)]),
        "rf_destroy": (ctypes.c_int, [_h]),
        "rf_create_sharded": (ctypes.c_int, [P, _dp, _dp, ctypes.c_char_p, ctypes.POINTER(_h)]),
        "rf_shard_unique_id": (ctypes.c_int, [ctypes.c_char_p]),
        "rf_shard_range": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
        "rf_step": (ctypes.c_int, [_h, ctypes.c_size_t]),
        "rf_assemble_system": (ctypes.c_int, [_h]),
        "rf_solve_system": (ctypes.c_int, [_h]),
        "rf_update_velocities": (ctypes.c_int, [_h]),
        "rf_update_fibers": (ctypes.c_int, [_h, ctypes.c_int]),
        "rf_get_state": (ctypes.c_int, [_h, _dp, _dp]),
        "rf_set_state": (ctypes.c_int, [_h, _dp, _dp]),
        "rf_get_velocities": (ctypes.c_int, [_h, _dp, _dp]),
        "rf_get_coeffs": (ctypes.c_int, [_h, _dp]),
        "rf_get_rhs": (ctypes.c_int, [_h, _dp]),
        "rf_get_matrix": (ctypes.c_int, [_h, _dp]),
        "rf_get_matrix_rows": (ctypes.c_int, [_h, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, _dp]),
        "rf_matvec": (ctypes.c_int, [_h, _dp, _dp]),
        "rf_matvec_free": (ctypes.c_int, [_h, _dp, _dp]),
        "rf_get_solve_stats": (ctypes.c_int, [_h, ctypes.POINTER(RfSolveStats)]),
        "rf_matvec_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p]),
        "rf_dgesv": (ctypes.c_int, [ctypes.c_int64, _dp, ctypes.c_int64, _dp, _dp, ctypes.c_void_p,
                                    ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
        "rf_get_history": (ctypes.c_int, [_h, _dp, _dp, _dp, _dp]),
        "rf_set_history": (ctypes.c_int, [_h, _dp, _dp, _dp, _dp, _dp]),
        "rf_timer_mark": (ctypes.c_int, [_h, ctypes.c_int32]),
        "rf_timer_elapsed_ms": (ctypes.c_double, [_h, ctypes.c_int32, ctypes.c_int32]),
        "rf_profile_matvec": (ctypes.c_int, [_h, ctypes.c_int32, _dp, _dp]),
        "rf_gemv_timer": (ctypes.c_int, [_h, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64), _dp, _dp]),
        "rf_system_size": (ctypes.c_int64, [_h]),
        "rf_matrix_ld": (ctypes.c_int64, [_h]),
        "rf_get_stream": (ctypes.c_void_p, [_h]),
        "rf_kernel_launches": (ctypes.c_int64, [_h]),
        "rf_last_error": (ctypes.c_char_p, [_h]),
        "rf_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "rf_generate_layout": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_uint64, _dp, _dp]),
        "rf_min_segment_distance": (ctypes.c_double, [ctypes.c_int32, _dp, _dp]),
        "rf_mlp_num_params": (ctypes.c_int64, []),
        "rf_set_mlp_weights": (ctypes.c_int, [_h, _fp, ctypes.c_int64]),
        "rf_compute_features": (ctypes.c_int, [_h, _fp]),
        "rf_compute_cluster_targets": (ctypes.c_int, [_h, _fp]),
        "rf_mlp_predict": (ctypes.c_int, [ctypes.c_int32, _fp, _fp, ctypes.c_int64, _fp]),
        "rf_trainer_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(_h)]),
        "rf_trainer_destroy": (ctypes.c_int, [_h]),
        "rf_trainer_add_samples": (ctypes.c_int, [_h, _fp, _fp, ctypes.c_int64]),
        "rf_trainer_train": (ctypes.c_int, [_h, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, _fp]),
        "rf_trainer_get_weights": (ctypes.c_int, [_h, _fp]),
        "rf_trainer_set_weights": (ctypes.c_int, [_h, _fp]),
        "rf_trainer_loss_grad": (ctypes.c_int, [_h, _fp, _fp, ctypes.c_int64, _fp, _fp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def declared_symbols(header=HEADER):
    """Names of the functions declared in include/rigidfibers.h."""
    import re

    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rf_[a-z0-9_]+)\s*\(", text)))


def check(status, handle=None):
    if status != RF_OK:
        msg = lib().rf_last_error(handle)
        raise RfError(status, msg.decode() if msg else "")
    return status
