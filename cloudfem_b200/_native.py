"""ctypes binding of libcfem (include/cfem.h) and the per-process runtime.

The CUDA library is the only compute path: importing this module does not
need a GPU, but every call that reaches ``runtime()`` requires the built
``libcfem.so`` and a compute-capability-10 device, and raises otherwise.
There is no CPU fallback.
"""

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcfem.so")

CFEM_OK = 0
CFEM_ERR_INVALID = 1
CFEM_ERR_CUDA = 2
CFEM_ERR_NOMEM = 3
CFEM_ERR_NOT_CONVERGED = 4
CFEM_ERR_BREAKDOWN = 5
CFEM_ERR_TIMEOUT = 6
CFEM_ERR_UNSUPPORTED = 7
CFEM_SLOT_RUNNING = -1

OP_P1_STIFF, OP_P1_MASS, OP_T10_STIFF, OP_T10_MASS = 1, 2, 3, 4
OP_P1_ELAST, OP_T10_ELAST = 5, 6
OP_T10_CURLCURL, OP_T10_NGRAD_X, OP_T10_NGRAD_Y, OP_T10_NGRAD_Z = 7, 8, 9, 10
COEF_CONST, COEF_ELEM, COEF_QP, COEF_NODAL = 0, 1, 2, 3
SOLVE_FP64, SOLVE_MIXED = 0, 1
PRECOND_JACOBI, PRECOND_BLOCK = 0, 1
SCHED_AUTO, SCHED_PERSISTENT, SCHED_GRAPH, SCHED_GRAPH_POLLED = 0, 1, 2, 3
PARAM_T10_WARPS, PARAM_P1_THREADS, PARAM_GRAPH_ITERS, PARAM_PDL, PARAM_SPMV_STAGE = 1, 2, 3, 4, 5
PARAM_BARRIER_TIMEOUT_US, PARAM_BARRIER_HOLD, PARAM_SELL_SORT = 6, 7, 8
PARAM_SELL3_LANES = 9
PARAM_SELL3_STAGED = 10
PARAM_SLOT_SELL3 = 11

STATUS_NAMES = {
    CFEM_OK: "ok", CFEM_ERR_INVALID: "invalid argument",
    CFEM_ERR_CUDA: "CUDA error", CFEM_ERR_NOMEM: "out of device memory",
    CFEM_ERR_NOT_CONVERGED: "not converged",
    CFEM_ERR_BREAKDOWN: "breakdown (matrix not SPD or non-finite values)",
    CFEM_ERR_TIMEOUT: "device wait timed out",
    CFEM_ERR_UNSUPPORTED: "unsupported device",
}

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_f64 = ctypes.c_double


class Coef(ctypes.Structure):
    _fields_ = [("d_values", _vp), ("constant", _f64), ("mode", _i32),
                ("pad_", _i32)]


class AssemblyJob(ctypes.Structure):
    _fields_ = [("pattern", _vp), ("d_nodes", _vp), ("d_elems", _vp),
                ("coef", Coef), ("load", Coef), ("d_vals", _vp),
                ("d_rhs", _vp)]


class MixedJob(ctypes.Structure):
    _fields_ = [("n_rows", _i64), ("bs", _i32), ("reserved", _i32), ("row_ptr", _vp),
                ("col", _vp), ("vals64", _vp), ("vals32", _vp)]


class LinSys(ctypes.Structure):
    _fields_ = [("n_rows", _i64), ("bs", _i32), ("precond", _i32),
                ("d_row_ptr", _vp), ("d_col", _vp), ("d_vals64", _vp),
                ("d_vals32", _vp), ("d_b", _vp), ("d_x", _vp),
                ("d_fixed", _vp), ("rtol", _f64), ("max_iter", _i32),
                ("mode", _i32), ("reliable_delta", _f64), ("max_stall", _i32),
                ("history_cap", _i32), ("d_history", _vp)]


class SolveStats(ctypes.Structure):
    _fields_ = [("status", _i32), ("iterations", _i32),
                ("residual_updates", _i32), ("pad_", _i32),
                ("relres", _f64), ("bnorm", _f64), ("kernel_ms", _f64),
                ("spmv_ms", _f64), ("spmv_samples", _i32), ("pad2_", _i32)]


# (name, restype, argtypes) of every symbol in include/cfem.h
SIGNATURES = [
    ("cfem_last_error", ctypes.c_char_p, []),
    ("cfem_version", ctypes.c_int, []),
    ("cfem_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    ("cfem_ctx_destroy", ctypes.c_int, [_vp]),
    ("cfem_ctx_launch_count", _i64, [_vp]),
    ("cfem_ctx_trim", _i32, [_vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("cfem_ctx_set_param", _i32, [_vp, ctypes.c_int, ctypes.c_int]),
    ("cfem_ctx_get_param", _i32, [_vp, ctypes.c_int]),
    ("cfem_ctx_set_scheduler", ctypes.c_int, [_vp, ctypes.c_int]),
    ("cfem_pattern_create", ctypes.c_int,
     [_vp, _vp, _i64, _i32, _i64, _vp, ctypes.POINTER(_vp)]),
    ("cfem_pattern_destroy", ctypes.c_int, [_vp]),
    ("cfem_pattern_info", ctypes.c_int,
     [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    ("cfem_pattern_node_csr", ctypes.c_int,
     [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    ("cfem_pattern_expand", ctypes.c_int, [_vp, _i32, _vp, _vp, _vp]),
    ("cfem_block_to_csr", ctypes.c_int, [_vp, _i32, _vp, _vp, _vp]),
    ("cfem_assemble", ctypes.c_int,
     [_vp, _vp, _i32, _vp, _vp, ctypes.POINTER(Coef), ctypes.POINTER(Coef),
      _vp, _vp, _i32, _vp]),
    ("cfem_element_stress", ctypes.c_int,
     [_vp, _vp, _vp, _i64, _i32, _vp, _f64, _f64, ctypes.POINTER(Coef), _f64,
      _f64, _vp, _vp, _vp]),
    ("cfem_face_geometry", ctypes.c_int,
     [_vp, _i32, _i64, _vp, _vp, _i32, _vp, _vp, _vp, _vp]),
    ("cfem_face_integrate", ctypes.c_int,
     [_vp, _i32, _i64, _vp, _vp, _i32, _vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _i64,
      _vp, _vp]),
    ("cfem_t10_joule_power", ctypes.c_int,
     [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f64, _vp, _vp, _vp, _vp, _vp]),
    ("cfem_assemble_curlcurl", ctypes.c_int,
     [_vp, _vp, _vp, _vp, Coef, _vp, ctypes.c_int, _vp]),
    ("cfem_assemble_batch", ctypes.c_int,
     [_vp, _i32, ctypes.POINTER(AssemblyJob), _i32, _vp]),
    ("cfem_assemble_elastic", ctypes.c_int,
     [_vp, _vp, _i32, _vp, _vp, _f64, _f64, ctypes.POINTER(Coef),
      ctypes.POINTER(Coef), _f64, _f64, _vp, _vp, _i32, _vp]),
    ("cfem_face_candidates", ctypes.c_int,
     [_vp, _vp, _i64, _i32, _i32, _vp, _i64, _vp, ctypes.POINTER(_i64), _vp]),
    ("cfem_face_exterior", ctypes.c_int,
     [_vp, _vp, _i32, _i32, _vp, _i64, _i64, _vp, _vp, ctypes.POINTER(_i64), _vp]),
    ("cfem_axpby", ctypes.c_int, [_vp, _i64, _f64, _vp, _f64, _vp, _vp, _vp]),
    ("cfem_spmv", ctypes.c_int,
     [_vp, _i64, _i32, _vp, _vp, _vp, _f64, _vp, _f64, _vp, _vp]),
    ("cfem_dirichlet_csr", ctypes.c_int,
     [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
      ctypes.POINTER(_i64), _vp]),
    ("cfem_mixed_matrix", ctypes.c_int,
     [_vp, _i64, _i32, _vp, _vp, _vp, _vp, _vp]),
    ("cfem_mixed_matrix_batch", ctypes.c_int, [_vp, ctypes.POINTER(MixedJob), _i32, _vp]),
    ("cfem_pcg_solve", ctypes.c_int,
     [_vp, ctypes.POINTER(LinSys), _i32, ctypes.POINTER(SolveStats), _vp]),
    ("cfem_pcg_plan_create", ctypes.c_int,
     [_vp, ctypes.POINTER(LinSys), ctypes.c_int32, _vp, ctypes.POINTER(_vp)]),
    ("cfem_pcg_plan_refresh", ctypes.c_int, [_vp, _vp]),
    ("cfem_pcg_plan_solve", ctypes.c_int, [_vp, ctypes.POINTER(SolveStats), _vp]),
    ("cfem_pcg_plan_destroy", ctypes.c_int, [_vp]),
    ("cfem_cocg_solve", ctypes.c_int,
     [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _f64, _i32, ctypes.POINTER(SolveStats), _vp]),
    ("cfem_pcg_noalloc_capacity", ctypes.c_size_t, []),
    ("cfem_pcg_slots_create", ctypes.c_int,
     [_vp, _i32, _i32, _i32, _i64, _i64, _vp, ctypes.POINTER(_vp)]),
    ("cfem_pcg_slots_assign", ctypes.c_int, [_vp, _i32, ctypes.POINTER(LinSys), _vp]),
    ("cfem_pcg_slots_run", ctypes.c_int, [_vp, _i32, _vp]),
    ("cfem_pcg_slots_ready", ctypes.c_int, [_vp]),
    ("cfem_pcg_slots_poll", ctypes.c_int, [_vp, ctypes.POINTER(SolveStats)]),
    ("cfem_pcg_slots_release", ctypes.c_int, [_vp, _i32, _vp]),
    ("cfem_pcg_solve_noalloc", ctypes.c_int,
     [_vp, ctypes.POINTER(LinSys), ctypes.POINTER(SolveStats), _vp]),
]

_lib = None
_lib_lock = threading.Lock()


def load_library(path=LIB_PATH):
    """Load libcfem.so and declare its C ABI. Raises if it is missing."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(
                f"libcfem.so not found at {path}; build it with "
                "`python -m cloudfem_b200.csrc.build` (needs nvcc, sm_100a)")
        lib = ctypes.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


class CfemError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"libcfem: {STATUS_NAMES.get(status, status)}: "
                         f"{message}")
        self.status = status


def check(status):
    if status == CFEM_OK:
        return
    msg = _lib.cfem_last_error().decode(errors="replace") if _lib else ""
    if status == CFEM_ERR_INVALID:
        raise ValueError(f"libcfem: {msg}")
    raise CfemError(status, msg)


class Runtime:
    """One libcfem context per CUDA device, created on first use."""

    def __init__(self, device):
        import torch
        self.torch = torch
        self.lib = load_library()
        self.device = device
        ctx = _vp()
        check(self.lib.cfem_ctx_create(int(device), ctypes.byref(ctx)))
        self.ctx = ctx

    def stream(self):
        return _vp(self.torch.cuda.current_stream(self.device).cuda_stream)

    def launches(self):
        return int(self.lib.cfem_ctx_launch_count(self.ctx))

    def set_param(self, param, value):
        check(self.lib.cfem_ctx_set_param(self.ctx, int(param), int(value)))

    def get_param(self, param):
        return int(self.lib.cfem_ctx_get_param(self.ctx, int(param)))

    def trim(self, keep_bytes=0):
        """Return the library pool's unused device memory beyond keep_bytes
        to the driver; returns the bytes the pool still reserves."""
        out = ctypes.c_uint64()
        check(self.lib.cfem_ctx_trim(self.ctx, int(keep_bytes), ctypes.byref(out)))
        return int(out.value)

    def __del__(self):
        try:
            if self.ctx:
                self.lib.cfem_ctx_destroy(self.ctx)
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


_runtimes = {}


def runtime(device=None):
    """The runtime of ``device`` (default: torch's current CUDA device)."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError(
            "cloudfem_b200 needs a CUDA device (B200, sm_100a); none is "
            "visible. There is no CPU fallback.")
    if device is None:
        device = torch.cuda.current_device()
    rt = _runtimes.get(device)
    if rt is None:
        rt = Runtime(device)
        _runtimes[device] = rt
    return rt


def ptr(t):
    """Device (or host) address of a torch tensor / numpy array, or NULL."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return _vp(t.ctypes.data)
    return _vp(t.data_ptr())
