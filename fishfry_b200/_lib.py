"""ctypes binding of the fishfry_b200 C ABI (include/fishfry.h).

The native library is required: importing the solver API without
lib/libfishfry.so raises instead of falling back to anything else.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfishfry.so")

FF_OK = 0
FF_ERR_INVALID = 1
FF_ERR_UNSUPPORTED = 2
FF_ERR_BYTES = 3
FF_ERR_CUDA = 4
FF_ERR_NOMEM = 5
FF_ERR_TIMEOUT = 6
FF_ERR_TASKS = 7

FF_FP64 = 0
FF_FP32 = 1
FF_MAX_PHASES = 5
FF_MAX_AXIS = 4096

# Every symbol include/fishfry.h declares.
EXPORTS = [
    "ff_phase_name", "ff_plan_phases", "ff_plan_create", "ff_plan_bytes", "ff_plan_info", "ff_solve", "ff_plan_check",
    "ff_plan_destroy", "ff_solve_passes", "ff_plan_set_wait_limit",
    "ff_init_field", "ff_error_sums", "ff_error_sums_noalloc", "ff_modes_generate", "ff_status_string",
    "ff_last_error", "ff_version",
    "ff_batch_create", "ff_batch_bytes", "ff_batch_solve", "ff_batch_tune", "ff_batch_shape", "ff_batch_check",
    "ff_batch_destroy", "ff_batch_radices",
    "ff_server_create", "ff_server_submit", "ff_server_wait", "ff_server_next", "ff_server_fetch",
    "ff_server_release",
    "ff_server_stats", "ff_server_reset_stats", "ff_server_check", "ff_server_destroy",
    "ff_slab_create", "ff_slab_layout", "ff_slab_forward", "ff_slab_xpass", "ff_slab_backward", "ff_slab_check",
    "ff_slab_destroy",
]


class FFError(RuntimeError):
    """A non-zero ff_status from the C ABI; .status holds the code."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class Mode(ctypes.Structure):
    _fields_ = [("kx", ctypes.c_int), ("ky", ctypes.c_int), ("kz", ctypes.c_int),
                ("a", ctypes.c_double), ("theta", ctypes.c_double)]


class PhaseTimes(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int), ("ms", ctypes.c_double * FF_MAX_PHASES), ("total_ms", ctypes.c_double)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_active", ctypes.c_int)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double)]


class ServerReport(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("solves_per_s", ctypes.c_double), ("points_per_s", ctypes.c_double),
                ("peak_bytes", ctypes.c_size_t), ("budget_bytes", ctypes.c_size_t), ("steps", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("max_active", ctypes.c_int)]


_lib = None


def _declare(L):
    i3 = ctypes.POINTER(ctypes.c_int)
    d3 = ctypes.POINTER(ctypes.c_double)
    vp = ctypes.c_void_p
    L.ff_phase_name.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.ff_phase_name.restype = ctypes.c_char_p
    L.ff_plan_phases.argtypes = [ctypes.c_void_p]
    L.ff_plan_phases.restype = ctypes.c_int
    L.ff_plan_create.argtypes = [i3, d3, d3, ctypes.c_int, ctypes.POINTER(vp)]
    L.ff_plan_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
    L.ff_plan_info.argtypes = [vp, i3, i3]
    L.ff_solve.argtypes = [vp, ctypes.c_size_t, vp, vp, vp, ctypes.POINTER(PhaseTimes)]
    L.ff_plan_check.argtypes = [vp, vp]
    L.ff_solve_passes.argtypes = [vp, ctypes.c_size_t, vp, vp, vp, ctypes.c_int]
    L.ff_plan_destroy.argtypes = [vp]
    L.ff_plan_set_wait_limit.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.ff_init_field.argtypes = [i3, d3, d3, ctypes.c_int, vp, ctypes.c_int, vp, vp]
    L.ff_error_sums.argtypes = [i3, d3, d3, ctypes.c_int, vp, ctypes.c_int, vp, d3, vp]
    L.ff_error_sums_noalloc.argtypes = [i3, d3, d3, ctypes.c_int, vp, ctypes.c_int, vp, d3, vp]
    L.ff_modes_generate.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, i3, ctypes.c_double, vp]
    L.ff_status_string.argtypes = [ctypes.c_int]
    L.ff_status_string.restype = ctypes.c_char_p
    L.ff_last_error.restype = ctypes.c_char_p
    L.ff_version.restype = ctypes.c_char_p
    pp = ctypes.POINTER(ctypes.c_void_p)
    ip = ctypes.POINTER(ctypes.c_int)
    L.ff_batch_create.argtypes = [ctypes.c_int, ip, d3, d3, ctypes.c_int, ctypes.POINTER(vp)]
    L.ff_batch_bytes.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
    L.ff_batch_solve.argtypes = [vp, pp, pp, vp, ctypes.POINTER(PhaseTimes)]
    L.ff_batch_tune.argtypes = [vp, pp, pp, vp, ctypes.c_int]
    L.ff_batch_shape.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, ip, ip]
    L.ff_batch_check.argtypes = [vp, vp]
    L.ff_batch_radices.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, ip]
    L.ff_batch_destroy.argtypes = [vp]
    L.ff_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
    L.ff_server_submit.argtypes = [vp, i3, ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
    L.ff_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(RequestInfo)]
    L.ff_server_next.argtypes = [vp, ctypes.c_double, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(RequestInfo)]
    L.ff_server_fetch.argtypes = [vp, ctypes.c_uint64, vp, ctypes.c_int]
    L.ff_server_release.argtypes = [vp, ctypes.c_uint64]
    L.ff_server_stats.argtypes = [vp, ctypes.POINTER(ServerReport)]
    L.ff_server_check.argtypes = [vp]
    L.ff_server_reset_stats.argtypes = [vp]
    L.ff_server_destroy.argtypes = [vp]
    L.ff_slab_create.argtypes = [i3, d3, d3, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.ff_slab_layout.argtypes = [vp, i3, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    L.ff_slab_forward.argtypes = [vp, vp, vp, ctypes.POINTER(vp), vp]
    L.ff_slab_xpass.argtypes = [vp, vp, ctypes.POINTER(vp), vp]
    L.ff_slab_backward.argtypes = [vp, vp, vp, vp, vp]
    L.ff_slab_check.argtypes = [vp, vp]
    L.ff_slab_destroy.argtypes = [vp]
    for name in ("ff_slab_create", "ff_slab_layout", "ff_slab_forward", "ff_slab_xpass", "ff_slab_backward",
                 "ff_slab_check", "ff_slab_destroy"):
        getattr(L, name).restype = ctypes.c_int
    for name in ("ff_server_create", "ff_server_submit", "ff_server_wait", "ff_server_next", "ff_server_fetch",
                 "ff_server_release",
                 "ff_server_stats", "ff_server_reset_stats", "ff_server_check", "ff_server_destroy"):
        getattr(L, name).restype = ctypes.c_int
    for name in ("ff_plan_create", "ff_plan_bytes", "ff_plan_info", "ff_solve", "ff_plan_check", "ff_plan_destroy",
                 "ff_solve_passes", "ff_plan_set_wait_limit",
                 "ff_init_field", "ff_error_sums", "ff_error_sums_noalloc", "ff_modes_generate", "ff_batch_create",
                 "ff_batch_bytes", "ff_batch_solve", "ff_batch_tune", "ff_batch_shape", "ff_batch_check",
                 "ff_batch_destroy", "ff_batch_radices"):
        getattr(L, name).restype = ctypes.c_int


def lib():
    """The loaded native library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"fishfry_b200 native library missing: {LIB_PATH} "
                              "(build it with `python -m fishfry_b200.build`)")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def check(status, what=""):
    if status != FF_OK:
        L = lib()
        raise FFError(status, f"{what}: {L.ff_status_string(status).decode()}: {L.ff_last_error().decode()}")


def int3(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def dbl3(v):
    return (ctypes.c_double * 3)(*[float(x) for x in v])


def modes_array(modes):
    """(count, void*, keepalive) for a list of (kx, ky, kz, a, theta)."""
    if not modes:
        return 0, None, None
    arr = (Mode * len(modes))()
    for q, m in enumerate(modes):
        arr[q] = Mode(int(m[0]), int(m[1]), int(m[2]), float(m[3]), float(m[4]))
    return len(modes), ctypes.cast(arr, ctypes.c_void_p), arr
