"""ctypes binding of libmfgpu.so (the C ABI declared in include/mfgpu.h)."""
import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libmfgpu.so")

MFGPU_OK = 0
MFGPU_ERR_ARG = 1
MFGPU_ERR_DEPTH = 2
MFGPU_ERR_LEAF = 3
MFGPU_ERR_OOM = 4
MFGPU_ERR_CUDA = 5
MFGPU_ERR_PIVOT = 6
MFGPU_ERR_TIMEOUT = 7
MFGPU_ERR_STATE = 8
MFGPU_ERR_NOT_CONVERGED = 9

MFGPU_FP64 = 0
MFGPU_MIXED = 1

# Every symbol include/mfgpu.h declares.
EXPORTED = [
    "mfgpu_default_options", "mfgpu_status_string", "mfgpu_create", "mfgpu_factor",
    "mfgpu_update", "mfgpu_solve", "mfgpu_apply", "mfgpu_solve_device", "mfgpu_apply_device",
    "mfgpu_set_stream", "mfgpu_get_info", "mfgpu_last_stats", "mfgpu_last_error",
    "mfgpu_destroy", "mfgpu_symbolic_create", "mfgpu_symbolic_destroy", "mfgpu_symbolic_error",
    "mfgpu_symbolic_sizes", "mfgpu_symbolic_front", "mfgpu_symbolic_sep", "mfgpu_symbolic_tasks",
    "mfgpu_symbolic_layout", "mfgpu_update_device", "mfgpu_refactor", "mfgpu_refactor_device",
    "mfgpu_profile_enable", "mfgpu_profile_reset", "mfgpu_profile_read", "mfgpu_kernel_launches",
    "mfgpu_symbolic_dirty", "mfgpu_batch_create", "mfgpu_batch_info",
    "mfgpu_symbolic_batch_create", "mfgpu_stencil_assemble_device", "mfgpu_stencil_update_device",
    "mfgpu_server_create", "mfgpu_server_submit", "mfgpu_server_wait", "mfgpu_server_last_error",
    "mfgpu_server_destroy", "mfgpu_save", "mfgpu_load", "mfgpu_autotune", "mfgpu_symbolic_create_full",
    "mfgpu_solve_device_noalloc", "mfgpu_set_wait_limit", "mfgpu_inject_alloc_failure",
    "mfgpu_graphs",
]

KERNEL_CLASSES = ["assemble", "potrf", "trsm", "syrk", "solve", "apply", "front", "coop", "tc"]


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("refine_tol", C.c_double),
                ("refine_maxit", C.c_int), ("reserved", C.c_int * 7)]


class Info(C.Structure):
    _fields_ = [("dim", C.c_int), ("levels", C.c_int), ("n_fronts", C.c_int), ("n_seps", C.c_int),
                ("ndof", C.c_int64), ("nnz", C.c_int64), ("leaf_box", C.c_int * 3),
                ("max_front", C.c_int), ("factor_flops", C.c_double), ("front_bytes", C.c_int64),
                ("sep_bytes", C.c_int64), ("device_bytes", C.c_int64)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("fronts", C.c_int), ("iterations", C.c_int), ("batch", C.c_int),
                ("queued_seconds", C.c_double), ("latency_seconds", C.c_double),
                ("residual", C.c_double), ("pool_bytes", C.c_int64), ("reserved", C.c_int64 * 4)]


class Stats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("flops", C.c_double), ("fronts", C.c_int),
                ("iterations", C.c_int), ("residual", C.c_double)]


# numpy view of mfgpu::Task (csrc/schedule.hpp), 56 bytes
TASK_DTYPE = np.dtype([("dst_off", "<i8"), ("src_off", "<i8"), ("dst_ld", "<i4"),
                       ("src_ld", "<i4"), ("rows", "<i4"), ("cols", "<i4"), ("kind", "<i4"),
                       ("dst_arena", "<i2"), ("src_arena", "<i2"), ("row_dof", "<i4"),
                       ("col_dof", "<i4"), ("trans", "<i2"), ("lower", "<i2"), ("owner", "<i4")])
assert TASK_DTYPE.itemsize == 56

_lib = None


def load(path=None):
    """Load the library once; raises OSError when it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.isfile(p):
        raise OSError(f"libmfgpu.so not built at {p}; run __graft_entry__.build()")
    lib = C.CDLL(p)
    P = C.c_void_p
    i32p = C.POINTER(C.c_int)
    dp = C.POINTER(C.c_double)
    lib.mfgpu_default_options.argtypes = [C.POINTER(Options)]
    lib.mfgpu_default_options.restype = None
    lib.mfgpu_status_string.argtypes = [C.c_int]
    lib.mfgpu_status_string.restype = C.c_char_p
    lib.mfgpu_create.argtypes = [C.c_int] * 7 + [C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.POINTER(Options), C.POINTER(P)]
    lib.mfgpu_create.restype = C.c_int
    lib.mfgpu_batch_create.argtypes = [C.c_int] + [C.c_void_p] * 6 + [
        C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Options), C.POINTER(P)]
    lib.mfgpu_batch_create.restype = C.c_int
    lib.mfgpu_batch_info.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int64)]
    lib.mfgpu_batch_info.restype = C.c_int
    lib.mfgpu_factor.argtypes = [P]
    lib.mfgpu_factor.restype = C.c_int
    lib.mfgpu_update.argtypes = [P, C.c_void_p, C.c_int64, C.c_void_p, C.c_int]
    lib.mfgpu_update.restype = C.c_int
    for nm in ("mfgpu_solve", "mfgpu_apply", "mfgpu_solve_device", "mfgpu_apply_device"):
        f = getattr(lib, nm)
        f.argtypes = [P, C.c_void_p, C.c_void_p, C.c_int, C.c_int64]
        f.restype = C.c_int
    lib.mfgpu_update_device.argtypes = [P, C.c_void_p, C.c_int64, C.c_void_p, C.c_int]
    lib.mfgpu_update_device.restype = C.c_int
    lib.mfgpu_refactor.argtypes = [P, C.c_void_p, C.c_int64]
    lib.mfgpu_refactor.restype = C.c_int
    lib.mfgpu_refactor_device.argtypes = [P, C.c_void_p, C.c_int64]
    lib.mfgpu_refactor_device.restype = C.c_int
    lib.mfgpu_profile_enable.argtypes = [P, C.c_int]
    lib.mfgpu_profile_enable.restype = C.c_int
    lib.mfgpu_profile_reset.argtypes = [P]
    lib.mfgpu_profile_reset.restype = C.c_int
    lib.mfgpu_profile_read.argtypes = [P, C.c_int, C.POINTER(C.c_int64), dp, dp, dp]
    lib.mfgpu_profile_read.restype = C.c_int
    lib.mfgpu_kernel_launches.argtypes = []
    lib.mfgpu_kernel_launches.restype = C.c_longlong
    lib.mfgpu_set_stream.argtypes = [P, C.c_void_p]
    lib.mfgpu_solve_device_noalloc.argtypes = [P, C.c_void_p, C.c_void_p, C.c_int, C.c_int64]
    lib.mfgpu_solve_device_noalloc.restype = C.c_int
    lib.mfgpu_set_wait_limit.argtypes = [P, C.c_uint]
    lib.mfgpu_set_wait_limit.restype = C.c_int
    lib.mfgpu_inject_alloc_failure.argtypes = [C.c_longlong]
    lib.mfgpu_inject_alloc_failure.restype = None
    lib.mfgpu_graphs.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.mfgpu_graphs.restype = C.c_int
    lib.mfgpu_save.argtypes = [P, C.c_char_p]
    lib.mfgpu_save.restype = C.c_int
    lib.mfgpu_load.argtypes = [P, C.c_char_p]
    lib.mfgpu_load.restype = C.c_int
    lib.mfgpu_autotune.argtypes = [P, C.c_int, C.c_void_p]
    lib.mfgpu_autotune.restype = C.c_int
    lib.mfgpu_set_stream.restype = C.c_int
    lib.mfgpu_get_info.argtypes = [P, C.POINTER(Info)]
    lib.mfgpu_get_info.restype = C.c_int
    lib.mfgpu_last_stats.argtypes = [P, C.POINTER(Stats)]
    lib.mfgpu_last_stats.restype = C.c_int
    lib.mfgpu_last_error.argtypes = [P]
    lib.mfgpu_last_error.restype = C.c_char_p
    lib.mfgpu_destroy.argtypes = [P]
    lib.mfgpu_destroy.restype = None
    lib.mfgpu_symbolic_create.argtypes = [C.c_int] * 6 + [C.POINTER(P)]
    lib.mfgpu_symbolic_create.restype = C.c_int
    lib.mfgpu_symbolic_create_full.argtypes = [C.c_int] * 6 + [C.POINTER(P)]
    lib.mfgpu_symbolic_create_full.restype = C.c_int
    lib.mfgpu_symbolic_batch_create.argtypes = [C.c_int] + [C.c_void_p] * 6 + [C.POINTER(P)]
    lib.mfgpu_symbolic_batch_create.restype = C.c_int
    lib.mfgpu_server_create.argtypes = [P, C.c_void_p, C.c_void_p, C.c_int, C.c_int64,
                                        C.POINTER(P)]
    lib.mfgpu_server_create.restype = C.c_int
    lib.mfgpu_server_submit.argtypes = [P, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int,
                                        C.c_int64, C.c_void_p, C.POINTER(C.c_int64)]
    lib.mfgpu_server_submit.restype = C.c_int
    lib.mfgpu_server_wait.argtypes = [P, C.c_int64, C.POINTER(RequestInfo)]
    lib.mfgpu_server_wait.restype = C.c_int
    lib.mfgpu_server_last_error.argtypes = [P]
    lib.mfgpu_server_last_error.restype = C.c_char_p
    lib.mfgpu_server_destroy.argtypes = [P]
    lib.mfgpu_server_destroy.restype = None
    lib.mfgpu_stencil_assemble_device.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.mfgpu_stencil_assemble_device.restype = C.c_int
    lib.mfgpu_stencil_update_device.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_void_p, C.c_int,
                                                C.POINTER(C.c_int)]
    lib.mfgpu_stencil_update_device.restype = C.c_int
    lib.mfgpu_symbolic_destroy.argtypes = [P]
    lib.mfgpu_symbolic_destroy.restype = None
    lib.mfgpu_symbolic_error.argtypes = []
    lib.mfgpu_symbolic_error.restype = C.c_char_p
    lib.mfgpu_symbolic_sizes.argtypes = [P, i32p, i32p, i32p, C.POINTER(C.c_int64)]
    lib.mfgpu_symbolic_sizes.restype = C.c_int
    lib.mfgpu_symbolic_front.argtypes = [P, C.c_int, i32p, i32p, i32p, i32p, C.POINTER(i32p)]
    lib.mfgpu_symbolic_front.restype = C.c_int
    lib.mfgpu_symbolic_sep.argtypes = [P, C.c_int, i32p, i32p, i32p, C.POINTER(i32p), i32p, i32p]
    lib.mfgpu_symbolic_sep.restype = C.c_int
    lib.mfgpu_symbolic_tasks.argtypes = [P, C.c_int, C.POINTER(C.c_void_p)]
    lib.mfgpu_symbolic_tasks.restype = C.c_int64
    lib.mfgpu_symbolic_dirty.argtypes = [P, C.c_void_p, C.c_int, C.c_void_p, dp]
    lib.mfgpu_symbolic_dirty.restype = C.c_int64
    lib.mfgpu_symbolic_layout.argtypes = [P, C.c_int, C.c_int, C.POINTER(C.c_int64), i32p]
    lib.mfgpu_symbolic_layout.restype = C.c_int
    _lib = lib
    return lib


def default_options(precision=MFGPU_FP64, device=0, refine_tol=1e-10, refine_maxit=50):
    o = Options()
    load().mfgpu_default_options(C.byref(o))
    o.precision = precision
    o.device = device
    o.refine_tol = refine_tol
    o.refine_maxit = refine_maxit
    return o


def status_string(st):
    return load().mfgpu_status_string(st).decode()


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)
