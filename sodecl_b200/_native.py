"""ctypes binding of libsodecl_cuda.so (include/sodecl_cuda.h).

Loads the in-tree library and declares every entry point.  There is no
fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsodecl_cuda.so")

OK = 0
ERR_INVALID_ARG = -1
ERR_COMPILE = -2
ERR_CUDA = -3
ERR_NO_DEVICE = -4
ERR_STATE = -5
ERR_NO_JACOBIAN = -6
ERR_NO_STOCH = -7
ERR_OUT_OF_MEMORY = -8
ERR_UNSUPPORTED = -9

# include/sodecl_cuda.h's SODECL_CUDA_ABI_VERSION, which the structures below follow
ABI_VERSION = 4
STOCHASTIC_EULER, EULER, RUNGE_KUTTA, IMPLICIT_EULER, IMPLICIT_MIDPOINT, DORMAND_PRINCE = range(6)
FP64, FP32 = 0, 1
DIV_RECIPROCAL, DIV_IEEE, DIV_DEFAULT = 0, 1, 2
STORE_DIRECT, STORE_PAIRS = 0, 1
FLAG_NEWTON_CAP = 1
FLAG_NONFINITE = 2


class Cfg(C.Structure):
    _fields_ = [
        ("solver", C.c_int32),
        ("dt", C.c_double),
        ("int_time", C.c_double),
        ("kernel_steps", C.c_int32),
        ("num_equat", C.c_int32),
        ("num_params", C.c_int32),
        ("num_noi", C.c_int32),
        ("list_size", C.c_int64),
        ("device", C.c_int32),
        ("local_group_size", C.c_int32),
        ("precision", C.c_int32),
        ("fmad", C.c_int32),
        ("newton_tol", C.c_double),
        ("newton_max_iter", C.c_int32),
        ("record_f32", C.c_int32),
        ("min_blocks_per_sm", C.c_int32),
        ("division", C.c_int32),
        ("lanes_per_orbit", C.c_int32),
        ("rtol", C.c_double),
        ("atol", C.c_double),
        ("max_steps", C.c_int32),
        ("record_store", C.c_int32),
    ]


class Launch(C.Structure):
    _fields_ = [
        ("t", C.c_void_p),
        ("y", C.c_void_p),
        ("params", C.c_void_p),
        ("counters", C.c_void_p),
        ("records", C.c_void_p),
        ("n", C.c_int64),
        ("orbit_offset", C.c_int64),
        ("rec_stride", C.c_int64),
        ("rec_col0", C.c_int64),
        ("chunk_begin", C.c_int32),
        ("chunk_end", C.c_int32),
        ("rec_first", C.c_int32),
        ("write_final", C.c_int32),
        ("newton_passes", C.c_void_p),
        ("flags", C.c_void_p),
    ]


class ClassCfg(C.Structure):
    _fields_ = [
        ("solver", C.c_int32),
        ("num_equat", C.c_int32),
        ("num_params", C.c_int32),
        ("num_noi", C.c_int32),
        ("dt", C.c_double),
        ("newton_tol", C.c_double),
        ("newton_max_iter", C.c_int32),
        ("lanes_per_orbit", C.c_int32),
    ]


class AdjointIO(C.Structure):
    _fields_ = [
        ("t0", C.c_void_p),
        ("y0", C.c_void_p),
        ("params", C.c_void_p),
        ("targets", C.c_void_p),
        ("loss", C.c_void_p),
        ("grad_params", C.c_void_p),
        ("grad_y0", C.c_void_p),
        ("flags", C.c_void_p),
        ("n", C.c_int64),
        ("ckpt_every", C.c_int32),
        ("tape_entries", C.c_int32),
        ("use_tape", C.c_int32),
    ]


FLAG_TAPE_OVERFLOW = 4


class BatchIO(C.Structure):
    _fields_ = [
        ("t", C.c_void_p),
        ("y", C.c_void_p),
        ("params", C.c_void_p),
        ("counters", C.c_void_p),
        ("nsteps", C.c_void_p),
        ("newton_passes", C.c_void_p),
        ("flags", C.c_void_p),
        ("class_count", C.c_void_p),
    ]

_P = C.c_void_p
# name -> (restype, argtypes); every function include/sodecl_cuda.h declares
SIGNATURES = {
    "sodecl_cfg_init": (None, [C.POINTER(Cfg)]),
    "sodecl_cuda_create": (C.c_int, [C.POINTER(Cfg), C.POINTER(C.c_void_p)]),
    "sodecl_cuda_compile": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "sodecl_cuda_upload": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sodecl_cuda_num_records": (C.c_int64, [C.c_void_p]),
    "sodecl_cuda_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "sodecl_cuda_download_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sodecl_cuda_status": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "sodecl_cuda_last_run_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "sodecl_cuda_last_error": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "sodecl_cuda_build_log": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "sodecl_cuda_program_source": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "sodecl_cuda_destroy": (None, [C.c_void_p]),
    "sodecl_cuda_strerror": (C.c_char_p, [C.c_int]),
    "sodecl_cuda_abi_version": (C.c_int, []),
    "sodecl_cuda_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "sodecl_cuda_release_scratch": (C.c_int, [C.c_void_p]),
    "sodecl_cuda_release_cached": (C.c_int, [C.c_int]),
    "sodecl_cuda_device_describe": (C.c_int, [C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_int),
                                              C.POINTER(C.c_int)]),
    "sodecl_cuda_launch": (C.c_int, [C.c_void_p, C.POINTER(Launch), C.c_void_p]),
    "sodecl_cuda_program_division": (C.c_int, [C.c_void_p]),
    "sodecl_cuda_get_cfg": (C.c_int, [C.c_void_p, C.POINTER(Cfg)]),
    "sodecl_cuda_adjoint": (C.c_int, [C.c_void_p, C.POINTER(AdjointIO), C.c_void_p]),
    "sodecl_cuda_autotune": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "sodecl_cuda_kernel_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "sodecl_cuda_noise_stream": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_double,
                                           C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sodecl_cuda_division_check": (C.c_int, [C.c_int, C.c_int64, C.c_uint64, C.POINTER(C.c_int64),
                                             C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "sodecl_cuda_division_check_f32": (C.c_int, [C.c_int, C.c_int64, C.c_uint64, C.POINTER(C.c_int64),
                                                 C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "sodecl_class_cfg_init": (None, [C.POINTER(ClassCfg)]),
    "sodecl_batch_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(_P)]),
    "sodecl_batch_add_class": (C.c_int, [_P, C.c_char_p, C.c_size_t, C.POINTER(ClassCfg), C.POINTER(C.c_int32)]),
    "sodecl_batch_compile": (C.c_int, [_P]),
    "sodecl_batch_set_items": (C.c_int, [_P, C.c_int64, _P, _P, _P, _P, _P, _P]),
    "sodecl_batch_set_launch": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "sodecl_batch_tune": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "sodecl_batch_class_lanes": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "sodecl_batch_run": (C.c_int, [_P, C.c_int32]),
    "sodecl_batch_results": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "sodecl_batch_last_ms": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "sodecl_batch_kernel_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "sodecl_batch_last_error": (C.c_size_t, [_P, C.c_char_p, C.c_size_t]),
    "sodecl_batch_program_source": (C.c_size_t, [_P, C.c_char_p, C.c_size_t]),
    "sodecl_batch_destroy": (None, [_P]),
    "sodecl_batch_run_noalloc": (C.c_int, [_P, C.POINTER(BatchIO), _P]),
    "sodecl_cuda_fma_peak": (C.c_int, [C.c_int, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "sodecl_cuda_sin_peak": (C.c_int, [C.c_int, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("%s is not built: run `python -c 'import __graft_entry__ as g; g.build()'` "
                          "or `python sodecl_b200/build.py`" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.sodecl_cuda_abi_version() != ABI_VERSION:
        raise ImportError("%s has ABI version %d, these bindings %d: rebuild it" %
                          (LIB_PATH, lib.sodecl_cuda_abi_version(), ABI_VERSION))
    return lib


lib = _load()


class SodeclError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (%d): %s" % (lib.sodecl_cuda_strerror(status).decode(), status, message))
        self.status = status


def _string(fn, ctx):
    n = fn(ctx, None, 0)
    buf = C.create_string_buffer(n + 1)
    fn(ctx, buf, n + 1)
    return buf.value.decode(errors="replace")


def last_error(ctx):
    return _string(lib.sodecl_cuda_last_error, ctx)


def build_log(ctx):
    return _string(lib.sodecl_cuda_build_log, ctx)


def program_source(ctx):
    return _string(lib.sodecl_cuda_program_source, ctx)


def check(status, ctx=None):
    if status != OK:
        raise SodeclError(status, last_error(ctx) if ctx else "")
    return status


def device_count():
    n = C.c_int(0)
    lib.sodecl_cuda_device_count(C.byref(n))
    return n.value
