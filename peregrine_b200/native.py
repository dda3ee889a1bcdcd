"""The ctypes binding of libpgb200.so (include/pgb200.h).

Every call is checked: a non-zero status raises the exception class of its
code with the library's message, as the reference's driver wrapper turns a
CUDA status into a typed exception (peregrine/backend/base/wrapper.py:53-57,
peregrine/backend/cuda/driver.py:7-55).  The library must be built
(``python -m peregrine_b200.build``); there is no other implementation to
fall back on.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libpgb200.so")

OK, ERR_ARG, ERR_STATE, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_TIMEOUT = range(7)
EULER, NAVIER_STOKES = 0, 1
EOS_CPG, EOS_TPG = 0, 1
FLUX_KEPAEC, FLUX_HLLC, FLUX_RUSANOV, FLUX_AUSMUP = 0, 1, 2, 3
RECON_CONSTANT, RECON_MUSCL = 0, 1
LIMITERS = {"koren": 1, "minmod": 2, "mc": 3, "superbee": 4, "vanleer": 5}
TRANS_NONE, TRANS_CONSTANT, TRANS_KINETIC = 0, 1, 2
PATH_BATCHED, PATH_PER_BLOCK = 0, 1
ARR_XCC, ARR_DETJINV, ARR_JINV, ARR_IS, ARR_JS, ARR_KS, ARR_IXC, ARR_JXC, ARR_KXC = range(9)
METRIC_IDS = {"xcc": ARR_XCC, "detJinv": ARR_DETJINV, "Jinv": ARR_JINV, "iS": ARR_IS, "jS": ARR_JS,
              "kS": ARR_KS, "ixc": ARR_IXC, "jxc": ARR_JXC, "kxc": ARR_KXC}


class PgbError(RuntimeError):
    code = None


class PgbArgumentError(PgbError, ValueError):
    code = ERR_ARG


class PgbStateError(PgbError):
    code = ERR_STATE


class PgbCudaError(PgbError):
    code = ERR_CUDA


class PgbOutOfMemory(PgbError, MemoryError):
    code = ERR_NOMEM


class PgbUnsupported(PgbError, NotImplementedError):
    code = ERR_UNSUPPORTED


class PgbTimeout(PgbError, TimeoutError):
    code = ERR_TIMEOUT


_ERRORS = {c.code: c for c in (PgbArgumentError, PgbStateError, PgbCudaError, PgbOutOfMemory, PgbUnsupported, PgbTimeout)}


class Physics(ctypes.Structure):
    _fields_ = [("simulator", ctypes.c_int), ("eos", ctypes.c_int), ("primary", ctypes.c_int),
                ("recon", ctypes.c_int), ("limiter", ctypes.c_int), ("trans", ctypes.c_int),
                ("ns", ctypes.c_int), ("nregs", ctypes.c_int), ("alpha", ctypes.c_double)]


class Combine(ctypes.Structure):
    _fields_ = [("out", ctypes.c_int), ("own", ctypes.c_int), ("wout", ctypes.c_double),
                ("nterms", ctypes.c_int), ("reg", ctypes.c_int * 3), ("w", ctypes.c_double * 3),
                ("step", ctypes.c_int)]


class Stage(ctypes.Structure):
    _fields_ = [("q", ctypes.c_int), ("dq", ctypes.c_int), ("ncombine", ctypes.c_int),
                ("combine", Combine * 2)]


# every symbol include/pgb200.h declares, with its argument types
SIGNATURES = {
    "pgb_last_error": ([], ctypes.c_char_p),
    "pgb_version": ([], ctypes.c_int),
    "pgb_device_init": ([ctypes.c_int], ctypes.c_int),
    "pgb_device_count": ([ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_device_sync": ([], ctypes.c_int),
    "pgb_mem_info": ([ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "pgb_case_create": ([ctypes.POINTER(Physics), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "pgb_case_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "pgb_case_set_table": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_case_add_block": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_case_connect": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_case_set_stages": ([ctypes.c_void_p, ctypes.POINTER(Stage), ctypes.c_int], ctypes.c_int),
    "pgb_case_finalize": ([ctypes.c_void_p], ctypes.c_int),
    "pgb_case_halo": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_case_device_bytes": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "pgb_metric_set": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_array_set": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_array_get": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_set_prims": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_rhs": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_step": ([ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_case_stream": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "pgb_last_step_ms": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "pgb_launches_per_step": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_set_tile": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_get_tile": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_state_set": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_state_get": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_host_register": ([ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
    "pgb_host_unregister": ([ctypes.c_void_p], ctypes.c_int),
    "pgb_step_timed": ([ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                        ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_set_fused_shape": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_fused_shapes": ([ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_rhs_block_noalloc": ([ctypes.POINTER(Physics), ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                              ctypes.c_int),
    "pgb_rhs_block_noalloc_max_cells": ([ctypes.c_int], ctypes.c_longlong),
    "pgb_block_uniform": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
}

_lib = None


def load():
    """The library, loaded once; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise ImportError(f"{LIBPATH} is not built: run `python -m peregrine_b200.build`")
    lib = ctypes.CDLL(LIBPATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(status):
    if status != OK:
        msg = load().pgb_last_error().decode(errors="replace")
        raise _ERRORS.get(status, PgbError)(msg)


def call(name, *args):
    check(getattr(load(), name)(*args))
