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
EULER, NAVIER_STOKES, EULER_DF, NAVIER_STOKES_DF = 0, 1, 2, 3
EOS_CPG, EOS_TPG, EOS_REALGAS, EOS_REALGAS_DF = 0, 1, 2, 3
FLUX_KEPAEC, FLUX_HLLC, FLUX_RUSANOV, FLUX_AUSMUP = 0, 1, 2, 3
RECON_CONSTANT, RECON_MUSCL = 0, 1
LIMITERS = {"koren": 1, "minmod": 2, "mc": 3, "superbee": 4, "vanleer": 5}
CHEM_NONE, CHEM_COUPLED, CHEM_SUBSTEPPED = 0, 1, 2
# boundary kinds, by the reference's bcvals names
BC_KINDS = {"slp-adia-wall": 1, "slp-isot-wall": 2, "no-slp-adia-wall": 3, "mov-adia-wall": 4,
            "no-slp-isot-wall": 5, "mov-isot-wall": 6, "sub-in-fvt": 7, "sup-in-fa": 8, "sub-in-ftptt": 9,
            "sub-in-fmt": 10, "sub-out-fp": 11, "sup-out-fn": 12}
# the boundary value programs' operations
OPS = {name: n for n, name in enumerate(("const", "x", "y", "z", "t", "add", "sub", "mul", "div", "neg", "pow", "sin",
                                         "cos", "tan", "exp", "log", "sqrt", "tanh", "abs", "min", "max"))}
BC_STACK = 16


def mechanism(consts):
    """The C ABI's mechanism struct from a mixture's tables (the columns of the
    reference's FiniteRateModel.rxnconsts and its third-body sets); returns
    the struct and the arrays it points into, which must outlive the call."""
    import numpy as np

    def side(sp, val):
        return [(int(a), float(b)) for a, b in zip(sp, val) if b != 0.0]

    nr = int(consts["rxn_nr"])
    rxns = (Reaction * max(nr, 1))()
    for k in range(nr):
        r = rxns[k]
        r.kind, r.reversible, r.product = (int(consts["rxn_kind"][k]), int(consts["rxn_reversible"][k]),
                                           int(consts["rxn_product"][k]))
        r.tb, r.troe, r.nfcent = int(consts["rxn_tb"][k]), int(consts["rxn_troeidx"][k]), int(consts["rxn_nfcent"][k])
        for name, sp, val, coef in (("fwd", "rxn_fwdsp", "rxn_fwdorder", "fwdorder"),
                                    ("react", "rxn_reactsp", "rxn_reactnu", "reactnu"),
                                    ("prod", "rxn_prodsp", "rxn_prodnu", "prodnu")):
            row = side(consts[sp][k], consts[val][k])
            if len(row) > MAXSIDE:
                raise ValueError(f"reaction {k}: more than {MAXSIDE} species on a side")
            setattr(r, "n" + name, len(row))
            for j, (a, b) in enumerate(row):
                getattr(r, name + "sp")[j] = a
                getattr(r, coef)[j] = b
        net = [(int(a), float(b), float(c)) for a, b, c in
               zip(consts["rxn_netsp"][k], consts["rxn_netnu"][k], consts["rxn_netnuMW"][k]) if b != 0.0]
        if len(net) > MAXNET:
            raise ValueError(f"reaction {k}: more than {MAXNET} species change")
        r.nnet = len(net)
        for j, (a, b, c) in enumerate(net):
            r.netsp[j], r.netnu[j], r.netnuMW[j] = a, b, c
        for name in ("logA", "b", "EaR", "logprA", "prb", "prEaR", "nusum"):
            setattr(r, name, float(consts["rxn_" + name][k]))
    ntb = len(consts["tbdefeff"])
    tbs = (ThirdBody * max(ntb, 1))()
    for j in range(ntb):
        tbs[j].defeff = float(consts["tbdefeff"][j])
        n = int(consts["tb_neff"][j])
        tbs[j].neff = n
        for i in range(n):
            tbs[j].effsp[i] = int(consts["tb_effsp"][j][i])
            tbs[j].effdev[i] = float(consts["tbeffdev"][j][i])
    lfc = np.ascontiguousarray(consts["rxnlfcpoly"], dtype=np.float64)
    gpoly = np.ascontiguousarray(consts["gpoly"], dtype=np.float64)
    m = Mechanism()
    m.nr, m.ntb = nr, ntb
    m.ntroe = int(lfc.shape[0]) if lfc.ndim == 2 else 0
    m.nlfc = int(lfc.shape[1]) if lfc.ndim == 2 else 0
    m.ng = int(gpoly.shape[1])
    m.rxn, m.tb = ctypes.cast(rxns, ctypes.POINTER(Reaction)), ctypes.cast(tbs, ctypes.POINTER(ThirdBody))
    m.lfcpoly = lfc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    m.gpoly = gpoly.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for name in ("logprefRu", "prefRu", "Rupref", "logcfloor", "maxgain", "troeuc", "troeuhinv"):
        setattr(m, name, float(consts[name]))
    return m, (rxns, tbs, lfc, gpoly)
TRANS_NONE, TRANS_CONSTANT, TRANS_KINETIC = 0, 1, 2
PATH_BATCHED, PATH_PER_BLOCK, PATH_PACKED = 0, 1, 2
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
                ("ns", ctypes.c_int), ("nregs", ctypes.c_int), ("alpha", ctypes.c_double),
                ("chemistry", ctypes.c_int)]


MAXSIDE, MAXNET = 4, 8


class Reaction(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("kind", "reversible", "product", "tb", "troe", "nfcent", "nfwd",
                                            "nreact", "nprod", "nnet")] + \
               [("fwdsp", ctypes.c_int * MAXSIDE), ("reactsp", ctypes.c_int * MAXSIDE),
                ("prodsp", ctypes.c_int * MAXSIDE), ("netsp", ctypes.c_int * MAXNET),
                ("fwdorder", ctypes.c_double * MAXSIDE), ("reactnu", ctypes.c_double * MAXSIDE),
                ("prodnu", ctypes.c_double * MAXSIDE), ("netnu", ctypes.c_double * MAXNET),
                ("netnuMW", ctypes.c_double * MAXNET)] + \
               [(n, ctypes.c_double) for n in ("logA", "b", "EaR", "logprA", "prb", "prEaR", "nusum")]


class ThirdBody(ctypes.Structure):
    _fields_ = [("defeff", ctypes.c_double), ("neff", ctypes.c_int), ("effsp", ctypes.c_int * 12),
                ("effdev", ctypes.c_double * 12)]


class Mechanism(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("nr", "ntb", "ntroe", "nlfc", "ng")] + \
               [("rxn", ctypes.POINTER(Reaction)), ("tb", ctypes.POINTER(ThirdBody)),
                ("lfcpoly", ctypes.POINTER(ctypes.c_double)), ("gpoly", ctypes.POINTER(ctypes.c_double))] + \
               [(n, ctypes.c_double) for n in ("logprefRu", "prefRu", "Rupref", "logcfloor", "maxgain", "troeuc",
                                               "troeuhinv")]


class Combine(ctypes.Structure):
    _fields_ = [("out", ctypes.c_int), ("own", ctypes.c_int), ("wout", ctypes.c_double),
                ("nterms", ctypes.c_int), ("reg", ctypes.c_int * 3), ("w", ctypes.c_double * 3),
                ("step", ctypes.c_int)]


class Stage(ctypes.Structure):
    _fields_ = [("q", ctypes.c_int), ("dq", ctypes.c_int), ("ncombine", ctypes.c_int),
                ("combine", Combine * 2), ("tfrac", ctypes.c_double)]


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
    "pgb_pool_create": ([ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "pgb_pool_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "pgb_pool_admit_reactor": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_case_set_generated_chemistry": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "pgb_case_generated_chemistry": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_char_p,
                                      ctypes.c_longlong], ctypes.c_int),
    "pgb_case_rates_source": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_longlong,
                               ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "pgb_case_rates_compile": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_longlong], ctypes.c_int),
    "pgb_pool_admit": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_pool_metric_set": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_pool_set_prims": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_pool_start": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_pool_step": ([ctypes.c_void_p, ctypes.c_double, ctypes.c_int], ctypes.c_int),
    "pgb_pool_done": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_pool_get": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_pool_release": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "pgb_pool_info": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_pool_last": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_case_set_mechanism": ([ctypes.c_void_p, ctypes.POINTER(Mechanism)], ctypes.c_int),
    "pgb_case_set_substeps": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double], ctypes.c_int),
    "pgb_substeps_get": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_long], ctypes.c_int),
    "pgb_stiff_head": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint), ctypes.c_int], ctypes.c_int),
    "pgb_production": ([ctypes.c_void_p, ctypes.c_long] + [ctypes.POINTER(ctypes.c_double)] * 4, ctypes.c_int),
    "pgb_case_add_block": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_case_connect": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_case_add_bc": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_case_set_face_bc": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_set_time": ([ctypes.c_void_p, ctypes.c_double], ctypes.c_int),
    "pgb_get_time": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "pgb_case_set_stages": ([ctypes.c_void_p, ctypes.POINTER(Stage), ctypes.c_int], ctypes.c_int),
    "pgb_case_finalize": ([ctypes.c_void_p], ctypes.c_int),
    "pgb_case_halo": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_case_device_bytes": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "pgb_metric_set": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_array_set": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_array_get": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_array_get_full": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_case_connect_oriented": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                   ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "pgb_exchange": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "pgb_advance": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "pgb_eos_get": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_set_prims": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long], ctypes.c_int),
    "pgb_rhs": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_rhs_path": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_step": ([ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_step_cfl": ([ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pgb_cflmax": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "pgb_set_dt": ([ctypes.c_void_p, ctypes.c_double], ctypes.c_int),
    "pgb_last_dt": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
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
    "pgb_case_set_halo_pull": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "pgb_case_halo_pull": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_rhs_block_noalloc": ([ctypes.POINTER(Physics), ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                              ctypes.c_int),
    "pgb_rhs_block_noalloc_max_cells": ([ctypes.c_int], ctypes.c_longlong),
    "pgb_block_uniform": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_case_batched_form": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_fp64_fma_rate": ([ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "pgb_case_halo_entries": ([ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong),
                               ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "pgb_case_halo_boxes": ([ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong),
                             ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "pgb_case_set_exchange": ([ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_int), ctypes.c_longlong, ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "pgb_exchange_pack": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "pgb_exchange_unpack": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "pgb_step_stage": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
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
