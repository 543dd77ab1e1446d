"""ctypes binding of ``libglp_b200.so`` (the C ABI declared in include/glp.h).

The library is the product path: importing this module never falls back to
anything else.  If the shared object is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libglp_b200.so")

GLP_OK = 0
GLP_EINVAL = -1
GLP_ENOMEM = -2
GLP_ECUDA = -3
GLP_ENOTSUP = -4
GLP_ENODEV = -5
GLP_ETIMEOUT = -6
GLP_ECANCELED = -7
GLP_EKERNEL = -8
GLP_EAGAIN = -9

METHOD_CLASSIC, METHOD_LAYERED, METHOD_SLPA, METHOD_USER, METHOD_SEEDED = 1, 2, 3, 4, 5
BACKEND_EXACT, BACKEND_CM, BACKEND_FA = 0, 1, 2
HOOKS_CLASSIC, HOOKS_LAYERED, HOOKS_WEIGHTED_DEGREE = 0, 1, 2
GRAPH_SYMMETRIC = 1
EDGES_DIRECTED, EDGES_KEEP_IDS = 1, 2
MAX_LAYERS = 32

_ERRNAMES = {
    GLP_EINVAL: "EINVAL", GLP_ENOMEM: "ENOMEM", GLP_ECUDA: "ECUDA", GLP_ENOTSUP: "ENOTSUP",
    GLP_ENODEV: "ENODEV", GLP_ETIMEOUT: "ETIMEOUT", GLP_ECANCELED: "ECANCELED",
    GLP_EKERNEL: "EKERNEL", GLP_EAGAIN: "EAGAIN",
}


class GlpError(RuntimeError):
    """A negative status returned by the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"glp error {code} ({_ERRNAMES.get(code, '?')}): {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32),
        ("backend", C.c_int32),
        ("nlayers", C.c_int32),
        ("dstar", C.c_int32 * MAX_LAYERS),
        ("slpa_T", C.c_int32),
        ("slpa_r", C.c_double),
        ("seed", C.c_uint64),
        ("hooks", C.c_int32),
        ("tiny_max", C.c_int32),
        ("mid_max", C.c_int32),
        ("big_max", C.c_int32),
        ("hub_chunk", C.c_int32),
        ("use_graph", C.c_int32),
        ("async_", C.c_int32),
        ("batch_threads", C.c_int32),
        ("barrier_limit_us", C.c_int32),
        ("fault_skip_cta", C.c_int32),
        ("majority_permille", C.c_int32),
        ("frontier_permille", C.c_int32),
        ("l2_window", C.c_int32),
        ("cycle_stop", C.c_int32),
        ("serial_step", C.c_int32),
        ("mid_prefetch", C.c_int32),
        ("batch_blocks", C.c_int32),
        ("big_staged", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class Outputs(C.Structure):
    _fields_ = [
        ("labels", C.c_void_p),
        ("slpa_comm", C.c_void_p),
        ("slpa_ncomm", C.c_void_p),
        ("slpa_mem", C.c_void_p),
        ("vol", C.c_void_p),
        ("changed", C.c_void_p),
        ("tier_ms", C.c_void_p),
        ("launches", C.c_void_p),
        ("iter_ms", C.c_void_p),
        ("step_tier_ms", C.c_void_p),
        ("on_device", C.c_int32),
    ]


ITER_CB = C.CFUNCTYPE(C.c_int, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_void_p)

# exported entry points and their ctypes signatures (include/glp.h)
SIGNATURES = {
    "glp_last_error": (C.c_char_p, []),
    "glp_version": (C.c_char_p, []),
    "glp_params_default": (C.c_int, [C.POINTER(Params)]),
    "glp_graph_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32,
                                   C.POINTER(C.c_void_p)]),
    "glp_graph_create_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32,
                                      C.c_uint32, C.POINTER(C.c_void_p)]),
    "glp_graph_destroy": (None, [C.c_void_p]),
    "glp_graph_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "glp_graph_plan": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(C.c_int64)]),
    "glp_graph_check": (C.c_int, [C.c_void_p]),
    "glp_graph_device_view": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "glp_graph_set_cancel_flag": (C.c_int, [C.c_void_p, C.c_void_p]),
    "glp_graph_set_seeds": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "glp_graph_from_edges": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_uint32,
                                       C.c_void_p, C.POINTER(C.c_void_p)]),
    "glp_graph_export": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "glp_graph_cm_sketch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_void_p]),
    "glp_graph_fa_summary": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32,
                                       C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "glp_plan_offsets": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Params), C.POINTER(C.c_int64)]),
    "glp_run": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Params), C.c_int32, C.POINTER(Outputs), ITER_CB,
                          C.c_void_p, C.c_void_p]),
    "glp_sample_rmat": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int64, C.c_int64,
                                  C.c_void_p, C.c_void_p, C.c_int32]),
    "glp_sample_planted": (C.c_int, [C.c_int32, C.c_int32, C.c_int64, C.c_uint64, C.c_int64, C.c_int64, C.c_void_p,
                                     C.c_void_p, C.c_int32]),
    "glp_sample_overlap": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_uint64, C.c_int64, C.c_int64,
                                     C.c_void_p, C.c_void_p, C.c_int32]),
    "glp_edge_weights": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_uint64, C.c_void_p,
                                   C.c_int32]),
    "glp_load_edgelist_bin": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "glp_free_host": (None, [C.c_void_p]),
    "glp_batch_create": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                   C.POINTER(C.c_void_p)]),
    "glp_batch_create_ex": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                      C.c_void_p, C.POINTER(C.c_void_p)]),
    "glp_batch_repack": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                   C.c_void_p]),
    "glp_batch_destroy": (None, [C.c_void_p]),
    "glp_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32)]),
    "glp_batch_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "glp_batch_tune": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "glp_server_config_default": (C.c_int, [C.c_void_p]),
    "glp_server_start": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "glp_server_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32,
                                    C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int64)]),
    "glp_server_add_graph": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64,
                                       C.c_int32, C.POINTER(C.c_int64)]),
    "glp_server_add_edges": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                                       C.c_uint32, C.c_void_p, C.POINTER(C.c_int64)]),
    "glp_server_submit_graph": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                          C.POINTER(C.c_int64)]),
    "glp_server_remove_graph": (C.c_int, [C.c_void_p, C.c_int64]),
    "glp_server_poll": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p]),
    "glp_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p]),
    "glp_server_release": (C.c_int, [C.c_void_p, C.c_int64]),
    "glp_server_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
    "glp_server_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                  C.POINTER(C.c_int64)]),
    "glp_server_stop": (C.c_int, [C.c_void_p]),
    "glp_run_classic_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
}

OPTIONAL_SIGNATURES: dict = {}

_lib = None


def load() -> C.CDLL:
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m glp_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in {**SIGNATURES, **OPTIONAL_SIGNATURES}.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> int:
    if rc < 0:
        msg = load().glp_last_error()
        raise GlpError(rc, msg.decode() if msg else "")
    return rc


def default_params() -> Params:
    p = Params()
    check(load().glp_params_default(C.byref(p)))
    return p
