"""ctypes binding of libphem.so (include/phem.h).

The library is the product: if it is missing this module raises instead of
falling back to anything else.  The seeded input generators (phem_gen_*,
host-only code) are also built alone into libphem_gen.so, which gen_lib()
loads, so that generating an input does not map the solver library (the
reference arm of the benchmark generates its input without it).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libphem.so"
GEN_LIB_PATH = PKG / "libphem_gen.so"

PHEM_OK = 0
PHEM_ERR_INVALID = 1
PHEM_ERR_CUDA = 2
PHEM_ERR_NOMEM = 3
PHEM_ERR_NONCONVERGED = 4
PHEM_ERR_TIMEOUT = 5
PHEM_ERR_UNSUPPORTED = 6
PHEM_ERR_NO_DEVICE = 7
PHEM_FOREST_EMPTY = 0x7FFFFFFF
PHEM_MAX_ROUNDS = 64
PHEM_CC_DEFAULT = 0
PHEM_CC_CANONICAL = 1
PHEM_CC_NOALLOC_MAX_VERTICES = 1 << 20
PHEM_BATCH_MSF = 0
PHEM_BATCH_CC = 1
PHEM_PATH_BATCHED = 0
PHEM_PATH_DEVICE = 1


class PhemError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: status {status}: {detail}")
        self.status = status


class PhemEdge(C.Structure):
    _fields_ = [("u", C.c_uint32), ("v", C.c_uint32), ("w", C.c_uint32)]


class CCStats(C.Structure):
    _fields_ = [("forest_edges", C.c_uint64), ("components", C.c_uint32), ("rounds", C.c_uint32),
                ("device_ms", C.c_float)]


class MSFStats(C.Structure):
    _fields_ = [("rounds", C.c_uint32), ("light_rounds", C.c_uint32),
                ("m_r", C.c_uint64 * PHEM_MAX_ROUNDS), ("n_r", C.c_uint64 * PHEM_MAX_ROUNDS),
                ("msf_edges", C.c_uint64), ("total_weight", C.c_uint64), ("threshold", C.c_uint64),
                ("device_ms", C.c_float)]


class KernelProfile(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_uint64), ("timed_launches", C.c_uint64),
                ("total_ms", C.c_double)]


class LaunchRecord(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("ms", C.c_float)]


class BatchGraph(C.Structure):
    _fields_ = [("edge_offset", C.c_uint64), ("num_edges", C.c_uint32), ("num_vertices", C.c_uint32),
                ("vertex_offset", C.c_uint32), ("kind", C.c_uint32)]


class ServerConfig(C.Structure):
    _fields_ = [("memory_budget", C.c_uint64), ("slots", C.c_uint32), ("max_batch_graphs", C.c_uint32),
                ("large_edges", C.c_uint64), ("large_workers", C.c_uint32), ("reserved", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("num_vertices", C.c_uint32), ("num_edges", C.c_uint64),
                ("edges", C.c_void_p), ("pairs", C.c_void_p), ("forest", C.c_void_p), ("labels", C.c_void_p)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("path", C.c_uint32), ("forest_edges", C.c_uint64),
                ("total_weight", C.c_uint64), ("submit_ns", C.c_uint64), ("start_ns", C.c_uint64),
                ("done_ns", C.c_uint64)]


class BatchStats(C.Structure):
    _fields_ = [("max_rounds", C.c_uint32), ("block_size", C.c_uint32), ("items", C.c_uint32),
                ("compact_ratio", C.c_float), ("grid", C.c_uint32), ("smem_vertices", C.c_uint32),
                ("device_ms", C.c_float)]


_VP = C.c_void_p
_lib = None

# name -> (restype, argtypes); mirrors include/phem.h
SIGNATURES = {
    "phem_version": (C.c_int, []),
    "phem_status_string": (C.c_char_p, [C.c_int]),
    "phem_last_error": (C.c_char_p, []),
    "phem_context_create": (C.c_int, [C.c_int, C.POINTER(_VP)]),
    "phem_context_destroy": (None, [_VP]),
    "phem_context_set_stream": (C.c_int, [_VP, _VP]),
    "phem_context_stream": (_VP, [_VP]),
    "phem_context_set_timeout_ms": (C.c_int, [_VP, C.c_uint32]),
    "phem_context_trim": (C.c_int, [_VP]),
    "phem_context_set_tuning": (C.c_int, [_VP, C.c_char_p, C.c_double]),
    "phem_context_get_tuning": (C.c_int, [_VP, C.c_char_p, C.POINTER(C.c_double)]),
    "phem_context_set_profiling": (C.c_int, [_VP, C.c_int]),
    "phem_context_profile": (C.c_int, [_VP, C.POINTER(KernelProfile), C.c_uint32, C.POINTER(C.c_uint32)]),
    "phem_context_profile_reset": (C.c_int, [_VP]),
    "phem_context_launch_log": (C.c_int, [_VP, C.POINTER(LaunchRecord), C.c_uint32, C.POINTER(C.c_uint32)]),
    "phem_cc_solve": (C.c_int, [_VP, _VP, C.c_int64, C.c_int32, _VP, _VP, C.c_uint32, C.POINTER(CCStats)]),
    "phem_cc_init": (C.c_int, [_VP, C.c_int32, _VP, _VP, _VP]),
    "phem_cc_unite": (C.c_int, [_VP, _VP, C.c_int64, C.c_int32, _VP, _VP]),
    "phem_cc_label": (C.c_int, [_VP, C.c_int32, _VP, _VP]),
    "phem_cc_stream": (C.c_int, [_VP, _VP, C.c_int64, C.c_int32, C.c_int64, _VP, _VP, _VP,
                                 C.POINTER(C.c_float)]),
    "phem_cc_stream_begin": (C.c_int, [_VP, C.c_int32, _VP, _VP, _VP]),
    "phem_cc_stream_push": (C.c_int, [_VP, _VP, C.c_int64]),
    "phem_cc_stream_end": (C.c_int, [_VP, C.POINTER(C.c_float)]),
    "phem_cc_merge": (C.c_int, [_VP, _VP, _VP, C.c_int32, _VP, _VP, _VP, C.POINTER(C.c_float)]),
    "phem_cc_solve_noalloc": (C.c_int, [_VP, C.c_int64, C.c_int32, _VP, _VP, _VP]),
    "phem_msf_solve": (C.c_int, [_VP, _VP, C.c_uint64, C.c_uint32, _VP, C.POINTER(C.c_uint64),
                                 C.POINTER(C.c_uint64), C.POINTER(MSFStats)]),
    "phem_msf_solve_device": (C.c_int, [_VP, _VP, C.c_uint64, C.c_uint32, _VP, _VP, C.POINTER(MSFStats)]),
    "phem_msf_stream": (C.c_int, [_VP, _VP, C.c_uint64, C.c_uint32, C.c_uint64, _VP, C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_float)]),
    "phem_msf_solve_csr": (C.c_int, [_VP, _VP, _VP, C.c_uint32, _VP, C.c_uint64, _VP, C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_uint64), C.POINTER(MSFStats)]),
    "phem_csr_to_coo": (C.c_int, [_VP, _VP, _VP, C.c_int32, _VP, C.POINTER(C.c_int64)]),
    "phem_gen_mix64": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint64]),
    "phem_gen_er": (C.c_int, [C.c_uint32, C.c_uint64, C.c_uint64, _VP, C.POINTER(C.c_uint64)]),
    "phem_gen_rmat": (C.c_int, [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64, _VP,
                                C.POINTER(C.c_uint64)]),
    "phem_gen_weights": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint32, _VP]),
    "phem_pack_msf_edges": (C.c_int, [_VP, _VP, C.c_uint64, _VP]),
    "phem_csr_from_sorted_pairs": (C.c_int, [_VP, C.c_uint64, C.c_uint32, _VP, _VP]),
    "phem_gen_rmat_range": (C.c_int, [C.c_uint32, C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                      C.c_uint64, _VP, C.POINTER(C.c_uint64)]),
    "phem_read_mtx": (C.c_int, [C.c_char_p, C.c_int, _VP, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "phem_read_ecl": (C.c_int, [C.c_char_p, _VP, _VP, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "phem_read_graph_pairs": (C.c_int, [C.c_char_p, _VP, C.c_uint64, C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint64)]),
    "phem_io_last_error": (C.c_char_p, []),
    "phem_gen_rgg": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint64, _VP, _VP, C.POINTER(C.c_uint64)]),
    "phem_gen_rmat_range_device": (C.c_int, [_VP, C.c_uint32, C.c_uint64, C.c_uint64, C.c_double, C.c_double,
                                             C.c_double, C.c_uint64, _VP, C.POINTER(C.c_uint64)]),
    "phem_batch_solve": (C.c_int, [_VP, _VP, C.c_uint32, _VP, C.c_uint64, C.c_uint32, _VP, _VP, _VP, _VP,
                                   C.POINTER(BatchStats)]),
    "phem_batch_plan_create": (C.c_int, [_VP, C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(_VP)]),
    "phem_batch_plan_destroy": (None, [_VP]),
    "phem_batch_plan_upload": (C.c_int, [_VP, _VP, C.c_uint32, _VP, C.c_uint64, C.c_uint32]),
    "phem_batch_plan_run": (C.c_int, [_VP]),
    "phem_batch_plan_download": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "phem_batch_plan_device": (C.c_int, [_VP, C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                                         C.POINTER(_VP)]),
    "phem_batch_autotune": (C.c_int, [_VP, _VP, C.c_uint32, _VP, C.c_uint64, C.c_uint32, C.c_uint32,
                                      C.POINTER(BatchStats)]),
    "phem_server_create": (C.c_int, [C.c_int, C.POINTER(ServerConfig), C.POINTER(_VP)]),
    "phem_server_destroy": (None, [_VP]),
    "phem_server_submit": (C.c_int, [_VP, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "phem_server_wait": (C.c_int, [_VP, C.c_uint64, C.c_uint32, C.POINTER(RequestResult)]),
    "phem_server_replay": (C.c_int, [_VP, C.POINTER(Request), _VP, C.c_uint32, C.POINTER(RequestResult)]),
}


def lib() -> C.CDLL:
    """The loaded libphem.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m phem_graph_b200.build` "
                              "(there is no fallback implementation)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


_GEN_NAMES = ("phem_gen_mix64", "phem_gen_er", "phem_gen_rmat", "phem_gen_weights", "phem_pack_msf_edges",
              "phem_csr_from_sorted_pairs", "phem_gen_rmat_range", "phem_gen_rgg")
_gen_lib = None


def gen_lib() -> C.CDLL:
    """The loaded libphem_gen.so (the generators alone); raises if it has not been built."""
    global _gen_lib
    if _gen_lib is None:
        if not GEN_LIB_PATH.exists():
            raise ImportError(f"{GEN_LIB_PATH} is missing: build it with `python -m phem_graph_b200.build`")
        L = C.CDLL(str(GEN_LIB_PATH))
        for name in _GEN_NAMES:
            res, args = SIGNATURES[name]
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _gen_lib = L
    return _gen_lib


def check_gen(status: int, where: str) -> None:
    """check() for the generator library (which keeps no error text)."""
    if status != PHEM_OK:
        raise PhemError(status, where, "invalid generator arguments")


def check(status: int, where: str) -> None:
    if status != PHEM_OK:
        detail = lib().phem_last_error()
        raise PhemError(status, where, detail.decode() if detail else "")


def ptr(a) -> int | None:
    """Address of a numpy array, a torch tensor or an int; None for None."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a)!r}")
