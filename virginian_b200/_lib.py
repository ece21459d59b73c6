"""ctypes bindings of ``libvirginian_b200.so`` (declared in include/virginian_b200.h).

The library is loaded with RTLD_GLOBAL so a Virginian host library loaded
afterwards binds its ``virg_vm_gpu`` call to it, as the reference's build links
its GPU VM object into the same archive (src/Makefile:52).  There is no CPU
fallback: importing fails if the CUDA library has not been built.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvirginian_b200.so")

VIRG_OPS = 32
VIRG_MAX_COLUMNS = 16


class VirgVar(ctypes.Union):
    """virg_var, src/virginian.h:309-317."""
    _fields_ = [("i", ctypes.c_int), ("f", ctypes.c_float), ("li", ctypes.c_longlong),
                ("d", ctypes.c_double), ("c", ctypes.c_char), ("s", ctypes.c_void_p)]


class VirgOp(ctypes.Structure):
    """virg_op, src/virginian.h:327-333."""
    _fields_ = [("op", ctypes.c_int), ("p1", ctypes.c_int), ("p2", ctypes.c_int),
                ("p3", ctypes.c_int), ("p4", VirgVar)]


class Schema(ctypes.Structure):
    _fields_ = [("key_type", ctypes.c_int), ("ncols", ctypes.c_uint),
                ("col_type", ctypes.c_int * VIRG_MAX_COLUMNS)]


class Segment(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint32), ("key", ctypes.c_void_p),
                ("col", ctypes.c_void_p * VIRG_MAX_COLUMNS)]


class StreamStats(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("copy_seconds", ctypes.c_double),
                ("h2d_bytes", ctypes.c_uint64), ("chunks", ctypes.c_uint)]


class ServeConfig(ctypes.Structure):
    _fields_ = [("result_budget_bytes", ctypes.c_uint64), ("max_queries", ctypes.c_uint),
                ("idle_us", ctypes.c_uint), ("max_load_bytes_per_row", ctypes.c_uint),
                ("max_row_vector_bytes", ctypes.c_uint), ("max_sel_vector_bytes", ctypes.c_uint),
                ("wait_limit_ms", ctypes.c_uint)]


class ServeStatus(ctypes.Structure):
    _fields_ = [("done", ctypes.c_int), ("rows", ctypes.c_uint64), ("readmits", ctypes.c_uint),
                ("queue_us", ctypes.c_double), ("latency_us", ctypes.c_double)]


class ServeCounters(ctypes.Structure):
    _fields_ = [("sessions", ctypes.c_uint), ("admitted", ctypes.c_ulonglong),
                ("readmitted", ctypes.c_ulonglong), ("pending", ctypes.c_ulonglong),
                ("inflight", ctypes.c_ulonglong), ("arena_used", ctypes.c_ulonglong),
                ("device_error", ctypes.c_uint), ("shape", ctypes.c_uint * 4),
                ("restarts", ctypes.c_ulonglong), ("work_items", ctypes.c_ulonglong),
                ("status_ring", ctypes.c_ulonglong), ("sampled", ctypes.c_ulonglong)]


class ProgramInfo(ctypes.Structure):
    _fields_ = [("nload", ctypes.c_uint), ("load_column", ctypes.c_int * (VIRG_MAX_COLUMNS + 1)),
                ("load_bytes_per_row", ctypes.c_uint), ("nout", ctypes.c_uint),
                ("out_type", ctypes.c_int * VIRG_MAX_COLUMNS),
                ("out_stride", ctypes.c_uint * VIRG_MAX_COLUMNS),
                ("out_bytes_per_row", ctypes.c_uint), ("nuops", ctypes.c_uint),
                ("row_vector_bytes", ctypes.c_uint), ("sel_vector_bytes", ctypes.c_uint)]


def _bind(lib: ctypes.CDLL) -> ctypes.CDLL:
    vp, u, i, u64 = ctypes.c_void_p, ctypes.c_uint, ctypes.c_int, ctypes.c_uint64
    P = ctypes.POINTER
    sig = {
        "virg_gpu_last_error": (ctypes.c_char_p, []),
        "virg_gpu_getsizes": (P(ctypes.c_size_t), []),
        "virg_vm_gpu": (i, [vp, vp, vp, vp, u]),
        "virg_gpu_dropin_cache": (i, [u64]),
        "virg_gpu_dropin_cache_stats": (i, [P(u64), P(u64), P(u64)]),
        "virg_gpu_engine_create": (i, [i, P(vp)]),
        "virg_gpu_engine_destroy": (None, [vp]),
        "virg_gpu_engine_stream": (vp, [vp]),
        "virg_gpu_engine_check": (i, [vp, P(u)]),
        "virg_gpu_engine_set_shape": (i, [vp, u, u, u, u]),
        "virg_gpu_engine_set_chunk_rows": (i, [vp, u]),
        "virg_gpu_engine_set_full_mode": (i, [vp, u]),
        "virg_gpu_engine_set_shared_scan": (i, [vp, i]),
        "virg_gpu_engine_launches": (ctypes.c_ulonglong, [vp]),
        "virg_gpu_engine_timing": (i, [vp, u]),
        "virg_gpu_engine_kernel_times": (i, [vp, P(ctypes.c_float), u, P(u)]),
        "virg_gpu_engine_last_launch": (i, [vp, P(u), P(u), P(u)]),
        "virg_gpu_program_create": (i, [P(VirgOp), u, u, P(Schema), P(vp)]),
        "virg_gpu_program_info_get": (i, [vp, P(ProgramInfo)]),
        "virg_gpu_program_flags": (i, [vp]),
        "virg_gpu_program_destroy": (None, [vp]),
        "virg_gpu_table_create": (i, [vp, P(Schema), P(vp)]),
        "virg_gpu_table_append": (i, [vp, P(Segment), u]),
        "virg_gpu_table_rows": (u64, [vp]),
        "virg_gpu_table_bytes": (u64, [vp]),
        "virg_gpu_table_destroy": (None, [vp]),
        "virg_gpu_table_estimate": (i, [vp, vp, P(u64)]),
        "virg_gpu_table_load_db": (i, [vp, ctypes.c_char_p, ctypes.c_char_p, P(u64)]),
        "virg_gpu_table_read_ceiling": (i, [vp, P(ctypes.c_int), u, u, u, P(ctypes.c_double),
                                            P(ctypes.c_ulonglong)]),
        "virg_gpu_query": (i, [vp, vp, vp, P(vp)]),
        "virg_gpu_query_tune": (i, [vp, vp, vp, P(u)]),
        "virg_gpu_result_rows": (i, [vp, P(u64)]),
        "virg_gpu_result_column": (vp, [vp, u]),
        "virg_gpu_result_download": (i, [vp, P(vp), u64, u64]),
        "virg_gpu_result_destroy": (None, [vp]),
        "virg_gpu_query_host": (i, [vp, vp, P(Segment), u, P(vp), u64, P(u64)]),
        "virg_gpu_query_prealloc": (i, [vp, P(Segment), P(vp), u64, P(u64), vp]),
        "virg_gpu_query_streamed": (i, [vp, vp, P(Segment), u, u, P(vp), P(StreamStats)]),
        "virg_gpu_batch_create": (i, [vp, P(vp)]),
        "virg_gpu_batch_add": (i, [vp, vp, vp, P(u)]),
        "virg_gpu_batch_set_autotune": (i, [vp, i]),
        "virg_gpu_batch_run": (i, [vp, i]),
        "virg_gpu_batch_wait": (i, [vp]),
        "virg_gpu_batch_rows": (i, [vp, u, P(u64)]),
        "virg_gpu_batch_column": (vp, [vp, u, u]),
        "virg_gpu_batch_download": (i, [vp, u, P(vp), u64, u64]),
        "virg_gpu_batch_shape": (i, [vp, P(u), P(u64)]),
        "virg_gpu_batch_destroy": (None, [vp]),
        "virg_serve_create": (i, [vp, P(ServeConfig), P(vp)]),
        "virg_serve_submit": (i, [vp, vp, vp, u64, P(u64)]),
        "virg_serve_poll": (i, [vp, u64, ctypes.c_int, P(ServeStatus)]),
        "virg_serve_download": (i, [vp, u64, P(vp)]),
        "virg_serve_column": (vp, [vp, u64, u]),
        "virg_serve_release": (i, [vp, u64]),
        "virg_serve_stats": (i, [vp, P(ServeCounters)]),
        "virg_serve_destroy": (None, [vp]),
        "virg_gpu_catalog_create": (i, [P(vp)]),
        "virg_gpu_catalog_add_table": (i, [vp, ctypes.c_char_p, i, u, P(ctypes.c_char_p),
                                           P(ctypes.c_int), P(u)]),
        "virg_gpu_catalog_destroy": (None, [vp]),
        "virg_gpu_sql_compile": (i, [vp, ctypes.c_char_p, P(VirgOp), P(u), P(u), ctypes.c_char_p,
                                     P(u)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m virginian_b200.build` "
                "(the VM has no CPU fallback)")
        _lib = _bind(ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL))
    return _lib


def last_error() -> str:
    e = lib().virg_gpu_last_error()
    return e.decode() if e else ""


class VirgError(RuntimeError):
    pass


def check(rc: int, what: str) -> None:
    if not rc:
        raise VirgError(f"{what}: {last_error()}")
