"""B200-native query VM for Virginian (sm_100a), Python side.

The product is the C ABI in include/virginian_b200.h, implemented in CUDA in
``csrc/`` and built into ``libvirginian_b200.so``.  This package wraps it with
ctypes for tests, benchmarks and Python callers:

* :class:`Engine` - one per device (stream, scratch, caches);
* :class:`Program` - a validated, decoded data-parallel section of a
  Virginian opcode program (``virg_op`` array, src/virginian.h:327-377);
* :class:`Table` - an HBM-resident table made of segments (tablets);
* :class:`Result` - an ordered, HBM-resident result stream.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import ProgramInfo, Schema, Segment, VirgError, VirgOp, check, lib

# virg_t numbering, src/virginian.h:196-204
VIRG_INT, VIRG_INT64, VIRG_FLOAT, VIRG_DOUBLE, VIRG_CHAR = 0, 1, 2, 3, 4
NP_OF = {VIRG_INT: np.int32, VIRG_INT64: np.int64, VIRG_FLOAT: np.float32,
         VIRG_DOUBLE: np.float64, VIRG_CHAR: np.int8}
TYPE_OF = {np.dtype(v): k for k, v in NP_OF.items()}

__all__ = ["Engine", "Program", "Table", "Result", "Batch", "Serve", "VirgError", "make_schema", "ops_array",
           "VIRG_INT", "VIRG_INT64", "VIRG_FLOAT", "VIRG_DOUBLE", "VIRG_CHAR", "NP_OF"]


def make_schema(col_types: Sequence[int], key_type: int = VIRG_INT) -> Schema:
    s = Schema()
    s.key_type = key_type
    s.ncols = len(col_types)
    for i, t in enumerate(col_types):
        s.col_type[i] = t
    return s


def ops_array(ops) -> Tuple[ctypes.Array, int]:
    """Accepts a ctypes virg_op array/structure sequence or (op,p1,p2,p3,p4) tuples."""
    n = len(ops)
    arr = (VirgOp * max(n, 1))()
    for k, o in enumerate(ops):
        if isinstance(o, tuple):
            op, p1, p2, p3 = o[:4]
            arr[k].op, arr[k].p1, arr[k].p2, arr[k].p3 = op, p1, p2, p3
            if len(o) > 4:
                p4 = o[4]
                if isinstance(p4, float):
                    arr[k].p4.f = p4
                else:
                    arr[k].p4.i = int(p4)
        else:
            ctypes.memmove(ctypes.byref(arr[k]), ctypes.byref(o), ctypes.sizeof(VirgOp))
    return arr, n


class Engine:
    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(lib().virg_gpu_engine_create(device, ctypes.byref(h)), "engine create")
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().virg_gpu_engine_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self) -> int:
        return lib().virg_gpu_engine_stream(self.h)

    def set_shared_scan(self, enable: bool) -> None:
        """Shared scans (off by default): in a launch of several queries, the
        queries over one table claim its chunks interleaved, so a chunk's
        columns come from device memory once and from L2 for the others."""
        check(lib().virg_gpu_engine_set_shared_scan(self.h, 1 if enable else 0), "set shared scan")

    def set_shape(self, threads: int = 0, stage_kb: int = 0, stages: int = 0,
                  ctas_per_sm: int = 0, chunk_rows: int = 0, full_mode: int = 0) -> None:
        """Launch shape of later queries: compute threads per CTA, KB per
        staging buffer, buffers, CTAs per SM, the chunk bound and the full
        phase's mode (0 reads staged tiles in place, 1 gathers the selected
        rows from device memory, 2 runs the projection over every row of a
        staged group); 0 in a field keeps the automatic choice."""
        check(lib().virg_gpu_engine_set_shape(self.h, threads, stage_kb, stages,
                                              ctas_per_sm), "set shape")
        check(lib().virg_gpu_engine_set_chunk_rows(self.h, chunk_rows), "set chunk rows")
        check(lib().virg_gpu_engine_set_full_mode(self.h, full_mode), "set full mode")

    def device_error(self) -> int:
        e = ctypes.c_uint()
        check(lib().virg_gpu_engine_check(self.h, ctypes.byref(e)), "engine check")
        return e.value

    def timing(self, slots: int) -> None:
        """Record events around each of the next launches (ring of `slots`)."""
        check(lib().virg_gpu_engine_timing(self.h, slots), "engine timing")

    def kernel_times(self, n: int) -> List[float]:
        """Device milliseconds of up to the last n timed kernel launches."""
        buf = (ctypes.c_float * max(n, 1))()
        got = ctypes.c_uint()
        check(lib().virg_gpu_engine_kernel_times(self.h, buf, n, ctypes.byref(got)), "kernel times")
        return [buf[i] for i in range(got.value)]

    @property
    def launches(self) -> int:
        return int(lib().virg_gpu_engine_launches(self.h))

    def last_launch(self) -> Dict[str, int]:
        s = (ctypes.c_uint * 4)()
        g, m = ctypes.c_uint(), ctypes.c_uint()
        check(lib().virg_gpu_engine_last_launch(self.h, s, ctypes.byref(g), ctypes.byref(m)),
              "last launch")
        return {"threads": s[0], "stage_kb": s[1], "stages": s[2], "ctas_per_sm": s[3],
                "grid": g.value, "smem": m.value}

    def query_host(self, program: "Program", segments: Sequence[dict], capacity: Optional[int] = None):
        """End to end from host arrays: returns the result columns as numpy arrays."""
        segs, keep = _segments(segments, program.col_types)
        total = sum(int(s["rows"]) for s in segments)
        cap = total if capacity is None else capacity
        info = program.info
        outs = [np.empty(max(cap, 1), dtype=NP_OF[info.out_type[j]]) for j in range(info.nout)]
        ptrs = (ctypes.c_void_p * max(1, info.nout))(*[o.ctypes.data for o in outs])
        rows = ctypes.c_uint64()
        check(lib().virg_gpu_query_host(self.h, program.h, segs, len(segments), ptrs, cap,
                                        ctypes.byref(rows)), "query_host")
        del keep
        return [o[:rows.value] for o in outs]


class Program:
    def __init__(self, ops, pc: int, col_types: Sequence[int], key_type: int = VIRG_INT):
        arr, n = ops_array(ops)
        self.col_types = list(col_types)
        self.key_type = key_type
        self.schema = make_schema(col_types, key_type)
        h = ctypes.c_void_p()
        check(lib().virg_gpu_program_create(arr, n, pc, ctypes.byref(self.schema), ctypes.byref(h)),
              "program create")
        self.h = h
        self.info = ProgramInfo()
        check(lib().virg_gpu_program_info_get(self.h, ctypes.byref(self.info)), "program info")

    @property
    def maybe_undefined(self) -> bool:
        return lib().virg_gpu_program_flags(self.h) == 1

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().virg_gpu_program_destroy(self.h)
        except Exception:
            pass


def _segments(segments: Sequence[dict], col_types: Sequence[int]):
    """Builds virg_gpu_segment structs from dicts {rows, key, cols} of numpy arrays."""
    arr = (Segment * max(1, len(segments)))()
    keep = []
    for i, s in enumerate(segments):
        arr[i].rows = int(s["rows"])
        k = s.get("key")
        if isinstance(k, int):
            arr[i].key = k
        elif k is not None:
            k = np.ascontiguousarray(k)
            keep.append(k)
            arr[i].key = k.ctypes.data
        for c, col in enumerate(s["cols"]):
            if col is None:
                continue
            if isinstance(col, int):
                arr[i].col[c] = col
                continue
            col = np.ascontiguousarray(col)
            if c < len(col_types):
                assert col.dtype == NP_OF[col_types[c]], (c, col.dtype)
            keep.append(col)
            arr[i].col[c] = col.ctypes.data
    return arr, keep


class Table:
    def __init__(self, engine: Engine, col_types: Sequence[int], key_type: int = VIRG_INT):
        self.engine = engine
        self.col_types = list(col_types)
        self.schema = make_schema(col_types, key_type)
        h = ctypes.c_void_p()
        check(lib().virg_gpu_table_create(engine.h, ctypes.byref(self.schema), ctypes.byref(h)),
              "table create")
        self.h = h

    def append(self, segments: Sequence[dict]) -> None:
        segs, keep = _segments(segments, self.col_types)
        check(lib().virg_gpu_table_append(self.h, segs, len(segments)), "table append")
        del keep

    @property
    def rows(self) -> int:
        return int(lib().virg_gpu_table_rows(self.h))

    @property
    def nbytes(self) -> int:
        return int(lib().virg_gpu_table_bytes(self.h))

    def load_db(self, path: str, table: str) -> int:
        """Appends every tablet of a table of a Virginian database file (read
        straight into pinned buffers and copied to the device); returns the
        rows appended."""
        n = ctypes.c_uint64()
        check(lib().virg_gpu_table_load_db(self.h, path.encode(), table.encode(), ctypes.byref(n)), "table load_db")
        return n.value

    def estimate(self, program: "Program") -> int:
        """Rows the program's filter keeps in a host sample of this table,
        scaled to the table (an estimate for sizing reservations)."""
        n = ctypes.c_uint64()
        check(lib().virg_gpu_table_estimate(self.h, program.h, ctypes.byref(n)), "table estimate")
        return n.value

    def read_ceiling(self, columns: Sequence[int], mode: int = 0, reps: int = 5) -> Tuple[float, int]:
        """Device time (ms, best of `reps`) and bytes of a kernel that only
        reads the given columns (-1: the key) of every segment: mode 0 with
        16-byte loads, 1-3 with bulk copies into 4, 6 or 2 shared-memory
        stages.  A measurement aid: the read bandwidth a scan of those
        columns could reach."""
        cols = (ctypes.c_int * max(1, len(columns)))(*columns)
        ms, nbytes = ctypes.c_double(), ctypes.c_ulonglong()
        check(lib().virg_gpu_table_read_ceiling(self.h, cols, len(columns), mode, reps, ctypes.byref(ms),
                                                ctypes.byref(nbytes)), "read ceiling")
        return ms.value, nbytes.value

    def query(self, program: Program) -> "Result":
        r = ctypes.c_void_p()
        check(lib().virg_gpu_query(self.engine.h, program.h, self.h, ctypes.byref(r)), "query")
        return Result(r, program)

    def close(self) -> None:
        if self.h:
            lib().virg_gpu_table_destroy(self.h)
            self.h = None


class Result:
    def __init__(self, h: ctypes.c_void_p, program: Program):
        self.h = h
        self.program = program

    @property
    def rows(self) -> int:
        n = ctypes.c_uint64()
        check(lib().virg_gpu_result_rows(self.h, ctypes.byref(n)), "result rows")
        return n.value

    def column_ptr(self, c: int) -> int:
        return lib().virg_gpu_result_column(self.h, c)

    def download(self, first: int = 0, count: Optional[int] = None) -> List[np.ndarray]:
        n = self.rows
        count = n - first if count is None else count
        info = self.program.info
        outs = [np.empty(max(count, 1), dtype=NP_OF[info.out_type[j]]) for j in range(info.nout)]
        ptrs = (ctypes.c_void_p * max(1, info.nout))(*[o.ctypes.data for o in outs])
        check(lib().virg_gpu_result_download(self.h, ptrs, first, count), "result download")
        return [o[:count] for o in outs]

    def close(self) -> None:
        if self.h:
            lib().virg_gpu_result_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many (program, table) queries run by one persistent launch."""

    def __init__(self, engine: Engine, autotune: bool = False):
        self.engine = engine
        h = ctypes.c_void_p()
        check(lib().virg_gpu_batch_create(engine.h, ctypes.byref(h)), "batch create")
        self.h = h
        self.programs: List[Program] = []
        if autotune:
            check(lib().virg_gpu_batch_set_autotune(self.h, 1), "batch autotune")

    def add(self, program: Program, table: Table) -> int:
        slot = ctypes.c_uint()
        check(lib().virg_gpu_batch_add(self.h, program.h, table.h, ctypes.byref(slot)), "batch add")
        self.programs.append(program)
        return slot.value

    def run(self, graph: bool = True) -> None:
        check(lib().virg_gpu_batch_run(self.h, 1 if graph else 0), "batch run")

    def wait(self) -> None:
        check(lib().virg_gpu_batch_wait(self.h), "batch wait")

    def rows(self, slot: int) -> int:
        n = ctypes.c_uint64()
        check(lib().virg_gpu_batch_rows(self.h, slot, ctypes.byref(n)), "batch rows")
        return n.value

    def download(self, slot: int) -> List[np.ndarray]:
        n = self.rows(slot)
        info = self.programs[slot].info
        outs = [np.empty(max(n, 1), dtype=NP_OF[info.out_type[j]]) for j in range(info.nout)]
        ptrs = (ctypes.c_void_p * max(1, info.nout))(*[o.ctypes.data for o in outs])
        check(lib().virg_gpu_batch_download(self.h, slot, ptrs, 0, n), "batch download")
        return [o[:n] for o in outs]

    def shape(self) -> Dict[str, int]:
        s = (ctypes.c_uint * 4)()
        w = ctypes.c_uint64()
        check(lib().virg_gpu_batch_shape(self.h, s, ctypes.byref(w)), "batch shape")
        return {"threads": s[0], "stage_kb": s[1], "stages": s[2], "grid": s[3],
                "chunks": w.value}

    def close(self) -> None:
        if self.h:
            lib().virg_gpu_batch_destroy(self.h)
            self.h = None


class Serve:
    """Serving loop: queries folded into one running persistent kernel
    (continuous batching), admitted by estimated result memory."""

    def __init__(self, engine: Engine, result_budget_bytes: int = 0, max_queries: int = 0,
                 idle_us: int = 0, max_load_bytes_per_row: int = 0, max_row_vector_bytes: int = 0,
                 max_sel_vector_bytes: int = 0, wait_limit_ms: int = 0):
        from ._lib import ServeConfig
        cfg = ServeConfig(result_budget_bytes, max_queries, idle_us, max_load_bytes_per_row,
                          max_row_vector_bytes, max_sel_vector_bytes, wait_limit_ms)
        h = ctypes.c_void_p()
        check(lib().virg_serve_create(engine.h, ctypes.byref(cfg), ctypes.byref(h)), "serve create")
        self.h = h
        self.engine = engine
        self._programs: Dict[int, Program] = {}

    def submit(self, program: Program, table: Table, estimated_rows: int = 0) -> int:
        t = ctypes.c_uint64()
        check(lib().virg_serve_submit(self.h, program.h, table.h, estimated_rows, ctypes.byref(t)),
              "serve submit")
        self._programs[t.value] = program
        return t.value

    def poll(self, ticket: int, wait_ms: int = 0) -> Dict[str, float]:
        from ._lib import ServeStatus
        st = ServeStatus()
        check(lib().virg_serve_poll(self.h, ticket, wait_ms, ctypes.byref(st)), "serve poll")
        return {"done": bool(st.done), "rows": st.rows, "readmits": st.readmits,
                "queue_us": st.queue_us, "latency_us": st.latency_us}

    def wait(self, ticket: int, timeout_s: float = 600.0) -> Dict[str, float]:
        import time
        deadline = time.monotonic() + timeout_s
        while True:
            st = self.poll(ticket, 100)
            if st["done"]:
                return st
            if time.monotonic() > deadline:
                raise VirgError(f"serve wait: query {ticket} not done after {timeout_s} s: {self.stats()}")

    def download(self, ticket: int) -> List[np.ndarray]:
        n = self.wait(ticket)["rows"]
        info = self._programs[ticket].info
        outs = [np.empty(max(n, 1), dtype=NP_OF[info.out_type[j]]) for j in range(info.nout)]
        ptrs = (ctypes.c_void_p * max(1, info.nout))(*[o.ctypes.data for o in outs])
        check(lib().virg_serve_download(self.h, ticket, ptrs), "serve download")
        return [o[:n] for o in outs]

    def release(self, ticket: int) -> None:
        check(lib().virg_serve_release(self.h, ticket), "serve release")
        self._programs.pop(ticket, None)

    def stats(self) -> Dict[str, int]:
        from ._lib import ServeCounters
        c = ServeCounters()
        check(lib().virg_serve_stats(self.h, ctypes.byref(c)), "serve stats")
        return {"sessions": c.sessions, "admitted": c.admitted, "readmitted": c.readmitted,
                "pending": c.pending, "inflight": c.inflight, "arena_used": c.arena_used,
                "device_error": c.device_error, "restarts": c.restarts,
                "work_items": c.work_items, "status_ring": c.status_ring, "sampled": c.sampled,
                "shape": {"threads": c.shape[0], "stage_kb": c.shape[1], "stages": c.shape[2],
                          "grid": c.shape[3]}}

    def close(self) -> None:
        if self.h:
            lib().virg_serve_destroy(self.h)
            self.h = None


def query_streamed(engine: Engine, program: Program, segments: Sequence[dict],
                   segs_per_chunk: int = 8):
    """Runs a program over host-resident segments, streaming the columns it
    reads through a staging ring; returns (Result, stats dict)."""
    from ._lib import StreamStats
    segs, keep = _segments(segments, program.col_types)
    r = ctypes.c_void_p()
    st = StreamStats()
    check(lib().virg_gpu_query_streamed(engine.h, program.h, segs, len(segments), segs_per_chunk,
                                        ctypes.byref(r), ctypes.byref(st)), "query_streamed")
    del keep
    return Result(r, program), {"seconds": st.seconds, "copy_seconds": st.copy_seconds,
                                "h2d_bytes": st.h2d_bytes, "chunks": st.chunks}


def tune(engine: Engine, program: Program, table: Table) -> Dict[str, int]:
    """Times the launch shapes for this query and caches the fastest."""
    s = (ctypes.c_uint * 4)()
    check(lib().virg_gpu_query_tune(engine.h, program.h, table.h, s), "query tune")
    return {"threads": s[0], "stage_kb": s[1], "stages": s[2], "ctas_per_sm": s[3]}
