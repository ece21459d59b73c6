"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes wrapper over ``oracle/_ref/libvirg_ref.so``: the reference's own
single-thread CPU VM (``virginia_single``, src/vm/virginia.c:228-891) and
multi-core VM, built unmodified from the reference sources by
``oracle/Makefile``, with a hand-written SQL front end (``oracle/sql_parse.c``)
feeding the reference's code generator (src/sql/generate.c).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module, as the checker or as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libvirg_ref.so")
REFGPU_LIB = os.path.join(HERE, "_ref", "libvirg_refgpu.so")
HOST_LIB = os.path.join(HERE, "_ref", "libvirg_host.so")

# virg_t (src/virginian.h:196-204)
VIRG_INT, VIRG_INT64, VIRG_FLOAT, VIRG_DOUBLE, VIRG_CHAR = 0, 1, 2, 3, 4
NP_TYPES = {VIRG_INT: np.int32, VIRG_INT64: np.int64, VIRG_FLOAT: np.float32,
            VIRG_DOUBLE: np.float64, VIRG_CHAR: np.int8}

VIRG_OPS = 32
VIRG_MAX_COLUMN_NAME = 16


class VirgVar(ctypes.Union):
    """virg_var (src/virginian.h:309-317), 8-byte aligned union."""
    _fields_ = [("i", ctypes.c_int), ("f", ctypes.c_float), ("li", ctypes.c_longlong),
                ("d", ctypes.c_double), ("c", ctypes.c_char), ("s", ctypes.c_void_p)]


class VirgOp(ctypes.Structure):
    """virg_op (src/virginian.h:327-333)."""
    _fields_ = [("op", ctypes.c_int), ("p1", ctypes.c_int), ("p2", ctypes.c_int),
                ("p3", ctypes.c_int), ("p4", VirgVar)]


class VirgVM(ctypes.Structure):
    """virg_vm (src/virginian.h:356-377)."""
    _fields_ = [("pc", ctypes.c_uint), ("stmt", VirgOp * VIRG_OPS), ("num_ops", ctypes.c_uint),
                ("global_reg", VirgVar * 16), ("type", ctypes.c_int * 16),
                ("table", ctypes.c_uint * 1), ("num_tables", ctypes.c_uint),
                ("head_result", ctypes.c_void_p), ("tail_result", ctypes.c_void_p),
                ("timing1", ctypes.c_float), ("timing2", ctypes.c_float),
                ("timing3", ctypes.c_float)]


def ref_root() -> str:
    """The reference checkout the oracle compiles from: $VIRGINIAN_REF, else
    the path it is mounted at on the build machine."""
    return os.environ.get("VIRGINIAN_REF", "/root/reference")


def build(root: str = "") -> None:
    """Compile the oracle libraries from the reference sources (needs them)."""
    subprocess.run(["make", "-s", "-C", HERE, f"REF={root or ref_root()}"], check=True)


def _bind(lib: ctypes.CDLL) -> ctypes.CDLL:
    vp, u, ull, i = ctypes.c_void_p, ctypes.c_uint, ctypes.c_ulonglong, ctypes.c_int
    lib.orc_open.restype = vp
    lib.orc_open.argtypes = [ctypes.c_char_p]
    lib.orc_close.argtypes = [vp]
    lib.orc_create_table.argtypes = [vp, ctypes.c_char_p, i, u, ctypes.POINTER(ctypes.c_char_p),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint)]
    lib.orc_insert.argtypes = [vp, u, ull, vp, u, u, ctypes.POINTER(vp), ctypes.POINTER(u)]
    lib.orc_loadmem.argtypes = [vp, u]
    lib.orc_compile.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(VirgVM), ctypes.c_char_p]
    lib.orc_query.restype = vp
    lib.orc_query.argtypes = [vp, ctypes.c_char_p, i, u, u]
    lib.orc_query_ops.restype = vp
    lib.orc_query_ops.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(VirgOp), u]
    lib.orc_result_rows.restype = ull
    lib.orc_result_rows.argtypes = [vp]
    lib.orc_result_ncols.restype = u
    lib.orc_result_ncols.argtypes = [vp]
    lib.orc_result_ntablets.restype = u
    lib.orc_result_ntablets.argtypes = [vp]
    lib.orc_result_seconds.restype = ctypes.c_double
    lib.orc_result_seconds.argtypes = [vp]
    lib.orc_result_timing.restype = ctypes.c_double
    lib.orc_result_timing.argtypes = [vp, ctypes.c_int]
    lib.orc_result_type.restype = i
    lib.orc_result_type.argtypes = [vp, u]
    lib.orc_result_stride.restype = u
    lib.orc_result_stride.argtypes = [vp, u]
    lib.orc_result_tablet_rows.argtypes = [vp, vp, ctypes.POINTER(u)]
    lib.orc_result_copy.argtypes = [vp, vp, ctypes.POINTER(vp)]
    lib.orc_result_free.argtypes = [vp, vp]
    lib.orc_reader_walk.restype = ull
    lib.orc_reader_walk.argtypes = [vp, ctypes.c_char_p, vp, u, ull, ctypes.POINTER(ull)]
    lib.orc_set_gpu_flags.argtypes = [vp, i, i, i]
    lib.orc_close_keep.restype = i
    lib.orc_close_keep.argtypes = [vp, ctypes.c_char_p, u]
    lib.orc_testsizes.restype = ctypes.POINTER(ctypes.c_size_t)
    lib.orc_sizeof_vm.restype = u
    lib.orc_sizeof_meta.restype = u
    lib.orc_mem_tablets.restype = u
    lib.orc_max_tables.restype = u
    return lib


_LIBS: Dict[str, ctypes.CDLL] = {}


def lib(path: str = REF_LIB, mode: int = ctypes.RTLD_LOCAL) -> ctypes.CDLL:
    if path not in _LIBS:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` first")
        _LIBS[path] = _bind(ctypes.CDLL(path, mode=mode))
    return _LIBS[path]


class Result:
    """Concatenated result stream of one query (all result tablets in order)."""

    def __init__(self, columns: List[np.ndarray], types: List[int], tablet_rows: List[int],
                 seconds: float):
        self.columns = columns
        self.types = types
        self.tablet_rows = tablet_rows
        self.seconds = seconds

    @property
    def rows(self) -> int:
        return 0 if not self.columns else int(self.columns[0].shape[0])


class OracleDB:
    """One reference database instance (virg_init + virg_db_create)."""

    def __init__(self, path: str = REF_LIB, mode: int = ctypes.RTLD_LOCAL):
        self.lib = lib(path, mode)
        self._tmp = tempfile.mkdtemp(prefix="virg_oracle_")
        self.h = self.lib.orc_open(self._tmp.encode())
        if not self.h:
            raise RuntimeError("virg_init/virg_db_create failed")
        self.tables: Dict[str, int] = {}

    def close(self) -> None:
        if self.h:
            self.lib.orc_close(self.h)
            self.h = None
            try:
                os.rmdir(self._tmp)
            except OSError:
                pass

    def close_keep(self) -> str:
        """Closes the database, writing every tablet to its file, and keeps
        the file; returns its path (the caller removes it and its folder)."""
        buf = ctypes.create_string_buffer(1024)
        if not self.lib.orc_close_keep(self.h, buf, 1024):
            raise RuntimeError("virg_close failed")
        self.h = None
        return buf.value.decode()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def create_table(self, name: str, columns: Sequence[tuple], key_type: int = VIRG_INT) -> int:
        names = (ctypes.c_char_p * max(1, len(columns)))(*[c[0].encode() for c in columns])
        types = (ctypes.c_int * max(1, len(columns)))(*[c[1] for c in columns])
        tid = ctypes.c_uint()
        if not self.lib.orc_create_table(self.h, name.encode(), key_type, len(columns), names, types,
                                         ctypes.byref(tid)):
            raise RuntimeError("table create failed")
        self.tables[name] = tid.value
        return tid.value

    def insert(self, table: str, keys: np.ndarray, cols: Sequence[np.ndarray]) -> None:
        keys = np.ascontiguousarray(keys)
        cols = [np.ascontiguousarray(c) for c in cols]
        n = keys.shape[0]
        ptrs = (ctypes.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
        strides = (ctypes.c_uint * max(1, len(cols)))(*[c.itemsize for c in cols])
        self.lib.orc_insert(self.h, self.tables[table], n, keys.ctypes.data, keys.itemsize,
                            len(cols), ptrs, strides)

    def compile(self, sql: str):
        vm = VirgVM()
        names = ctypes.create_string_buffer(VIRG_OPS * VIRG_MAX_COLUMN_NAME)
        if not self.lib.orc_compile(self.h, sql.encode(), ctypes.byref(vm), names):
            raise ValueError(f"oracle could not compile: {sql}")
        raw = names.raw
        colnames = {}
        for k in range(vm.num_ops):
            if vm.stmt[k].op == 1:
                s = raw[k * VIRG_MAX_COLUMN_NAME:(k + 1) * VIRG_MAX_COLUMN_NAME]
                colnames[k] = s.split(b"\0", 1)[0].decode()
        return vm, colnames

    def query(self, sql: str, mode: int = 0, threads: int = 0, repeat: int = 1) -> Result:
        r = self.lib.orc_query(self.h, sql.encode(), mode, threads, repeat)
        if not r:
            raise ValueError(f"oracle query failed: {sql}")
        return self._result(r)

    def query_ops(self, sql: str, ops: Sequence[VirgOp]) -> Result:
        """A hand-assembled program on the single-core CPU VM: `sql` gives
        the result layout (Table, ResultColumn, Parallel), `ops` the whole
        program (see orc_query_ops in harness.c)."""
        arr = (VirgOp * max(1, len(ops)))(*ops)
        r = self.lib.orc_query_ops(self.h, sql.encode(), arr, len(ops))
        if not r:
            raise ValueError(f"oracle could not run the program for: {sql}")
        return self._result(r)

    def _result(self, r) -> Result:
        try:
            n = self.lib.orc_result_rows(r)
            ncols = self.lib.orc_result_ncols(r)
            types = [self.lib.orc_result_type(r, c) for c in range(ncols)]
            cols = [np.empty(n, dtype=NP_TYPES[t]) for t in types]
            ptrs = (ctypes.c_void_p * max(1, ncols))(*[c.ctypes.data for c in cols])
            self.lib.orc_result_copy(self.h, r, ptrs)
            nt = self.lib.orc_result_ntablets(r)
            trows = (ctypes.c_uint * max(1, nt))()
            self.lib.orc_result_tablet_rows(self.h, r, trows)
            res = Result(cols, types, list(trows)[:nt], self.lib.orc_result_seconds(r))
            res.gpu_timing = tuple(self.lib.orc_result_timing(r, k) for k in (1, 2, 3))
            return res
        finally:
            self.lib.orc_result_free(self.h, r)

    def reader_walk(self, sql: str, row_bytes: int, max_rows: int):
        buf = np.zeros(max(1, max_rows) * row_bytes, dtype=np.uint8)
        g = ctypes.c_ulonglong()
        n = self.lib.orc_reader_walk(self.h, sql.encode(), buf.ctypes.data, row_bytes, max_rows,
                                     ctypes.byref(g))
        return n, g.value, buf


def sizes() -> List[int]:
    p = lib().orc_testsizes()
    return [p[k] for k in range(15)]
