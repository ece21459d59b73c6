"""Python side of the re-entrant SQL front end (virg_gpu_sql_compile)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, List, Sequence, Tuple

from ._lib import VirgOp, check, lib

VIRG_OPS = 32
VIRG_MAX_COLUMN_NAME = 16


@dataclass
class Compiled:
    ops: ctypes.Array        # VirgOp * VIRG_OPS
    num_ops: int
    pc: int                  # first op of the data-parallel section
    table_id: int
    names: Dict[int, str]    # ResultColumn op index -> result column name

    def op_list(self):
        return [self.ops[k] for k in range(self.num_ops)]


class Catalog:
    """Table names, column names and types the compiler resolves against."""

    def __init__(self):
        h = ctypes.c_void_p()
        check(lib().virg_gpu_catalog_create(ctypes.byref(h)), "catalog create")
        self.h = h
        self.tables: Dict[str, int] = {}

    def add_table(self, name: str, columns: Sequence[Tuple[str, int]], key_type: int = 0) -> int:
        n = len(columns)
        names = (ctypes.c_char_p * max(n, 1))(*[c[0].encode() for c in columns])
        types = (ctypes.c_int * max(n, 1))(*[c[1] for c in columns])
        tid = ctypes.c_uint()
        check(lib().virg_gpu_catalog_add_table(self.h, name.encode(), key_type, n, names, types,
                                               ctypes.byref(tid)), "catalog add table")
        self.tables[name] = tid.value
        return tid.value

    def compile(self, sql: str) -> Compiled:
        ops = (VirgOp * VIRG_OPS)()
        n, pc, tid = ctypes.c_uint(), ctypes.c_uint(), ctypes.c_uint()
        names = ctypes.create_string_buffer(VIRG_OPS * VIRG_MAX_COLUMN_NAME)
        check(lib().virg_gpu_sql_compile(self.h, sql.encode(), ops, ctypes.byref(n), ctypes.byref(pc),
                                         names, ctypes.byref(tid)), "sql compile")
        raw = names.raw
        out = {}
        for k in range(n.value):
            if ops[k].op == 1:
                out[k] = raw[k * 16:(k + 1) * 16].split(b"\0", 1)[0].decode()
        return Compiled(ops, n.value, pc.value, tid.value, out)

    def __del__(self):
        try:
            if self.h:
                lib().virg_gpu_catalog_destroy(self.h)
        except Exception:
            pass
