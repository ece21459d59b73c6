"""Seeded synthetic tables with the benchmark schema.

Schema A (the 7-column benchmark table): key ``id`` int32 = 0..N-1 plus
``uniformi`` int32 U[0,100), ``normali5`` int32 round(N(0,5)), ``normali20``
int32 round(N(0,20)), ``uniformf`` float32 U[0,100), ``normalf5`` float32
N(0,5), ``normalf20`` float32 N(0,20).  Schema B adds ``uniforml`` int64
uniform over the full range and ``normald`` float64 N(0,1).

The reference generates its benchmark table with GSL's ranlxd2 seeded by
time(0) (db/generate.c:35-48), so its data cannot be reproduced; here every
column comes from numpy's counter-based Philox generator keyed by
(seed, table, column), so any slice of rows can be regenerated independently
and CPU and GPU paths see identical bytes.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import VIRG_DOUBLE, VIRG_FLOAT, VIRG_INT, VIRG_INT64

SCHEMA_A: List[Tuple[str, int]] = [
    ("uniformi", VIRG_INT), ("normali5", VIRG_INT), ("normali20", VIRG_INT),
    ("uniformf", VIRG_FLOAT), ("normalf5", VIRG_FLOAT), ("normalf20", VIRG_FLOAT),
]
SCHEMA_B: List[Tuple[str, int]] = SCHEMA_A + [("uniforml", VIRG_INT64), ("normald", VIRG_DOUBLE)]

# rows in one full tablet of these schemas as the reference lays them out
# (8 MB tablets, 704-byte header, key + 8-byte key pointer + fixed columns):
# measured from the reference host library for 1M rows of schema A
TABLET_ROWS_A = 232992


def _gen(seed: int, table: int, col: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(key=[seed & 0xFFFFFFFF, (table << 8) | col]))


def column(name: str, n: int, seed: int = 0, table: int = 0, start: int = 0) -> np.ndarray:
    """Rows [start, start+n) of one column; chunks are generated in blocks of
    2^20 rows so any slice regenerates the same bytes."""
    names = [c[0] for c in SCHEMA_B]
    if name == "id":
        return np.arange(start, start + n, dtype=np.int32)
    ci = names.index(name) + 1
    if n == 0:
        return _block(name, np.random.Generator(np.random.Philox(0)), 0)
    block = 1 << 20
    out = []
    b0, b1 = start // block, (start + n + block - 1) // block
    for b in range(b0, b1):
        g = np.random.Generator(np.random.Philox(key=[seed & 0xFFFFFFFF, (table << 8) | ci],
                                                 counter=[0, 0, 0, b]))
        out.append(_block(name, g, block))
    arr = np.concatenate(out) if len(out) > 1 else out[0]
    lo = start - b0 * block
    return np.ascontiguousarray(arr[lo:lo + n])


def _block(name: str, g: np.random.Generator, n: int) -> np.ndarray:
    if name == "uniformi":
        return g.integers(0, 100, size=n, dtype=np.int32)
    if name == "normali5":
        return np.rint(g.normal(0.0, 5.0, size=n)).astype(np.int32)
    if name == "normali20":
        return np.rint(g.normal(0.0, 20.0, size=n)).astype(np.int32)
    if name == "uniformf":
        return (g.random(size=n, dtype=np.float32) * np.float32(100.0)).astype(np.float32)
    if name == "normalf5":
        return (g.standard_normal(size=n, dtype=np.float32) * np.float32(5.0)).astype(np.float32)
    if name == "normalf20":
        return (g.standard_normal(size=n, dtype=np.float32) * np.float32(20.0)).astype(np.float32)
    if name == "uniforml":
        return g.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, size=n,
                          dtype=np.int64, endpoint=True)
    if name == "normald":
        return g.standard_normal(size=n)
    raise KeyError(name)


def table(n: int, schema: Sequence[Tuple[str, int]] = SCHEMA_A, seed: int = 0,
          table_no: int = 0) -> Dict[str, np.ndarray]:
    cols = {"id": column("id", n)}
    for name, _ in schema:
        cols[name] = column(name, n, seed, table_no)
    return cols


def segments(cols: Dict[str, np.ndarray], schema: Sequence[Tuple[str, int]],
             rows_per_segment: int = TABLET_ROWS_A) -> List[dict]:
    """Splits columns into tablet-sized segments for Table.append/query_host."""
    n = cols["id"].shape[0]
    out = []
    for s in range(0, max(n, 1), rows_per_segment):
        e = min(n, s + rows_per_segment)
        if e <= s:
            break
        out.append({"rows": e - s, "key": cols["id"][s:e],
                    "cols": [cols[name][s:e] for name, _ in schema]})
    return out
