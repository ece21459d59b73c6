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


def device_table(n: int, schema: Sequence[Tuple[str, int]] = SCHEMA_A, seed: int = 0,
                 seg_rows: int = TABLET_ROWS_A, device: str = "cuda"):
    """A table of n rows generated on the GPU with torch, for workloads too
    large to generate on the host (tens of GB): the same column
    distributions as column(), from torch's own seeded generator, so the
    bytes differ from the host generator's.  Returns (segments with device
    pointers, tensors to keep alive while they are used)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    cols = {"id": torch.arange(n, dtype=torch.int32, device=device)}
    for name, _ in schema:
        if name == "uniformi":
            t = torch.floor(torch.rand(n, generator=g, device=device) * 100).to(torch.int32)
        elif name in ("normali5", "normali20"):
            sd = 5.0 if name == "normali5" else 20.0
            t = torch.round(torch.randn(n, generator=g, device=device) * sd).to(torch.int32)
        elif name == "uniformf":
            t = torch.rand(n, generator=g, device=device) * 100.0
        elif name in ("normalf5", "normalf20"):
            t = torch.randn(n, generator=g, device=device) * (5.0 if name == "normalf5" else 20.0)
        elif name == "uniforml":
            t = torch.randint(-(2 ** 63), 2 ** 63 - 1, (n,), generator=g, device=device, dtype=torch.int64)
        elif name == "normald":
            t = torch.randn(n, generator=g, device=device, dtype=torch.float64)
        else:
            raise ValueError(name)
        cols[name] = t.contiguous()
    segs = []
    for a in range(0, n, seg_rows):
        b = min(n, a + seg_rows)
        segs.append({"rows": b - a, "key": cols["id"][a:].data_ptr(),
                     "cols": [cols[c][a:].data_ptr() for c, _ in schema]})
    return segs, list(cols.values())
