"""Checker helper for the benchmark's parity lines: the reference CPU VM's
(virginia_single, src/vm/virginia.c) result streams on seeded synthetic
tables, reduced to digests so a worker process can hand them back cheaply.

Test infrastructure.  The benchmark runs these functions in worker processes
after its timed sections, only to check the results its GPU path produced
against the reference's; nothing here is timed or shipped.
"""
from __future__ import annotations

import hashlib
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, List, Sequence, Tuple

import numpy as np

Digest = Tuple[int, Tuple[str, ...]]


def digest(columns: Sequence[np.ndarray]) -> Digest:
    """Row count and the SHA-256 of each column's bytes, in order."""
    rows = int(columns[0].shape[0]) if len(columns) else 0
    return rows, tuple(hashlib.sha256(np.ascontiguousarray(c).view(np.uint8)).hexdigest() for c in columns)


def host_table(n: int, seed: int, table_no: int = 0, threads: int = 8, schema: str = "A") -> Dict[str, np.ndarray]:
    """The seeded table of n rows (virginian_b200.datagen), generated by
    column slices on a few threads (the generator releases the interpreter
    lock); the same bytes as datagen.table(n, schema, seed, table_no)."""
    from virginian_b200 import datagen
    sch = datagen.SCHEMA_A if schema == "A" else datagen.SCHEMA_B
    names = [c for c, _ in sch]
    piece = 1 << 23  # a multiple of the generator's 2^20-row blocks
    cols = {"id": np.arange(n, dtype=np.int32)}
    if n == 0:
        for nm in names:
            cols[nm] = datagen.column(nm, 0, seed, table_no)
        return cols
    with ThreadPoolExecutor(max(1, threads)) as ex:
        futs = {nm: [ex.submit(datagen.column, nm, min(piece, n - a), seed, table_no, a)
                     for a in range(0, n, piece)] for nm in names}
        for nm in names:
            parts = [f.result() for f in futs[nm]]
            cols[nm] = parts[0] if len(parts) == 1 else np.concatenate(parts)
    return cols


def table_digests(n: int, seed: int, table_no: int, queries: Sequence[str],
                  threads: int = 1) -> List[Digest]:
    """Builds table `test` (n seeded rows of the 7-column schema) in a fresh
    reference database and returns the digest of virginia_single's result
    stream for each query, in order."""
    from oracle import oracle
    from virginian_b200 import datagen
    cols = host_table(n, seed, table_no, threads)
    db = oracle.OracleDB()
    try:
        db.create_table("test", datagen.SCHEMA_A)
        if n:
            db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
        del cols
        return [digest(db.query(q, mode=0).columns) for q in queries]
    finally:
        db.close()


def table_digests_star(args) -> List[Digest]:
    return table_digests(*args)
