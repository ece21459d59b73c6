"""Shared test helpers: query corpus, oracle databases, result comparison."""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from virginian_b200 import datagen

# the reference's 10-query suite (src/test/queries.h:1-13), on this schema
SUITE = [
    "select id, uniformi, normali5 from test where uniformi > 60 and normali5 < 0",
    "select id, uniformf, normalf5 from test where uniformf > 60.0 and normalf5 < 0.0",
    "select id, uniformi, normali5 from test where uniformi > -60 and normali5 < 5",
    "select id, uniformf, normalf5 from test where uniformf > -60.0 and normalf5 < 5.0",
    "select id, uniformi, normali20 from test where (normali20 + 40) > (uniformi - 10)",
    "select id, uniformf, normalf20 from test where (normalf20 + 40.0) > (uniformf - 10.0)",
    "select id, normali5, normali20 from test where normali5 * normali20 >= -5 and normali5 * normali20 <= 5",
    "select id, normalf5, normalf20 from test where normalf5 * normalf20 >= -5.0 and normalf5 * normalf20 <= 5.0",
    "select id, uniformi, normali5, normali20 from test where uniformi >= -1 and uniformi <= 1 or normali5 >= -1 and normali5 <= 1 or normali20 >= -1 and normali20 <= 1",
    "select id, uniformf, normalf5, normalf20 from test where uniformf >= -1.0 and uniformf <= 1.0 or normalf5 >= -1.0 and normalf5 <= 1.0 or normalf20 >= -1.0 and normalf20 <= 1.0",
]

# the plain CPU-runnable filter of the benchmark
CONFIG1 = "SELECT id, uniformi, normali5 FROM test WHERE uniformi > 60 AND normali5 < 0"


def config2(c: float, d: float) -> str:
    """Scan plus arithmetic; aliases keep result names within 15 characters
    (the reference's name printer overruns its 16-byte buffer otherwise,
    src/sql/node.c:55-99)."""
    return ("SELECT id, uniformf + normalf5 * 2.5 AS fsum, normali20 / 3 AS idiv, "
            f"uniformi - normali5 AS isub FROM test WHERE uniformf < {c:.6f} OR normalf20 > {d:.6f}")


EXTRA = [
    "select id from test",
    "select uniformi, uniformf from test where uniformi = 50",
    "select id, normali20 from test where normali20 != 0 and uniformi >= 95",
    "select id, uniformi from test where uniformi < 5 and (normali5 = 2 or normali5 = -3)",
    "select id, uniformi from test where uniformi < 5 or normali20 > 40 or normalf5 < -10.0",
    "select normalf20 * normalf5 - uniformf as m, id from test where normalf20 > 30.0",
    "select id, uniformi - normali5 - normali20 as r from test where uniformi > 90",
    "select uniformi * 3 + 7 as q, id from test where (uniformi > 20 and uniformi < 30)",
    "select id, normalf5 / 3.0 as dq from test where normalf5 > 9.0 or normalf5 < -9.0",
    "select id, uniformi from test where uniformi > 1000",
    "select id, uniformi from test where uniformi >= 0",
    "select id, uniformi + 5 * 20 as k from test where id < 3000",
    "select id, uniformi from test where id < 500 and (id >= 100 or id = 7)",
]


def build_oracle_db(oracle, n: int, seed: int = 0, schema=datagen.SCHEMA_A, name: str = "test"):
    cols = datagen.table(n, schema, seed)
    db = oracle.OracleDB()
    db.create_table(name, schema)
    db.insert(name, cols["id"], [cols[c] for c, _ in schema])
    return db, cols


def col_types(schema) -> List[int]:
    return [t for _, t in schema]


def assert_same_stream(got: Sequence[np.ndarray], want: Sequence[np.ndarray], what: str = ""):
    assert len(got) == len(want), f"{what}: {len(got)} columns vs {len(want)}"
    for j, (g, w) in enumerate(zip(got, want)):
        assert g.shape == w.shape, f"{what}: column {j} has {g.shape[0]} rows, oracle {w.shape[0]}"
        gb, wb = g.view(np.uint8), w.view(np.uint8)
        if not np.array_equal(gb, wb):
            bad = np.nonzero(g.view(f"u{g.itemsize}") != w.view(f"u{w.itemsize}"))[0]
            raise AssertionError(f"{what}: column {j} differs at {bad.size} rows, first {bad[:5]}: "
                                 f"{g[bad[:5]]} vs {w[bad[:5]]}")
