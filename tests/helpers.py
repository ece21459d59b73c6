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


# ---- hand-assembled programs: opcodes the code generator never emits ----
# virg_op_t numbering (src/virginian.h:166-193)
OP = dict(Table=0, ResultColumn=1, Parallel=2, Finish=3, Column=4, Rowid=5, Result=6, Converge=7, Invalid=8,
          Integer=10, Float=11, Le=12, Lt=13, Ge=14, Gt=15, Eq=16, Neq=17, Add=18, Sub=19, Mul=20, Div=21,
          And=22, Or=23, Not=24)
# column indices of the benchmark schema
U, N5, N20, UF, NF5, NF20 = 0, 1, 2, 3, 4, 5


def _b(name, p1=0, p2=0, p3=0, p4=0):
    return (OP[name], p1, p2, p3, p4)


# (skeleton query giving the result layout, data-parallel body starting at op
# 4, numpy selection over the columns, the result columns' names).  Jump
# targets are absolute op indices; a jump keeps validity when p4 = 1 and
# clears it when p4 = 0 (src/vm/virginia.c:48-130); Not jumps when its
# register is zero (src/vm/virginia.c:598-680).
HAND_PROGRAMS = [
    ("select id, uniformi from test where uniformi > 0",
     [_b("Column", 0, U), _b("Column", 1, N5), _b("And", 0, 1, 8, 1), _b("Invalid"),
      _b("Rowid", 2), _b("Column", 3, U), _b("Result", 2, 2), _b("Converge")],
     lambda c: (c["uniformi"] != 0) & (c["normali5"] != 0), ("id", "uniformi")),
    ("select id, uniformi from test where uniformi > 0",
     [_b("Column", 0, N5), _b("Column", 1, N20), _b("Or", 0, 1, 7, 0),
      _b("Rowid", 2), _b("Column", 3, N5), _b("Result", 2, 2), _b("Converge")],
     lambda c: (c["normali5"] == 0) & (c["normali20"] == 0), ("id", "normali5")),
    ("select id, uniformi from test where uniformi > 0",
     [_b("Column", 0, N5), _b("Not", 0, 0, 7, 1), _b("Invalid"),
      _b("Rowid", 2), _b("Column", 3, N20), _b("Result", 2, 2), _b("Converge")],
     lambda c: c["normali5"] == 0, ("id", "normali20")),
    ("select id, uniformi from test where uniformi > 0",
     [_b("Column", 0, U), _b("Integer", 1, 50), _b("Lt", 0, 1, 11, 1), _b("Column", 2, N5), _b("Column", 3, N20),
      _b("Or", 2, 3, 14, 0), _b("Not", 2, 0, 14, 1), _b("Column", 4, N5), _b("And", 4, 0, 14, 1), _b("Invalid"),
      _b("Rowid", 5), _b("Column", 6, U), _b("Result", 5, 2), _b("Converge")],
     lambda c: (((c["uniformi"] < 50) & (c["normali5"] != 0) & (c["uniformi"] != 0)) |
                ((c["uniformi"] >= 50) & (c["normali5"] == 0) & (c["normali20"] == 0))), ("id", "uniformi")),
    ("select id, uniformf from test where uniformf > 0.0",
     [_b("Column", 0, NF5), _b("Column", 1, UF), _b("And", 0, 1, 9, 1), _b("Not", 0, 0, 9, 0), _b("Invalid"),
      _b("Rowid", 2), _b("Column", 3, NF20), _b("Result", 2, 2), _b("Converge")],
     lambda c: (c["normalf5"] != 0) & (c["uniformf"] != 0), ("id", "normalf20")),
    ("select id, uniformf from test where uniformf > 0.0",
     [_b("Column", 0, NF5), _b("Column", 1, NF20), _b("Or", 0, 1, 8, 0),
      _b("Rowid", 2), _b("Column", 3, UF), _b("Result", 2, 2), _b("Converge")],
     lambda c: (c["normalf5"] == 0) & (c["normalf20"] == 0), ("id", "uniformf")),
]


def assemble(skeleton_ops, body):
    """The skeleton's Table, ResultColumn and Parallel ops, the body, then
    Finish; Parallel's p3 (where the serial VM resumes,
    src/vm/execute.c:80-90) points at the Finish."""
    head = list(skeleton_ops[:4])
    ops = [(o.op, o.p1, o.p2, o.p3, o.p4.i) for o in head] + list(body)
    ops.append(_b("Finish"))
    op, p1, p2, _, p4 = ops[3]
    assert op == OP["Parallel"]
    ops[3] = (op, p1, p2, len(ops) - 1, p4)
    return ops, 4


def hand_table(n: int, seed: int):
    """Columns with many zeros (so And, Or and Not take every branch):
    integer columns in [-2, 2], float columns from {0, -0, 1.5, -2, NaN}."""
    rng = np.random.default_rng(seed)
    cols = {"id": np.arange(n, dtype=np.int32)}
    fl = np.array([0.0, -0.0, 1.5, -2.0, np.nan], dtype=np.float32)
    for name, ty in datagen.SCHEMA_A:
        if ty == 2:
            cols[name] = rng.choice(fl, size=n).astype(np.float32)
        else:
            cols[name] = rng.integers(-2, 3, size=n).astype(np.int32)
    return cols
