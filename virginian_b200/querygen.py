"""Seeded random SELECT queries over the benchmark schema.

Each query is a random predicate tree of depth 1-4 over the int32/float32
columns, with constants drawn from each column's distribution, and 1-5
projected or computed result columns.  Queries stay inside what the
reference's front end and CPU VM handle to a defined result:
  - operands of a comparison or arithmetic op have the same type (the CPU VM
    asserts equal types, src/vm/virginia.c:52/:143; no Cast is emitted);
  - no integer division by a column or by zero (SIGFPE in the CPU VM);
  - no float constant-op-constant (the code generator folds it through int
    truncation, src/sql/generate.c:336-337);
  - result columns are distinct expressions with short aliases (the
    register reordering at src/sql/generate.c:651-674 assumes distinct
    registers, and names over 15 characters overrun a 16-byte buffer);
  - the program fits 32 ops and 16 registers, and no still-valid row reads a
    register its path skipped (checked by the caller with the VM decoder).
Parenthesised groups only end a condition list, as the grammar requires
(src/sql/sql.y:126-149), so a tree of depth d is a list whose last element is
a group of depth d-1.
"""
from __future__ import annotations

import random
from typing import List, Optional, Sequence, Tuple

INT_COLS = ["uniformi", "normali5", "normali20"]
FLOAT_COLS = ["uniformf", "normalf5", "normalf20"]

# approximate value ranges for drawing constants (column distributions)
INT_RANGE = {"uniformi": (0, 99), "normali5": (-12, 12), "normali20": (-45, 45)}
FLOAT_RANGE = {"uniformf": (0.0, 100.0), "normalf5": (-12.0, 12.0), "normalf20": (-45.0, 45.0)}


class QueryGen:
    def __init__(self, seed: int):
        self.r = random.Random(seed)

    def _const(self, col: str) -> str:
        if col in INT_RANGE:
            lo, hi = INT_RANGE[col]
            return str(self.r.randint(lo, hi))
        lo, hi = FLOAT_RANGE[col]
        return f"{self.r.uniform(lo, hi):.2f}"

    def _leaf(self) -> str:
        is_int = self.r.random() < 0.5
        cols = INT_COLS if is_int else FLOAT_COLS
        a = self.r.choice(cols)
        op = self.r.choice(["<", "<=", ">", ">=", "=", "!="] if is_int else ["<", "<=", ">", ">="])
        kind = self.r.random()
        if kind < 0.7:
            rhs = self._const(a)
        elif kind < 0.85:
            rhs = self.r.choice(cols)
        else:
            b = self.r.choice(cols)
            rhs = f"({b} + {self._const(b)})"
        return f"{a} {op} {rhs}"

    def _list(self, depth: int, min_leaves: int = 1) -> str:
        n = self.r.randint(min_leaves, 3)
        parts = [self._leaf() for _ in range(n)]
        out = parts[0]
        for p in parts[1:]:
            out += f" {self.r.choice(['and', 'or'])} {p}"
        if depth > 1:
            out += f" {self.r.choice(['and', 'or'])} ({self._list(depth - 1, 2)})"
        return out

    def _proj(self, i: int, used: set) -> str:
        for _ in range(20):
            kind = self.r.random()
            if kind < 0.45:
                e = self.r.choice(INT_COLS + FLOAT_COLS + ["id"])
            else:
                is_int = self.r.random() < 0.5
                cols = INT_COLS if is_int else FLOAT_COLS
                a = self.r.choice(cols)
                op = self.r.choice(["+", "-", "*", "/"])
                if op == "/" and is_int:
                    b = str(self.r.choice([2, 3, 5, 7, -4]))
                elif self.r.random() < 0.5:
                    b = self.r.choice(cols)
                else:
                    b = self._const(a) if not is_int else str(self.r.randint(1, 9))
                e = f"{a} {op} {b}"
            if e not in used:
                used.add(e)
                return f"{e} as c{i}"
        return f"id as c{i}" if "id" not in used else "uniformi as cz"

    def query(self, table: str = "test") -> str:
        depth = self.r.randint(1, 4)
        nproj = self.r.randint(1, 5)
        used: set = set()
        proj = ", ".join(self._proj(i, used) for i in range(nproj))
        return f"select {proj} from {table} where {self._list(depth)}"


def generate(n: int, seed: int, accept=None, table: str = "test") -> List[str]:
    """n queries; `accept(sql) -> bool` filters (e.g. compile + decoder checks)."""
    g = QueryGen(seed)
    out: List[str] = []
    tries = 0
    while len(out) < n:
        tries += 1
        if tries > n * 50:
            raise RuntimeError("query generator could not satisfy the filter")
        q = g.query(table)
        if accept is None or accept(q):
            out.append(q)
    return out
