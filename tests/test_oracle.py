"""The oracle (the reference's own CPU VM, built from its sources) against the
reference's known-answer tests, src/test/sql.cc."""
import numpy as np
import pytest

from tests.helpers import build_oracle_db

VIRG_INT = 0
OP_Table, OP_ResultColumn, OP_Parallel, OP_Integer = 0, 1, 2, 10

# src/test/sql.cc:14-37
CONDITIONS = [
    "select col0 from test where col0 < 9 and col0 >= 7 or col0 = 3",
    "select col0 from test where col0 >= 8 or col0 = 3 and col0 < 1",
    "select col0 from test where col0 = 8 and col0 = 8",
    "select col0 from test where col0 = 8 or col0 = 8",
    "select col0 from test where col0 = 2",
    "select col0 from test where (col0 = 2)",
    "select col0 from test where col0 < 5 and (col0 = 7 or col0 = 2)",
    "select col0 from test where col0 = 7 or col0 = 2 or col0 = 8",
    "select col0 from test where col0 < 5 and (col0 = 2 or col0 = 8 or col0 = 1)",
]
CONDITION_ROWS = [3, 2, 1, 1, 1, 1, 1, 3, 2]


def simpledb(oracle, n):
    """src/test/test.cc:26-54: table test(col0, col1, col2) = (i, i+1, i+2)."""
    db = oracle.OracleDB()
    db.create_table("test", [("col0", VIRG_INT), ("col1", VIRG_INT), ("col2", VIRG_INT)])
    x = np.arange(n, dtype=np.int32)
    db.insert("test", x, [x, x + 1, x + 2])
    return db


def test_condition_row_counts(oracle_mod):
    with simpledb(oracle_mod, 10) as db:
        for q, n in zip(CONDITIONS, CONDITION_ROWS):
            r = db.query(q)
            assert r.rows == n, q
        assert set(db.query(CONDITIONS[0]).columns[0]) == {3, 7, 8}
        assert set(db.query(CONDITIONS[1]).columns[0]) == {8, 9}


def test_expression_folding_and_names(oracle_mod):
    # src/test/sql.cc:129-155
    with simpledb(oracle_mod, 1) as db:
        vm, names = db.compile("select col0 + 5 * 20 from test")
        assert vm.stmt[0].op == OP_Table
        assert vm.stmt[1].op == OP_ResultColumn and names[1] == "(col0+(5*20))"
        assert vm.stmt[2].op == OP_Parallel
        assert vm.stmt[4].op == OP_Integer and vm.stmt[4].p2 == 100
        # sql.cc:157-223
        for mode in (0, 1):
            assert db.query("select col0 + 5 * 20 from test", mode=mode, threads=2).columns[0][0] == 100
        assert db.query("select col0 + 10 * (1 + 2) from test").columns[0][0] == 30


def test_columns_result_registers(oracle_mod):
    # src/test/sql.cc:355-412
    with simpledb(oracle_mod, 1) as db:
        vm, _ = db.compile("select col0, col1 from test")
        col0 = col1 = -1
        for k in range(1, vm.num_ops):
            o = vm.stmt[k]
            if o.op == 4:
                if o.p2 == 0:
                    col0 = o.p1
                if o.p2 == 1:
                    col1 = o.p1
            if o.op == 6:
                assert o.p1 == col0 and o.p2 == 2
        assert col0 < col1
        r = db.query("select col0, col1 from test")
        assert r.columns[0][0] == 0 and r.columns[1][0] == 1


def test_reader_drops_last_row(oracle_mod):
    # the reference reader returns VIRG_FAIL on the last row (src/reader/row.c:42-47)
    with simpledb(oracle_mod, 10) as db:
        n, getrows, _ = db.reader_walk("select col0 from test where col0 >= 5", 4, 16)
        assert getrows == 5 and n == 4


def test_single_is_ordered_and_multi_is_a_permutation(oracle_mod):
    db, cols = build_oracle_db(oracle_mod, 300_000)
    with db:
        q = "select id, uniformi, normali5 from test where uniformi > 60 and normali5 < 0"
        single = db.query(q)
        ids = single.columns[0]
        assert np.all(np.diff(ids) > 0)
        want = np.nonzero((cols["uniformi"] > 60) & (cols["normali5"] < 0))[0]
        assert np.array_equal(ids, want.astype(np.int32))
        multi = db.query(q, mode=1, threads=4)
        assert np.array_equal(np.sort(multi.columns[0]), ids)


def test_result_tablets_roll_over(oracle_mod):
    db, _ = build_oracle_db(oracle_mod, 600_000)
    with db:
        r = db.query("select id, uniformi from test")
        assert r.rows == 600_000
        assert len(r.tablet_rows) >= 2 and sum(r.tablet_rows) == 600_000


def test_group_must_end_condition_list(oracle_mod):
    # `( c OR rest )` is a whole condition list (sql.y:144-148): it cannot be
    # followed by AND, so the reference grammar rejects this query
    with simpledb(oracle_mod, 10) as db:
        with pytest.raises(ValueError):
            db.compile("select col0 from test where (col0 = 1 or col0 = 2) and col0 < 5")
        assert db.query("select col0 from test where col0 < 5 and (col0 = 1 or col0 = 2)").rows == 2


def test_hand_programs_and_or_not(oracle_mod):
    """The CPU VM on hand-assembled And / Or / Not programs equals an
    independent numpy evaluation (pins the oracle for opcodes the code
    generator never emits)."""
    from virginian_b200 import datagen
    from tests.helpers import HAND_PROGRAMS, assemble, hand_table
    from oracle.oracle import VirgOp
    cols = hand_table(20_000, seed=4)
    db = oracle_mod.OracleDB()
    with db:
        db.create_table("test", datagen.SCHEMA_A)
        db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
        for skel, body, sel, names in HAND_PROGRAMS:
            vm, _ = db.compile(skel)
            ops, _ = assemble([vm.stmt[k] for k in range(vm.num_ops)], body)
            vops = []
            for t in ops:
                o = VirgOp()
                o.op, o.p1, o.p2, o.p3, o.p4.i = t
                vops.append(o)
            got = db.query_ops(skel, vops).columns
            m = sel(cols)
            assert m.sum() > 0 and (~m).sum() > 0
            for g, name in zip(got, names):
                want = cols[name][m]
                assert np.array_equal(g.view(np.uint8), want.view(np.uint8)), (skel, body, name)
