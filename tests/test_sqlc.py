"""The product SQL front end emits exactly the reference's programs: every op
(opcode, p1-p3, p4) and result column name, compared with the reference's
parser+generator (oracle) on a fixed corpus and on seeded random queries."""
import ctypes
import struct

import pytest

import virginian_b200 as vb
from virginian_b200 import datagen, querygen, sql
from tests.helpers import CONFIG1, EXTRA, SUITE, build_oracle_db, col_types, config2

TYPES = col_types(datagen.SCHEMA_A)


@pytest.fixture(scope="module")
def both(oracle_mod):
    db, _ = build_oracle_db(oracle_mod, 10)
    cat = sql.Catalog()
    cat.add_table("test", datagen.SCHEMA_A)
    yield db, cat
    db.close()


def p4_bits(o):
    """The defined part of p4: the code generator sets p4.i or p4.f (4 bytes,
    src/sql/generate.c:125, :418); the upper half is uninitialised there."""
    return ctypes.cast(ctypes.pointer(o.p4), ctypes.POINTER(ctypes.c_uint32))[0]


def same_program(ref_vm, ref_names, mine):
    assert ref_vm.num_ops == mine.num_ops
    for k in range(mine.num_ops):
        a, b = ref_vm.stmt[k], mine.ops[k]
        assert (a.op, a.p1, a.p2, a.p3) == (b.op, b.p1, b.p2, b.p3), k
        if a.op != 1:  # ResultColumn p4 is a heap pointer in the reference
            assert p4_bits(a) == p4_bits(b), k
    assert ref_names == mine.names


FIXED = SUITE + EXTRA + [CONFIG1, config2(12.5, -3.0),
    "select col + 1 from test".replace("col", "uniformi"),
    "select uniformi - normali5 - normali20 as x from test",
    "select uniformi * 3 + 7 as q from test",
    "select 2.5 * 2.0 as k, id from test",
    "select 7 / 2 as k, id from test where 10 - 3 > uniformi",
    "select id from test where uniformi > 1 or normali5 > 1 and normali20 > 1",
    "select id from test where (uniformi > 1 and normali5 > 1)",
    "select id from test where (uniformi > 1 or normali5 > 1)",
    "select id from test where uniformi > 1 and (normali5 > 1 or (normali20 > 1 and uniformi < 50))",
    "SELECT id, uniformi FROM test WHERE uniformi>=50",
    "select uniformi a, normali5 as b from test",
]


@pytest.mark.parametrize("q", FIXED)
def test_fixed_corpus(both, q):
    db, cat = both
    vm, names = db.compile(q)
    same_program(vm, names, cat.compile(q))


def test_random_queries(both):
    db, cat = both
    qs = querygen.generate(400, seed=7)
    for q in qs:
        try:
            mine = cat.compile(q)
        except vb.VirgError:
            # too many ops/registers: the reference would overflow its fixed arrays
            continue
        vm, names = db.compile(q)
        same_program(vm, names, mine)


def test_errors_are_reported(both):
    _, cat = both
    with pytest.raises(vb.VirgError, match="parse error"):
        cat.compile("select from test")
    with pytest.raises(vb.VirgError, match="no column"):
        cat.compile("select nosuch from test")
    with pytest.raises(vb.VirgError, match="could not find table"):
        cat.compile("select id from nosuch")
    with pytest.raises(vb.VirgError, match="division by zero"):
        cat.compile("select 1 / 0 as z from test")
    with pytest.raises(vb.VirgError, match="parse error"):
        cat.compile("select id from test where (id = 1 or id = 2) and id < 5")
