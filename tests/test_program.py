"""Host-side decoder of the data-parallel section (no GPU): accepts every
program the reference code generator emits for the test corpus, and refuses
the programs the reference CPU VM cannot run to a defined result."""
import numpy as np
import pytest

import virginian_b200 as vb
from virginian_b200 import datagen
from tests.helpers import CONFIG1, EXTRA, SUITE, build_oracle_db, col_types, config2

TYPES = col_types(datagen.SCHEMA_A)
OPS = {"Column": 4, "Rowid": 5, "Result": 6, "Converge": 7, "Invalid": 8, "Cast": 9,
       "Integer": 10, "Float": 11, "Le": 12, "Lt": 13, "Ge": 14, "Gt": 15, "Eq": 16,
       "Neq": 17, "Add": 18, "Sub": 19, "Mul": 20, "Div": 21, "Not": 24, "Table": 0}


@pytest.fixture(scope="module")
def db(oracle_mod):
    d, _ = build_oracle_db(oracle_mod, 100)
    yield d
    d.close()


def section_start(vm):
    return next(k for k in range(vm.num_ops) if vm.stmt[k].op == 2) + 1


def test_corpus_decodes(db):
    for q in SUITE + EXTRA + [CONFIG1, config2(1.0, 40.0)]:
        vm, _ = db.compile(q)
        p = vb.Program([vm.stmt[k] for k in range(vm.num_ops)], section_start(vm), TYPES)
        assert p.info.nout >= 1
        assert not p.maybe_undefined, q


def test_config1_program_shape(db):
    vm, _ = db.compile(CONFIG1)
    p = vb.Program([vm.stmt[k] for k in range(vm.num_ops)], section_start(vm), TYPES)
    info = p.info
    # id, uniformi, normali5: 12 bytes read per row, 12 written per result row
    assert info.nload == 3 and info.load_bytes_per_row == 12
    assert info.nout == 3 and info.out_bytes_per_row == 12
    # two compares and the Invalid + Result survive; loads and constants fold away
    assert info.nuops == 4


def test_config2_program_shape(db):
    vm, _ = db.compile(config2(50.0, 10.0))
    p = vb.Program([vm.stmt[k] for k in range(vm.num_ops)], section_start(vm), TYPES)
    assert p.info.load_bytes_per_row == 28
    assert p.info.out_bytes_per_row == 16


def prog(ops, pc=1):
    full = [(OPS["Table"], 0, 0, 0)] + ops
    return vb.Program(full, pc, TYPES)


def test_rejects_cast():
    with pytest.raises(vb.VirgError, match="Cast"):
        prog([(OPS["Column"], 0, 0, 0), (OPS["Cast"], 2, 0, 0), (OPS["Result"], 0, 1, 0),
              (OPS["Converge"], 0, 0, 0)])


def test_rejects_backward_jump():
    with pytest.raises(vb.VirgError, match="forward"):
        prog([(OPS["Column"], 0, 0, 0), (OPS["Integer"], 1, 5, 0), (OPS["Lt"], 0, 1, 1, 0),
              (OPS["Result"], 0, 1, 0), (OPS["Converge"], 0, 0, 0)])


def test_rejects_mixed_types():
    # uniformi (int) compared with uniformf (float): the CPU VM asserts
    with pytest.raises(vb.VirgError, match="types differ"):
        prog([(OPS["Column"], 0, 0, 0), (OPS["Column"], 1, 3, 0), (OPS["Lt"], 0, 1, 5, 0),
              (OPS["Result"], 0, 1, 0), (OPS["Converge"], 0, 0, 0)])


def test_rejects_missing_converge_and_result():
    with pytest.raises(vb.VirgError, match="Converge"):
        prog([(OPS["Column"], 0, 0, 0), (OPS["Result"], 0, 1, 0)])
    with pytest.raises(vb.VirgError, match="Result"):
        prog([(OPS["Column"], 0, 0, 0), (OPS["Converge"], 0, 0, 0)])


def test_rejects_serial_op_in_section():
    with pytest.raises(vb.VirgError, match="not a data-parallel op"):
        prog([(OPS["Column"], 0, 0, 0), (OPS["Table"], 0, 0, 0), (OPS["Result"], 0, 1, 0),
              (OPS["Converge"], 0, 0, 0)])


def test_rejects_unset_register_and_bad_column():
    with pytest.raises(vb.VirgError, match="before it is set"):
        prog([(OPS["Column"], 0, 0, 0), (OPS["Lt"], 0, 3, 4, 0), (OPS["Result"], 0, 1, 0),
              (OPS["Converge"], 0, 0, 0)])
    with pytest.raises(vb.VirgError, match="not in table"):
        prog([(OPS["Column"], 0, 9, 0), (OPS["Result"], 0, 1, 0), (OPS["Converge"], 0, 0, 0)])


def test_maybe_undefined_flag():
    # r2 = normali5 * 2 is computed only on the OR branch, then read by every
    # valid row: rows that took the first branch read a register their path
    # never set (stale in the reference CPU VM)
    ops = [(OPS["Column"], 0, 0, 0), (OPS["Integer"], 1, 60, 0), (OPS["Gt"], 0, 1, 9, 1),
           (OPS["Column"], 3, 1, 0), (OPS["Integer"], 4, 2, 0), (OPS["Mul"], 2, 3, 4),
           (OPS["Lt"], 2, 4, 9, 1), (OPS["Invalid"], 0, 0, 0),
           (OPS["Result"], 2, 1, 0), (OPS["Converge"], 0, 0, 0)]
    p = vb.Program([(OPS["Table"], 0, 0, 0)] + ops, 1, TYPES)
    assert p.maybe_undefined
    # the same program with the first jump invalidating (p4 = 0) is well defined
    ops[2] = (OPS["Gt"], 0, 1, 9, 0)
    assert not vb.Program([(OPS["Table"], 0, 0, 0)] + ops, 1, TYPES).maybe_undefined
