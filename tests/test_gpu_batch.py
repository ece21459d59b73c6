"""Batched persistent execution: many queries over tables of uneven size in
one launch give, for every query, the reference CPU VM's result stream; graph
replays and autotuned shapes give the same bytes."""
import numpy as np
import pytest

import virginian_b200 as vb
from virginian_b200 import datagen, querygen, sql
from tests.helpers import assert_same_stream, col_types

pytestmark = pytest.mark.gpu

TYPES = col_types(datagen.SCHEMA_A)
SIZES = [1, 100, 5000, 70_001, 250_000, 0, 2049, 131_072]


def accepted(cat):
    def ok(q):
        try:
            c = cat.compile(q)
            return not vb.Program(c.op_list(), c.pc, TYPES).maybe_undefined
        except vb.VirgError:
            return False
    return ok


@pytest.fixture(scope="module")
def setup(oracle_mod):
    eng = vb.Engine(0)
    db = oracle_mod.OracleDB()
    cat = sql.Catalog()
    tables, data = [], []
    for i, n in enumerate(SIZES):
        cols = datagen.table(n, datagen.SCHEMA_A, seed=100 + i)
        name = f"t{i}"
        db.create_table(name, datagen.SCHEMA_A)
        if n:
            db.insert(name, cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
        cat.add_table(name, datagen.SCHEMA_A)
        t = vb.Table(eng, TYPES)
        if n:
            t.append(datagen.segments(cols, datagen.SCHEMA_A, 40_000))
        tables.append(t)
    check = sql.Catalog()
    check.add_table("test", datagen.SCHEMA_A)
    qs = querygen.generate(48, seed=3, accept=accepted(check))
    rng = np.random.default_rng(4)
    work = [(q.replace(" from test ", f" from t{int(k)} "), int(k))
            for q, k in zip(qs, rng.integers(0, len(SIZES), size=len(qs)))]
    yield eng, db, cat, tables, work
    for t in tables:
        t.close()
    db.close()
    eng.close()


def build_batch(eng, cat, tables, work, autotune=False):
    b = vb.Batch(eng, autotune=autotune)
    for q, k in work:
        c = cat.compile(q)
        b.add(vb.Program(c.op_list(), c.pc, TYPES), tables[k])
    return b


def test_batch_matches_oracle(setup):
    eng, db, cat, tables, work = setup
    b = build_batch(eng, cat, tables, work)
    b.run(graph=False)
    b.wait()
    for slot, (q, k) in enumerate(work):
        assert_same_stream(b.download(slot), db.query(q).columns, q)
    b.close()


def test_graph_replay_and_per_query_agree(setup):
    eng, db, cat, tables, work = setup
    b = build_batch(eng, cat, tables, work)
    first = None
    for rep in range(3):
        b.run(graph=True)
        b.wait()
        got = [b.download(s) for s in range(len(work))]
        if first is None:
            first = got
        else:
            for s in range(len(work)):
                assert_same_stream(got[s], first[s], f"replay {rep} slot {s}")
    # one launch per query through the single-query path
    for s, (q, k) in enumerate(work):
        c = cat.compile(q)
        r = tables[k].query(vb.Program(c.op_list(), c.pc, TYPES))
        assert_same_stream(r.download(), first[s], q)
        r.close()
    b.close()


def test_autotuned_batch(setup):
    eng, db, cat, tables, work = setup
    b = build_batch(eng, cat, tables, work[:16], autotune=True)
    b.run(graph=True)
    b.wait()
    shape = b.shape()
    assert shape["threads"] in (128, 256, 320, 448, 512)
    for s, (q, k) in enumerate(work[:16]):
        assert_same_stream(b.download(s), db.query(q).columns, q)
    b.close()
    # the tuned shape is cached: a second batch of the same shape key reuses it
    b2 = build_batch(eng, cat, tables, work[:16], autotune=True)
    b2.run(graph=False)
    b2.wait()
    assert b2.shape()["threads"] == shape["threads"]
    b2.close()


@pytest.mark.parametrize("chunk_rows", [0, 1024])
def test_shared_scans_give_the_same_bytes(setup, chunk_rows):
    """Queries over one table claim its chunks interleaved (a shared scan);
    with it turned off each query's chunks are claimed in one run.  Both give
    every query the CPU VM's stream, also with small chunks (many chunks per
    table, so the interleaved claims cross many CTAs)."""
    eng, db, cat, tables, work = setup
    # every table scanned by several queries, empty ones included
    many = work + [(q, k) for q, k in work[:24]]
    results = {}
    try:
        eng.set_shape(chunk_rows=chunk_rows)
        for shared in (True, False):
            eng.set_shared_scan(shared)
            b = build_batch(eng, cat, tables, many)
            b.run(graph=False)
            b.wait()
            results[shared] = [b.download(s) for s in range(len(many))]
            b.close()
    finally:
        eng.set_shared_scan(False)
        eng.set_shape(0, 0, 0, 0)
    for s, (q, k) in enumerate(many):
        assert_same_stream(results[True][s], results[False][s], f"shared vs one run: {q}")
        assert_same_stream(results[True][s], db.query(q).columns, q)


WIDE_FILTER = ("select id from {t} where uniformi + normali5 > normali20 - uniformi and uniformi * normali5 < 1000 "
               "and normali20 * 2 > uniformi - 7 and normali5 + normali20 < uniformi * 3")
MANY_RESULTS = ("select uniformi + normali5 as a, uniformi - normali5 as b, uniformi * normali5 as c, "
                "normali20 + 1 as d, normali20 * 3 as e, uniformf * 2.0 as f from {t} where uniformi > 20")


@pytest.mark.parametrize("graph", [False, True])
def test_batch_with_a_wide_program_runs_as_two_launches(setup, graph):
    """A program whose filter needs more row-vector bytes than three 48 KB
    data buffers leave room for runs in a launch of its own (besides the
    launches of the narrow programs, split by sampled selectivity); every
    query still gets the CPU VM's stream."""
    eng, db, cat, tables, work = setup
    many = [(WIDE_FILTER.format(t="t4"), 4), (MANY_RESULTS.format(t="t4"), 4),
            (WIDE_FILTER.format(t="t6"), 6)] + work[:12] + [(MANY_RESULTS.format(t="t7"), 7)]
    b = build_batch(eng, cat, tables, many)
    b.run(graph=graph)
    b.wait()
    l0 = eng.launches
    b.run(graph=graph)
    b.wait()
    assert eng.launches - l0 in (2, 3)
    for slot, (q, k) in enumerate(many):
        assert_same_stream(b.download(slot), db.query(q).columns, q)
    b.close()
