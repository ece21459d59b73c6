"""Parity of the sm_100a VM with the reference single-core CPU VM (the
oracle) on the same seeded tables: result streams must be byte-identical and
in the same order."""
import numpy as np
import pytest

import virginian_b200 as vb
from virginian_b200 import datagen
from tests.helpers import (CONFIG1, EXTRA, HAND_PROGRAMS, SUITE, assemble, assert_same_stream, build_oracle_db,
                           col_types, config2, hand_table)

pytestmark = pytest.mark.gpu

TYPES_A = col_types(datagen.SCHEMA_A)
TYPES_B = col_types(datagen.SCHEMA_B)
N = 500_000


def section_start(vm):
    return next(k for k in range(vm.num_ops) if vm.stmt[k].op == 2) + 1


def program(db, sql, types):
    vm, _ = db.compile(sql)
    return vb.Program([vm.stmt[k] for k in range(vm.num_ops)], section_start(vm), types)


@pytest.fixture(scope="module")
def engine():
    e = vb.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def data_a(oracle_mod, engine):
    db, cols = build_oracle_db(oracle_mod, N, seed=11)
    t = vb.Table(engine, TYPES_A)
    t.append(datagen.segments(cols, datagen.SCHEMA_A))
    yield db, cols, t
    t.close()
    db.close()


def run_both(db, t, sql, types):
    # decode first: a program the decoder refuses may abort the reference CPU
    # VM (its type asserts, src/vm/virginia.c:52)
    p = program(db, sql, types)
    want = db.query(sql).columns
    r = t.query(p)
    got = r.download()
    r.close()
    return got, want, p


@pytest.mark.parametrize("sql", SUITE + EXTRA + [CONFIG1])
def test_resident_query_matches_oracle(data_a, sql, engine):
    db, _, t = data_a
    got, want, _ = run_both(db, t, sql, TYPES_A)
    assert_same_stream(got, want, sql)
    assert engine.device_error() == 0


@pytest.mark.parametrize("sel", [0.001, 0.01, 0.1, 0.5, 0.99])
def test_config2_selectivity_sweep(data_a, sel):
    db, cols, t = data_a
    # c and d from the empirical distributions so the OR of two independent
    # conditions, each keeping q of the rows, keeps 1 - (1 - q)^2 = sel
    q = 1 - (1 - sel) ** 0.5
    c = float(np.quantile(cols["uniformf"], q))
    d = float(np.quantile(cols["normalf20"], 1 - q))
    sql = config2(c, d)
    got, want, _ = run_both(db, t, sql, TYPES_A)
    assert_same_stream(got, want, sql)
    frac = got[0].shape[0] / N
    assert abs(frac - sel) < max(0.02, sel * 0.2)


@pytest.mark.parametrize("mode", [1, 2])
def test_full_modes_across_selectivity(data_a, engine, mode):
    """The gathering and dense full phases on the config-2 query at low,
    middle and high selectivity and on the query suite."""
    db, cols, t = data_a
    engine.set_shape(full_mode=mode)
    try:
        for sel in (0.01, 0.5, 0.99):
            q = 1 - (1 - sel) ** 0.5
            sql = config2(float(np.quantile(cols["uniformf"], q)), float(np.quantile(cols["normalf20"], 1 - q)))
            got, want, _ = run_both(db, t, sql, TYPES_A)
            assert_same_stream(got, want, f"mode={mode} {sql}")
        for sql in SUITE + EXTRA:
            got, want, _ = run_both(db, t, sql, TYPES_A)
            assert_same_stream(got, want, f"mode={mode} {sql}")
    finally:
        engine.set_shape(0, 0, 0, 0, 0, 0)


def test_query_host_end_to_end(data_a, engine):
    db, cols, _ = data_a
    p = program(db, CONFIG1, TYPES_A)
    got = engine.query_host(p, datagen.segments(cols, datagen.SCHEMA_A))
    assert_same_stream(got, db.query(CONFIG1).columns, "query_host")


def test_query_host_pieces_and_chunks(oracle_mod, engine):
    """End to end over 3.2M rows whose segments are partly back to back in
    host memory (merged into one copy per column) and partly separate
    arrays, one of them longer than a staging chunk (split across chunks),
    with a short segment and an empty one between them; called twice, so
    the second call reuses the engine's staging ring."""
    n = 3_200_000
    db, cols = build_oracle_db(oracle_mod, n, seed=12)
    try:
        segs = datagen.segments({k: v[:900_000] for k, v in cols.items()}, datagen.SCHEMA_A, 300_000)
        rest = {k: np.copy(v[900_000:]) for k, v in cols.items()}
        segs += datagen.segments({k: v[:7] for k, v in rest.items()}, datagen.SCHEMA_A, 7)
        segs.append({"rows": 0, "key": rest["id"][:0], "cols": [rest[c][:0] for c, _ in datagen.SCHEMA_A]})
        segs += datagen.segments({k: np.copy(v[7:]) for k, v in rest.items()}, datagen.SCHEMA_A, n)
        for sql in (CONFIG1, config2(30.0, 20.0)):
            p = program(db, sql, TYPES_A)
            want = db.query(sql).columns
            for _ in range(2):
                assert_same_stream(engine.query_host(p, segs), want, f"query_host pieces {sql}")
    finally:
        db.close()


# (compute threads, stage KB, buffers (0: as many as fit), CTAs per SM, chunk rows, full-phase mode)
@pytest.mark.parametrize("shape", [(320, 16, 0, 1, 1024, 0), (448, 32, 3, 1, 2048, 0), (256, 16, 0, 1, 8192, 0),
                                   (256, 32, 0, 1, 4096, 0), (256, 48, 2, 2, 4096, 0), (512, 24, 0, 1, 2048, 0),
                                   (512, 32, 4, 1, 8192, 0), (256, 8, 0, 1, 256, 0), (256, 24, 0, 1, 4096, 1),
                                   (320, 48, 0, 1, 8192, 1), (256, 8, 0, 1, 256, 1), (448, 16, 0, 1, 1024, 1),
                                   (128, 24, 0, 2, 4096, 0), (128, 32, 0, 2, 8192, 1), (256, 32, 0, 1, 4096, 2),
                                   (128, 24, 0, 2, 8192, 2), (256, 16, 0, 1, 1024, 2)])
def test_every_launch_shape(data_a, engine, shape):
    db, _, t = data_a
    engine.set_shape(*shape)
    try:
        for sql in (CONFIG1, config2(30.0, 20.0), SUITE[8], REFILTER[0]):
            try:
                got, want, _ = run_both(db, t, sql, TYPES_A)
            except vb.VirgError as e:
                if "shared memory" in str(e) or "cannot hold" in str(e):
                    continue  # this stage size cannot stage the program's columns
                raise
            assert_same_stream(got, want, f"{shape} {sql}")
        assert engine.last_launch()["threads"] == shape[0]
    finally:
        engine.set_shape(0, 0, 0, 0, 0, 0)


# result columns that reuse a register the filter computed (the code
# generator's expression reuse): the full phase runs the filter again
REFILTER = ["select uniformf + normalf5 as s, id from test where uniformf + normalf5 > 50.0",
            "select normali5 * normali20 as p from test where normali5 * normali20 > 10 and uniformi < 50",
            "select id, uniformi - normali5 as d, normalf20 from test where uniformi - normali5 < 20 or normalf20 > 30.0"]


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_filter_vectors_in_results(data_a, engine, mode):
    db, _, t = data_a
    engine.set_shape(full_mode=mode)
    try:
        for sql in REFILTER + ["select id, uniformi, normali5, normali20, uniformf, normalf5, normalf20 "
                               "from test where uniformi > 90"]:
            got, want, _ = run_both(db, t, sql, TYPES_A)
            assert_same_stream(got, want, sql)
    finally:
        engine.set_shape(0, 0, 0, 0, 0, 0)


@pytest.mark.parametrize("n", [0, 1, 63, 64, 65, 1023, 1024, 1025, 4097, 70_001])
def test_edge_sizes(oracle_mod, engine, n):
    db, cols = build_oracle_db(oracle_mod, n, seed=n)
    with db:
        t = vb.Table(engine, TYPES_A)
        if n:
            t.append(datagen.segments(cols, datagen.SCHEMA_A))
        for sql in (CONFIG1, "select id, uniformi from test", SUITE[9]):
            got, want, _ = run_both(db, t, sql, TYPES_A)
            assert_same_stream(got, want, f"n={n} {sql}")
        t.close()


def test_ragged_segments(oracle_mod, engine):
    n = 30_000
    db, cols = build_oracle_db(oracle_mod, n, seed=5)
    with db:
        t = vb.Table(engine, TYPES_A)
        cuts = [0, 1, 2, 100, 4096, 4097, 9000, 17_777, 30_000]
        for a, b in zip(cuts[:-1], cuts[1:]):
            t.append([{"rows": b - a, "key": cols["id"][a:b],
                       "cols": [cols[c][a:b] for c, _ in datagen.SCHEMA_A]}])
        for sql in (CONFIG1, SUITE[5], config2(10.0, 10.0)):
            got, want, _ = run_both(db, t, sql, TYPES_A)
            assert_same_stream(got, want, sql)
        t.close()


def test_int64_and_double_columns(oracle_mod, engine):
    n = 300_000
    db, cols = build_oracle_db(oracle_mod, n, seed=3, schema=datagen.SCHEMA_B)
    with db:
        t = vb.Table(engine, TYPES_B)
        t.append(datagen.segments(cols, datagen.SCHEMA_B, 161_000))
        for sql in ["select id, uniforml, normald from test where normali20 > 15 and uniformf < 50.0",
                    "select normald * normald - normald / normald as dd, id from test where normald > normald * normald",
                    "select uniforml + uniforml as l2, uniforml * uniforml as l3 from test where uniforml < uniforml - uniforml",
                    "select id, normald from test where normald >= normald + normald or uniformi = 3",
                    # 36 result bytes per row: read from the staged tile in place
                    "select id, uniforml, normald, uniformi, uniformf, normalf5, normalf20 from test "
                    "where normali20 > 10 or uniformf < 5.0"]:
            for mode in (0, 1, 2):
                engine.set_shape(full_mode=mode)
                try:
                    got, want, _ = run_both(db, t, sql, TYPES_B)
                finally:
                    engine.set_shape(0, 0, 0, 0, 0, 0)
                assert_same_stream(got, want, f"mode={mode} {sql}")
        t.close()


def test_float_edge_values(oracle_mod, engine):
    """Signed zeros, subnormals, infinities and NaN through compares and
    arithmetic (no flush-to-zero, IEEE division)."""
    specials = np.array([0.0, -0.0, 1e-45, -1e-45, 1.17549435e-38, 3.4e38, -3.4e38, np.inf, -np.inf,
                         np.nan, 1.0, -1.0, 0.1, 1e-30], dtype=np.float32)
    n = 4096
    rng = np.random.default_rng(9)
    cols = {"id": np.arange(n, dtype=np.int32)}
    for name, ty in datagen.SCHEMA_A:
        if ty == vb.VIRG_FLOAT:
            cols[name] = rng.choice(specials, size=n).astype(np.float32)
        else:
            # no zero: the reference CPU VM evaluates result expressions of
            # rows already filtered out too, and an integer divide by zero
            # traps it
            cols[name] = rng.choice(np.array([-3, -2, -1, 1, 2, 3], dtype=np.int32), size=n)
    db = oracle_mod.OracleDB()
    with db:
        db.create_table("test", datagen.SCHEMA_A)
        db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
        t = vb.Table(engine, TYPES_A)
        t.append(datagen.segments(cols, datagen.SCHEMA_A))
        for sql in ["select id, uniformf / normalf5 as q, normalf20 * uniformf as m from test where uniformf >= normalf5 or normalf20 != normalf20",
                    "select uniformf - normalf5 as s, normalf20 + normalf20 as a from test where uniformf = 0.0 or normalf5 < 0.0",
                    "select id, uniformi / normali5 as iq from test where normali5 > 0",
                    "select normali5 * normali20 - uniformi as z from test"]:
            got, want, _ = run_both(db, t, sql, TYPES_A)
            assert_same_stream(got, want, sql)
        t.close()


@pytest.mark.parametrize("per_chunk", [1, 2, 7])
def test_streamed_matches_oracle(oracle_mod, engine, per_chunk):
    """Host-resident tablets streamed through the staging ring, chunk by chunk,
    continue one ordered result stream."""
    n = 700_001
    db, cols = build_oracle_db(oracle_mod, n, seed=17, schema=datagen.SCHEMA_B)
    with db:
        segs = datagen.segments(cols, datagen.SCHEMA_B, 100_000)
        # ragged: an empty and a tiny segment in the middle
        segs.insert(3, {"rows": 0, "key": cols["id"][:0], "cols": [cols[c][:0] for c, _ in datagen.SCHEMA_B]})
        for sql in ["select id, uniforml, normald from test where normali20 > 15 and uniformf < 50.0",
                    "select id from test where uniformi >= 0",
                    "select id, uniformi from test where uniformi > 1000"]:
            p = program(db, sql, TYPES_B)
            r, stats = vb.query_streamed(engine, p, segs, per_chunk)
            assert_same_stream(r.download(), db.query(sql).columns, f"{per_chunk} {sql}")
            assert stats["h2d_bytes"] == n * p.info.load_bytes_per_row
            r.close()


@pytest.mark.parametrize("k", range(len(HAND_PROGRAMS)))
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_hand_programs_and_or_not(oracle_mod, engine, k, mode):
    """Hand-assembled programs with And, Or and Not (which the code
    generator never emits) on both VMs, over a table with many zeros, NaN and
    signed zeros in its columns."""
    from oracle.oracle import VirgOp
    skel, body, _, _ = HAND_PROGRAMS[k]
    cols = hand_table(300_001, seed=6)
    db = oracle_mod.OracleDB()
    with db:
        db.create_table("test", datagen.SCHEMA_A)
        db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
        vm, _ = db.compile(skel)
        ops, pc = assemble([vm.stmt[j] for j in range(vm.num_ops)], body)
        vops = []
        for t in ops:
            o = VirgOp()
            o.op, o.p1, o.p2, o.p3, o.p4.i = t
            vops.append(o)
        want = db.query_ops(skel, vops).columns
        t = vb.Table(engine, TYPES_A)
        t.append(datagen.segments(cols, datagen.SCHEMA_A))
        engine.set_shape(full_mode=mode)
        try:
            r = t.query(vb.Program(ops, pc, TYPES_A))
            got = r.download()
            r.close()
        finally:
            engine.set_shape(0, 0, 0, 0, 0, 0)
            t.close()
        assert_same_stream(got, want, f"hand program {k}")


def test_config1_at_one_million_rows(oracle_mod, engine):
    """The plain CPU-runnable filter at its stated size: 1,000,000 rows."""
    db, cols = build_oracle_db(oracle_mod, 1_000_000, seed=21)
    with db:
        t = vb.Table(engine, TYPES_A)
        t.append(datagen.segments(cols, datagen.SCHEMA_A))
        got, want, _ = run_both(db, t, CONFIG1, TYPES_A)
        assert_same_stream(got, want, "config 1, 1M rows")
        assert len(want[0]) > 100_000
        t.close()
