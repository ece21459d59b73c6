"""Serving loop (continuous batching): queries submitted while others run are
folded into the running persistent kernel; every query's result stream is
the same as the query run alone, and the same as the reference CPU VM's.
Short result estimates are admitted again with their exact size, and an
idle loop ends its kernel session and starts a new one for later queries."""
import time

import numpy as np
import pytest

import virginian_b200 as vb
from virginian_b200 import datagen, querygen, sql
from tests.helpers import assert_same_stream, col_types

pytestmark = pytest.mark.gpu

TYPES = col_types(datagen.SCHEMA_A)
SIZES = [250_000, 0, 1, 70_001, 1_100_000, 5000, 131_072]


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
    tables = []
    for i, n in enumerate(SIZES):
        cols = datagen.table(n, datagen.SCHEMA_A, seed=300 + i)
        name = f"t{i}"
        db.create_table(name, datagen.SCHEMA_A)
        if n:
            db.insert(name, cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
        cat.add_table(name, datagen.SCHEMA_A)
        t = vb.Table(eng, TYPES)
        if n:
            t.append(datagen.segments(cols, datagen.SCHEMA_A, 60_000))
        tables.append(t)
    check = sql.Catalog()
    check.add_table("test", datagen.SCHEMA_A)
    qs = querygen.generate(40, seed=11, accept=accepted(check))
    rng = np.random.default_rng(12)
    work = []
    for q, k in zip(qs, rng.integers(0, len(SIZES), size=len(qs))):
        q = q.replace(" from test ", f" from t{int(k)} ")
        c = cat.compile(q)
        work.append((q, int(k), vb.Program(c.op_list(), c.pc, TYPES)))
    # each query alone: one launch, one result
    alone = []
    for q, k, p in work:
        r = tables[k].query(p)
        alone.append(r.download())
        r.close()
    yield eng, db, tables, work, alone
    for t in tables:
        t.close()
    db.close()
    eng.close()


def test_mix_equals_alone_and_oracle(setup):
    eng, db, tables, work, alone = setup
    s = vb.Serve(eng, result_budget_bytes=1 << 30)
    try:
        tickets = []
        # arrivals in bursts while earlier queries are on the GPU
        for i, (q, k, p) in enumerate(work):
            tickets.append(s.submit(p, tables[k]))
            if i % 7 == 6:
                time.sleep(0.002)
        for t, (q, k, p), want in zip(tickets, work, alone):
            got = s.download(t)
            assert_same_stream(got, want, f"mix vs alone: {q}")
            assert_same_stream(got, db.query(q).columns, f"mix vs oracle: {q}")
            s.release(t)
        st = s.stats()
        assert st["admitted"] == len(work)
        assert st["device_error"] == 0
        assert st["inflight"] == 0 and st["pending"] == 0 and st["arena_used"] == 0
    finally:
        s.close()


def test_single_queries_of_other_shapes_beside_a_session(setup):
    """Single queries of other launch shapes (other shared-memory sizes of the
    same kernel) launched from this thread while the serving thread starts
    sessions: neither side's launch may fail, and every result stays the
    query's own."""
    eng, db, tables, work, alone = setup
    s = vb.Serve(eng, result_budget_bytes=1 << 30, idle_us=1000)
    shapes = [(256, 24, 2, 1), (256, 48, 3, 1), (256, 32, 0, 1), (0, 0, 0, 0)]
    try:
        for rnd in range(3):
            tickets = []
            for i, (q, k, p) in enumerate(work):
                tickets.append(s.submit(p, tables[k]))
                eng.set_shape(*shapes[i % len(shapes)])
                try:
                    r = tables[k].query(p)
                    got = r.download()
                    r.close()
                finally:
                    eng.set_shape(0, 0, 0, 0)
                assert_same_stream(got, alone[i], f"single beside a session: {q}")
                if i % 5 == 4:
                    time.sleep(0.003)  # let the session go idle and restart
            for t, (q, k, p), want in zip(tickets, work, alone):
                assert_same_stream(s.download(t), want, f"session beside singles: {q}")
                s.release(t)
        st = s.stats()
        assert st["device_error"] == 0 and st["restarts"] == 0
    finally:
        s.close()


def test_short_estimates_are_admitted_again(setup):
    eng, db, tables, work, alone = setup
    s = vb.Serve(eng, result_budget_bytes=256 << 20)
    try:
        tickets = [s.submit(p, tables[k], estimated_rows=1) for q, k, p in work]
        readmits = 0
        for t, want, (q, k, p) in zip(tickets, alone, work):
            got = s.download(t)
            readmits += s.poll(t)["readmits"]
            assert_same_stream(got, want, f"readmitted: {q}")
            s.release(t)
        assert readmits > 0
        assert s.stats()["readmitted"] == readmits
    finally:
        s.close()


def test_idle_loop_restarts_its_session(setup):
    eng, db, tables, work, alone = setup
    s = vb.Serve(eng, result_budget_bytes=256 << 20, idle_us=1000)
    try:
        for rnd in range(3):
            tickets = [s.submit(p, tables[k]) for q, k, p in work[rnd * 5:rnd * 5 + 5]]
            for t, want in zip(tickets, alone[rnd * 5:rnd * 5 + 5]):
                assert_same_stream(s.download(t), want, f"round {rnd}")
                s.release(t)
            time.sleep(0.02)
        assert s.stats()["sessions"] >= 3
    finally:
        s.close()


def test_session_rollover_keeps_results(setup):
    """A session takes at most max_queries queries; later ones run in the
    next session."""
    eng, db, tables, work, alone = setup
    s = vb.Serve(eng, result_budget_bytes=1 << 30, max_queries=8)
    try:
        tickets = [s.submit(p, tables[k]) for q, k, p in work]
        for t, want, (q, k, p) in zip(tickets, alone, work):
            assert_same_stream(s.download(t), want, f"rollover: {q}")
            s.release(t)
        assert s.stats()["sessions"] >= len(work) // 8
    finally:
        s.close()


def test_rejects_program_beyond_layout(setup):
    eng, db, tables, work, alone = setup
    s = vb.Serve(eng, result_budget_bytes=64 << 20, max_load_bytes_per_row=4)
    try:
        wide = next(p for q, k, p in work if p.info.load_bytes_per_row > 4)
        with pytest.raises(vb.VirgError, match="serving layout"):
            s.submit(wide, tables[0])
    finally:
        s.close()


def test_bounded_wait_ends_an_idle_session(setup):
    """A session kernel whose producer waits for the doorbell longer than the
    session's wait limit stops by itself and reports a stage-wait timeout
    (no fault, no hang); the loop notices, keeps finished results and runs
    later queries in a new session."""
    eng, db, tables, work, alone = setup
    s = vb.Serve(eng, result_budget_bytes=256 << 20, idle_us=2_000_000, wait_limit_ms=5)
    try:
        q, k, p = work[0]
        t = s.submit(p, tables[k])
        assert_same_stream(s.download(t), alone[0], "before the timeout")
        s.release(t)
        # no submissions for far longer than the wait limit
        time.sleep(0.3)
        st = s.stats()
        assert st["device_error"] == 2, st   # DE_STAGE_TIMEOUT
        assert st["restarts"] >= 1, st
        for i in range(1, 4):
            q, k, p = work[i]
            t = s.submit(p, tables[k])
            assert_same_stream(s.download(t), alone[i], "after the timeout")
            s.release(t)
        assert s.stats()["sessions"] >= 2
    finally:
        s.close()


def test_result_larger_than_budget_fails_cleanly(setup):
    """A query admitted with a short estimate whose exact result needs more
    memory than the whole result budget fails with an error (it cannot be
    admitted again), and the loop goes on serving other queries."""
    eng, db, tables, work, alone = setup
    big = max(range(len(work)), key=lambda i: len(alone[i][0]) * work[i][2].info.out_bytes_per_row)
    need = len(alone[big][0]) * work[big][2].info.out_bytes_per_row
    assert need > 64 << 10
    s = vb.Serve(eng, result_budget_bytes=32 << 10)
    try:
        q, k, p = work[big]
        t = s.submit(p, tables[k], estimated_rows=1)
        with pytest.raises(vb.VirgError, match="result budget"):
            s.wait(t, timeout_s=60)
        s.release(t)
        small = min(range(len(work)), key=lambda i: len(alone[i][0]) * work[i][2].info.out_bytes_per_row)
        assert len(alone[small][0]) * work[small][2].info.out_bytes_per_row < 8 << 10
        q, k, p = work[small]
        t = s.submit(p, tables[k], estimated_rows=max(1, len(alone[small][0])))
        assert_same_stream(s.download(t), alone[small], "after the rejected query")
        s.release(t)
    finally:
        s.close()


def test_sample_estimates_track_selectivity(oracle_mod):
    """The host row sample behind serving reservations: the estimate of a
    filter's rows stays within a few percent of the table's actual share,
    across selectivities, and a submission without a caller's estimate is
    sized from it."""
    import numpy as np
    from tests.helpers import config2
    n = 2_000_000
    cols = datagen.table(n, datagen.SCHEMA_A, seed=61)
    types = [t for _, t in datagen.SCHEMA_A]
    cat = sql.Catalog()
    cat.add_table("test", datagen.SCHEMA_A)
    with vb.Engine(0) as eng:
        t = vb.Table(eng, types)
        t.append(datagen.segments(cols, datagen.SCHEMA_A, 100_000))
        for c, d in ((1.0, 60.0), (30.0, 20.0), (90.0, -30.0)):
            comp = cat.compile(config2(c, d))
            p = vb.Program(comp.op_list(), comp.pc, types)
            want = int(((cols["uniformf"] < c) | (cols["normalf20"] > d)).sum())
            est = t.estimate(p)
            assert abs(est - want) <= 0.05 * n, (c, d, est, want)
        srv = vb.Serve(eng, result_budget_bytes=1 << 30)
        comp = cat.compile(config2(30.0, 20.0))
        p = vb.Program(comp.op_list(), comp.pc, types)
        tk = srv.submit(p, t)
        st = srv.wait(tk, timeout_s=60)
        assert st["rows"] == int(((cols["uniformf"] < 30.0) | (cols["normalf20"] > 20.0)).sum())
        assert srv.stats()["sampled"] >= 1
        srv.release(tk)
        srv.close()
        t.close()
