"""virg_gpu_query_prealloc, the entry point that allocates nothing (its
scratch is a fixed device array), against the engine's virg_gpu_query on the
same rows: identical result streams on two calls in a row, the second on a
smaller segment, so a counter, status word or row count left over from the
first call would show, and both against the reference CPU VM (the oracle).
Collected last on purpose; it must also pass alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import virginian_b200 as vb
from virginian_b200 import _lib, datagen, sql
from tests.helpers import CONFIG1, config2

pytestmark = pytest.mark.gpu

TYPES = [t for _, t in datagen.SCHEMA_A]
MAX_ROWS = 1 << 26  # the entry point's stated limit

DTYPES = {vb.VIRG_INT: np.int32, vb.VIRG_FLOAT: np.float32, vb.VIRG_INT64: np.int64,
          vb.VIRG_DOUBLE: np.float64, vb.VIRG_CHAR: np.uint8}


def compile_program(text):
    cat = sql.Catalog()
    cat.add_table("test", datagen.SCHEMA_A)
    comp = cat.compile(text)
    return vb.Program(comp.op_list(), comp.pc, TYPES)


def host_columns(n, seed):
    return {name: datagen.column(name, n, seed=seed) for name in ["id"] + [c for c, _ in datagen.SCHEMA_A]}


def engine_result(engine, cols, prog):
    t = vb.Table(engine, TYPES)
    t.append(datagen.segments(cols, datagen.SCHEMA_A))
    r = t.query(prog)
    out = r.download()
    r.close()
    t.close()
    return out


def oracle_result(oracle_mod, cols, text):
    db = oracle_mod.OracleDB()
    try:
        db.create_table("test", datagen.SCHEMA_A)
        db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
        return db.query(text).columns
    finally:
        db.close()


def prealloc_result(torch, cols, prog, capacity, default_stream=False):
    """Runs the no-allocation entry point on device copies of `cols`; the
    caller (this test) owns every device buffer.  default_stream passes a
    null stream (the legacy default stream)."""
    n = len(cols["id"])
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in cols.items()}
    seg = _lib.Segment()
    seg.rows = n
    seg.key = dev["id"].data_ptr()
    for c, (name, _) in enumerate(datagen.SCHEMA_A):
        seg.col[c] = dev[name].data_ptr()
    info = prog.info
    outs = [torch.empty(max(capacity, 1), dtype=getattr(torch, np.dtype(DTYPES[info.out_type[j]]).name),
                        device="cuda") for j in range(info.nout)]
    ptrs = (ctypes.c_void_p * max(1, info.nout))(*[o.data_ptr() for o in outs])
    rows = ctypes.c_uint64(0)
    stream = None if default_stream else ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ok = _lib.lib().virg_gpu_query_prealloc(prog.h, ctypes.byref(seg), ptrs, capacity, ctypes.byref(rows),
                                            stream)
    err = None if ok else _lib.lib().virg_gpu_last_error().decode()
    got = [o[:min(rows.value, capacity)].cpu().numpy() for o in outs]
    return ok, rows.value, got, err


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


@pytest.fixture(scope="module")
def engine():
    e = vb.Engine(0)
    yield e
    e.close()


def assert_same(got, want, what):
    assert len(got) == len(want), what
    for j, (g, w) in enumerate(zip(got, want)):
        assert g.shape == w.shape, f"{what}: column {j} has {g.shape[0]} rows, want {w.shape[0]}"
        assert g.tobytes() == w.tobytes(), f"{what}: column {j} differs"


def test_two_calls_in_a_row_match_engine(torch, engine, oracle_mod):
    big = host_columns(300_001, seed=21)
    small = host_columns(70_001, seed=22)
    q1 = config2(40.0, 15.0)
    q2 = CONFIG1
    p1, p2 = compile_program(q1), compile_program(q2)
    want1 = engine_result(engine, big, p1)
    want2 = engine_result(engine, small, p2)
    ok, n1, got1, err = prealloc_result(torch, big, p1, 300_001)
    assert ok, err
    assert n1 == want1[0].shape[0]
    assert_same(got1, want1, "first call")
    ok, n2, got2, err = prealloc_result(torch, small, p2, 70_001)
    assert ok, err
    assert n2 == want2[0].shape[0]
    assert_same(got2, want2, "second call")
    assert_same(got1, oracle_result(oracle_mod, big, q1), "first call against the oracle")
    assert_same(got2, oracle_result(oracle_mod, small, q2), "second call against the oracle")


def test_null_stream(torch, oracle_mod):
    cols = host_columns(120_000, seed=24)
    prog = compile_program(CONFIG1)
    ok, n, got, err = prealloc_result(torch, cols, prog, 120_000, default_stream=True)
    assert ok, err
    assert_same(got, oracle_result(oracle_mod, cols, CONFIG1), "null stream")


def test_refuses_more_rows_than_its_scratch(torch):
    prog = compile_program(CONFIG1)
    seg = _lib.Segment()
    seg.rows = MAX_ROWS + 1
    rows = ctypes.c_uint64(0)
    ptrs = (ctypes.c_void_p * 16)()
    ok = _lib.lib().virg_gpu_query_prealloc(prog.h, ctypes.byref(seg), ptrs, 0, ctypes.byref(rows), None)
    assert not ok
    assert "at most 67108864 rows" in _lib.lib().virg_gpu_last_error().decode()


def test_refuses_host_and_misaligned_columns(torch):
    """Columns outside the current device's memory, or not 16-byte aligned,
    are refused on the host before anything is launched."""
    n = 4096
    cols = host_columns(n, seed=25)
    prog = compile_program(CONFIG1)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in cols.items()}
    outs = [torch.empty(n, dtype=torch.int32, device="cuda") for _ in range(prog.info.nout)]
    rows = ctypes.c_uint64(0)

    def call(seg, out_ptrs):
        ptrs = (ctypes.c_void_p * max(1, len(out_ptrs)))(*out_ptrs)
        ok = _lib.lib().virg_gpu_query_prealloc(prog.h, ctypes.byref(seg), ptrs, n, ctypes.byref(rows), None)
        return ok, ("" if ok else _lib.lib().virg_gpu_last_error().decode())

    def segment(override=None):
        seg = _lib.Segment()
        seg.rows = n
        seg.key = dev["id"].data_ptr()
        for c, (name, _) in enumerate(datagen.SCHEMA_A):
            seg.col[c] = dev[name].data_ptr()
        if override:
            for c, p in override.items():
                seg.col[c] = p
        return seg

    good = [o.data_ptr() for o in outs]
    host = np.ascontiguousarray(cols["uniformi"])
    ci = [name for name, _ in datagen.SCHEMA_A].index("uniformi")
    ok, err = call(segment({ci: host.ctypes.data}), good)
    assert not ok and "current device's memory" in err, err
    ok, err = call(segment({ci: dev["uniformi"].data_ptr() + 4}), good)
    assert not ok and "16-byte aligned" in err, err
    host_out = np.empty(n, dtype=np.int32)
    ok, err = call(segment(), [host_out.ctypes.data] + good[1:])
    assert not ok and "result columns must be in the current device's memory" in err, err
    # the same call with its own buffers runs
    ok, err = call(segment(), good)
    assert ok, err


def test_small_capacity_reports_overflow(torch, engine):
    cols = host_columns(50_000, seed=23)
    prog = compile_program("SELECT id, uniformi FROM test WHERE uniformi > 10")
    want = engine_result(engine, cols, prog)
    need = want[0].shape[0]
    assert need > 100
    ok, n, got, err = prealloc_result(torch, cols, prog, 100)
    assert not ok and "buffers hold 100" in err
    assert n == need
    # the rows that fit are the first rows of the full result
    assert_same(got, [w[:100] for w in want], "truncated")
    # an overflowed call leaves nothing behind: the next call with room
    # returns the whole result
    ok, n, got, err = prealloc_result(torch, cols, prog, need)
    assert ok, err
    assert n == need
    assert_same(got, want, "after the overflow")
