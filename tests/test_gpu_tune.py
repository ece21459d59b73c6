"""The persistent tuned-shape cache: a shape tuned by one engine is written
to the cache file and picked up by an engine created afterwards, which then
launches the query with it without tuning; lines of another build or device
are ignored."""
import os

import pytest

import virginian_b200 as vb
from virginian_b200 import datagen, sql
from tests.helpers import col_types, config2

pytestmark = pytest.mark.gpu

TYPES = col_types(datagen.SCHEMA_A)


def test_tuned_shape_persists(tmp_path, monkeypatch):
    path = tmp_path / "shapes.txt"
    path.write_text("other build|other device/1|some key\t512 16 2 1 1024 0\n")
    monkeypatch.setenv("VIRGINIAN_B200_TUNE_CACHE", str(path))
    cols = datagen.table(400_000, datagen.SCHEMA_A, seed=31)
    cat = sql.Catalog()
    cat.add_table("test", datagen.SCHEMA_A)
    c = cat.compile(config2(30.0, 20.0))
    with vb.Engine(0) as e1:
        t1 = vb.Table(e1, TYPES)
        t1.append(datagen.segments(cols, datagen.SCHEMA_A))
        p1 = vb.Program(c.op_list(), c.pc, TYPES)
        vb.tune(e1, p1, t1)
        r = t1.query(p1)
        want_rows = r.rows
        want = r.download()
        r.close()
        tuned = e1.last_launch()
        t1.close()
    lines = path.read_text().splitlines()
    assert len(lines) >= 2 and lines[0].startswith("other build|")
    fields = lines[-1].split("\t")[1].split()
    assert [int(x) for x in fields[:2]] == [tuned["threads"], tuned["stage_kb"]]
    # a new engine reads the file and launches the same query with the shape
    with vb.Engine(0) as e2:
        t2 = vb.Table(e2, TYPES)
        t2.append(datagen.segments(cols, datagen.SCHEMA_A))
        p2 = vb.Program(c.op_list(), c.pc, TYPES)
        r = t2.query(p2)
        assert r.rows == want_rows
        got = r.download()
        r.close()
        launch = e2.last_launch()
        assert (launch["threads"], launch["stage_kb"]) == (tuned["threads"], tuned["stage_kb"])
        assert all(a.tobytes() == b.tobytes() for a, b in zip(got, want))
        t2.close()
