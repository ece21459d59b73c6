"""Tablet ingest: a table written to a Virginian database file by the
unmodified reference host library (virg_close writes every tablet,
src/db/close.c:20-50) is read straight into a resident table; the rows, and
query results over them, equal the same rows appended from host arrays.
Runs in a child process so the reference host library and this repository's
library share nothing else."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import ctypes, os, sys
import numpy as np
sys.path.insert(0, ROOT)
import virginian_b200 as vb
from virginian_b200 import _lib, datagen, sql
_lib.lib()                                   # the GPU VM first, RTLD_GLOBAL
from oracle import oracle as O
from tests.helpers import CONFIG1, config2, assert_same_stream
n = int(sys.argv[1])
cols = datagen.table(n, datagen.SCHEMA_A, seed=77)
db = O.OracleDB(path=O.HOST_LIB, mode=ctypes.RTLD_GLOBAL)
db.create_table("test", datagen.SCHEMA_A)
db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
path = db.close_keep()
types = [t for _, t in datagen.SCHEMA_A]
cat = sql.Catalog()
cat.add_table("test", datagen.SCHEMA_A)
try:
    with vb.Engine(0) as eng:
        t1 = vb.Table(eng, types)
        got_rows = t1.load_db(path, "test")
        assert got_rows == n, (got_rows, n)
        t2 = vb.Table(eng, types)
        t2.append(datagen.segments(cols, datagen.SCHEMA_A))
        for q in (CONFIG1, config2(20.0, 15.0), "select id, uniformi, normalf20 from test"):
            c = cat.compile(q)
            p = vb.Program(c.op_list(), c.pc, types)
            r1, r2 = t1.query(p), t2.query(p)
            a, b = r1.download(), r2.download()
            r1.close(); r2.close()
            assert_same_stream(a, b, q)
        keep = (cols["uniformi"] > 60) & (cols["normali5"] < 0)
        c = cat.compile(CONFIG1)
        r = t1.query(vb.Program(c.op_list(), c.pc, types))
        assert np.array_equal(r.download()[0], cols["id"][keep])
        r.close()
        t1.close(); t2.close()
finally:
    os.unlink(path)
    os.rmdir(os.path.dirname(path))
print("OK", n)
"""


@pytest.mark.parametrize("n", [1, 600_000])
def test_load_db_equals_appended_rows(n):
    code = "ROOT = %r\n" % ROOT + SCRIPT
    out = subprocess.run([sys.executable, "-c", code, str(n)], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert "OK" in out.stdout
