"""The drop-in virg_vm_gpu inside the unmodified reference host library
(stock virginian.h, real CUDA runtime): virg_query with use_gpu must build the
same result-tablet chain as the single-core CPU VM, tablet by tablet."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, ROOT)
from virginian_b200 import _lib, datagen
_lib.lib()                                   # GPU VM first, RTLD_GLOBAL
from oracle import oracle as O
from tests.helpers import SUITE, CONFIG1, EXTRA, config2, assert_same_stream
db = O.OracleDB(path=O.HOST_LIB, mode=ctypes.RTLD_GLOBAL)
n = int(sys.argv[1])
cols = datagen.table(n, datagen.SCHEMA_A, seed=21)
db.create_table("test", datagen.SCHEMA_A)
db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
# the last query keeps every row of 28 bytes: several result tablets roll over
WIDE = "select id, uniformi, normali5, normali20, uniformf, normalf5, normalf20 from test"
for q in [CONFIG1, config2(20.0, 15.0), "select id, uniformi from test"] + SUITE[:4] + EXTRA[:4] + [WIDE]:
    cpu = db.query(q, mode=0)
    gpu = db.query(q, mode=2)
    assert_same_stream(gpu.columns, cpu.columns, q)
    assert gpu.tablet_rows == cpu.tablet_rows, (q, gpu.tablet_rows, cpu.tablet_rows)
# the reference reader API on top of GPU results
n1, g1, b1 = db.reader_walk(CONFIG1, 12, 1000)
print("OK", n1, g1)
"""


@pytest.mark.parametrize("n", [10, 600_000])
def test_dropin_matches_single_core_vm(n):
    code = "ROOT = %r\n" % ROOT + SCRIPT
    out = subprocess.run([sys.executable, "-c", code, str(n)], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert "OK" in out.stdout


CACHE_SCRIPT = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, ROOT)
from virginian_b200 import _lib, datagen
lib = _lib.lib()                             # GPU VM first, RTLD_GLOBAL
from oracle import oracle as O
from tests.helpers import CONFIG1, config2, assert_same_stream
lib.virg_gpu_dropin_cache(1 << 30)
db = O.OracleDB(path=O.HOST_LIB, mode=ctypes.RTLD_GLOBAL)
n = int(sys.argv[1])
cols = datagen.table(n, datagen.SCHEMA_A, seed=24)
db.create_table("test", datagen.SCHEMA_A)
db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
queries = [CONFIG1, config2(20.0, 15.0), "select id, uniformi from test where uniformi < 7"]
h, m, b = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
for rep in range(2):
    for q in queries:
        cpu = db.query(q, mode=0)
        gpu = db.query(q, mode=2)
        assert_same_stream(gpu.columns, cpu.columns, q)
        assert gpu.tablet_rows == cpu.tablet_rows, (q, gpu.tablet_rows, cpu.tablet_rows)
lib.virg_gpu_dropin_cache_stats(ctypes.byref(h), ctypes.byref(m), ctypes.byref(b))
assert h.value > 0 and b.value > 0, (h.value, m.value, b.value)
misses_before = m.value
# appended rows change the last tablet's row count: it is copied again
more = datagen.table(5000, datagen.SCHEMA_A, seed=25)
more["id"] = more["id"] + n
db.insert("test", more["id"], [more[c] for c, _ in datagen.SCHEMA_A])
for q in queries:
    cpu = db.query(q, mode=0)
    gpu = db.query(q, mode=2)
    assert_same_stream(gpu.columns, cpu.columns, q)
lib.virg_gpu_dropin_cache_stats(ctypes.byref(h), ctypes.byref(m), ctypes.byref(b))
assert m.value > misses_before, (m.value, misses_before)
# a capacity below two tablets: every tablet evicts the one before it,
# which the previous tablet's kernel may still be reading
lib.virg_gpu_dropin_cache(12 << 20)
for q in queries:
    cpu = db.query(q, mode=0)
    gpu = db.query(q, mode=2)
    assert_same_stream(gpu.columns, cpu.columns, q)
    assert gpu.tablet_rows == cpu.tablet_rows, (q, gpu.tablet_rows, cpu.tablet_rows)
lib.virg_gpu_dropin_cache(0)
lib.virg_gpu_dropin_cache_stats(ctypes.byref(h), ctypes.byref(m), ctypes.byref(b))
assert b.value == 0, b.value
print("OK", h.value, m.value)
"""


def test_dropin_residency_cache_hits_and_refreshes_appended_tablets():
    code = "ROOT = %r\n" % ROOT + CACHE_SCRIPT
    out = subprocess.run([sys.executable, "-c", code, "600000"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert "OK" in out.stdout
