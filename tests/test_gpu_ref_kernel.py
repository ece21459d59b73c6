"""The reference's own GPU VM (src/vm/vm_gpu.cu, compiled unmodified for
sm_100a into oracle/_ref/libvirg_refgpu.so) on the same seeded tables: its
results are unordered (block-level atomics, src/vm/vm_gpu.cu:893-1126), so
they are compared with the single-core CPU VM's as a multiset of rows; its
own kernel timing (serial transfer mode, vm->timing2) is the existing-kernel
bar the sm_100a VM is measured against.  Runs in a child process so the
reference's library and this repository's never share a process."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, ROOT)
from virginian_b200 import datagen
from oracle import oracle as O
from tests.helpers import CONFIG1, config2
n = int(sys.argv[1])
cols = datagen.table(n, datagen.SCHEMA_A, seed=31)
db = O.OracleDB(path=O.REFGPU_LIB)
db.create_table("test", datagen.SCHEMA_A)
db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
q = 1 - (1 - 0.10) ** 0.5
c = float(np.quantile(cols["uniformf"], q)); d = float(np.quantile(cols["normalf20"], 1 - q))
out = []
for sql in (CONFIG1, config2(c, d)):
    cpu = db.query(sql, mode=0)
    gpu = db.query(sql, mode=2, repeat=3)
    rows_c = np.rec.fromarrays([x.view(f"u{x.itemsize}") for x in cpu.columns])
    rows_g = np.rec.fromarrays([x.view(f"u{x.itemsize}") for x in gpu.columns])
    same = rows_c.shape == rows_g.shape and bool(np.array_equal(np.sort(rows_c), np.sort(rows_g)))
    out.append({"sql": sql, "rows": int(cpu.rows), "gpu_rows": int(gpu.rows), "multiset_equal": same,
                "kernel_s": gpu.gpu_timing[1], "h2d_s": gpu.gpu_timing[0], "d2h_s": gpu.gpu_timing[2]})
db.close()
print("JSON " + json.dumps(out))
"""


def run_ref(n):
    lib = os.path.join(ROOT, "oracle", "_ref", "libvirg_refgpu.so")
    if not os.path.exists(lib):
        pytest.fail("oracle/_ref/libvirg_refgpu.so is missing (built by __graft_entry__.build())")
    p = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + SCRIPT, str(n)], capture_output=True,
                       text=True, timeout=900)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    line = [x for x in p.stdout.splitlines() if x.startswith("JSON ")][-1]
    return json.loads(line[5:])


def test_reference_gpu_vm_rows_match_cpu_vm_as_multiset():
    for r in run_ref(1_000_000):
        assert r["gpu_rows"] == r["rows"], r
        assert r["multiset_equal"], r["sql"]
