"""The C-ABI library loads and exports every entry point its header declares;
struct sizes match the reference's (src/test/virgstate.cc:64-80).  No GPU."""
import ctypes
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(virg_\w+)\s*\(", text, re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "virg_vm_gpu" in names and "virg_gpu_getsizes" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from virginian_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_sizes_match_reference(oracle_mod):
    """virg_gpu_getsizes (this library) against virg_testsizes of the stock
    reference header, read from the reference host library in a clean process."""
    code = f"""
import ctypes, sys
sys.path.insert(0, {ROOT!r})
from virginian_b200 import _lib
mine = _lib.lib().virg_gpu_getsizes()
host = ctypes.CDLL({os.path.join(ROOT, 'oracle', '_ref', 'libvirg_host.so')!r}, mode=ctypes.RTLD_GLOBAL)
host.orc_testsizes.restype = ctypes.POINTER(ctypes.c_size_t)
ref = host.orc_testsizes()
print([mine[i] for i in range(15)] == [ref[i] for i in range(15)], [mine[i] for i in range(15)], [ref[i] for i in range(15)])
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("True"), out.stdout


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    from virginian_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(ImportError):
        _lib.lib()
