"""Builds ``virginian_b200/libvirginian_b200.so`` (the VM kernels and the C ABI)
with nvcc for sm_100a only.  Runs without a GPU (nvcc cross-compiles).

    python -m virginian_b200.build [--verbose-ptxas]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvirginian_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["vm_kernel.cu", "engine.cu", "batch.cu", "stream.cu", "dropin.cu", "noalloc.cu", "serve.cu",
           "ceiling.cu", "tunecache.cpp", "estimate.cpp", "ingest.cu", "program.cpp", "sqlc.cpp"]
EXTRA_SOURCES: List[str] = []

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # bit-exact float arithmetic: no FMA contraction, IEEE division
    "-fmad=false", "-prec-div=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-O2,-fno-strict-aliasing",
    "-I", os.path.join(os.path.dirname(HERE), "include"),
]


def _stale(obj: str, deps: List[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "virginian_b200.h"))
    objs = []
    procs = []
    for src in SOURCES + EXTRA_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.rsplit(".", 1)[0] + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [NVCC] + FLAGS + ["-c", path, "-o", obj]
            if verbose_ptxas and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if src.endswith(".cpp"):
                cmd = [NVCC, "-x", "cu"] + FLAGS + ["-c", path, "-o", obj]
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.STDOUT, text=True)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if out.strip():
            sys.stderr.write(f"--- {src}\n{out}")
        if p.returncode != 0:
            failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    if force or _stale(LIB, objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + [
            "-ldl", "-lpthread"]
        subprocess.run(cmd, check=True)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose_ptxas, a.force))


if __name__ == "__main__":
    main()
