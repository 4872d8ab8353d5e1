"""Build recipe for the test-infrastructure libraries under oracle/.

* ``oracle/_build/libcfa_oracle.so``: the C restatement (gcc, OpenMP, no FP contraction so the
  host arithmetic matches the reference's host code operation for operation).
* ``oracle/_ref/libcfa_ref.so``: the reference's own solver translation unit compiled for
  sm_100a behind ``ref_harness.cu`` (nvcc, read from the reference source tree at build time;
  nothing of it is copied into this repository). Built only where that tree exists; the built
  library travels with the repository to GPU machines.

Run as ``python oracle/build.py [oracle|ref|all]``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE_SRC = "/root/reference/src"
ORACLE_LIB = os.path.join(HERE, "_build", "libcfa_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libcfa_ref.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "cfa_oracle.c")
    hdr = os.path.join(HERE, "cfa_oracle.h")
    if force or _stale(ORACLE_LIB, [src, hdr]):
        os.makedirs(os.path.dirname(ORACLE_LIB), exist_ok=True)
        cmd = ["gcc", "-O2", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
               "-o", ORACLE_LIB, src, "-lm"]
        subprocess.check_call(cmd)
    return ORACLE_LIB


def build_ref(force: bool = False) -> str | None:
    """Returns the library path, or None when the reference tree is absent (GPU machines use the
    prebuilt library)."""
    main = os.path.join(REFERENCE_SRC, "cylinder_fem_amr.cu")
    if not os.path.exists(main):
        return REF_LIB if os.path.exists(REF_LIB) else None
    harness = os.path.join(HERE, "ref_harness.cu")
    deps = [harness, main] + [os.path.join(REFERENCE_SRC, "cfa", f) for f in os.listdir(os.path.join(REFERENCE_SRC, "cfa"))]
    if force or _stale(REF_LIB, deps):
        os.makedirs(os.path.dirname(REF_LIB), exist_ok=True)
        cmd = [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
               "-Xcompiler", "-fopenmp,-fPIC", "-shared", "-I", REFERENCE_SRC,
               "-o", REF_LIB, harness, "-lgomp"]
        subprocess.check_call(cmd)
    return REF_LIB


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("oracle", "all"):
        print(build_oracle(force=True))
    if what in ("ref", "all"):
        print(build_ref(force=True))
