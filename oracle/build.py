"""Build recipe for the test-infrastructure libraries under oracle/.

* ``oracle/_build/libcfa_oracle.so``: the C restatement (gcc, OpenMP, no FP contraction so the
  host arithmetic matches the reference's host code operation for operation).
* ``oracle/_ref/libcfa_ref.so``: the reference's own solver translation unit compiled for
  sm_100a behind ``ref_harness.cu`` (nvcc, read from the reference source tree at build time;
  nothing of it is copied into this repository). Built only where that tree exists; the built
  library travels with the repository to GPU machines.

* ``oracle/_ref/cfa_ref_driver``: the reference's application, built by the one-line recipe of
  its README (``nvcc -O3 -std=c++17 ... src/cylinder_fem_amr.cu``) for sm_100a.
* ``oracle/_ref/cfa_dropin_driver``: the same unmodified application source built against this
  repository's solvers: a temporary mirror of the reference's ``src/`` whose files are links to
  the originals except ``cfa/linalg.cuh``, which links to ``cylinder-fem-amr_b200/shim/cfa/
  linalg.cuh``; linked with ``libcfa_b200.so``. The mirror is removed after the build.
* ``oracle/_ref/cfa_swap_driver``: as the drop-in, with the driver's Step A and B call sites
  (assembly, boundary conditions, OSS terms and the PPE solve) switched to the shim's
  ``cfa_swap`` functions: the mirror's ``cylinder_fem_amr.cu`` is a copy of the reference's with
  the eight call-site substitutions of ``SWAP_SITES`` applied (each anchor must occur exactly
  once), removed with the mirror after the build.

Run as ``python oracle/build.py [oracle|ref|drivers|all]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference project's src/ tree; CFA_REFERENCE_SRC overrides the default location.
REFERENCE_SRC = os.environ.get("CFA_REFERENCE_SRC", os.path.join(os.sep, "root", "reference", "src"))
ORACLE_LIB = os.path.join(HERE, "_build", "libcfa_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libcfa_ref.so")
REF_DRIVER = os.path.join(HERE, "_ref", "cfa_ref_driver")
DROPIN_DRIVER = os.path.join(HERE, "_ref", "cfa_dropin_driver")
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "cylinder-fem-amr_b200")
SHIM = os.path.join(PKG, "shim", "cfa", "linalg.cuh")
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


SWAP_DRIVER = os.path.join(HERE, "_ref", "cfa_swap_driver")
# call sites of the driver's Steps A and B -> the shim's cfa_swap functions (same arguments,
# the driver's DeviceMeshBuffers in front)
SWAP_SITES = [
    ("k_assemble_momentum_fem<<<blocks_elems, threads>>>(", "cfa_swap::assemble_momentum(gpu_buf, "),
    ("k_apply_bc_momentum<<<blocks_nodes, threads>>>(", "cfa_swap::apply_bc_momentum(gpu_buf, "),
    ("k_compute_oss_weights<<<blocks_elems, threads>>>(", "cfa_swap::oss_weights(gpu_buf, "),
    ("k_accumulate_scalar_gradient<<<blocks_elems, threads>>>(", "cfa_swap::scalar_gradient(gpu_buf, "),
    ("k_assemble_pressure_poisson<<<blocks_elems, threads>>>(", "cfa_swap::assemble_pressure_poisson(gpu_buf, "),
    ("apply_bc_pressure(n_nodes, gpu_buf.d_bc_tag", "cfa_swap::apply_bc_pressure(gpu_buf, n_nodes, gpu_buf.d_bc_tag"),
    ("if (oss) assemble_oss_projection(gpu_buf);", "if (oss) cfa_swap::assemble_oss_projection(gpu_buf);"),
    ("int it_p = solver.solve_pcg(", "int it_p = cfa_swap::solve_pcg(solver, gpu_buf, "),
]


def _driver_cmd(src: str, out: str, extra: list[str]) -> list[str]:
    return [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "shared",
            "-Xcompiler", "-fopenmp", *extra, src, "-o", out, "-lgomp"]


# The application's solver tolerances (CG and BiCGSTAB stop at |r| < 1e-7 |b|, the re-projection
# CG at 1e-8) written as literals at the call sites. The *_tight builds replace them by 1e-10 in
# both the stock program and the drop-in, so that two builds whose solvers differ only in rounding
# can be compared where the stopping tolerance no longer sets the size of the difference.
TIGHT_SITES = {
    "cylinder_fem_amr.cu": [
        ("gpu_buf.d_u, gpu_buf.d_v, 150, 1.0e-7, mom_ilu);", "gpu_buf.d_u, gpu_buf.d_v, 150, 1.0e-10, mom_ilu);"),
        ("gpu_buf.d_Kp_val, gpu_buf.d_rhs_p, gpu_buf.d_dp, 4000, 1.0e-7,",
         "gpu_buf.d_Kp_val, gpu_buf.d_rhs_p, gpu_buf.d_dp, 4000, 1.0e-10,"),
    ],
    "device.cuh": [
        ("g.d_Kp_val, g.d_rhs_p, g.d_dp, 4000, 1.0e-8,\n                                  oss ?",
         "g.d_Kp_val, g.d_rhs_p, g.d_dp, 4000, 1.0e-10,\n                                  oss ?"),
        ("g.d_Kp_val, g.d_rhs_p, g.d_dp, 4000, 1.0e-8,\n                                 nullptr,",
         "g.d_Kp_val, g.d_rhs_p, g.d_dp, 4000, 1.0e-10,\n                                 nullptr,"),
    ],
}
REF_TIGHT_DRIVER = os.path.join(HERE, "_ref", "cfa_ref_driver_tight")
DROPIN_TIGHT_DRIVER = os.path.join(HERE, "_ref", "cfa_dropin_driver_tight")


def _substitute(text: str, sites: list[tuple[str, str]]) -> str:
    for anchor, repl in sites:
        if text.count(anchor) != 1:
            raise RuntimeError(f"call site not found exactly once: {anchor}")
        text = text.replace(anchor, repl)
    return text


def _build_mirrored(out: str, shim: bool, swap: bool, tight: bool) -> None:
    """Builds the application from a temporary mirror of the reference's src/: links to the
    original files, except cfa/linalg.cuh -> the shim (shim=True) and the files edited at the
    call sites of SWAP_SITES (swap=True) or TIGHT_SITES (tight=True), which are written as
    copies. The mirror is removed afterwards."""
    main = os.path.join(REFERENCE_SRC, "cylinder_fem_amr.cu")
    cfa_dir = os.path.join(REFERENCE_SRC, "cfa")
    mirror = os.path.join(HERE, "_ref", "mirror")
    if os.path.isdir(mirror):
        shutil.rmtree(mirror)
    os.makedirs(os.path.join(mirror, "cfa"))
    try:
        sites = {}
        if swap:
            sites.setdefault("cylinder_fem_amr.cu", []).extend(SWAP_SITES)
        if tight:
            for f, s in TIGHT_SITES.items():
                sites.setdefault(f, []).extend(s)
        files = [("cylinder_fem_amr.cu", main)] + [(os.path.join("cfa", f), os.path.join(cfa_dir, f))
                                                  for f in os.listdir(cfa_dir)]
        for rel, src in files:
            dst = os.path.join(mirror, rel)
            if shim and rel == os.path.join("cfa", "linalg.cuh"):
                os.symlink(SHIM, dst)
            elif os.path.basename(rel) in sites:
                with open(dst, "w") as f:
                    f.write(_substitute(open(src).read(), sites[os.path.basename(rel)]))
            else:
                os.symlink(src, dst)
        extra = []
        if shim:
            extra = ["-I", os.path.join(ROOT, "include"), "-L", PKG, "-lcfa_b200",
                     "-Xlinker", "-rpath,$ORIGIN/../../cylinder-fem-amr_b200"]
        subprocess.check_call(_driver_cmd(os.path.join(mirror, "cylinder_fem_amr.cu"), out, extra))
    finally:
        shutil.rmtree(mirror)


def build_drivers(force: bool = False) -> tuple[str | None, str | None]:
    """The reference application as it ships, and the same source on this repository's solvers
    (plus the call-site-swapped build and the two tight-tolerance builds). Returns (stock, drop-in)
    paths, None where neither the reference tree nor a prebuilt binary exists."""
    main = os.path.join(REFERENCE_SRC, "cylinder_fem_amr.cu")
    if not os.path.exists(main):
        return (REF_DRIVER if os.path.exists(REF_DRIVER) else None,
                DROPIN_DRIVER if os.path.exists(DROPIN_DRIVER) else None)
    cfa_dir = os.path.join(REFERENCE_SRC, "cfa")
    deps = [main] + [os.path.join(cfa_dir, f) for f in os.listdir(cfa_dir)]
    os.makedirs(os.path.dirname(REF_DRIVER), exist_ok=True)
    if force or _stale(REF_DRIVER, deps):
        subprocess.check_call(_driver_cmd(main, REF_DRIVER, []))
    if force or _stale(REF_TIGHT_DRIVER, deps + [os.path.abspath(__file__)]):
        _build_mirrored(REF_TIGHT_DRIVER, shim=False, swap=False, tight=True)
    lib = os.path.join(PKG, "libcfa_b200.so")
    header = os.path.join(ROOT, "include", "cfa_b200.h")
    for out, swap, tight in ((DROPIN_DRIVER, False, False), (SWAP_DRIVER, True, False),
                             (DROPIN_TIGHT_DRIVER, False, True)):
        if force or _stale(out, deps + [SHIM, lib, header, os.path.abspath(__file__)]):
            _build_mirrored(out, shim=True, swap=swap, tight=tight)
    return REF_DRIVER, DROPIN_DRIVER


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("oracle", "all"):
        print(build_oracle(force=True))
    if what in ("ref", "all"):
        print(build_ref(force=True))
    if what in ("drivers", "all"):
        print(build_drivers(force=True))
