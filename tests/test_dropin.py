"""The reference application, unmodified, on this repository's solvers.

``oracle/_ref/cfa_ref_driver`` is the reference's own program (src/cylinder_fem_amr.cu built by
its README recipe); ``oracle/_ref/cfa_dropin_driver`` is the same source compiled against the
shim header ``cylinder-fem-amr_b200/shim/cfa/linalg.cuh`` and linked with ``libcfa_b200.so``;
``oracle/_ref/cfa_swap_driver`` additionally has the driver's Step A and B call sites switched to
this library's assembly and handle-based PPE solve; ``oracle/_ref/cfa_ref_driver_tight`` and
``oracle/_ref/cfa_dropin_driver_tight`` are the stock program and the drop-in with the solver
tolerances at the call sites set to 1e-10 instead of the application's 1e-7 / 1e-8
(``oracle/build.py drivers``). Each runs the
DFG 2D-2 cylinder case on a uniform level-3 mesh (the reference's U3 run, 29k nodes) and with
adaptive refinement (its A1 settings, a remesh every 10 steps), and the force histories
(``<prefix>_forces.csv``, 10 significant digits), meshes and iteration counts are compared with
the stock program's row by row.
"""
import csv
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
STOCK = os.path.join(REF_DIR, "cfa_ref_driver")
DROPIN = os.path.join(REF_DIR, "cfa_dropin_driver")
SWAP = os.path.join(REF_DIR, "cfa_swap_driver")
STOCK_TIGHT = os.path.join(REF_DIR, "cfa_ref_driver_tight")
DROPIN_TIGHT = os.path.join(REF_DIR, "cfa_dropin_driver_tight")

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
if not (os.path.exists(STOCK) and os.path.exists(DROPIN)):
    pytest.skip("application binaries not built (python oracle/build.py drivers)", allow_module_level=True)

CASES = {
    # the reference's campaign settings (scripts/campaign.sh: U3 and A1), 400 steps of dt = 1e-3
    "U3": ["--uniform-level", "3"],
    "A1": ["--amr-tol-vort", "0.1", "--amr-tol-interp", "0.01", "--max-level", "4", "--max-elems", "200000",
           "--min-level", "2"],
}
STEPS = 400
ITERS = re.compile(r"\[Step\s+(\d+).*Iters\(u,v,p\): \((\d+),(\d+),(\d+)\)")


def run(binary, case, tmp, env=None):
    prefix = os.path.join(str(tmp), os.path.basename(binary))
    cmd = [binary, "--steps", str(STEPS), "--print-interval", "10", "--prefix", prefix, *CASES[case]]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env={**os.environ, **(env or {})})
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    with open(prefix + "_forces.csv") as f:
        rows = list(csv.DictReader(f))
    iters = {int(m.group(1)): tuple(int(g) for g in m.groups()[1:]) for m in ITERS.finditer(p.stdout)}
    wall = re.search(r"\[Timing\] ([0-9.eE+-]+) s wall", p.stdout)
    return rows, iters, float(wall.group(1)) if wall else None, p.stdout


def compare(a, b):
    """Largest relative difference of the drag and lift histories (scaled by the series' own
    magnitude) and whether every row has the same mesh."""
    assert len(a) == len(b) == STEPS
    same_mesh = all(ra["nodes"] == rb["nodes"] and ra["elements"] == rb["elements"] for ra, rb in zip(a, b))
    out = {}
    for key in ("C_D", "C_L", "delta_p"):
        xa = [float(r[key]) for r in a]
        xb = [float(r[key]) for r in b]
        scale = max(abs(v) for v in xa[20:])   # past the impulsive start
        out[key] = max(abs(u - v) for u, v in zip(xa, xb)) / scale
    return out, same_mesh


_STOCK_RUNS = {}


def stock(case, tmp_path_factory, binary=STOCK):
    key = (case, binary)
    if key not in _STOCK_RUNS:
        _STOCK_RUNS[key] = run(binary, case, tmp_path_factory.mktemp("stock"))
    return _STOCK_RUNS[key]


# Largest force difference allowed, relative to the series' scale. At the application's own
# tolerances (CG and BiCGSTAB stop at |r| < 1e-7 |b|) a PPE solve that stops one iteration earlier
# or later than the stock program's moves the solution by about the tolerance, and on A1 that
# shows in the lift from the first step after the remesh at step 65 on (31 against 32 CG
# iterations there): measured C_D 3.1e-10, C_L 4.5e-9, dp 4.2e-10. With both programs' tolerances
# at 1e-10 the same comparison measures C_D 0, C_L 1.1e-11, dp 0 -- the stock program's own
# run-to-run spread (its assembly sums with atomics), so there the north star's 1e-9 holds.
FORCE_TOL = {"dropin": 1e-8, "swap": 1e-8, "dropin_tight": 1e-9}


@pytest.mark.parametrize("case", ["U3", "A1"])
@pytest.mark.parametrize("build", ["dropin", "swap", "dropin_tight"])
def test_unmodified_application_on_b200_solvers(build, case, tmp_path, tmp_path_factory):
    binary = {"dropin": DROPIN, "swap": SWAP, "dropin_tight": DROPIN_TIGHT}[build]
    ref_binary = STOCK_TIGHT if build == "dropin_tight" else STOCK
    if not (os.path.exists(binary) and os.path.exists(ref_binary)):
        pytest.skip(f"{binary} not built")
    ref_rows, ref_it, ref_wall, _ = stock(case, tmp_path_factory, ref_binary)
    new_rows, new_it, new_wall, out = run(binary, case, tmp_path)
    diff, same_mesh = compare(ref_rows, new_rows)
    print(f"{case}: wall {ref_wall} s (reference) vs {new_wall} s ({build}); max rel diff {diff}; "
          f"same meshes {same_mesh}")
    assert same_mesh
    # Iteration counts of the printed steps. Momentum: within one of the reference's at every
    # step. PPE: CG stops at |r| < 1e-7 |b|, and the 2-norm of a CG residual is not monotone;
    # where it oscillates about the tolerance, rounding decides whether a dip crosses it (on A1
    # the counts differ at 111 of 400 steps at 1e-7 and at 153 at 1e-10, by one or two). So:
    # within one at 90 % of the printed steps, and the totals within 1 %.
    assert ref_it.keys() == new_it.keys()
    close = 0
    for s in ref_it:
        (ru, rv, rp), (nu, nv, np_) = ref_it[s], new_it[s]
        assert abs(ru - nu) <= 1 and abs(rv - nv) <= 1, (s, ref_it[s], new_it[s])
        close += abs(rp - np_) <= 1
    assert close >= 0.9 * len(ref_it)
    tot_ref, tot_new = sum(v[2] for v in ref_it.values()), sum(v[2] for v in new_it.values())
    assert abs(tot_ref - tot_new) <= 0.01 * tot_ref
    # forces (the histories are printed with 10 significant digits)
    for key, d in diff.items():
        assert d <= FORCE_TOL[build], (key, d)
