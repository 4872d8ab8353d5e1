"""Benchmark of the per-timestep solve path: pressure + momentum solve ms/step, mixed precision
(FP32 SA-AMG / ILU inside FP64 Krylov) and plain FP64, at 1e-10 relative residual.

Workload (default): the adaptive ~400k-vertex mesh (seeded Delaunay + NVB, refined near the disc
and in the wake band), BDF2 step with dt = 1e-3, nu = 1e-3, SUPG T = 1 ms, OSS stab 0.3, inflow
U = 1.5; u^n = u^{n-1} and p^n are seeded Fourier fields (synthetic data). One step = momentum
assembly + BCs, ILU(0) factor, BiCGSTAB2 (u, v) to 1e-10, OSS weights, G(p^n), pressure system
assembly (PPE + BCs + OSS operator), PCG (K + OSS, SA-AMG) to 1e-10. The AMG setup is timed
separately and amortised over 50 steps, the reference driver's rebuild interval.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c1]

With N > 1 (torchrun) each rank solves its own replica (the single-system path does not shard):
`value` is then the job's aggregate time per step (max over ranks / (N K)).
`--impl reference` runs the reference's own CUDA build (oracle/_ref, compiled from the
reference sources) on the same workload on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cylinder-fem-amr_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

AMG_REBUILD = 50          # src/cfa/options.cuh:26
SETUP_REPS = 5
STAB, DT, NU, U_MAX, TOL = 0.3, 1e-3, 1e-3, 1.5, 1e-10
METRIC = "pressure+momentum solve ms/step & HBM GB/s, mixed vs FP64 at 1e-10 rel res"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling (every 100 ms) while the timed regions run: one sampler process for
    the whole run; samples taken between start() and pause() are kept."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"cfa_clocks_{os.getpid()}.csv")
        self.windows = []
        self.t0 = None

    def start(self):
        if self.proc is None:
            q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            try:
                self.f = open(self.path, "w")
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=self.f, stderr=subprocess.DEVNULL)
                time.sleep(0.3)
            except Exception:
                self.proc = False
        self.t0 = time.time()

    def pause(self):
        if self.t0 is not None:
            self.windows.append((self.t0, time.time() + 0.1))
            self.t0 = None

    def stop(self):
        self.pause()
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        import datetime
        sm, mx, reasons, n_all = [], 0.0, set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                clk, cmax = float(f[1]), float(f[2])
            except ValueError:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                ts = None   # unknown format: keep the sample
            n_all += 1
            if ts is not None and not any(a <= ts <= b for a, b in self.windows):
                continue
            sm.append(clk)
            mx = max(mx, cmax)
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "samples_total": n_all}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def workload_inputs(name):
    import fixtures as F
    m = F.make_mesh(name)
    u = F.fourier_field(m.x, m.y, 1)
    v = F.fourier_field(m.x, m.y, 2)
    p = 0.3 * F.fourier_field(m.x, m.y, 3)
    return m, u, v, p


def workload_name(name, n, nnz):
    """The workload string both arms print (the same mesh, the same step)."""
    kind = "uniform" if name in ("c0", "c2") else "adaptive"
    return f"{name}: {kind} NVB mesh n={n}, nnz={nnz}, BDF2 step, OSS 0.3, tol 1e-10"


def l2_flush(buf):
    buf.add_(1.0)


# ------------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------------
def operator_bytes(n, nnz, passes, stored_nnz):
    """Algorithmic bytes of one application y = A x of the pressure operator (K + OSS) as the
    standalone entry point runs it (pn = x is written back for the own row, as in the CG).
    One pass (K - B^T M^-1 B stored on the two-ring pattern): col_ind + values (12 B per stored
    entry), row_ptr, x read, pn and y written. Two passes: pass 1 reads col_ind + Bx + By
    (20 B/nnz), row_ptr, x, inv_m, writes pn and g (x, y); pass 2 reads col_ind + K + BTx + BTy
    (28 B/nnz), row_ptr, pn, g, tags, writes y."""
    if passes == 1:
        return stored_nnz * 12 + 4 * (n + 1) + n * 24
    p1 = nnz * 20 + 4 * (n + 1) + n * (8 + 8 + 8 + 16)
    p2 = nnz * 28 + 4 * (n + 1) + n * (8 + 16 + 4 + 8)
    return p1 + p2


def time_operator(cfa, st, reps, flush):
    """Live CUDA-event timing of the dominant kernel pair: the pressure operator passes."""
    import torch
    x = st.dp.clone().normal_()
    y = torch.empty_like(x)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    cfa.pressure_operator_prepare(st.ctx, st.dm.rp, st.dm.ci, st.Kp, st.oss)
    layout = cfa.pressure_operator_layout(st.ctx)
    for _ in range(3):
        cfa.pressure_operator(st.ctx, st.dm.rp, st.dm.ci, st.Kp, x, y, st.oss)
    total = 0.0
    for _ in range(reps):
        l2_flush(flush)
        ev[0].record()
        cfa.pressure_operator(st.ctx, st.dm.rp, st.dm.ci, st.Kp, x, y, st.oss)
        ev[1].record()
        ev[1].synchronize()
        total += ev[0].elapsed_time(ev[1])
    return total / reps, layout


def run_ours(args, rank, world):
    import torch
    import cfa_b200 as cfa
    import step as S

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    m, u, v, p = workload_inputs(args.workload)
    ctx = cfa.Context()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    res = {}
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", 0)))
    for prec_name, prec in (("fp64", cfa.FP64), ("mixed", cfa.MIXED)):
        if args.profile and args.profile_precision not in ("both", prec_name):
            continue
        st = S.SolveStep(m, u, v, p, precision=prec, ctx=ctx, dt=DT, nu=NU, stab=STAB, u_max=U_MAX, tol=TOL)
        # AMG setup: one untimed setup (first-touch allocations), then the median of SETUP_REPS
        # (a setup runs host loops and synchronises; on a shared host one of them now and then
        # stalls for tens of ms, which a mean would spread over every step)
        st.amg_setup()
        ph0 = dict(st.amg.phase_ms)
        setup_ms = float(np.median([st.amg_setup() for _ in range(SETUP_REPS)]))
        phases = {k: (v - ph0.get(k, 0.0)) / SETUP_REPS for k, v in st.amg.phase_ms.items()}
        if args.profile:
            for _ in range(args.warmup):
                st.run()
            torch.cuda.synchronize()
            torch.cuda.profiler.start()
            st.run()
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
            print(json.dumps({"profile": prec_name, "report": st.report(), "launches": ctx.launches}))
            del st
            continue
        for _ in range(args.warmup):
            st.run()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        total = 0.0
        l0 = ctx.launches
        reports = []
        clk.start()
        for _ in range(args.steps):
            l2_flush(flush)
            ev[0].record()
            st.run()
            ev[1].record()
            ev[1].synchronize()
            total += ev[0].elapsed_time(ev[1])
            reports.append(st.report())
        clk.pause()
        launches = ctx.launches - l0
        torch.cuda.synchronize()
        step_ms = total / args.steps
        # end-to-end through the API with host buffers: H2D of the step inputs, D2H of the results
        hu = torch.from_numpy(u).pin_memory()
        hv = torch.from_numpy(v).pin_memory()
        hp = torch.from_numpy(p).pin_memory()
        outs = [torch.empty(m.n, dtype=torch.float64).pin_memory() for _ in range(3)]
        e2e_total = 0.0
        clk.start()
        for _ in range(args.steps):
            l2_flush(flush)
            ev[0].record()
            st.u_n.copy_(hu, non_blocking=True)
            st.v_n.copy_(hv, non_blocking=True)
            st.p_n.copy_(hp, non_blocking=True)
            st.u_prev.copy_(st.u_n)
            st.v_prev.copy_(st.v_n)
            st.run(host_out=outs)   # u, v copied out during the pressure solve, dp after it
            ev[1].record()
            ev[1].synchronize()
            e2e_total += ev[0].elapsed_time(ev[1])
        clk.pause()
        e2e_ms = e2e_total / args.steps
        clk.start()
        op_ms, op_layout = time_operator(cfa, st, 20, flush) if prec == cfa.FP64 else (None, None)
        kern = kernel_table(cfa, st, flush)[0] if prec == cfa.MIXED else None
        clk.pause()
        res[prec_name] = dict(step_ms=step_ms, setup_ms=setup_ms, e2e_ms=e2e_ms, launches=launches,
                              report=reports[-1], op_ms=op_ms, op_layout=op_layout, levels=st.amg.num_levels(), phases=phases,
                              composite=st.amg.composite(),
                              colours=st.ilu.n_colours, nnz=st.nnz, n=st.n, kernels=kern)
        del st
    clk.stop()
    res["clocks"] = clk.summary()
    return m, res


def cpu_baseline(m, u, v, p):
    """The oracle (C restatement, OpenMP) on one full step of the same workload, host cores."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    rp, ci = O.csr_build(m.n, m.elem_v)
    t_pattern = time.perf_counter() - t0
    t0 = time.perf_counter()
    A, ru, rv, mass = O.assemble_momentum(m, rp, ci, u, v, u, v, p, O.bdf2_params())
    uu, vv = u.copy(), v.copy()
    O.apply_bc_momentum(m, rp, ci, A, ru, rv, uu, vv)
    ilu = O.Ilu(rp, ci)
    ilu.factor(A)
    xu, xv, _ = O.bicgstab2(rp, ci, A, ru, rv, uu, vv, ilu, 1000, TOL)
    dt_proj = 2 * DT / 3
    s = O.oss_weights(m, xu, xv, dt_proj, 1.0, NU, STAB)
    gx, gy = O.scalar_gradient(m, p, s)
    Kp, rhs, div = O.assemble_ppe(m, rp, ci, xu, xv, p, gx, gy, mass, s, dt_proj, 1.0, STAB)
    dp = np.zeros(m.n)
    O.apply_bc_pressure(m, rp, ci, Kp, rhs, dp, mass)
    oss, inv_m = O.assemble_oss(m, rp, ci, s, mass)
    t_solve_start = time.perf_counter()
    amg = O.Amg(rp, ci, Kp)
    t_setup = time.perf_counter() - t_solve_start
    O.pcg(rp, ci, Kp, rhs, dp, 4000, TOL, oss, inv_m, m.tag, amg)
    t_step = time.perf_counter() - t0 - t_setup
    ms = 1e3 * t_step + 1e3 * t_setup / AMG_REBUILD
    return dict(value=ms, unit="ms/step", cores=O.lib().or_num_threads(), kind="port",
                sample=f"1 full FP64 step of the same workload (n={m.n}) by the oracle port, OpenMP; "
                       f"AMG setup {1e3 * t_setup:.0f} ms amortised over {AMG_REBUILD} steps")


# ------------------------------------------------------------------------------------------------
# reference arm: the reference's own CUDA build (oracle/_ref)
# ------------------------------------------------------------------------------------------------
def run_reference(args):
    import ctypes as C
    import torch
    from oracle import oracle as O
    m, u, v, p = workload_inputs(args.workload)
    R = O.ref()
    if not R.ref_gpu_available():
        return {"impl": "reference", "unavailable": "no GPU visible to the reference build"}
    ev = np.ascontiguousarray(m.elem_v, np.int32)
    tag = np.ascontiguousarray(m.tag, np.int32)
    h = C.c_void_p(R.ref_step_create(m.n, m.ne, O._p(ev), O._p(m.x), O._p(m.y), O._p(tag), O._p(u), O._p(v),
                                     O._p(p), C.c_double(DT), C.c_double(NU), C.c_double(1.0), C.c_double(U_MAX),
                                     C.c_double(1.0), C.c_double(1e-3), C.c_double(STAB), C.c_double(TOL), 1000, 4000))
    setup_ms = R.ref_step_amg_setup(h)
    its, conv, rel = np.zeros(3, np.int32), np.zeros(3, np.int32), np.zeros(3)
    for _ in range(args.warmup):
        R.ref_step_run(h, O._p(its), O._p(conv), O._p(rel), None, None, None)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    total = 0.0
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", 0)))
    clk.start()
    for _ in range(args.steps):
        flush.add_(1.0)
        torch.cuda.synchronize()
        total += R.ref_step_run(h, O._p(its), O._p(conv), O._p(rel), None, None, None)
    clk.stop()
    nnz = R.ref_step_nnz(h)
    R.ref_step_free(h)
    step_ms = total / args.steps
    value = step_ms + setup_ms / AMG_REBUILD
    threads = int(R.ref_omp_threads())
    return {
        "metric": METRIC, "value": round(value, 4), "unit": "ms/step", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(value, 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(args.workload, m.n, nnz),
                   "precision": "fp64 (the reference has no mixed mode)", "l2": "flushed between steps",
                   "amg_setup_ms": round(setup_ms, 3), "amg_rebuild": AMG_REBUILD,
                   "step_ms_without_setup": round(step_ms, 4), "omp_threads": threads,
                   "iterations": {"u": int(its[0]), "v": int(its[1]), "p": int(its[2])},
                   "converged": [bool(c) for c in conv]},
        "cpu_baseline": {"value": round(value, 4), "unit": "ms/step", "cores": threads, "kind": "reference",
                         "sample": "the reference's own CUDA build (nvcc sm_100a, host-timed steps with its "
                                   "device syncs) on the same workload; AMG setup on the host with the "
                                   "reference application's OpenMP thread rule (half the logical CPUs, at most 8)"},
        "e2e": {"value": round(value, 4), "unit": "ms/step", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    }


# ------------------------------------------------------------------------------------------------
# bandwidth stress (c2): ~4M vertices, repeated solves with perturbed right-hand sides
# ------------------------------------------------------------------------------------------------
def vcycle_bytes(levels, coarse_n, vb, eb=8):
    """Algorithmic bytes of one V(2,2) cycle of the tile kernels: per level with n rows, z entries
    of A and q of P (= of R), values of vb bytes, vectors of eb bytes (8, or 4 for the FP32 V-cycle
    of mixed precision, whose level 0 still reads the FP64 right-hand side and writes the FP64
    result): pre-smoothing (initial guess fused), residual, restriction, prolongation-add and two
    post-smoothing sweeps, each reading its matrix once (column index + value, row offsets) and
    its vectors once per entry read or written; the dense coarse solve reads its FP64 inverse.
    These are the bytes of the V(2,2) level chain as the reference runs it; the composite coarse
    operator and the fused transfers do the same arithmetic with other reads, which the model
    does not follow, so its fraction is the chain's bytes over the time taken."""
    total = 0
    for lvl, (n, z, nc, q) in enumerate(levels):
        bb = 8 if lvl == 0 else eb                       # the level's right-hand side
        zb = 8 if lvl == 0 else eb                       # the last sweep's output
        mat_a = z * (vb + 4) + 4 * (n + 1)
        total += mat_a + n * (bb + eb + bb + eb)         # pre: b, dinv (gathered), b (own), x write
        total += mat_a + n * (eb + bb + eb)              # residual: x, b, r write
        total += q * (vb + 4) + 4 * (nc + 1) + eb * n + eb * nc          # restriction
        total += q * (vb + 4) + 4 * (n + 1) + eb * nc + 2 * eb * n       # prolongation-add
        total += mat_a + n * (eb + bb + eb + eb)         # Jacobi sweep: x, b, dinv, out
        total += mat_a + n * (eb + bb + eb + zb)         # last sweep
    return total + 8 * coarse_n * coarse_n + 2 * eb * coarse_n


def ilu_bytes(n, nnz, vb, wb):
    """Algorithmic bytes of one two-right-hand-side ILU apply (forward and backward colour sweeps,
    both right-hand sides interleaved per row): the split factors once ((nnz - n) column indices
    and values of vb bytes), the diagonal inverse, the row order and the split offsets; the FP64
    right-hand side read once and the FP64 result written once (16 bytes a row each), the work
    vector (wb bytes a row for the pair: 16 in FP64, where it is the result itself, 8 in FP32)
    written by the forward sweep and read and written by the backward sweep."""
    base = (nnz - n) * (vb + 4) + n * vb + 4 * n + 8 * (n + 1)
    if wb == 16:                      # in place in the FP64 result: r read, y written, y read, z written
        return base + 4 * 16 * n
    return base + 16 * n + wb * n + 2 * wb * n + 16 * n


def kernel_table(cfa, st, flush, reps=20):
    """Per-kernel bandwidth of the four paths the solves spend their time in, each applied alone
    on the step's own operators, repeated, timed by CUDA events on the context's stream with the
    L2 flushed before each repetition: the pressure operator (FP64, one pass), the V-cycle (the
    handle's precision), the momentum ILU apply (interleaved pair, the handle's precision) and the
    two-right-hand-side momentum SpMV (FP64)."""
    import torch
    ctx = st.ctx
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        acc = 0.0
        for _ in range(reps):
            flush.add_(1.0)
            ev[0].record()
            fn()
            ev[1].record()
            ev[1].synchronize()
            acc += ev[0].elapsed_time(ev[1])
        return acc / reps * 1e3

    hbm, _ = peaks()
    n, nnz = st.n, st.nnz
    mixed = st.precision == cfa.MIXED
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    cfa.pressure_operator_prepare(ctx, st.dm.rp, st.dm.ci, st.Kp, st.oss)
    passes, stored = cfa.pressure_operator_layout(ctx)
    t_op = timed(lambda: cfa.pressure_operator(ctx, st.dm.rp, st.dm.ci, st.Kp, x, y, st.oss))
    b_op = operator_bytes(n, nnz, passes, stored)
    z = torch.empty_like(x)
    t_vc = timed(lambda: st.amg.apply(x, z))
    levels = []
    for lvl in range(st.amg.num_levels() - 1):
        d = st.amg.level(lvl)
        levels.append((d["rows"], int(d["A"][1].numel()), d["pcols"], int(d["P"][1].numel())))
    fp32_vectors = mixed and os.environ.get("CFA_VCYCLE_FP64", "0") != "1"
    b_vc = vcycle_bytes(levels, st.amg.coarse_n, 4 if mixed else 8, 4 if fp32_vectors else 8)
    x2 = torch.randn(2 * n, dtype=torch.float64, device="cuda")
    z2 = torch.empty_like(x2)
    t_ilu = timed(lambda: st.ilu.apply_interleaved(x2, z2))
    b_ilu = ilu_bytes(n, nnz, 4 if mixed else 8, 8 if mixed else 16)
    t_spmv = timed(lambda: cfa.spmv_multi(ctx, st.dm.rp, st.dm.ci, st.A, x2, z2, 2))
    b_spmv = nnz * 12 + 4 * (n + 1) + 4 * n * 8
    tag = "fp32" if mixed else "fp64"
    kern = {}
    for name, b, t in (("pressure_operator_fp64", b_op, t_op), (f"vcycle_{tag}", b_vc, t_vc),
                       (f"ilu_apply_2rhs_{tag}", b_ilu, t_ilu), ("momentum_spmv_2rhs_fp64", b_spmv, t_spmv)):
        gbs = b / (t * 1e-6) / 1e9
        kern[name] = {"bytes": int(b), "us": round(t, 2), "gbs": round(gbs, 1), "frac": round(gbs / hbm, 4)}
    return kern, passes


def run_stress(args, rank, world):
    """c2: repeated momentum + pressure solve pairs on the ~4M-vertex mesh with seeded N(0, 1e-3)
    right-hand-side noise, mixed precision (the headline) and plain FP64, and the per-kernel
    bandwidth table of each precision. With --profile, one mixed solve pair runs between
    cudaProfilerStart/Stop (for ncu --profile-from-start off) and no line is printed."""
    import torch
    import cfa_b200 as cfa
    import step as S

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    m, u, v, p = workload_inputs("c2")
    ctx = cfa.Context()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    solves = max(args.steps, 1)
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", 0)))
    legs = {}
    for prec_name, prec in (("mixed", cfa.MIXED), ("fp64", cfa.FP64)):
        st = S.SolveStep(m, u, v, p, precision=prec, ctx=ctx, dt=DT, nu=NU, stab=STAB, u_max=U_MAX, tol=TOL)
        st.amg_setup()
        base_u, base_v, base_p = st.rhs_u.clone(), st.rhs_v.clone(), st.rhs_p.clone()
        n, nnz = st.n, st.nnz

        def perturbed(k):
            g = torch.Generator(device="cuda")
            g.manual_seed(k)
            st.rhs_u.copy_(base_u + 1e-3 * torch.randn(n, generator=g, device="cuda", dtype=torch.float64))
            st.rhs_v.copy_(base_v + 1e-3 * torch.randn(n, generator=g, device="cuda", dtype=torch.float64))
            st.rhs_p.copy_(base_p + 1e-3 * torch.randn(n, generator=g, device="cuda", dtype=torch.float64))
            st.u.copy_(st.u_n)
            st.v.copy_(st.v_n)
            st.dp.zero_()

        for k in range(args.warmup):
            perturbed(1000 + k)
            st.solve_momentum()
            st.solve_pressure()
        torch.cuda.synchronize()
        if args.profile:
            perturbed(0)
            torch.cuda.synchronize()
            torch.cuda.profiler.start()
            st.solve_momentum()
            st.solve_pressure()
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
            print(json.dumps({"profile": "c2 " + prec_name, "report": st.report(), "launches": ctx.launches}))
            return
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        clk.start()
        total, its = 0.0, []
        l0 = ctx.launches
        for k in range(solves):
            perturbed(k)
            ev[0].record()
            st.solve_momentum()
            st.solve_pressure()
            ev[1].record()
            ev[1].synchronize()
            total += ev[0].elapsed_time(ev[1])
            r = st.report()
            its.append((r["it_u"], r["it_v"], r["it_p"]))
        launches = ctx.launches - l0
        kern, passes = kernel_table(cfa, st, flush)
        clk.pause()
        legs[prec_name] = dict(ms=total / solves, its=its, launches=launches, kernels=kern, passes=passes,
                               levels=st.amg.num_levels(), n=n, nnz=nnz)
        del st
        torch.cuda.synchronize()
    clk.stop()
    hbm, peak_kind = peaks()
    mx, f64 = legs["mixed"], legs["fp64"]
    n, nnz = mx["n"], mx["nnz"]
    kern = mx["kernels"]
    line = {
        "metric": "pressure+momentum solve ms per repeated solve & HBM GB/s per kernel (c2, mixed, 1e-10 rel res)",
        "value": round(mx["ms"], 3), "unit": "ms/solve pair", "n_gpus": 1, "steps": solves, "warmup": args.warmup,
        "ms_per_step": round(mx["ms"], 3), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 outer / f32 preconditioners", "data": "synthetic",
        "config": {"workload": f"c2: uniform NVB mesh n={n}, nnz={nnz}; {solves} solves, RHS + N(0, 1e-3) noise "
                               "seeded by the solve index (momentum BiCGSTAB2 + pressure PCG)",
                   "l2": "inputs larger than L2; kernels timed alone with a 256 MB L2 flush before each",
                   "iterations_median": [int(np.median([i[c] for i in mx["its"]])) for c in range(3)],
                   "fp64_ms_per_solve_pair": round(f64["ms"], 3),
                   "mixed_speedup_vs_fp64": round(f64["ms"] / mx["ms"], 3),
                   "iterations_median_fp64": [int(np.median([i[c] for i in f64["its"]])) for c in range(3)],
                   "amg_levels": mx["levels"], "pressure_operator_passes": mx["passes"]},
        "kernels": kern,
        "kernels_fp64": f64["kernels"],
        "roofline": {"bound": "hbm", "kernel": "pressure operator (K - B^T M^-1 B, one pass), FP64",
                     "achieved": kern["pressure_operator_fp64"]["gbs"], "peak": hbm, "unit": "GB/s",
                     "frac": kern["pressure_operator_fp64"]["frac"], "traffic": None, "peak_kind": peak_kind},
        "e2e": {"value": round(mx["ms"], 3), "unit": "ms/solve pair", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 48},
        "gpu_launches": int(mx["launches"]),
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


# ------------------------------------------------------------------------------------------------
# adjoint (c3): gradient of the mean drag over 200 BDF2 steps on the c1 mesh
# ------------------------------------------------------------------------------------------------
def run_adjoint(args):
    import torch
    import adjoint as AD
    import cfa_b200 as cfa
    import fixtures as F

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    m = F.make_mesh("c1")
    steps = 200
    u0 = 4 * U_MAX * m.y * (1 - m.y)
    z = np.zeros(m.n)
    nu_node = np.full(m.n, NU)

    stab = args.stab

    def make(prec):
        return AD.DragAdjoint(m, u0, z, z, nu_node, u_max=U_MAX, steps=steps, dt=5e-3, nu=NU, precision=prec,
                              checkpoint=20, tol=1e-12, stab=stab)

    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", 0)))
    adj = make(cfa.MIXED)
    adj.objective()                                   # warm-up: setup, graphs
    torch.cuda.synchronize()
    clk.start()
    t0 = time.perf_counter()
    J = adj.objective()
    torch.cuda.synchronize()
    t_fwd = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    J2, g_nu, g_u = adj.gradient()
    torch.cuda.synchronize()
    t_grad = (time.perf_counter() - t0) * 1e3
    clk.stop()
    # central differences with h = 1e-6 U (the workload's step) and h = 1e-4 U: at 1e-6 the
    # solves' 1e-12 noise in J divided by h is about 1e-7 of dJ/dU; at 1e-4 it and the truncation
    # error (h^2 J'''/6) are both near 1e-8
    fds = {}
    for rel in (1e-6, 1e-4):
        h = rel * U_MAX
        fds[rel] = (adj.objective(U_MAX + h) - adj.objective(U_MAX - h)) / (2 * h)
    ref = make(cfa.FP64)
    J64, g64, gu64 = ref.gradient()
    line = {
        "metric": "adjoint gradient of the mean drag over 200 BDF2 steps (c1 mesh), wall ms per gradient",
        "value": round(t_grad, 1), "unit": "ms/gradient", "n_gpus": 1, "steps": steps, "warmup": 1,
        "ms_per_step": round(t_grad / steps, 3), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 outer / f32 preconditioners", "data": "synthetic",
        "config": {"workload": f"c3: c1 mesh n={m.n}, dt 5e-3, U 1.5, nu 1e-3, from the inflow profile, "
                               f"OSS stab {stab:g}, checkpoints every 20 steps, solves to 1e-12",
                   "forward_ms": round(t_fwd, 1), "J_mean_drag": J,
                   "dJ_dU": g_u, "dJ_dU_central_fd_h1e-6": fds[1e-6], "dJ_dU_central_fd_h1e-4": fds[1e-4],
                   "fd_rel_diff": abs(g_u - fds[1e-6]) / abs(fds[1e-6]),
                   "fd_rel_diff_h1e-4": abs(g_u - fds[1e-4]) / abs(fds[1e-4]),
                   "dJ_dnu_norm": float(torch.linalg.norm(g_nu)),
                   "fp64_grad_rel_diff": float(torch.abs(g_nu - g64).max() / torch.abs(g64).max()),
                   "fp64_dJ_dU_rel_diff": abs(g_u - gu64) / abs(gu64)},
        "e2e": {"value": round(t_grad, 1), "unit": "ms/gradient", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 8},
        "gpu_launches": None,
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


# ------------------------------------------------------------------------------------------------
# batched systems (c4): 64 independent system pairs, 5k-500k vertices, LPT over GPUs
# ------------------------------------------------------------------------------------------------
def run_batch(args, rank, world):
    import torch
    import batch as BT
    import cfa_b200 as cfa

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    count = 64
    targets = [BT.batch_target(s) for s in range(1, count + 1)]
    mine = BT.lpt_partition(targets, world)[rank]
    systems = [BT.batch_system(i + 1) for i in mine]
    # keep=True: every system's solution (u*, v*, dp) is read back to the host inside the timed
    # region, as a caller of the batch would
    solver = BT.BatchSolver(precision=cfa.MIXED, streams=args.streams, keep=True)
    if args.autotune:
        cfa.autotune(True)   # tile heights timed in the warm-up's setups, cached per pattern class
    # warm-up: whole batches (module loading, the worker contexts' first allocations)
    for _ in range(max(1, args.warmup)):
        solver.solve(systems)
    if world > 1:
        torch.distributed.barrier()
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", 0)))
    clk.start()
    walls, reps, launches = [], None, 0
    for _ in range(args.steps):
        rep = solver.solve(systems)
        walls.append(rep.wall_ms)
        reps = rep.systems
        launches += rep.launches
    clk.stop()
    wall = float(np.mean(walls))
    h2d = sum(s.mesh.n * (8 * 2 + 4 + 24) + s.mesh.ne * 12 for s in systems)
    if world > 1:
        t = torch.tensor([wall], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        wall = float(t.item())
    allr = BT.gather_reports(reps)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    value = count / (wall * 1e-3)
    ms = np.array([r.solve_ms for r in allr])
    line = {
        "metric": "batched pressure+momentum system pairs solved per second (64 systems, 5k-500k vertices, "
                  "mixed precision, 1e-10 rel res)",
        "value": round(value, 3), "unit": "systems/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(wall, 3), "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64 outer / f32 preconditioners", "data": "synthetic",
        "config": {"workload": "c4: 64 independent system pairs, seeds 1..64, log-uniform 5k-500k vertices, "
                               "nu log-uniform [5e-4, 5e-3]; per system: assembly, ILU(0), BiCGSTAB2, AMG setup, PCG",
                   "parallelism": f"LPT split over {world} GPU(s), {args.streams} streams per GPU",
                   "l2": "inputs larger than L2 in aggregate (each system's mesh and fields uploaded per solve)",
                   "vertices_total": int(sum(r.n for r in allr)),
                   "p50_ms": round(float(np.percentile(ms, 50)), 3), "p99_ms": round(float(np.percentile(ms, 99)), 3),
                   "converged": int(sum(r.converged for r in allr)),
                   "iterations_p_median": int(np.median([r.it_p for r in allr])),
                   "autotune": {"on": bool(args.autotune), "classes": len(cfa.autotune_log()),
                                "row_shifts": [rec["row_shift"] for rec in cfa.autotune_log()]}},
        "e2e": {"value": round(value, 3), "unit": "systems/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(sum(r.n for r in allr) * 24)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--streams", type=int, default=4, help="concurrent streams per GPU (c4)")
    ap.add_argument("--stab", type=float, default=STAB,
                    help="c3: OSS pressure stabilisation of the differentiated loop (0.3, the reference's default)")
    ap.add_argument("--autotune", action="store_true",
                    help="c4: time the V-cycle tile heights per pattern class (cfa_autotune_set)")
    ap.add_argument("--step", action="store_true",
                    help="c2: time the whole step path (as c1 does) instead of the repeated solve pairs")
    ap.add_argument("--profile-precision", default="both", choices=["both", "fp64", "mixed"],
                    help="--profile: the precision(s) whose step is profiled")
    ap.add_argument("--profile", action="store_true",
                    help="one step per precision between cudaProfilerStart/Stop (for ncu --profile-from-start off); no JSON line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    import torch
    if args.impl == "reference":
        if rank != 0:
            return
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        print(json.dumps(run_reference(args)))
        return
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.workload == "c4":
        run_batch(args, rank, world)
        return
    if args.workload == "c2" and not args.step:
        if rank == 0:
            run_stress(args, rank, world)
        return
    if args.workload == "c3":
        if rank == 0:
            run_adjoint(args)
        return
    m, res = run_ours(args, rank, world)
    if args.profile:
        return
    mixed, fp64 = res["mixed"], res["fp64"]
    value = mixed["step_ms"] + mixed["setup_ms"] / AMG_REBUILD
    value64 = fp64["step_ms"] + fp64["setup_ms"] / AMG_REBUILD
    e2e = mixed["e2e_ms"] + mixed["setup_ms"] / AMG_REBUILD
    if world > 1:
        t = torch.tensor([value, e2e, value64], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        value, e2e, value64 = (float(x) / world for x in t.tolist())
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    n, nnz = mixed["n"], mixed["nnz"]
    hbm, peak_kind = peaks()
    passes, stored_nnz = fp64["op_layout"]
    op_bytes = operator_bytes(n, nnz, passes, stored_nnz)
    op_ms = fp64["op_ms"]
    achieved = op_bytes / (op_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(f"pressure_operator_{args.workload}")
    cpu = None if args.no_cpu else cpu_baseline(m, *workload_inputs(args.workload)[1:])
    clocks = res["clocks"]
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "ms/step", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(value, 4), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 outer / f32 preconditioners", "data": "synthetic",
        "config": {"workload": workload_name(args.workload, n, nnz),
                   "parallelism": "replicas" if world > 1 else "single GPU", "l2": "flushed between steps (256 MB write)",
                   "fp64_ms_per_step": round(value64, 4), "mixed_speedup_vs_fp64": round(value64 / value, 3),
                   "amg_setup_ms": {"mixed": round(mixed["setup_ms"], 3), "fp64": round(fp64["setup_ms"], 3)},
                   "amg_rebuild": AMG_REBUILD, "amg_setup_stat": f"median of {SETUP_REPS} warm setups",
                   "step_ms_without_setup": round(mixed["step_ms"], 4),
                   "iterations_mixed": {"u": mixed["report"]["it_u"], "v": mixed["report"]["it_v"], "p": mixed["report"]["it_p"]},
                   "iterations_fp64": {"u": fp64["report"]["it_u"], "v": fp64["report"]["it_v"], "p": fp64["report"]["it_p"]},
                   "converged": mixed["report"]["conv"] + fp64["report"]["conv"],
                   "amg_levels": mixed["levels"], "ilu_colours": mixed["colours"],
                   "vcycle": {"composite_level": mixed["composite"][0], "composite_rows": mixed["composite"][1],
                              "fused_transfers": os.environ.get("CFA_VC_FUSE", "1")},
                   "amg_setup_phases_ms": {k: round(v, 2) for k, v in mixed["phases"].items()}},
        "e2e": {"value": round(e2e, 4), "unit": "ms/step", "h2d_bytes_per_step": 3 * 8 * n, "d2h_bytes_per_step": 3 * 8 * n},
        "gpu_launches": int(mixed["launches"]),
        "roofline": {"bound": "hbm",
                     "kernel": ("pressure operator K - B^T M^-1 B on the two-ring pattern (k_opt_k), FP64"
                                if passes == 1 else "pressure operator K + OSS, two passes (k_opt_b + k_opt_k), FP64"),
                     "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "traffic": traffic, "peak_kind": peak_kind,
                     "bytes_per_launch": op_bytes, "stored_nnz": stored_nnz, "launch_us": round(op_ms * 1e3, 2)},
        "kernels": mixed["kernels"],
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
