"""Batched solves: many independent pressure + momentum system pairs of uneven sizes.

One system = one time step's solve path on its own mesh (``step.SolveStep``): momentum assembly,
ILU(0) factor, two-component BiCGSTAB, pressure system assembly, SA-AMG setup and PCG, all to the
same relative tolerance.

On one GPU the systems run on ``streams`` concurrent CUDA streams (one host thread and one
``cfa_ctx`` per stream); each thread takes the largest remaining system, so small systems fill
the gaps that large ones leave (longest-processing-time list scheduling). Every solve inside is a
CUDA graph already; concurrency across streams is what lets many small systems share the 148 SMs.

Across GPUs (one process per GPU) the systems are split by an LPT partition on their estimated
cost; the partition needs no communication, and the per-system reports are gathered at the end
(``gather_reports``). Results do not depend on the schedule: each system's kernels run in order
on one stream and every reduction has a fixed order.
"""
from __future__ import annotations

import dataclasses
import heapq
import queue
import threading
import time

import numpy as np

import cfa_b200 as cfa
import fixtures as F
import step as S


@dataclasses.dataclass
class BatchSystem:
    seed: int
    mesh: F.Mesh
    nu: float
    u: np.ndarray
    v: np.ndarray
    p: np.ndarray

    @property
    def cost(self) -> float:
        """Estimated solve cost: matrix entries (about 7 per node on P1 meshes)."""
        return float(self.mesh.n) * 7.0


def batch_target(seed: int, n_min: int = 5_000, n_max: int = 500_000) -> float:
    """The target vertex count of system ``seed`` (its first random draw), known before the mesh
    is made: the cost estimate of the LPT split across GPUs."""
    rng = np.random.default_rng(seed)
    return float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))


def batch_system(seed: int, n_min: int = 5_000, n_max: int = 500_000) -> BatchSystem:
    """System ``seed``: target vertex count log-uniform in [n_min, n_max], reached by uniform NVB
    depth from a seeded base spacing plus bisection rounds inside a seeded radius around the disc;
    viscosity log-uniform in [5e-4, 5e-3]; velocity and pressure fields are seeded Fourier modes."""
    rng = np.random.default_rng(seed)
    target = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
    h = float(rng.uniform(0.045, 0.09))
    radius = float(rng.uniform(0.15, 0.5))
    nu = float(np.exp(rng.uniform(np.log(5e-4), np.log(5e-3))))
    m = F.base_mesh(h=h, seed=seed)
    # uniform rounds while the mesh stays below half the target, then rounds on the elements
    # within `radius` of the disc centre (one more bisection each) until the target is reached
    while m.n * 2 <= target:
        m = F.refine_uniform(m, 1)
    while m.n < target:
        t = m.tri
        cx = (m.x[t[:, 0]] + m.x[t[:, 1]] + m.x[t[:, 2]]) / 3.0
        cy = (m.y[t[:, 0]] + m.y[t[:, 1]] + m.y[t[:, 2]]) / 3.0
        mark = np.hypot(cx - F.XC, cy - F.YC) < radius
        if not mark.any():
            break
        m = F.nvb_round(m, mark)
    m = F.renumber(m)
    u = F.fourier_field(m.x, m.y, 3 * seed + 1)
    v = F.fourier_field(m.x, m.y, 3 * seed + 2)
    p = 0.3 * F.fourier_field(m.x, m.y, 3 * seed + 3)
    return BatchSystem(seed, m, nu, u, v, p)


def batch_systems(count: int = 64, first_seed: int = 1, n_min: int = 5_000, n_max: int = 500_000) -> list:
    return [batch_system(s, n_min, n_max) for s in range(first_seed, first_seed + count)]


def lpt_partition(costs, parts: int) -> list:
    """Longest-processing-time partition: items in decreasing cost (ties by index) each go to the
    currently least loaded part (ties by part index). Returns the item indices of every part."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, k) for k in range(parts)]
    out = [[] for _ in range(parts)]
    for i in order:
        load, k = heapq.heappop(heap)
        out[k].append(i)
        heapq.heappush(heap, (load + costs[i], k))
    return out


@dataclasses.dataclass
class SystemReport:
    seed: int
    n: int
    nnz: int
    solve_ms: float          # device time of the system's whole solve path on its stream
    it_u: int
    it_v: int
    it_p: int
    converged: bool
    rel: list


@dataclasses.dataclass
class BatchReport:
    systems: list
    wall_ms: float
    launches: int = 0        # kernels this library launched for the batch

    @property
    def systems_per_s(self) -> float:
        return len(self.systems) / (self.wall_ms * 1e-3) if self.wall_ms > 0 else 0.0

    def percentile_ms(self, q: float) -> float:
        return float(np.percentile([s.solve_ms for s in self.systems], q)) if self.systems else 0.0


def solve_system(ctx: cfa.Context, sysm: BatchSystem, precision: int, tol: float, reuse=None) -> tuple:
    """The system's solve path on ctx's stream; returns (SolveStep, device ms). ``reuse``: the
    previous system's SolveStep on this context, whose solver handles are taken over."""
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    st = S.SolveStep(sysm.mesh, sysm.u, sysm.v, sysm.p, precision=precision, nu=sysm.nu, tol=tol, ctx=ctx,
                     reuse=reuse)
    # one solve per hierarchy: the plain level chain, whose setup is cheapest (the composite
    # operator and the fused transfers pay back only over repeated solves)
    st.amg.set_vcycle(0, 0, 0)
    st.amg.set_aggregation(0)   # the device aggregation's waiting blocks would hold SMs the other streams use
    st.amg_setup()          # assembly, ILU factor, BiCGSTAB2, pressure system, AMG setup
    st.solve_pressure()
    ev1.record()
    ev1.synchronize()
    return st, ev0.elapsed_time(ev1)


class BatchSolver:
    """Solves batches of systems on ``streams`` worker threads, each with its own context (CUDA
    stream). The contexts live as long as the solver, so the device blocks and workspaces one
    batch grew serve the next one (``close()`` releases them)."""

    def __init__(self, precision: int = cfa.MIXED, streams: int = 4, tol: float = 1e-10, keep: bool = False):
        self.precision, self.streams, self.tol, self.keep = precision, streams, tol, keep
        self.results = {}     # seed -> (u, v, dp) host arrays when keep
        self._ctxs = [None] * max(1, streams)
        self._prev = [None] * max(1, streams)   # each worker's last SolveStep (its handles are reused)

    def close(self):
        self._prev = [None] * len(self._ctxs)
        for i, c in enumerate(self._ctxs):
            if c is not None:
                c.close()
                self._ctxs[i] = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, systems: list) -> BatchReport:
        import torch
        cfa.lib()                                   # load the library before the worker threads
        dev = torch.cuda.current_device()
        work = queue.Queue()
        for i in sorted(range(len(systems)), key=lambda i: (-systems[i].cost, i)):
            work.put(systems[i])
        reports, errors, lock = [], [], threading.Lock()
        launches = [0]

        def worker(k):
            torch.cuda.set_device(dev)
            if self._ctxs[k] is None:
                self._ctxs[k] = cfa.Context()       # own stream, made current in this thread
            ctx = self._ctxs[k]
            torch.cuda.set_stream(ctx.stream)
            launches0 = ctx.launches
            prev = self._prev[k]
            try:
                while True:
                    try:
                        sysm = work.get_nowait()
                    except queue.Empty:
                        return
                    st, ms = solve_system(ctx, sysm, self.precision, self.tol, reuse=prev)
                    prev = None
                    r = st.report()
                    rep = SystemReport(sysm.seed, st.n, st.nnz, ms, r["it_u"], r["it_v"], r["it_p"],
                                       all(r["conv"]), r["rel"])
                    res = (st.u.cpu().numpy(), st.v.cpu().numpy(), st.dp.cpu().numpy()) if self.keep else None
                    with lock:
                        reports.append(rep)
                        if self.keep:
                            self.results[sysm.seed] = res
                    prev = st
            except Exception as e:               # reported to the caller after the join
                with lock:
                    errors.append(e)
            finally:
                self._prev[k] = prev
                torch.cuda.current_stream().synchronize()
                with lock:
                    launches[0] += ctx.launches - launches0

        torch.cuda.synchronize()
        t0 = time.perf_counter()
        threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(self._ctxs))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        if errors:
            raise errors[0]
        reports.sort(key=lambda r: r.seed)
        return BatchReport(reports, wall, launches[0])


def gather_reports(local: list) -> list:
    """All ranks' SystemReports (torch.distributed initialised), sorted by seed."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return sorted(local, key=lambda r: r.seed)
    rows = [dataclasses.asdict(r) for r in local]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, rows)
    return sorted((SystemReport(**d) for part in out for d in part), key=lambda r: r.seed)
