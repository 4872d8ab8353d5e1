"""Batched solves of independent system pairs (config c4): the system generator, the LPT split
across GPUs and the report gather over two processes (gloo, CPU), and on a GPU the multi-stream
batch against one-at-a-time solves of the same systems."""
import os
import socket

import numpy as np
import pytest

import batch as B


def test_lpt_partition_balances_and_covers():
    costs = [9.0, 7.0, 6.0, 5.0, 4.0, 3.0, 2.0, 2.0, 1.0]
    parts = B.lpt_partition(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    # deterministic, largest first, ties by index
    assert parts == B.lpt_partition(costs, 3)
    assert parts[0][0] == 0 and parts[1][0] == 1 and parts[2][0] == 2
    assert B.lpt_partition([1.0, 1.0], 4) == [[0], [1], [], []]


def test_batch_systems_are_seeded_and_sized():
    a = B.batch_system(5, n_min=2_000, n_max=20_000)
    b = B.batch_system(5, n_min=2_000, n_max=20_000)
    assert np.array_equal(a.mesh.tri, b.mesh.tri) and a.nu == b.nu and np.array_equal(a.u, b.u)
    sizes = [B.batch_system(s, n_min=2_000, n_max=20_000).mesh.n for s in range(1, 7)]
    assert min(sizes) >= 2_000 and max(sizes) <= 2 * 20_000
    assert len(set(sizes)) > 3
    nus = [B.batch_system(s, n_min=2_000, n_max=4_000).nu for s in range(1, 5)]
    assert all(5e-4 <= nu <= 5e-3 for nu in nus)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [float(7 * (1000 + 37 * s)) for s in range(1, 11)]
        mine = B.lpt_partition(costs, world)[rank]
        local = [B.SystemReport(seed=i + 1, n=1000 + 37 * (i + 1), nnz=7, solve_ms=float(i), it_u=1, it_v=1,
                                it_p=2, converged=True, rel=[0.0, 0.0, 0.0]) for i in mine]
        allr = B.gather_reports(local)
        out.put((rank, [r.seed for r in allr], [r.seed for r in local]))
    finally:
        dist.destroy_process_group()


def test_lpt_split_and_gather_over_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    for _, allseeds, _ in got:
        assert allseeds == list(range(1, 11))
    assert sorted(got[0][2] + got[1][2]) == list(range(1, 11)) and not set(got[0][2]) & set(got[1][2])


@pytest.mark.gpu
def test_multistream_batch_matches_single_solves():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cfa_b200 as cfa
    systems = [B.batch_system(s, n_min=3_000, n_max=30_000) for s in range(1, 7)]
    solver = B.BatchSolver(precision=cfa.MIXED, streams=3, keep=True)
    rep = solver.solve(systems)
    assert [r.seed for r in rep.systems] == list(range(1, 7))
    assert all(r.converged for r in rep.systems)
    assert rep.systems_per_s > 0 and rep.percentile_ms(99) >= rep.percentile_ms(50) > 0
    ctx = cfa.default_context()
    for sysm in systems[:3]:
        st, _ = B.solve_system(ctx, sysm, cfa.MIXED, 1e-10)
        u, v, dp = solver.results[sysm.seed]
        assert np.array_equal(st.u.cpu().numpy(), u) and np.array_equal(st.v.cpu().numpy(), v)
        assert np.array_equal(st.dp.cpu().numpy(), dp)
