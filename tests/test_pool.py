"""The block cache behind the library's device buffers (csrc/pool.cu), through the C ABI.

A context's buffers return their blocks to the context's stream when a handle is destroyed or
grows; later allocations on that stream take them back, and the solve results do not depend on
which blocks they got. Results are compared bit for bit (same kernels, same reduction order).
"""
import numpy as np
import pytest

import fixtures as F

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import cfa_b200 as cfa  # noqa: E402
import step as S  # noqa: E402


def _solve(ctx, m, u, v, p, reuse=None):
    st = S.SolveStep(m, u, v, p, precision=cfa.MIXED, ctx=ctx, reuse=reuse)
    st.amg_setup()
    st.solve_pressure()
    torch.cuda.current_stream().synchronize()
    return st, (st.u.cpu().numpy(), st.v.cpu().numpy(), st.dp.cpu().numpy())


def _fields(m, seed):
    return (F.fourier_field(m.x, m.y, 3 * seed + 1), F.fourier_field(m.x, m.y, 3 * seed + 2),
            0.3 * F.fourier_field(m.x, m.y, 3 * seed + 3))


def test_cached_blocks_are_reused_and_results_do_not_change():
    small, medium = F.make_mesh("small"), F.make_mesh("medium")
    prev_stream = torch.cuda.current_stream()
    ctx = cfa.Context()                          # its own stream, made torch's current one
    try:
        st, first = _solve(ctx, medium, *_fields(medium, 1))
        before = cfa.mem_cached()[0]
        del st                                   # handles destroyed: their blocks go to ctx's stream
        held = cfa.mem_cached()[0]
        assert held > before
        # a smaller system, then the first one again, on the recycled blocks
        st, _ = _solve(ctx, small, *_fields(small, 2))
        st, again = _solve(ctx, medium, *_fields(medium, 1), reuse=st)
        for a, b in zip(first, again):
            assert np.array_equal(a, b)
        del st
        # the same system on another context (other blocks) gives the same bits
        ctx2 = cfa.Context()
        try:
            _, fresh = _solve(ctx2, medium, *_fields(medium, 1))
            for a, b in zip(first, fresh):
                assert np.array_equal(a, b)
        finally:
            ctx2.close()                         # its stream's blocks become idle
            torch.cuda.set_stream(ctx.stream)
        ctx.trim()                               # ctx's blocks and the idle ones go back to the device
        assert cfa.mem_cached()[0] < held
    finally:
        ctx.close()
        torch.cuda.set_stream(prev_stream)
