"""cfa_oss_apply_noalloc (static device scratch, no allocation) against cfa_oss_apply.

Both are called through the C ABI on the same assembled OSS operator. Two calls in a row with
different inputs check that the static scratch carries nothing from one call to the next.
Tolerance: 1e-13 relative to the largest |entry| (the two use the same per-row summation order,
so the results are expected to be identical). Around those two calls the device's free memory and
the library's block cache are unchanged: the entry point allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

import fixtures as F

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import cfa_b200 as cfa  # noqa: E402

TOL = 1e-13
MAX_ROWS = 1 << 19


def _oss_operator(ctx, m):
    dm = cfa.DeviceMesh(ctx, m)
    n, ne, nnz = m.n, m.ne, dm.nnz
    f64 = dict(dtype=torch.float64, device="cuda")
    u = torch.from_numpy(F.fourier_field(m.x, m.y, 1)).to("cuda")
    v = torch.from_numpy(F.fourier_field(m.x, m.y, 2)).to("cuda")
    mass = torch.zeros(n, **f64)
    cfa.lumped_mass(ctx, dm, mass)
    s = torch.zeros(ne, **f64)
    cfa.oss_weights(ctx, dm, u, v, 2e-3 / 3, 1.0, 1e-3, 0.3, s)
    oss, inv_m = torch.zeros(4 * nnz, **f64), torch.zeros(n, **f64)
    cfa.assemble_oss(ctx, dm, s, mass, oss, inv_m)
    return dm, oss, inv_m


def _last_error(ctx):
    return cfa.lib().cfa_ctx_last_error(ctx.h).decode()


def _noalloc(ctx, dm, oss, inv_m, x, out):
    return cfa.lib().cfa_oss_apply_noalloc(ctx.h, dm.h, cfa.ptr(oss), cfa.ptr(inv_m), cfa.ptr(x), cfa.ptr(out))


@pytest.mark.parametrize("name", ["small", "medium"])
def test_oss_apply_noalloc_matches_oss_apply(name):
    ctx = cfa.default_context()
    m = F.make_mesh(name)
    dm, oss, inv_m = _oss_operator(ctx, m)
    rng = np.random.default_rng(11)
    base = torch.from_numpy(rng.uniform(-1, 1, m.n)).to("cuda")
    xs = [torch.from_numpy(rng.uniform(-0.5, 0.5, m.n)).to("cuda") for _ in range(2)]
    want, got = [], []
    for x in xs:
        ref = base.clone()
        cfa.oss_apply(ctx, dm, oss, inv_m, x, ref)
        want.append(ref)
    outs = [base.clone() for _ in xs]
    torch.cuda.synchronize()
    # device memory and the library's block cache before and after: the calls allocate nothing
    free0, cached0 = torch.cuda.mem_get_info()[0], cfa.mem_cached()[0]
    for x, out in zip(xs, outs):   # two calls in a row on the same scratch
        st = _noalloc(ctx, dm, oss, inv_m, x, out)
        assert st == cfa.CFA_OK, _last_error(ctx)
        got.append(out)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert cfa.mem_cached()[0] == cached0
    for w, g in zip(want, got):
        w, g = w.cpu().numpy(), g.cpu().numpy()
        assert np.abs(g - w).max() <= TOL * np.abs(w).max()
    assert not np.array_equal(want[0].cpu().numpy(), want[1].cpu().numpy())


def test_oss_apply_noalloc_rejects_meshes_above_its_scratch():
    ctx = cfa.default_context()
    k = 730                                   # (k + 1)^2 = 534361 > 2^19 nodes
    assert (k + 1) ** 2 > MAX_ROWS
    i, j = np.meshgrid(np.arange(k), np.arange(k), indexing="ij")
    a = (i * (k + 1) + j).ravel()
    tri = np.concatenate([np.stack([a, a + k + 1, a + 1], 1), np.stack([a + 1, a + k + 1, a + k + 2], 1)])
    xs, ys = np.meshgrid(np.linspace(0, 1, k + 1), np.linspace(0, 1, k + 1), indexing="ij")
    mesh = F.Mesh(x=xs.ravel().copy(), y=ys.ravel().copy(), tag=np.zeros((k + 1) ** 2, np.int32),
                  tri=tri.astype(np.int32), gen=np.zeros(len(tri), np.int32))
    dm = cfa.DeviceMesh(ctx, mesh)
    n, nnz = mesh.n, dm.nnz
    oss = torch.zeros(4 * nnz, dtype=torch.float64, device="cuda")
    inv_m = torch.ones(n, dtype=torch.float64, device="cuda")
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    out = torch.full((n,), 2.0, dtype=torch.float64, device="cuda")
    st = _noalloc(ctx, dm, oss, inv_m, x, out)
    assert st == cfa.CFA_BAD_ARG
    assert "static scratch" in _last_error(ctx)
    torch.cuda.synchronize()
    assert bool((out == 2.0).all())
