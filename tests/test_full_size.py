"""The solve path at the workloads' full sizes, checked through properties that do not depend on
the size: c1 (adaptive mesh, 402k vertices) and c2 (uniform mesh, 4.23M vertices).

At these sizes the oracle takes minutes, so instead of comparing with it the test recomputes
every solve's true residual with an independent FP64 operator (torch sparse matrices built from
the assembled CSR arrays: the momentum matrix, and for the pressure K - diag(not Dirichlet)
(Bx^T M^-1 Bx + By^T M^-1 By), the fused OSS operator of the reference's apply_oss_projection)
and compares the mixed-precision solutions with the FP64 ones. Bars: true relative residuals
below 1e-9 for solves run to 1e-10 (the Krylov recurrences drift by less than a decade), mixed
and FP64 solutions within 1e-7 of each other relative to their size.
"""
import numpy as np
import pytest

import fixtures as F

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore:Sparse:UserWarning")]

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import cfa_b200 as cfa  # noqa: E402
import step as S  # noqa: E402

STAB, DT, NU, U_MAX, TOL = 0.3, 1e-3, 1e-3, 1.5, 1e-10   # the workloads' settings
BC_OUTLET = 2


def _csr(dm, vals):
    return torch.sparse_csr_tensor(dm.rp.long(), dm.ci.long(), vals, size=(dm.n, dm.n))


def _coo_t(dm, vals):
    """The transpose of the CSR matrix vals, as a sparse COO tensor."""
    rows = torch.repeat_interleave(torch.arange(dm.n, device=dm.rp.device), (dm.rp[1:] - dm.rp[:-1]).long())
    idx = torch.stack([dm.ci.long(), rows])
    return torch.sparse_coo_tensor(idx, vals, size=(dm.n, dm.n)).coalesce()


def _mv(A, x):
    return (A @ x.unsqueeze(1)).squeeze(1)


def _pressure_apply(st, x, non_dir):
    dm, nnz = st.dm, st.nnz
    K = _csr(dm, st.Kp)
    bx, by = st.oss_val[:nnz], st.oss_val[nnz:2 * nnz]
    gx = _mv(_csr(dm, bx), x)
    gy = _mv(_csr(dm, by), x)
    s = _mv(_coo_t(dm, bx), st.inv_m * gx) + _mv(_coo_t(dm, by), st.inv_m * gy)
    return _mv(K, x) - non_dir * s


def _rel(r, b):
    return (torch.linalg.norm(r) / torch.linalg.norm(b)).item()


def _solve(m, u, v, p, precision):
    st = S.SolveStep(m, u, v, p, precision=precision, dt=DT, nu=NU, stab=STAB, u_max=U_MAX, tol=TOL)
    st.amg_setup()          # momentum assembly + BiCGSTAB2, pressure system, AMG set-up
    st.solve_pressure()
    torch.cuda.synchronize()
    return st


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_full_size_solves_reach_their_true_residuals(name):
    m = F.make_mesh(name)
    u, v, p = (F.fourier_field(m.x, m.y, 1), F.fourier_field(m.x, m.y, 2), 0.3 * F.fourier_field(m.x, m.y, 3))
    non_dir = torch.from_numpy((np.asarray(m.tag) != BC_OUTLET).astype(np.float64)).to("cuda")
    sols = {}
    for prec in (cfa.MIXED, cfa.FP64):
        st = _solve(m, u, v, p, prec)
        r = st.report()
        assert all(r["conv"]), r
        A = _csr(st.dm, st.A)
        assert _rel(st.rhs_u - _mv(A, st.u), st.rhs_u) <= 1e-9
        assert _rel(st.rhs_v - _mv(A, st.v), st.rhs_v) <= 1e-9
        assert _rel(st.rhs_p - _pressure_apply(st, st.dp, non_dir), st.rhs_p) <= 1e-9
        sols[prec] = (st.u.clone(), st.v.clone(), st.dp.clone())
        del st
    for a, b in zip(sols[cfa.MIXED], sols[cfa.FP64]):
        assert _rel(a - b, b) <= 1e-7
