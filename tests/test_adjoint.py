"""Adjoint of the momentum predictor: transposed solves (BiCGSTAB2 on A^T with the transposed
multicolour ILU) and the dual-number element derivatives, checked against central finite
differences (h = 1e-6 relative) of J = c.u* + d.v*, and the mixed-precision gradient against the
FP64 one. The torch.autograd.Function wrapper lives here, in the test harness only."""
import numpy as np
import pytest

import fixtures as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import cfa_b200 as cfa  # noqa: E402

TOL = 1e-13
DT, U_MAX, H = 5e-3, 1.5, 1.0


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")


class MomentumStep:
    """Step A with parameters theta = (u_old, v_old, u_prev, v_prev, p_old, nu_node, u_max)."""

    def __init__(self, ctx, m, precision):
        self.ctx, self.m = ctx, m
        self.dm = cfa.DeviceMesh(ctx, m)
        rp, ci = self.dm.host_pattern()
        self.ilu = cfa.MulticolourIlu0(ctx, precision)
        self.ilu.set_pattern(m.n, rp, ci, self.dm.rp, self.dm.ci)
        self.solver = cfa.GpuBicgstab2(ctx)
        n, nnz = m.n, self.dm.nnz
        z = lambda k: torch.zeros(k, dtype=torch.float64, device="cuda")
        self.A, self.AT, self.ru, self.rv, self.mass = z(nnz), z(nnz), z(n), z(n), z(n)
        self.prm = cfa.bdf2_params(DT, 1e-3, 1.0, 1e-3, 0.5, True)

    def exact_J(self, th, c, d):
        """J = c.u* + d.v* with the system assembled on the device and solved by a sparse direct
        solver on the host (no iterative-solver tolerance in the finite differences)."""
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl
        u_old, v_old, u_prev, v_prev, p_old, nu, u_max = th
        x_u, x_v = u_old.clone(), v_old.clone()
        cfa.assemble_momentum(self.ctx, self.dm, u_old, v_old, u_prev, v_prev, p_old, self.prm, self.A, self.ru,
                              self.rv, self.mass, x_u, x_v, u_max=u_max, H=H, nu_node=nu)
        rp, ci = self.dm.host_pattern()
        A = sp.csr_matrix((self.A.cpu().numpy(), ci, rp), shape=(self.m.n, self.m.n)).tocsc()
        lu = spl.splu(A)
        xu, xv = lu.solve(self.ru.cpu().numpy()), lu.solve(self.rv.cpu().numpy())
        return float(c.cpu().numpy() @ xu + d.cpu().numpy() @ xv)

    def solve(self, th):
        u_old, v_old, u_prev, v_prev, p_old, nu, u_max = th
        x_u, x_v = u_old.clone(), v_old.clone()
        cfa.assemble_momentum(self.ctx, self.dm, u_old, v_old, u_prev, v_prev, p_old, self.prm, self.A, self.ru,
                              self.rv, self.mass, x_u, x_v, u_max=u_max, H=H, nu_node=nu)
        self.ilu.factor(self.A)
        self.solver.solve(self.m.n, self.dm.rp, self.dm.ci, self.A, self.ru, self.rv, x_u, x_v, 1000, TOL, self.ilu)
        assert all(self.solver.converged)
        return x_u, x_v

    def adjoint(self, th, x_u, x_v, gu, gv):
        u_old, v_old, u_prev, v_prev, p_old, nu, u_max = th
        cfa.transpose_values(self.ctx, self.ilu, self.A, self.AT)
        self.ilu.factor_transposed(self.A)
        lam_u, lam_v = torch.zeros_like(gu), torch.zeros_like(gv)
        self.solver.solve(self.m.n, self.dm.rp, self.dm.ci, self.AT, gu, gv, lam_u, lam_v, 1000, TOL, self.ilu)
        assert all(self.solver.converged)
        out = [torch.zeros_like(gu) for _ in range(6)]
        sc = torch.zeros(2, dtype=torch.float64, device="cuda")
        cfa.momentum_adjoint(self.ctx, self.dm, u_old, v_old, u_prev, v_prev, p_old, self.prm, u_max, H, x_u, x_v,
                             lam_u, lam_v, *out[:5], sc, nu_node=nu, g_nu_node=out[5])
        return lam_u, lam_v, out, float(sc[0].item())


class StepFunction(torch.autograd.Function):
    """x* = (u*, v*) of Step A as a differentiable function of its nodal inputs (u_max fixed)."""

    @staticmethod
    def forward(fctx, step, u_old, v_old, u_prev, v_prev, p_old, nu, u_max):
        th = (u_old, v_old, u_prev, v_prev, p_old, nu, u_max)
        x_u, x_v = step.solve(th)
        fctx.step, fctx.th = step, th
        fctx.save_for_backward(x_u, x_v)
        return x_u.clone(), x_v.clone()

    @staticmethod
    def backward(fctx, gu, gv):
        x_u, x_v = fctx.saved_tensors
        _, _, g, _ = fctx.step.adjoint(fctx.th, x_u, x_v, gu.contiguous(), gv.contiguous())
        return (None, *g, None)


def theta(m):
    f = lambda s: F.fourier_field(m.x, m.y, s)
    u0 = 0.8 + 0.3 * f(11)
    return [dev(u0), dev(0.3 * f(12)), dev(u0 + 0.05 * f(13)), dev(0.3 * f(12) + 0.05 * f(14)), dev(0.2 * f(15)),
            dev(1e-3 * (1.0 + 0.3 * np.sin(3 * m.x) * np.cos(2 * m.y))), U_MAX]


@pytest.mark.parametrize("precision", [cfa.FP64, cfa.MIXED])
def test_momentum_adjoint_matches_finite_differences(precision):
    ctx = cfa.default_context()
    m = F.make_mesh("small")
    st = MomentumStep(ctx, m, precision)
    th = theta(m)
    rng = np.random.default_rng(3)
    c, d = dev(rng.standard_normal(m.n)), dev(rng.standard_normal(m.n))
    x_u, x_v = st.solve(th)
    J0 = st.exact_J(th, c, d)
    st.solve(th)
    lam_u, lam_v, g, g_umax = st.adjoint(th, x_u, x_v, c, d)
    # the adjoint solution solves A^T lambda = c (oracle product with the transposed CSR)
    rp, ci = st.dm.host_pattern()
    A = st.A.cpu().numpy()
    AT = O.csr_transpose((m.n, m.n, rp, ci, A))
    r = O.spmv(AT[2], AT[3], AT[4], lam_u.cpu().numpy()) - c.cpu().numpy()
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(c.cpu().numpy())
    # directional derivatives, central differences (h = 1e-6 of the parameter's scale)
    for k in range(6):
        delta = dev(rng.standard_normal(m.n)) * float(th[k].abs().mean().clamp(min=1e-3))
        h = 1e-6
        tp = list(th); tp[k] = th[k] + h * delta
        tm = list(th); tm[k] = th[k] - h * delta
        fd = (st.exact_J(tp, c, d) - st.exact_J(tm, c, d)) / (2 * h)
        ad = float(torch.dot(g[k], delta))
        assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-6 * abs(J0)), (k, ad, fd)
    h = 1e-6 * U_MAX
    tp, tm = list(th), list(th)
    tp[6], tm[6] = U_MAX + h, U_MAX - h
    fd = (st.exact_J(tp, c, d) - st.exact_J(tm, c, d)) / (2 * h)
    assert abs(g_umax - fd) <= 1e-6 * abs(fd), (g_umax, fd)


def test_mixed_adjoint_matches_fp64_gradient_and_autograd():
    ctx = cfa.default_context()
    m = F.make_mesh("small")
    th = theta(m)
    rng = np.random.default_rng(4)
    c, d = dev(rng.standard_normal(m.n)), dev(rng.standard_normal(m.n))
    grads = []
    for prec in (cfa.FP64, cfa.MIXED):
        st = MomentumStep(ctx, m, prec)
        x_u, x_v = st.solve(th)
        grads.append(st.adjoint(th, x_u, x_v, c, d)[2])
    for a, b in zip(*grads):
        assert torch.abs(a - b).max().item() <= 1e-8 * torch.abs(a).max().item()
    # autograd through the wrapper gives the same gradient
    st = MomentumStep(ctx, m, cfa.FP64)
    leaves = [t.clone().requires_grad_(True) for t in th[:6]]
    xu, xv = StepFunction.apply(st, *leaves, U_MAX)
    (torch.dot(c, xu) + torch.dot(d, xv)).backward()
    for leaf, want in zip(leaves, grads[0]):
        assert torch.abs(leaf.grad - want).max().item() <= 1e-12 * torch.abs(want).max().item()


# ------------------------------------------------------------------------------------------------
# the time loop: gradient of the time-averaged drag
# ------------------------------------------------------------------------------------------------
def _loop_inputs(m):
    f = lambda s: F.fourier_field(m.x, m.y, s)
    u0 = 4 * U_MAX * m.y * (1 - m.y) + 0.1 * f(21)
    v0 = 0.1 * f(22)
    p0 = 0.05 * f(23)
    nu = 1e-3 * (1.0 + 0.2 * np.cos(2 * m.x) * np.sin(3 * m.y))
    return u0, v0, p0, nu


@pytest.mark.parametrize("stab", [0.0, 0.3])
def test_drag_adjoint_matches_finite_differences(stab):
    """dJ/dnu (per node) and dJ/dU of J = mean C_D over 5 BDF2 steps (the first backward Euler),
    with checkpoints every 2 steps, against central differences (h = 1e-6) of J computed with
    direct sparse solves; without and with the OSS pressure stabilisation (0.3, the reference's
    default)."""
    import adjoint as AD
    m = F.make_mesh("small")
    u0, v0, p0, nu = _loop_inputs(m)
    adj = AD.DragAdjoint(m, u0, v0, p0, nu, u_max=U_MAX, steps=5, dt=DT, precision=cfa.FP64, checkpoint=2,
                         direct=True, stab=stab)
    J, g_nu, g_u = adj.gradient()
    assert abs(J - adj.objective()) <= 1e-12 * abs(J)
    rng = np.random.default_rng(7)
    base = adj.nu_node.clone()
    for _ in range(2):
        delta = dev(rng.standard_normal(m.n)) * 1e-3
        # 1e-4 of nu: J's rounding (about 1e-14 through the direct solves) over 2h stays below
        # 1e-6 of the derivative, and the O(h^2) truncation far below it
        h = 1e-4
        adj.nu_node = base + h * delta
        jp = adj.objective()
        adj.nu_node = base - h * delta
        jm = adj.objective()
        adj.nu_node = base
        fd = (jp - jm) / (2 * h)
        ad = float(torch.dot(g_nu, delta))
        assert abs(ad - fd) <= 1e-6 * abs(fd) + 1e-9 * abs(J), (ad, fd)
    h = 1e-6 * U_MAX
    fd = (adj.objective(U_MAX + h) - adj.objective(U_MAX - h)) / (2 * h)
    assert abs(g_u - fd) <= 1e-6 * abs(fd), (g_u, fd)


@pytest.mark.parametrize("stab", [0.0, 0.3])
def test_drag_adjoint_iterative_mixed_matches_direct_fp64(stab):
    """The gradient through the device solvers (FP32 preconditioners, FP64 Krylov, solves to
    1e-12; with OSS the fused operator inside the CG) against the one with direct FP64 solves."""
    import adjoint as AD
    m = F.make_mesh("small")
    u0, v0, p0, nu = _loop_inputs(m)
    ref = AD.DragAdjoint(m, u0, v0, p0, nu, u_max=U_MAX, steps=4, dt=DT, precision=cfa.FP64, checkpoint=3,
                         direct=True, stab=stab)
    J0, g0, gu0 = ref.gradient()
    it = AD.DragAdjoint(m, u0, v0, p0, nu, u_max=U_MAX, steps=4, dt=DT, precision=cfa.MIXED, checkpoint=3,
                        tol=1e-12, stab=stab)
    J1, g1, gu1 = it.gradient()
    assert abs(J1 - J0) <= 1e-9 * abs(J0)
    assert torch.abs(g1 - g0).max().item() <= 1e-6 * torch.abs(g0).max().item()
    assert abs(gu1 - gu0) <= 1e-6 * abs(gu0)


@pytest.mark.parametrize("stab", [0.0, 0.3])
def test_drag_adjoint_pinned_outlet_matches_finite_differences(stab):
    """The same gradient with the application's --outlet dirichlet rule: the scaled inflow parabola
    on the outlet and the pressure increment pinned at the outlet node nearest mid-height, the
    PPE right-hand side losing its mass-weighted mean first (src/cfa/fem_kernels.cuh:493-531).
    Central differences (h = 1e-4 of nu, 1e-6 of U) of J with direct solves."""
    import adjoint as AD
    m = F.make_mesh("small")
    u0, v0, p0, nu = _loop_inputs(m)
    adj = AD.DragAdjoint(m, u0, v0, p0, nu, u_max=U_MAX, steps=4, dt=DT, precision=cfa.FP64, checkpoint=2,
                         direct=True, stab=stab, outlet_dirichlet=True)
    J, g_nu, g_u = adj.gradient()
    assert abs(J - adj.objective()) <= 1e-12 * abs(J)
    rng = np.random.default_rng(9)
    base = adj.nu_node.clone()
    for _ in range(2):
        delta = dev(rng.standard_normal(m.n)) * 1e-3
        h = 1e-4
        adj.nu_node = base + h * delta
        jp = adj.objective()
        adj.nu_node = base - h * delta
        jm = adj.objective()
        adj.nu_node = base
        fd = (jp - jm) / (2 * h)
        ad = float(torch.dot(g_nu, delta))
        assert abs(ad - fd) <= 1e-6 * abs(fd) + 1e-9 * abs(J), (ad, fd)
    h = 1e-6 * U_MAX
    fd = (adj.objective(U_MAX + h) - adj.objective(U_MAX - h)) / (2 * h)
    assert abs(g_u - fd) <= 1e-6 * abs(fd), (g_u, fd)
    # the iterative path (FP32 preconditioners, PCG on the pinned operator) agrees with it
    it = AD.DragAdjoint(m, u0, v0, p0, nu, u_max=U_MAX, steps=4, dt=DT, precision=cfa.MIXED, checkpoint=2,
                        tol=1e-12, stab=stab, outlet_dirichlet=True)
    J1, g1, gu1 = it.gradient()
    assert abs(J1 - J) <= 1e-9 * abs(J)
    assert torch.abs(g1 - g_nu).max().item() <= 1e-6 * torch.abs(g_nu).max().item()
    assert abs(gu1 - g_u) <= 1e-6 * abs(g_u)
