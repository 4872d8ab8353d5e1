"""Discrete adjoint of the BDF2 time loop: the gradient of the time-averaged volume-integral drag

    J = (1/N) sum_{n=1..N} C_D^n,   C_D = force_scale F_x  (k_volume_forces)

with respect to a per-node viscosity field of the momentum equation and the inflow amplitude U,
for the loop of ``step.TimeStepper`` (the rotational pressure update takes the scalar viscosity,
as do the OSS weights). Either outlet rule: p = 0 on the outlet (the default), or
``outlet_dirichlet``, the scaled inflow parabola there and the pressure increment pinned at one
node, whose right-hand side mean removal cfa_ppe_rhs_adjoint transposes. With the OSS pressure
stabilisation (stab > 0) the pressure operator is (1 + s_K) K - B^T M^-1 B with weights s_K of u*,
and its right-hand side carries the OSS terms of p^n; their derivatives go through
cfa_oss_adjoint.

Every solve's backward is the transposed solve: the pressure operator acts symmetrically on the
rows that are not Dirichlet (the adjoint right-hand side is zeroed on the Dirichlet rows, whose
multipliers no derivative uses), so the PCG with the same operator and AMG serves; the momentum system uses BiCGSTAB2 on A^T with the transposed
multicolour ILU. The assembly and the other kernels have adjoint kernels in the library
(cfa_momentum_adjoint, cfa_ppe_rhs_adjoint, cfa_projection_adjoint, cfa_volume_forces_adjoint).
The forward sweep keeps the state every ``checkpoint`` steps (and the records of the last segment,
which the backward sweep needs first); the backward sweep recomputes each earlier segment's steps
from its checkpoint and runs them in reverse. Every backward solve starts from the solution of
the step after it (the adjoint fields change little from step to step).

``direct=True`` solves both systems with a sparse LU on the host instead (for finite-difference
checks that must not carry an iterative tolerance).
"""
from __future__ import annotations

import numpy as np

import cfa_b200 as cfa


class DragAdjoint:
    def __init__(self, mesh, u0, v0, p0, nu_node, u_max=1.5, steps=10, dt=5e-3, nu=1e-3, rho=1.0, tau_time=1e-3,
                 H=1.0, u_mean=1.0, diameter=0.2, precision=cfa.MIXED, tol=1e-12, checkpoint=20, ctx=None,
                 direct=False, stab=0.0, outlet_dirichlet=False):
        import torch
        self.torch = torch
        self.ctx = ctx or cfa.default_context()
        self.dm = cfa.DeviceMesh(self.ctx, mesh)
        self.m = mesh
        n, ne, nnz = self.dm.n, self.dm.ne, self.dm.nnz
        self.n, self.nnz = n, nnz
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")
        self.u0, self.v0, self.p0 = t(u0), t(v0), t(p0)
        self.nu_node = t(nu_node)
        self.u_max, self.steps, self.dt, self.nu, self.rho = float(u_max), steps, dt, nu, rho
        self.tau_time, self.H = tau_time, H
        self.force_scale = -2.0 / (u_mean * u_mean * diameter)
        self.tol, self.checkpoint, self.direct = tol, max(1, checkpoint), direct
        z = lambda k: torch.zeros(k, dtype=torch.float64, device="cuda")
        self.z = z
        self.A, self.AT, self.ru, self.rv, self.mass = z(nnz), z(nnz), z(n), z(n), z(n)
        self.Kp, self.rhs_p, self.div, self.elem_s = z(nnz), z(n), z(n), z(ne)
        self.gdx, self.gdy, self.vort_num, self.vort, self.forces = z(n), z(n), z(n), z(n), z(2)
        self.stab = float(stab)
        self.oss_val, self.inv_m = z(4 * nnz), z(n)
        self.oss = cfa.oss_operator(self.dm, self.oss_val, self.inv_m) if self.stab > 0.0 else None
        tag = np.ascontiguousarray(mesh.tag)
        if outlet_dirichlet:
            # the application's --outlet dirichlet: the scaled inflow parabola at the outlet and the
            # pressure increment pinned at one outlet node (its only Dirichlet row)
            pin, scale = cfa.pinned_outlet(mesh.x, mesh.y, tag, H)
            self.dm.set_outlet(1, pin, scale)
            nd = np.ones(n)
            nd[pin] = 0.0
        else:
            nd = (tag != cfa.BC_OUTLET).astype(np.float64)   # p = 0 on the outlet (the default)
        self.non_dirichlet = t(nd)
        rp, ci = self.dm.host_pattern()
        self.rp_h, self.ci_h = rp, ci
        self.ilu = cfa.MulticolourIlu0(self.ctx, precision)
        self.ilu.set_pattern(n, rp, ci, self.dm.rp, self.dm.ci)
        self.mom = cfa.GpuBicgstab2(self.ctx)
        self.pcg = cfa.GpuLinearSolver(self.ctx)
        self.amg = cfa.AmgPreconditioner(self.ctx, precision)
        # the loop's solves start from the neighbouring step's solution, mostly below the FP64
        # phase's switch already, so the phase would add its setup and launches for nothing
        if precision == cfa.MIXED:
            self.amg.set_fp64_phase(0.0)
        self.amg_ready = False
        self.drag = []

    # -------------------------------------------------------------------------------------------
    def coefficients(self, k):
        """(dt', a0, a1, a2, c1, c2) of step k >= 1 (backward Euler first)."""
        dt = self.dt
        if k > 1:
            return (2.0 / 3.0) * dt, 1.5 / dt, 2.0 / dt, -0.5 / dt, 2.0, -1.0
        return dt, 1.0 / dt, 1.0 / dt, 0.0, 1.0, 0.0

    def _params(self, k):
        dt_p, a0, a1, a2, c1, c2 = self.coefficients(k)
        return cfa.MomentumParams(self.dt, self.nu, self.rho, a0, a1, a2, c1, c2, self.tau_time, 0.5)

    def _lu_solve(self, vals, rhs_list, oss=False):
        """Sparse direct solves with the matrix vals on the pattern; oss: the pressure operator,
        vals - [rows not Dirichlet] B^T M^-1 B from the assembled OSS arrays."""
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl
        shape = (self.n, self.n)
        A = sp.csr_matrix((vals.cpu().numpy(), self.ci_h, self.rp_h), shape=shape)
        if oss:
            o = self.oss_val.cpu().numpy()
            nnz = self.nnz
            Bx = sp.csr_matrix((o[:nnz], self.ci_h, self.rp_h), shape=shape)
            By = sp.csr_matrix((o[nnz:2 * nnz], self.ci_h, self.rp_h), shape=shape)
            Mi = sp.diags(self.inv_m.cpu().numpy())
            S = Bx.T @ Mi @ Bx + By.T @ Mi @ By
            A = A - sp.diags(self.non_dirichlet.cpu().numpy()) @ S
        lu = spl.splu(A.tocsc())
        return [self.torch.from_numpy(lu.solve(r.cpu().numpy())).to("cuda") for r in rhs_list]

    def _assemble_momentum(self, k, u_n, v_n, u_nm1, v_nm1, p_n, x_u, x_v, u_max):
        cfa.assemble_momentum(self.ctx, self.dm, u_n, v_n, u_nm1, v_nm1, p_n, self._params(k), self.A, self.ru,
                              self.rv, self.mass, x_u, x_v, u_max=u_max, H=self.H, nu_node=self.nu_node)

    def _pressure_system(self, k, x_u, x_v, p_n, dp):
        dt_p = self.coefficients(k)[0]
        if self.stab > 0.0:
            cfa.oss_weights(self.ctx, self.dm, x_u, x_v, dt_p, self.rho, self.nu, self.stab, self.elem_s)
            cfa.scalar_gradient(self.ctx, self.dm, p_n, self.elem_s, self.gdx, self.gdy)
        cfa.assemble_pressure_system(self.ctx, self.dm, x_u, x_v, p_n, self.gdx, self.gdy, self.mass, self.elem_s,
                                     dt_p, self.rho, self.stab, self.Kp, self.rhs_p, self.div, dp, self.oss_val,
                                     self.inv_m)
        if not self.amg_ready and not self.direct:
            # built once: the stiffness part of the operator of the first step (with OSS a fixed
            # SPD preconditioner for every step, as the reference reuses it between rebuilds)
            self.amg.setup(self.n, self.nnz, self.dm.rp, self.dm.ci, self.Kp)
            self.amg_ready = True

    def _pressure_solve(self, rhs, x):
        """x = A^-1 rhs with this step's pressure operator (iterative: warm start from x)."""
        if self.direct:
            (sol,) = self._lu_solve(self.Kp, [rhs], oss=self.stab > 0.0)
            x.copy_(sol)
        else:
            self.pcg.solve_pcg(self.n, self.dm.rp, self.dm.ci, self.Kp, rhs, x, 4000, self.tol, self.oss, self.amg)
        return x

    def step(self, k, state, u_max=None):
        """Step k from state (u^n, v^n, u^{n-1}, v^{n-1}, p^n, dp warm start); returns the new state
        and the step's record (its inputs, x*, dp and outputs)."""
        torch = self.torch
        u_max = self.u_max if u_max is None else u_max
        u_n, v_n, u_nm1, v_nm1, p_n, dp_prev = state
        dt_p, a0, a1, a2, c1, c2 = self.coefficients(k)
        x_u, x_v = u_n.clone(), v_n.clone()
        self._assemble_momentum(k, u_n, v_n, u_nm1, v_nm1, p_n, x_u, x_v, u_max)
        if self.direct:
            x_u, x_v = self._lu_solve(self.A, [self.ru, self.rv])
        else:
            self.ilu.factor(self.A)
            self.mom.solve(self.n, self.dm.rp, self.dm.ci, self.A, self.ru, self.rv, x_u, x_v, 2000, self.tol, self.ilu)
        dp = dp_prev.clone()
        self._pressure_system(k, x_u, x_v, p_n, dp)
        self._pressure_solve(self.rhs_p, dp)
        u, v, p = x_u.clone(), x_v.clone(), p_n.clone()
        cfa.project_step(self.ctx, self.dm, dt_p, self.rho, self.rho * self.nu, True, self.mass, dp, self.div, self.gdx,
                         self.gdy, self.vort_num, u, v, p, self.vort)
        cfa.volume_forces(self.ctx, self.dm, u, v, u_n, v_n, u_nm1, v_nm1, p, a0, -a1, -a2, self.nu, self.rho,
                          self.forces)
        drag = self.force_scale * float(self.forces[0].item())
        rec = dict(k=k, u_n=u_n, v_n=v_n, u_nm1=u_nm1, v_nm1=v_nm1, p_n=p_n, x_u=x_u, x_v=x_v, dp=dp, u=u, v=v, p=p)
        return (u, v, u_n, v_n, p, dp), rec, drag

    def initial_state(self):
        return (self.u0.clone(), self.v0.clone(), self.u0.clone(), self.v0.clone(), self.p0.clone(),
                self.z(self.n))

    def objective(self, u_max=None):
        """J alone (no checkpoints kept)."""
        state, total = self.initial_state(), 0.0
        for k in range(1, self.steps + 1):
            state, _, d = self.step(k, state, u_max)
            total += d
        return total / self.steps

    # -------------------------------------------------------------------------------------------
    def gradient(self):
        """(J, dJ/dnu_node [n], dJ/du_max)."""
        torch = self.torch
        N, K = self.steps, self.checkpoint
        checkpoints = {}
        last = 1 + K * ((N - 1) // K)     # first step of the last segment: taped in this sweep
        tape = []
        state, total = self.initial_state(), 0.0
        for k in range(1, N + 1):
            if (k - 1) % K == 0:
                checkpoints[k] = tuple(t.clone() for t in state)
            state, rec, d = self.step(k, state)
            if k >= last:
                tape.append(rec)
            total += d
        J = total / N
        z = self.z
        n = self.n
        gU, gV, gP = z(n), z(n), z(n)                 # adjoints of the outputs of step k
        gU1, gV1, gP1 = z(n), z(n), z(n)              # of step k-1
        gU2, gV2 = z(n), z(n)                         # of step k-2
        g_nu, g_umax = z(n), 0.0
        w = self.force_scale / N
        g_dp, lam_p = z(n), z(n)
        gu_o, gv_o, gu_p, gv_p, gp_o, gnu_k = (z(n) for _ in range(6))
        sc = z(2)
        lam_u, lam_v = z(n), z(n)   # warm starts: each backward solve starts from the later step's
        for start in sorted(checkpoints, reverse=True):
            stop = min(start + K - 1, N)
            if start == last:
                recs, tape = tape, []
            else:
                state = tuple(t.clone() for t in checkpoints[start])
                recs = []
                for k in range(start, stop + 1):
                    state, rec, _ = self.step(k, state)
                    recs.append(rec)
            for rec in reversed(recs):
                k = rec["k"]
                dt_p, a0, a1, a2, c1, c2 = self.coefficients(k)
                # D: the drag of this step
                cfa.volume_forces_adjoint(self.ctx, self.dm, rec["u"], rec["v"], rec["u_n"], rec["v_n"], rec["u_nm1"],
                                          rec["v_nm1"], rec["p"], a0, -a1, -a2, self.nu, self.rho, w, 0.0, gU, gV,
                                          gU1, gV1, gU2, gV2, gP)
                # C: projection
                cfa.projection_adjoint(self.ctx, self.dm, dt_p, self.rho, self.nu, self.mass, gU, gV, gP, g_dp)
                g_us, g_vs = gU.clone(), gV.clone()
                gP1 += gP
                # B: pressure solve (the operator on the rows that are not Dirichlet) and its
                # right-hand side; with OSS also the weights' and the OSS right-hand side's terms
                self._pressure_system(k, rec["x_u"], rec["x_v"], rec["p_n"], rec["dp"].clone())
                self._pressure_solve(g_dp * self.non_dirichlet, lam_p)
                cfa.ppe_rhs_adjoint(self.ctx, self.dm, lam_p, dt_p, self.rho, g_us, g_vs)
                if self.stab > 0.0:
                    cfa.oss_adjoint(self.ctx, self.dm, rec["x_u"], rec["x_v"], dt_p, self.rho, self.nu, self.stab,
                                    self.elem_s, self.mass, lam_p, rec["p_n"], rec["dp"], g_us, g_vs, gP1)
                # A: momentum, transposed solve and the assembly derivatives
                xu0, xv0 = rec["u_n"].clone(), rec["v_n"].clone()
                self._assemble_momentum(k, rec["u_n"], rec["v_n"], rec["u_nm1"], rec["v_nm1"], rec["p_n"], xu0, xv0,
                                        self.u_max)
                if self.direct:
                    import scipy.sparse as sp
                    import scipy.sparse.linalg as spl
                    A = sp.csr_matrix((self.A.cpu().numpy(), self.ci_h, self.rp_h), shape=(n, n)).T.tocsc()
                    lu = spl.splu(A)
                    lam_u = torch.from_numpy(lu.solve(g_us.cpu().numpy())).to("cuda")
                    lam_v = torch.from_numpy(lu.solve(g_vs.cpu().numpy())).to("cuda")
                else:
                    cfa.transpose_values(self.ctx, self.ilu, self.A, self.AT)
                    self.ilu.factor_transposed(self.A)
                    self.mom.solve(n, self.dm.rp, self.dm.ci, self.AT, g_us, g_vs, lam_u, lam_v, 2000, self.tol,
                                   self.ilu)
                cfa.momentum_adjoint(self.ctx, self.dm, rec["u_n"], rec["v_n"], rec["u_nm1"], rec["v_nm1"],
                                     rec["p_n"], self._params(k), self.u_max, self.H, rec["x_u"], rec["x_v"], lam_u,
                                     lam_v, gu_o, gv_o, gu_p, gv_p, gp_o, sc, nu_node=self.nu_node, g_nu_node=gnu_k)
                gU1 += gu_o
                gV1 += gv_o
                gU2 += gu_p
                gV2 += gv_p
                gP1 += gp_o
                g_nu += gnu_k
                g_umax += float(sc[0].item())
                # shift to the previous step
                gU, gV, gP = gU1, gV1, gP1
                gU1, gV1, gP1 = gU2, gV2, z(n)
                gU2, gV2 = z(n), z(n)
        return J, g_nu, g_umax
