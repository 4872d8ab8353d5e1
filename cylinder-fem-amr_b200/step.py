"""One time step's solve path through the C ABI, in the order of the reference driver's Steps A
and B (src/cylinder_fem_amr.cu:300-475):

  A. momentum assembly + BCs (one row pass), ILU(0) factor, two-component BiCGSTAB;
  B. OSS weights s_K, G(p^n), pressure system (PPE + BCs + OSS operator, one row pass), PCG with
     the OSS term and SA-AMG.

The AMG hierarchy is built by ``amg_setup()`` (the driver rebuilds it every ``amg_rebuild`` = 50
steps, src/cfa/options.cuh:26); ``run()`` does one step. Every ``run()`` starts from the same
state (u* = u^n, dp = 0), so repeated steps do identical work. All device memory is allocated
here once; ``run()`` allocates nothing.
"""
from __future__ import annotations

import numpy as np

import cfa_b200 as cfa


class SolveStep:
    def __init__(self, mesh, u_n, v_n, p_n, precision=cfa.FP64, dt=1e-3, nu=1e-3, rho=1.0, tau_time=1e-3,
                 stab=0.3, u_max=1.5, H=1.0, tol=1e-10, max_it_mom=1000, max_it_p=4000, ctx=None, dm=None,
                 reuse=None):
        """``reuse``: an earlier SolveStep on the same context whose ILU, AMG and Krylov handles
        this one takes over (their device buffers only grow, so a sequence of systems allocates
        nothing once the largest has been seen); the earlier step must not be used afterwards."""
        import torch
        self.ctx = ctx or cfa.default_context()
        self.dm = dm or cfa.DeviceMesh(self.ctx, mesh)
        n, ne, nnz = self.dm.n, self.dm.ne, self.dm.nnz
        self.n, self.ne, self.nnz = n, ne, nnz
        dev = "cuda"
        f64 = dict(dtype=torch.float64, device=dev)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
        self.u_n, self.v_n, self.p_n = t(u_n), t(v_n), t(p_n)
        self.u_prev, self.v_prev = self.u_n.clone(), self.v_n.clone()
        self.u, self.v = self.u_n.clone(), self.v_n.clone()      # u*, v* (initial guess u^n)
        self.A = torch.zeros(nnz, **f64)
        self.rhs_u, self.rhs_v, self.mass = torch.zeros(n, **f64), torch.zeros(n, **f64), torch.zeros(n, **f64)
        self.elem_s = torch.zeros(ne, **f64)
        self.gpx, self.gpy = torch.zeros(n, **f64), torch.zeros(n, **f64)
        self.Kp = torch.zeros(nnz, **f64)
        self.rhs_p, self.div, self.dp = torch.zeros(n, **f64), torch.zeros(n, **f64), torch.zeros(n, **f64)
        self.oss_val = torch.zeros(4 * nnz, **f64)
        self.inv_m = torch.zeros(n, **f64)
        self.prm = cfa.bdf2_params(dt, nu, rho, tau_time, 0.5, True)
        self.dt, self.nu, self.rho, self.stab, self.u_max, self.H = dt, nu, rho, stab, u_max, H
        self.dt_proj = (2.0 / 3.0) * dt
        self.tol, self.max_it_mom, self.max_it_p = tol, max_it_mom, max_it_p
        rp_h, ci_h = self.dm.host_pattern()
        if reuse is not None and reuse.ctx is self.ctx and reuse.precision == precision:
            self.ilu, self.mom, self.solver, self.amg = reuse.ilu, reuse.mom, reuse.solver, reuse.amg
            reuse.ilu = reuse.mom = reuse.solver = reuse.amg = None
        else:
            self.ilu = cfa.MulticolourIlu0(self.ctx, precision)
            self.mom = cfa.GpuBicgstab2(self.ctx)
            self.solver = cfa.GpuLinearSolver(self.ctx)
            self.amg = cfa.AmgPreconditioner(self.ctx, precision)
        self.ilu.set_pattern(n, rp_h, ci_h, self.dm.rp, self.dm.ci)
        self.oss = cfa.oss_operator(self.dm, self.oss_val, self.inv_m) if stab > 0.0 else None
        self.precision = precision
        self.it_p = 0

    def reset(self):
        self.u.copy_(self.u_n)
        self.v.copy_(self.v_n)
        self.dp.zero_()

    def assemble_momentum(self):
        c, d = self.ctx, self.dm
        cfa.assemble_momentum(c, d, self.u_n, self.v_n, self.u_prev, self.v_prev, self.p_n, self.prm, self.A,
                              self.rhs_u, self.rhs_v, self.mass, self.u, self.v, u_max=self.u_max, H=self.H)

    def solve_momentum(self):
        self.ilu.factor(self.A)
        self.mom.solve(self.n, self.dm.rp, self.dm.ci, self.A, self.rhs_u, self.rhs_v, self.u, self.v,
                       self.max_it_mom, self.tol, self.ilu)

    def assemble_pressure(self):
        c, d = self.ctx, self.dm
        if self.stab > 0.0:
            cfa.oss_weights(c, d, self.u, self.v, self.dt_proj, self.rho, self.nu, self.stab, self.elem_s)
            cfa.scalar_gradient(c, d, self.p_n, self.elem_s, self.gpx, self.gpy)
        cfa.assemble_pressure_system(c, d, self.u, self.v, self.p_n, self.gpx, self.gpy, self.mass, self.elem_s,
                                     self.dt_proj, self.rho, self.stab, self.Kp, self.rhs_p, self.div, self.dp,
                                     self.oss_val, self.inv_m)

    def solve_pressure(self):
        self.it_p = self.solver.solve_pcg(self.n, self.dm.rp, self.dm.ci, self.Kp, self.rhs_p, self.dp, self.max_it_p,
                                          self.tol, self.oss, self.amg)

    def amg_setup(self) -> float:
        """Assembles the pressure operator of this state and builds the hierarchy; returns ms."""
        self.reset()
        self.assemble_momentum()
        self.solve_momentum()
        self.assemble_pressure()
        self.amg.setup(self.n, self.nnz, self.dm.rp, self.dm.ci, self.Kp)
        return self.amg.setup_ms

    def run(self, host_out=None):
        """One step's solves. ``host_out`` = (u, v, dp) pinned host tensors: the momentum solution
        is copied out on a side stream while the pressure system is assembled and solved (both only
        read it), dp after its solve; the context's stream waits for the side copy, so one
        synchronisation of it covers all three."""
        import torch
        self.reset()
        self.assemble_momentum()
        self.solve_momentum()
        side = None
        if host_out is not None:
            if getattr(self, "_copy_stream", None) is None:
                self._copy_stream = torch.cuda.Stream()
            side = self._copy_stream
            ready = torch.cuda.Event()
            ready.record(self.ctx.stream)
            side.wait_event(ready)
            with torch.cuda.stream(side):
                host_out[0].copy_(self.u, non_blocking=True)
                host_out[1].copy_(self.v, non_blocking=True)
        self.assemble_pressure()
        self.solve_pressure()
        if side is not None:
            host_out[2].copy_(self.dp, non_blocking=True)
            joined = torch.cuda.Event()
            joined.record(side)
            self.ctx.stream.wait_event(joined)

    def report(self) -> dict:
        return dict(it_u=self.mom.iters[0], it_v=self.mom.iters[1], it_p=self.it_p,
                    conv=[bool(self.mom.converged[0]), bool(self.mom.converged[1]), bool(self.solver.converged)],
                    rel=[self.mom.last_rel_residual[0], self.mom.last_rel_residual[1], self.solver.last_rel_residual])


class TimeStepper:
    """The reference driver's time loop on one fixed mesh (src/cylinder_fem_amr.cu:276-520):
    BDF2 incremental pressure correction in rotational form, first step backward Euler.

      history: u_prev <- u_old <- u;
      A. momentum assembly + BCs, ILU(0), BiCGSTAB2 (u, v) from u^n;
      B. OSS weights, G(p^n), pressure system, AMG rebuilt every ``amg_rebuild`` steps, PCG from
         the last dp;
      C. div_num = -(dt'/rho) K dp (rotational term from the increment), grad dp, vorticity,
         u -= dt'/rho M^-1 grad dp, p += dp - rho nu M^-1 div_num;
      D. volume-integral drag and lift, C_D = force_scale F_x, C_L = force_scale F_y.

    Everything stays on the device; ``step()`` returns (C_D, C_L) (one 16-byte read per step)."""

    def __init__(self, mesh, u0, v0, p0, precision=cfa.FP64, dt=1e-3, nu=1e-3, rho=1.0, tau_time=1e-3, stab=0.3,
                 u_max=1.5, H=1.0, u_mean=1.0, diameter=0.2, tol_mom=1e-7, tol_p=1e-7, max_it_mom=150,
                 max_it_p=4000, amg_rebuild=50, rotational=True, bdf2=True, ctx=None, dm=None):
        import torch
        self.ctx = ctx or cfa.default_context()
        self.dm = dm or cfa.DeviceMesh(self.ctx, mesh)
        n, ne, nnz = self.dm.n, self.dm.ne, self.dm.nnz
        self.n, self.ne, self.nnz = n, ne, nnz
        f64 = dict(dtype=torch.float64, device="cuda")
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")
        self.u, self.v, self.p = t(u0), t(v0), t(p0)
        self.u_old, self.v_old = self.u.clone(), self.v.clone()
        self.u_prev, self.v_prev = self.u.clone(), self.v.clone()
        z = lambda k: torch.zeros(k, **f64)
        self.A, self.rhs_u, self.rhs_v, self.mass = z(nnz), z(n), z(n), z(n)
        self.elem_s, self.gpx, self.gpy = z(ne), z(n), z(n)
        self.Kp, self.rhs_p, self.div, self.dp = z(nnz), z(n), z(n), z(n)
        self.oss_val, self.inv_m = z(4 * nnz), z(n)
        self.vort_num, self.vort = z(n), z(n)
        self.forces = z(2)
        self.dt, self.nu, self.rho, self.tau_time, self.stab = dt, nu, rho, tau_time, stab
        self.u_max, self.H = u_max, H
        self.force_scale = -2.0 / (u_mean * u_mean * diameter)
        self.tol_mom, self.tol_p, self.max_it_mom, self.max_it_p = tol_mom, tol_p, max_it_mom, max_it_p
        self.amg_rebuild, self.rotational, self.bdf2 = amg_rebuild, rotational, bdf2
        rp_h, ci_h = self.dm.host_pattern()
        self.ilu = cfa.MulticolourIlu0(self.ctx, precision)
        self.ilu.set_pattern(n, rp_h, ci_h, self.dm.rp, self.dm.ci)
        self.mom = cfa.GpuBicgstab2(self.ctx)
        self.solver = cfa.GpuLinearSolver(self.ctx)
        self.amg = cfa.AmgPreconditioner(self.ctx, precision)
        self.oss = cfa.oss_operator(self.dm, self.oss_val, self.inv_m) if stab > 0.0 else None
        self.step_no = 0
        self.amg_built = None
        self.iters = []

    def coefficients(self):
        """(dt', a0, a1, a2, c1, c2) of this step (src/cylinder_fem_amr.cu:288-294)."""
        dt = self.dt
        bdf2 = self.bdf2 and self.step_no > 1
        if bdf2:
            return (2.0 / 3.0) * dt, 1.5 / dt, 2.0 / dt, -0.5 / dt, 2.0, -1.0
        return dt, 1.0 / dt, 1.0 / dt, 0.0, 1.0, 0.0

    def step(self):
        c, d = self.ctx, self.dm
        self.step_no += 1
        dt_proj, a0, a1, a2, c1, c2 = self.coefficients()
        self.u_prev.copy_(self.u_old)
        self.v_prev.copy_(self.v_old)
        self.u_old.copy_(self.u)
        self.v_old.copy_(self.v)
        # A
        prm = cfa.MomentumParams(self.dt, self.nu, self.rho, a0, a1, a2, c1, c2,
                            self.tau_time if self.tau_time > 0.0 else self.dt, 0.5)
        cfa.assemble_momentum(c, d, self.u_old, self.v_old, self.u_prev, self.v_prev, self.p, prm, self.A,
                              self.rhs_u, self.rhs_v, self.mass, self.u, self.v, u_max=self.u_max, H=self.H)
        self.ilu.factor(self.A)
        self.mom.solve(self.n, d.rp, d.ci, self.A, self.rhs_u, self.rhs_v, self.u, self.v, self.max_it_mom,
                       self.tol_mom, self.ilu)
        # B
        if self.stab > 0.0:
            cfa.oss_weights(c, d, self.u, self.v, dt_proj, self.rho, self.nu, self.stab, self.elem_s)
            cfa.scalar_gradient(c, d, self.p, self.elem_s, self.gpx, self.gpy)
        cfa.assemble_pressure_system(c, d, self.u, self.v, self.p, self.gpx, self.gpy, self.mass, self.elem_s,
                                     dt_proj, self.rho, self.stab, self.Kp, self.rhs_p, self.div, self.dp,
                                     self.oss_val, self.inv_m)
        if self.amg_built is None or self.step_no - self.amg_built >= self.amg_rebuild:
            self.amg.setup(self.n, self.nnz, d.rp, d.ci, self.Kp)
            self.amg_built = self.step_no
        it_p = self.solver.solve_pcg(self.n, d.rp, d.ci, self.Kp, self.rhs_p, self.dp, self.max_it_p, self.tol_p,
                                     self.oss, self.amg)
        self.iters.append((self.mom.iters[0], self.mom.iters[1], it_p))
        # C
        rot_coeff = self.rho * self.nu if self.rotational else 0.0
        cfa.project_step(c, d, dt_proj, self.rho, rot_coeff, True, self.mass, self.dp, self.div, self.gpx, self.gpy,
                         self.vort_num, self.u, self.v, self.p, self.vort)
        # D
        cfa.volume_forces(c, d, self.u, self.v, self.u_old, self.v_old, self.u_prev, self.v_prev, self.p, a0, -a1,
                          -a2, self.nu, self.rho, self.forces)
        f = self.forces.cpu().numpy()
        return self.force_scale * f[0], self.force_scale * f[1]


def project_divergence_free(ctx, dm, dt, u, v, p, mass, amg=None, tol=1e-8, rho=1.0):
    """project_divergence_free (src/cfa/device.cuh:413-461): K phi = -(rho/dt) (N_i, div u) with the
    outlet rows eliminated, then u -= (dt/rho) M^-1 grad phi (p unchanged). u, v updated in place;
    returns (PCG iterations, nodal vorticity of the projected field). amg: a hierarchy of K to
    reuse (set up here when it has none yet)."""
    import torch
    n, nnz, ne = dm.n, dm.nnz, dm.ne
    z = lambda k: torch.zeros(k, dtype=torch.float64, device="cuda")
    Kp, rhs, div, phi = z(nnz), z(n), z(n), z(n)
    gx, gy, vn, vort = z(n), z(n), z(n), z(n)
    cfa.lumped_mass(ctx, dm, mass)
    cfa.assemble_pressure_system(ctx, dm, u, v, p, gx, gy, mass, z(ne), dt, rho, 0.0, Kp, rhs, div, phi, z(4 * nnz),
                                 z(n))
    if amg is not None and amg.h is None:
        amg.setup(n, nnz, dm.rp, dm.ci, Kp)
    it = cfa.GpuLinearSolver(ctx).solve_pcg(n, dm.rp, dm.ci, Kp, rhs, phi, 4000, tol, None, amg)
    cfa.grad_dp_vorticity(ctx, dm, phi, u, v, gx, gy, vn)
    cfa.velocity_pressure_correction(ctx, dm, dt, rho, 0.0, 0.0, div, mass, gx, gy, vn, phi, u, v, p, vort)
    return it, vort


def project_scheme_consistent(ctx, dm, dt_proj, stab, nu, u_old, v_old, u, v, p, amg=None, both_levels=True,
                              tol=1e-8, rho=1.0):
    """project_scheme_consistent (src/cfa/device.cuh:337-405): after a remesh, each velocity level
    (u^{n-1} and u^n, or u^n only) is projected with the time step's own pressure operator (PPE
    with the OSS term for weights of the current u, G(p^n)), p unchanged. Fields updated in place;
    returns the PCG iterations. The AMG hierarchy is set up on the first level's operator."""
    import torch
    n, nnz, ne = dm.n, dm.nnz, dm.ne
    z = lambda k: torch.zeros(k, dtype=torch.float64, device="cuda")
    mass, elem_s, Kp, rhs, div, dp = z(n), z(ne), z(nnz), z(n), z(n), z(n)
    gpx, gpy, gx, gy, vn, vort = z(n), z(n), z(n), z(n), z(n), z(n)
    oss_val, inv_m = z(4 * nnz), z(n)
    cfa.lumped_mass(ctx, dm, mass)
    if stab > 0.0:
        cfa.oss_weights(ctx, dm, u, v, dt_proj, rho, nu, stab, elem_s)
    oss = cfa.oss_operator(dm, oss_val, inv_m) if stab > 0.0 else None
    solver = cfa.GpuLinearSolver(ctx)
    iters = 0
    levels = ((u_old, v_old), (u, v)) if both_levels else ((u, v),)
    for k, (fu, fv) in enumerate(levels):
        dp.zero_()
        if stab > 0.0:
            cfa.scalar_gradient(ctx, dm, p, elem_s, gpx, gpy)
        cfa.assemble_pressure_system(ctx, dm, fu, fv, p, gpx, gpy, mass, elem_s, dt_proj, rho, stab, Kp, rhs, div, dp,
                                     oss_val, inv_m)
        if amg is not None and k == 0:
            amg.setup(n, nnz, dm.rp, dm.ci, Kp)
        iters += solver.solve_pcg(n, dm.rp, dm.ci, Kp, rhs, dp, 4000, tol, oss, amg)
        cfa.grad_dp_vorticity(ctx, dm, dp, fu, fv, gx, gy, vn)
        cfa.velocity_pressure_correction(ctx, dm, dt_proj, rho, 0.0, 0.0, div, mass, gx, gy, vn, dp, fu, fv, p, vort)
    return iters
