"""ctypes access to the oracle (CPU restatement) and to the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` as the checker and
by bench.py's CPU-baseline and reference legs. Never imported by the product package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_I = np.int32
_D = np.float64


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.c_void_p)


def _load(path):
    lib = C.CDLL(path)
    return lib


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        from . import build as _b  # type: ignore
        _lib = _load(_b.build_oracle())
        _lib.or_dot.restype = C.c_double
        for name in ("or_ilu_create", "or_amg_setup"):
            getattr(_lib, name).restype = C.c_void_p
        for name in ("or_ilu_colours", "or_ilu_factor", "or_ilu_apply", "or_ilu_free", "or_ilu_export",
                     "or_amg_num_levels", "or_amg_level_info", "or_amg_level_agg", "or_amg_level_csr",
                     "or_amg_level_dinv", "or_amg_coarse_n", "or_amg_coarse", "or_amg_apply", "or_amg_free"):
            getattr(_lib, name).argtypes = None
    return _lib


def ref():
    """The reference's own code (host parts run anywhere; GPU parts need a GPU)."""
    global _ref
    if _ref is None:
        from . import build as _b  # type: ignore
        path = _b.build_ref()
        if path is None:
            raise RuntimeError("reference harness library not built")
        _ref = _load(path)
        _ref.ref_spectral_radius.restype = C.c_double
        _ref.ref_amg_host_setup.restype = C.c_void_p
        _ref.ref_amg_host_omega.restype = C.c_double
        _ref.ref_step_create.restype = C.c_void_p
        _ref.ref_step_amg_setup.restype = C.c_double
        _ref.ref_step_run.restype = C.c_double
        for name in ("ref_amg_host_levels", "ref_amg_host_level", "ref_amg_host_omega",
                     "ref_amg_host_coarse_inv", "ref_amg_host_free", "ref_step_amg_setup", "ref_step_run",
                     "ref_step_systems", "ref_step_free"):
            getattr(_ref, name).argtypes = None
    return _ref


def i32(a):
    return np.ascontiguousarray(a, dtype=_I)


def f64(a):
    return np.ascontiguousarray(a, dtype=_D)


# ---------------------------------------------------------------------------------------------
# CSR
# ---------------------------------------------------------------------------------------------
def csr_build(n, elem_v):
    ev = i32(elem_v)
    ne = ev.size // 3
    rp = np.zeros(n + 1, _I)
    nnz = lib().or_csr_count(n, ne, _p(ev), _p(rp))
    ci = np.zeros(nnz, _I)
    lib().or_csr_fill(n, ne, _p(ev), _p(rp), _p(ci))
    return rp, ci


def spmv(rp, ci, val, x):
    n = rp.size - 1
    y = np.zeros(n, _D)
    lib().or_spmv(n, _p(i32(rp)), _p(i32(ci)), _p(f64(val)), _p(f64(x)), _p(y))
    return y


def csr_multiply(A, B):
    """A, B: (rows, cols, rp, ci, v) tuples. Reference host SpGEMM order."""
    ar, ac, arp, aci, av = A
    br, bc, brp, bci, bv = B
    crp = np.zeros(ar + 1, _I)
    nnz = lib().or_csr_multiply(ar, ac, _p(arp), _p(aci), _p(av), bc, _p(brp), _p(bci), _p(bv), _p(crp), None, None)
    cci = np.zeros(nnz, _I)
    cv = np.zeros(nnz, _D)
    lib().or_csr_multiply(ar, ac, _p(arp), _p(aci), _p(av), bc, _p(brp), _p(bci), _p(bv), _p(crp), _p(cci), _p(cv))
    return (ar, bc, crp, cci, cv)


def csr_transpose(A):
    rows, cols, rp, ci, v = A
    trp = np.zeros(cols + 1, _I)
    tci = np.zeros(ci.size, _I)
    tv = np.zeros(ci.size, _D)
    lib().or_csr_transpose(rows, cols, _p(rp), _p(ci), _p(v), _p(trp), _p(tci), _p(tv))
    return (cols, rows, trp, tci, tv)


# ---------------------------------------------------------------------------------------------
# assembly
# ---------------------------------------------------------------------------------------------
class MomParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("dt", "nu", "rho", "a0", "a1", "a2", "c1", "c2", "tau_time", "skew_coef")]


def bdf2_params(dt=1e-3, nu=1e-3, rho=1.0, tau_time=1e-3, skew=0.5, bdf2=True):
    if bdf2:
        return MomParams(dt, nu, rho, 1.5 / dt, 2.0 / dt, -0.5 / dt, 2.0, -1.0, tau_time, skew)
    return MomParams(dt, nu, rho, 1.0 / dt, 1.0 / dt, 0.0, 1.0, 0.0, tau_time, skew)


def assemble_momentum(mesh, rp, ci, u_old, v_old, u_prev, v_prev, p_old, prm):
    n, ne = mesh.n, mesh.ne
    A = np.zeros(rp[-1], _D)
    ru, rv, m = np.zeros(n, _D), np.zeros(n, _D), np.zeros(n, _D)
    lib().or_assemble_momentum(n, ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(f64(u_old)),
                               _p(f64(v_old)), _p(f64(u_prev)), _p(f64(v_prev)), _p(f64(p_old)), C.byref(prm),
                               _p(rp), _p(ci), _p(A), _p(ru), _p(rv), _p(m))
    return A, ru, rv, m


def apply_bc_momentum(mesh, rp, ci, A, ru, rv, u, v, u_max=1.5, H=1.0, outlet_dirichlet=0, outlet_scale=1.0):
    lib().or_apply_bc_momentum(mesh.n, _p(i32(mesh.tag)), _p(f64(mesh.y)), C.c_double(u_max), C.c_double(H),
                               outlet_dirichlet, C.c_double(outlet_scale), _p(rp), _p(ci), _p(A), _p(ru), _p(rv),
                               _p(u), _p(v))


def oss_weights(mesh, u, v, dt, rho, nu, stab):
    s = np.zeros(mesh.ne, _D)
    lib().or_oss_weights(mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(f64(u)), _p(f64(v)),
                         C.c_double(dt), C.c_double(rho), C.c_double(nu), C.c_double(stab), _p(s))
    return s


def scalar_gradient(mesh, f, elem_s):
    gx, gy = np.zeros(mesh.n, _D), np.zeros(mesh.n, _D)
    lib().or_scalar_gradient(mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(f64(f)),
                             _p(f64(elem_s)) if elem_s is not None else None, _p(gx), _p(gy))
    return gx, gy


def lumped_mass(mesh):
    m = np.zeros(mesh.n, _D)
    lib().or_lumped_mass(mesh.n, mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(m))
    return m


def stiffness_apply(mesh, f, c, out):
    """out += c (grad N_i, grad f) (k_stiffness_apply)."""
    lib().or_stiffness_apply(mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(f64(f)), C.c_double(c),
                             _p(out))


def grad_dp_vorticity(mesh, dp, u, v):
    gdx, gdy, vn = np.zeros(mesh.n, _D), np.zeros(mesh.n, _D), np.zeros(mesh.n, _D)
    lib().or_grad_dp_vorticity(mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(f64(dp)), _p(f64(u)),
                               _p(f64(v)), _p(gdx), _p(gdy), _p(vn))
    return gdx, gdy, vn


def velocity_pressure_correction(mesh, dt, rho, p_update, rot_coeff, div_num, mass, gdx, gdy, vort_num, dp, u, v, p,
                                 outlet_dirichlet=0):
    """u, v, p updated in place (float64 arrays); returns vort."""
    vort = np.zeros(mesh.n, _D)
    lib().or_velocity_pressure_correction(mesh.n, _p(i32(mesh.tag)), outlet_dirichlet, C.c_double(dt),
                                          C.c_double(rho), C.c_double(p_update), C.c_double(rot_coeff),
                                          _p(f64(div_num)), _p(f64(mass)), _p(f64(gdx)), _p(f64(gdy)),
                                          _p(f64(vort_num)), _p(f64(dp)), _p(u), _p(v), _p(p), _p(vort))
    return vort


def volume_forces(mesh, u, v, u_old, v_old, u_prev, v_prev, p, b0, b1, b2, nu, rho):
    out = np.zeros(2, _D)
    lib().or_volume_forces(mesh.ne, _p(mesh.elem_v), _p(i32(mesh.tag)), _p(f64(mesh.x)), _p(f64(mesh.y)),
                           _p(f64(u)), _p(f64(v)), _p(f64(u_old)), _p(f64(v_old)), _p(f64(u_prev)), _p(f64(v_prev)),
                           _p(f64(p)), C.c_double(b0), C.c_double(b1), C.c_double(b2), C.c_double(nu),
                           C.c_double(rho), _p(out))
    return out


def amr_indicators(mesh, u, v, u_max, H, mass):
    """(grad_rec [4 n], elem_error [2 ne]) of k_accumulate_recovered_gradient and
    k_compute_amr_error_indicator."""
    g = np.zeros(4 * mesh.n, _D)
    lib().or_recovered_gradient(mesh.n, mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(f64(u)),
                                _p(f64(v)), C.c_double(u_max), C.c_double(H), _p(g))
    err = np.zeros(2 * mesh.ne, _D)
    lib().or_amr_error_indicator(mesh.n, mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(g),
                                 _p(f64(mass)), _p(err))
    return g, err


def assemble_ppe(mesh, rp, ci, u, v, p, gpx, gpy, mass, elem_s, dt, rho, stab):
    Kp = np.zeros(rp[-1], _D)
    rhs, div = np.zeros(mesh.n, _D), np.zeros(mesh.n, _D)
    lib().or_assemble_ppe(mesh.n, mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(f64(u)), _p(f64(v)),
                          _p(f64(p)), _p(f64(gpx)), _p(f64(gpy)), _p(f64(mass)), _p(f64(elem_s)), C.c_double(dt),
                          C.c_double(rho), C.c_double(stab), _p(rp), _p(ci), _p(Kp), _p(rhs), _p(div))
    return Kp, rhs, div


def apply_bc_pressure(mesh, rp, ci, Kp, rhs, dp, mass, outlet_dirichlet=0, pin=-1):
    lib().or_apply_bc_pressure(mesh.n, _p(i32(mesh.tag)), outlet_dirichlet, pin, _p(rp), _p(ci), _p(Kp), _p(rhs),
                               _p(dp), _p(f64(mass)))


def assemble_oss(mesh, rp, ci, elem_s, mass):
    oss = np.zeros(4 * rp[-1], _D)
    inv_m = np.zeros(mesh.n, _D)
    lib().or_assemble_oss(mesh.n, mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(f64(elem_s)),
                          _p(rp), _p(ci), _p(f64(mass)), _p(oss), _p(inv_m))
    return oss, inv_m


def oss_apply(mesh, rp, ci, oss, inv_m, x, out, outlet_dirichlet=0, pin=-1):
    lib().or_oss_apply(mesh.n, _p(rp), _p(ci), _p(oss), _p(inv_m), _p(i32(mesh.tag)), outlet_dirichlet, pin,
                       _p(f64(x)), _p(out))


def oss_matrix_free(mesh, elem_s, mass, x, out, outlet_dirichlet=0, pin=-1):
    lib().or_oss_matrix_free(mesh.n, mesh.ne, _p(mesh.elem_v), _p(f64(mesh.x)), _p(f64(mesh.y)), _p(i32(mesh.tag)),
                             outlet_dirichlet, pin, _p(f64(elem_s)), _p(f64(mass)), _p(f64(x)), _p(out))


# ---------------------------------------------------------------------------------------------
# ILU, AMG, Krylov
# ---------------------------------------------------------------------------------------------
class Report(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("rel_residual", C.c_double)]


class Ilu:
    def __init__(self, rp, ci):
        self.rp, self.ci = i32(rp), i32(ci)
        self.n = self.rp.size - 1
        self.h = lib().or_ilu_create(self.n, _p(self.rp), _p(self.ci))
        if not self.h:
            raise ValueError("row longer than 32 entries")
        self.h = C.c_void_p(self.h)
        self.nc = lib().or_ilu_colours(self.h)
        n = self.n
        nlnu = np.zeros(2, _I)
        lib().or_ilu_export(self.h, None, None, None, None, None, None, None, None, None, None, _p(nlnu))
        self.nl, self.nu = int(nlnu[0]), int(nlnu[1])
        self.colour = np.zeros(n, _I)
        self.colour_start = np.zeros(self.nc + 1, _I)
        self.rows = np.zeros(n, _I)
        self.lp, self.up = np.zeros(n + 1, _I), np.zeros(n + 1, _I)
        self.lc, self.uc = np.zeros(self.nl, _I), np.zeros(self.nu, _I)
        self.l_src, self.u_src = np.zeros(self.nl, _I), np.zeros(self.nu, _I)
        self.d_src = np.zeros(n, _I)
        lib().or_ilu_export(self.h, _p(self.colour), _p(self.colour_start), _p(self.rows), _p(self.lp), _p(self.up),
                            _p(self.lc), _p(self.uc), _p(self.l_src), _p(self.u_src), _p(self.d_src), None)

    def factor(self, val):
        lu = np.zeros(self.rp[-1], _D)
        lv, uv, dinv = np.zeros(self.nl, _D), np.zeros(self.nu, _D), np.zeros(self.n, _D)
        lib().or_ilu_factor(self.h, _p(f64(val)), _p(lu), _p(lv), _p(uv), _p(dinv))
        return lu, lv, uv, dinv

    def apply(self, r, nrhs=1):
        z = np.zeros(self.n * nrhs, _D)
        lib().or_ilu_apply(self.h, _p(f64(r)), _p(z), nrhs)
        return z

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_ilu_free(self.h)
            self.h = None


class Amg:
    def __init__(self, rp, ci, val, theta=0.08, smooth_steps=2, coarse_target=300, max_levels=15):
        self.opts = (theta, smooth_steps, coarse_target, max_levels)
        self.remaps = 0
        self._setup(rp, ci, val)

    def remap(self, rp, ci, val, new_to_old):
        """AmgPreconditioner::remap (src/cfa/linalg.cuh:1074-1157); sets up anew when nothing can be
        reused, as the reference does."""
        rp, ci, val, n2o = i32(rp), i32(ci), f64(val), i32(new_to_old)
        n = rp.size - 1
        if lib().or_amg_remap(self.h, n, _p(rp), _p(ci), _p(val), _p(n2o)):
            self.rp, self.ci, self.val, self.n = rp, ci, val, n
            self.remaps += 1
            return True
        lib().or_amg_free(self.h)
        self.h = None
        self._setup(rp, ci, val)
        return False

    def _setup(self, rp, ci, val):
        theta, smooth_steps, coarse_target, max_levels = self.opts
        self.rp, self.ci, self.val = i32(rp), i32(ci), f64(val)
        n = self.rp.size - 1
        h = lib().or_amg_setup(n, _p(self.rp), _p(self.ci), _p(self.val), C.c_double(theta), smooth_steps,
                               coarse_target, max_levels)
        if not h:
            raise ValueError("coarse operator not SPD")
        self.h = C.c_void_p(h)
        self.n = n
        self.nlev = lib().or_amg_num_levels(self.h)
        self.coarse_n = lib().or_amg_coarse_n(self.h)

    def level(self, l):
        info = np.zeros(4, _I)
        om = C.c_double()
        lib().or_amg_level_info(self.h, l, _p(info), C.byref(om))
        rows, annz, pcols, pnnz = (int(v) for v in info)
        out = {"rows": rows, "omega": om.value, "pcols": pcols}
        for which, name, r, c, z in ((0, "A", rows, rows, annz), (1, "P", rows, pcols, pnnz), (2, "R", pcols, rows, pnnz)):
            rp = np.zeros(r + 1, _I)
            ci = np.zeros(z, _I)
            v = np.zeros(z, _D)
            lib().or_amg_level_csr(self.h, l, which, _p(rp), _p(ci), _p(v))
            out[name] = (r, c, rp, ci, v)
        agg = np.zeros(rows, _I)
        lib().or_amg_level_agg(self.h, l, _p(agg))
        dinv = np.zeros(rows, _D)
        lib().or_amg_level_dinv(self.h, l, _p(dinv))
        out["agg"] = agg
        out["dinv"] = dinv
        return out

    def coarse(self):
        cn = self.coarse_n
        A = np.zeros(cn * cn, _D)
        inv = np.zeros(cn * cn, _D)
        lib().or_amg_coarse(self.h, _p(A), _p(inv))
        return A.reshape(cn, cn), inv.reshape(cn, cn)

    def apply(self, r):
        z = np.zeros(self.n, _D)
        lib().or_amg_apply(self.h, _p(f64(r)), _p(z))
        return z

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_amg_free(self.h)
            self.h = None


def pcg(rp, ci, val, b, x0, max_iter=4000, tol=1e-7, oss=None, inv_m=None, tag=None, amg=None,
        outlet_dirichlet=0, pin=-1):
    n = rp.size - 1
    x = f64(x0).copy()
    rep = Report()
    lib().or_pcg(n, _p(i32(rp)), _p(i32(ci)), _p(f64(val)), _p(f64(b)), _p(x), max_iter, C.c_double(tol),
                 _p(oss) if oss is not None else None, _p(inv_m) if inv_m is not None else None,
                 _p(i32(tag)) if tag is not None else None, outlet_dirichlet, pin,
                 amg.h if amg is not None else None, C.byref(rep))
    return x, rep


def bicgstab(rp, ci, val, b, x0, max_iter=200, tol=1e-7):
    n = rp.size - 1
    x = f64(x0).copy()
    rep = Report()
    lib().or_bicgstab(n, _p(i32(rp)), _p(i32(ci)), _p(f64(val)), _p(f64(b)), _p(x), max_iter, C.c_double(tol),
                      C.byref(rep))
    return x, rep


def bicgstab2(rp, ci, val, bu, bv, xu0, xv0, ilu, max_iter=150, tol=1e-7):
    n = rp.size - 1
    xu, xv = f64(xu0).copy(), f64(xv0).copy()
    reps = (Report * 2)()
    lib().or_bicgstab2(n, _p(i32(rp)), _p(i32(ci)), _p(f64(val)), _p(f64(bu)), _p(f64(bv)), _p(xu), _p(xv),
                       max_iter, C.c_double(tol), ilu.h, reps)
    return xu, xv, (reps[0], reps[1])


class Stepper:
    """The reference driver's time loop on a fixed mesh (src/cylinder_fem_amr.cu:276-520), CPU
    restatement: the oracle of the device time stepper (same steps, same order, same options:
    BDF2 after a backward Euler first step, rotational pressure update from the increment, OSS,
    AMG rebuilt every ``amg_rebuild`` steps)."""

    def __init__(self, mesh, u0, v0, p0, dt=1e-3, nu=1e-3, rho=1.0, tau_time=1e-3, stab=0.3, u_max=1.5, H=1.0,
                 u_mean=1.0, diameter=0.2, tol_mom=1e-7, tol_p=1e-7, max_it_mom=150, max_it_p=4000,
                 amg_rebuild=50, rotational=True, bdf2=True):
        self.m = mesh
        self.rp, self.ci = csr_build(mesh.n, mesh.elem_v)
        self.u, self.v, self.p = f64(u0).copy(), f64(v0).copy(), f64(p0).copy()
        self.u_old, self.v_old = self.u.copy(), self.v.copy()
        self.u_prev, self.v_prev = self.u.copy(), self.v.copy()
        self.dp = np.zeros(mesh.n)
        self.dt, self.nu, self.rho, self.tau_time, self.stab = dt, nu, rho, tau_time, stab
        self.u_max, self.H = u_max, H
        self.force_scale = -2.0 / (u_mean * u_mean * diameter)
        self.tol_mom, self.tol_p, self.max_it_mom, self.max_it_p = tol_mom, tol_p, max_it_mom, max_it_p
        self.amg_rebuild, self.rotational, self.bdf2 = amg_rebuild, rotational, bdf2
        self.ilu = Ilu(self.rp, self.ci)
        self.amg, self.amg_built, self.step_no = None, None, 0
        self.iters = []

    def step(self):
        m, rp, ci = self.m, self.rp, self.ci
        self.step_no += 1
        dt = self.dt
        if self.bdf2 and self.step_no > 1:
            dt_proj, a0, a1, a2, c1, c2 = (2.0 / 3.0) * dt, 1.5 / dt, 2.0 / dt, -0.5 / dt, 2.0, -1.0
        else:
            dt_proj, a0, a1, a2, c1, c2 = dt, 1.0 / dt, 1.0 / dt, 0.0, 1.0, 0.0
        self.u_prev, self.v_prev = self.u_old.copy(), self.v_old.copy()
        self.u_old, self.v_old = self.u.copy(), self.v.copy()
        prm = MomParams(dt, self.nu, self.rho, a0, a1, a2, c1, c2, self.tau_time if self.tau_time > 0 else dt, 0.5)
        A, ru, rv, mass = assemble_momentum(m, rp, ci, self.u_old, self.v_old, self.u_prev, self.v_prev, self.p, prm)
        u, v = self.u_old.copy(), self.v_old.copy()
        apply_bc_momentum(m, rp, ci, A, ru, rv, u, v, self.u_max, self.H)
        self.ilu.factor(A)
        u, v, (ru_rep, rv_rep) = bicgstab2(rp, ci, A, ru, rv, u, v, self.ilu, self.max_it_mom, self.tol_mom)
        s = oss_weights(m, u, v, dt_proj, self.rho, self.nu, self.stab) if self.stab > 0 else np.zeros(m.ne)
        gx, gy = scalar_gradient(m, self.p, s) if self.stab > 0 else (np.zeros(m.n), np.zeros(m.n))
        Kp, rhs, div = assemble_ppe(m, rp, ci, u, v, self.p, gx, gy, mass, s, dt_proj, self.rho, self.stab)
        apply_bc_pressure(m, rp, ci, Kp, rhs, self.dp, mass)
        oss, inv_m = assemble_oss(m, rp, ci, s, mass) if self.stab > 0 else (None, None)
        if self.amg_built is None or self.step_no - self.amg_built >= self.amg_rebuild:
            self.amg = Amg(rp, ci, Kp)
            self.amg_built = self.step_no
        self.dp, prep = pcg(rp, ci, Kp, rhs, self.dp, self.max_it_p, self.tol_p, oss, inv_m, m.tag, self.amg)
        self.iters.append((ru_rep.iterations, rv_rep.iterations, prep.iterations))
        div_num = np.zeros(m.n)
        stiffness_apply(m, self.dp, -dt_proj / self.rho, div_num)
        gdx, gdy, vn = grad_dp_vorticity(m, self.dp, u, v)
        rot = self.rho * self.nu if self.rotational else 0.0
        self.vort = velocity_pressure_correction(m, dt_proj, self.rho, 1.0, rot, div_num, mass, gdx, gdy, vn, self.dp,
                                                 u, v, self.p)
        self.u, self.v = u, v
        f = volume_forces(m, u, v, self.u_old, self.v_old, self.u_prev, self.v_prev, self.p, a0, -a1, -a2, self.nu,
                          self.rho)
        return self.force_scale * f[0], self.force_scale * f[1]


def project_divergence_free(mesh, rp, ci, dt, u, v, tol=1e-8, rho=1.0):
    """project_divergence_free (src/cfa/device.cuh:413-461): u, v updated in place; returns phi."""
    n = mesh.n
    mass = lumped_mass(mesh)
    z = np.zeros(n)
    Kp, rhs, div = assemble_ppe(mesh, rp, ci, u, v, z, z, z, mass, np.zeros(mesh.ne), dt, rho, 0.0)
    phi = np.zeros(n)
    apply_bc_pressure(mesh, rp, ci, Kp, rhs, phi, mass)
    phi, rep = pcg(rp, ci, Kp, rhs, phi, 4000, tol, amg=Amg(rp, ci, Kp))
    gx, gy, vn = grad_dp_vorticity(mesh, phi, u, v)
    velocity_pressure_correction(mesh, dt, rho, 0.0, 0.0, div, mass, gx, gy, vn, phi, u, v, np.zeros(n))
    return phi


def project_scheme_consistent(mesh, rp, ci, dt_proj, stab, nu, levels, p, tol=1e-8, rho=1.0):
    """project_scheme_consistent (src/cfa/device.cuh:337-405): each (u, v) pair of `levels`
    projected in place with the step's pressure operator; p unchanged."""
    n = mesh.n
    mass = lumped_mass(mesh)
    s = oss_weights(mesh, levels[-1][0], levels[-1][1], dt_proj, rho, nu, stab) if stab > 0 else np.zeros(mesh.ne)
    oss, inv_m = assemble_oss(mesh, rp, ci, s, mass) if stab > 0 else (None, None)
    amg = None
    for k, (u, v) in enumerate(levels):
        gx, gy = scalar_gradient(mesh, p, s) if stab > 0 else (np.zeros(n), np.zeros(n))
        Kp, rhs, div = assemble_ppe(mesh, rp, ci, u, v, p, gx, gy, mass, s, dt_proj, rho, stab)
        dp = np.zeros(n)
        apply_bc_pressure(mesh, rp, ci, Kp, rhs, dp, mass)
        if k == 0:
            amg = Amg(rp, ci, Kp)
        dp, rep = pcg(rp, ci, Kp, rhs, dp, 4000, tol, oss, inv_m, mesh.tag, amg)
        gdx, gdy, vn = grad_dp_vorticity(mesh, dp, u, v)
        velocity_pressure_correction(mesh, dt_proj, rho, 0.0, 0.0, div, mass, gdx, gdy, vn, dp, u, v, p.copy())
