"""Python host side of cfa_b200: ctypes bindings of the C ABI (include/cfa_b200.h) and classes
that mirror the reference's C++ solver interface (src/cfa/linalg.cuh): ``GpuLinearSolver``
(solve_pcg, solve_bicgstab), ``MulticolourIlu0`` (set_pattern, factor, apply), ``GpuBicgstab2``
(solve) and ``AmgPreconditioner`` (setup, apply), with the same argument meaning and result
fields (converged, last_rel_residual, iters ...). Device memory is torch CUDA tensors (plumbing);
every computation runs in the CUDA library, which must be built (``build.py``): importing this
module on a machine without it raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcfa_b200.so")

CFA_OK, CFA_NOT_CONVERGED, CFA_BREAKDOWN, CFA_ROW_TOO_LONG, CFA_COARSE_NOT_SPD = 0, 1, 2, 3, 4
CFA_CUDA_ERROR, CFA_TIMEOUT, CFA_BAD_ARG, CFA_NO_MEMORY = 5, 6, 7, 8
FP64, MIXED = 0, 1

_lib = None


def lib():
    """The CUDA library (loaded once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"cfa_b200 CUDA library missing: {LIB_PATH} (run build.py)")
        L = C.CDLL(LIB_PATH)
        L.cfa_ctx_last_error.restype = C.c_char_p
        L.cfa_status_string.restype = C.c_char_p
        L.cfa_ctx_kernel_launches.restype = C.c_longlong
        _lib = L
    return _lib


def mem_cached() -> tuple:
    """(device bytes, pinned host bytes) held by the library's block cache."""
    d, h = C.c_size_t(), C.c_size_t()
    s = lib().cfa_mem_cached(C.byref(d), C.byref(h))
    if s != CFA_OK:
        raise CfaError(s, "cfa_mem_cached")
    return d.value, h.value


class CfaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"cfa status {status}: {msg}")
        self.status = status


class MomentumParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("dt", "nu", "rho", "a0", "a1", "a2", "c1", "c2", "tau_time", "skew_coef")]


class MomentumBc(C.Structure):
    _fields_ = [("u_max", C.c_double), ("H", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("tol", C.c_double)]


class SolveReport(C.Structure):
    _fields_ = [("iterations", C.c_int * 2), ("converged", C.c_int * 2), ("rel_residual", C.c_double * 2),
                ("solve_ms", C.c_double)]


class AmgOpts(C.Structure):
    _fields_ = [("theta", C.c_double), ("smooth_steps", C.c_int), ("coarse_target", C.c_int),
                ("max_levels", C.c_int), ("precision", C.c_int)]


class OssOperator(C.Structure):
    _fields_ = [("mesh", C.c_void_p), ("d_oss_val", C.c_void_p), ("d_inv_m", C.c_void_p)]


def bdf2_params(dt=1e-3, nu=1e-3, rho=1.0, tau_time=1e-3, skew=0.5, bdf2=True):
    """Coefficients of the driver's time levels (src/cylinder_fem_amr.cu:284-289)."""
    if bdf2:
        return MomentumParams(dt, nu, rho, 1.5 / dt, 2.0 / dt, -0.5 / dt, 2.0, -1.0, tau_time, skew)
    return MomentumParams(dt, nu, rho, 1.0 / dt, 1.0 / dt, 0.0, 1.0, 0.0, tau_time, skew)


def ptr(t):
    """Device (or host numpy) address of a tensor/array, None passes NULL."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return C.c_void_p(t.ctypes.data)
    return C.c_void_p(t.data_ptr())


class Context:
    """One cfa_ctx bound to a CUDA stream (default: torch's current stream)."""

    def __init__(self, stream=None):
        import torch
        if stream is None:
            # a dedicated stream, made torch's current one so tensor work and library kernels
            # are ordered on it (solves are captured as CUDA graphs, which the legacy stream
            # does not allow)
            stream = torch.cuda.Stream()
            torch.cuda.set_stream(stream)
        self.stream = stream
        h = C.c_void_p()
        s = lib().cfa_ctx_create(C.c_void_p(stream.cuda_stream), C.byref(h))
        if s != CFA_OK:
            raise CfaError(s, "cfa_ctx_create failed")
        self.h = h

    def check(self, status, allow=(CFA_OK,)):
        if status not in allow:
            raise CfaError(status, lib().cfa_ctx_last_error(self.h).decode())
        return status

    @property
    def launches(self) -> int:
        return int(lib().cfa_ctx_kernel_launches(self.h))

    def sync(self):
        self.check(lib().cfa_ctx_sync(self.h))

    def trim(self):
        """Synchronises and returns this context's cached device blocks (and the idle ones)."""
        self.check(lib().cfa_mem_trim(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().cfa_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def autotune(enabled: bool = True):
    """Turns the V-cycle tile autotuner on or off for the AMG setups that follow."""
    lib().cfa_autotune_set(1 if enabled else 0)


def autotune_log() -> list:
    """The autotuner's choices so far, one dict per tuned pattern class."""
    import json
    n = C.c_size_t()
    lib().cfa_autotune_log(None, 0, C.byref(n))
    buf = C.create_string_buffer(n.value + 1)
    lib().cfa_autotune_log(buf, n.value + 1, C.byref(n))
    return [json.loads(line) for line in buf.value.decode().splitlines() if line.strip()]


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context()
    return _default_ctx


# ---------------------------------------------------------------------------------------------
# CSR pattern and mesh
# ---------------------------------------------------------------------------------------------
def csr_build(ctx: Context, n: int, d_elem_v):
    """build_csr_and_boundary_topology (src/cfa/mesh.cuh:198-249) on the device."""
    import torch
    dev = d_elem_v.device
    rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    nnz = C.c_int()
    ne = d_elem_v.numel() // 3
    ctx.check(lib().cfa_csr_count(ctx.h, n, ne, ptr(d_elem_v), ptr(rp), C.byref(nnz)))
    ci = torch.empty(nnz.value, dtype=torch.int32, device=dev)
    ctx.check(lib().cfa_csr_fill(ctx.h, n, ne, ptr(d_elem_v), ptr(rp), ptr(ci)))
    return rp, ci


# node tags (src/cfa/mesh.cuh:62-70)
BC_INTERIOR, BC_INLET, BC_OUTLET, BC_WALL, BC_CYLINDER = 0, 1, 2, 3, 4


def pinned_outlet(x, y, tag, H: float = 1.0):
    """(pin, scale) of the application's ``--outlet dirichlet`` rule (src/cfa/device.cuh:153-171):
    the pressure increment is pinned at the outlet node nearest mid-height, and the outlet
    parabola is scaled by the ratio of the trapezoidal fluxes of the unit parabola through the
    inlet and the outlet nodes (the corners y = 0, H counted with zero velocity)."""
    import numpy as np
    x, y, tag = np.asarray(x), np.asarray(y), np.asarray(tag)
    out = np.flatnonzero(tag == BC_OUTLET)
    if out.size == 0:
        raise ValueError("pinned outlet: the mesh has no outlet node")
    # first node of least distance in index order, as the application's strict '<' scan
    pin = int(out[np.argmin(np.abs(y[out] - 0.5 * H))])

    def flux(t):
        ys = np.sort(np.concatenate([[0.0, H], y[tag == t]]))
        prof = ys * (H - ys)
        q = 0.0
        for k in range(1, ys.size):
            q += 0.5 * (ys[k] - ys[k - 1]) * (prof[k] + prof[k - 1])
        return q

    return pin, flux(BC_INLET) / flux(BC_OUTLET)


class DeviceMesh:
    """The device mesh of DeviceMeshBuffers (src/cfa/device.cuh:21-59) plus the assembly plan."""

    def __init__(self, ctx: Context, mesh, rp=None, ci=None, device="cuda"):
        import torch
        self.ctx = ctx
        self.n, self.ne = mesh.n, mesh.ne
        self.elem_v = torch.from_numpy(np.ascontiguousarray(mesh.tri.reshape(-1).astype(np.int32))).to(device)
        self.x = torch.from_numpy(np.ascontiguousarray(mesh.x, dtype=np.float64)).to(device)
        self.y = torch.from_numpy(np.ascontiguousarray(mesh.y, dtype=np.float64)).to(device)
        self.tag = torch.from_numpy(np.ascontiguousarray(mesh.tag, dtype=np.int32)).to(device)
        if rp is None:
            rp, ci = csr_build(ctx, self.n, self.elem_v)
        self.rp, self.ci = rp, ci
        self.nnz = int(ci.numel())
        h = C.c_void_p()
        ctx.check(lib().cfa_mesh_create(ctx.h, self.n, self.ne, ptr(self.elem_v), ptr(self.x), ptr(self.y),
                                        ptr(self.tag), ptr(self.rp), ptr(self.ci), C.byref(h)))
        self.h = h

    def host_pattern(self):
        return self.rp.cpu().numpy(), self.ci.cpu().numpy()

    def set_outlet(self, outlet_dirichlet: int, pin: int, scale: float):
        s = lib().cfa_mesh_set_outlet(self.h, outlet_dirichlet, pin, C.c_double(scale))
        if s != CFA_OK:
            raise CfaError(s, "cfa_mesh_set_outlet")

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().cfa_mesh_destroy(self.h)
                self.h = None
        except Exception:
            pass


# ---------------------------------------------------------------------------------------------
# assembly
# ---------------------------------------------------------------------------------------------
def assemble_momentum(ctx, m: DeviceMesh, u_old, v_old, u_prev, v_prev, p_old, prm, A_val, rhs_u, rhs_v, mass,
                      u=None, v=None, u_max=None, H=1.0, nu_node=None):
    bc = MomentumBc(u_max, H) if u_max is not None else None
    if nu_node is None:
        ctx.check(lib().cfa_assemble_momentum(ctx.h, m.h, ptr(u_old), ptr(v_old), ptr(u_prev), ptr(v_prev), ptr(p_old),
                                              C.byref(prm), C.byref(bc) if bc is not None else None, ptr(A_val),
                                              ptr(rhs_u), ptr(rhs_v), ptr(mass), ptr(u), ptr(v)))
    else:
        ctx.check(lib().cfa_assemble_momentum_nu(ctx.h, m.h, ptr(u_old), ptr(v_old), ptr(u_prev), ptr(v_prev),
                                                 ptr(p_old), C.byref(prm), ptr(nu_node),
                                                 C.byref(bc) if bc is not None else None, ptr(A_val), ptr(rhs_u),
                                                 ptr(rhs_v), ptr(mass), ptr(u), ptr(v)))


def momentum_adjoint(ctx, m: DeviceMesh, u_old, v_old, u_prev, v_prev, p_old, prm, u_max, H, x_u, x_v, lam_u, lam_v,
                     g_u_old, g_v_old, g_u_prev, g_v_prev, g_p_old, scalars2, nu_node=None, g_nu_node=None):
    """cfa_momentum_adjoint: node gradients (overwritten) and scalars2 = [dJ/du_max, dJ/dnu]."""
    bc = MomentumBc(u_max, H)
    ctx.check(lib().cfa_momentum_adjoint(ctx.h, m.h, ptr(u_old), ptr(v_old), ptr(u_prev), ptr(v_prev), ptr(p_old),
                                         C.byref(prm), ptr(nu_node), C.byref(bc), ptr(x_u), ptr(x_v), ptr(lam_u),
                                         ptr(lam_v), ptr(g_u_old), ptr(g_v_old), ptr(g_u_prev), ptr(g_v_prev),
                                         ptr(g_p_old), ptr(g_nu_node), ptr(scalars2)))


def ppe_rhs_adjoint(ctx, m: DeviceMesh, lam_p, dt_proj, rho, g_u, g_v):
    ctx.check(lib().cfa_ppe_rhs_adjoint(ctx.h, m.h, ptr(lam_p), C.c_double(dt_proj), C.c_double(rho), ptr(g_u),
                                        ptr(g_v)))


def oss_adjoint(ctx, m: DeviceMesh, u_star, v_star, dt_proj, rho, nu, stab, elem_s, mass, lam_p, p_old, dp, g_u, g_v,
                g_p):
    """Adds the OSS terms' derivatives of lambda^T (rhs_p - A dp) to g_u, g_v (u*, v*) and g_p (p^n)."""
    ctx.check(lib().cfa_oss_adjoint(ctx.h, m.h, ptr(u_star), ptr(v_star), C.c_double(dt_proj), C.c_double(rho),
                                    C.c_double(nu), C.c_double(stab), ptr(elem_s), ptr(mass), ptr(lam_p), ptr(p_old),
                                    ptr(dp), ptr(g_u), ptr(g_v), ptr(g_p)))


def projection_adjoint(ctx, m: DeviceMesh, dt_proj, rho, nu, mass, g_u_new, g_v_new, g_p_new, g_dp):
    ctx.check(lib().cfa_projection_adjoint(ctx.h, m.h, C.c_double(dt_proj), C.c_double(rho), C.c_double(nu), ptr(mass),
                                           ptr(g_u_new), ptr(g_v_new), ptr(g_p_new), ptr(g_dp)))


def volume_forces_adjoint(ctx, m: DeviceMesh, u, v, u_old, v_old, u_prev, v_prev, p, b0, b1, b2, nu, rho, wx, wy,
                          g_u, g_v, g_u_old, g_v_old, g_u_prev, g_v_prev, g_p):
    ctx.check(lib().cfa_volume_forces_adjoint(ctx.h, m.h, ptr(u), ptr(v), ptr(u_old), ptr(v_old), ptr(u_prev),
                                              ptr(v_prev), ptr(p), C.c_double(b0), C.c_double(b1), C.c_double(b2),
                                              C.c_double(nu), C.c_double(rho), C.c_double(wx), C.c_double(wy),
                                              ptr(g_u), ptr(g_v), ptr(g_u_old), ptr(g_v_old), ptr(g_u_prev),
                                              ptr(g_v_prev), ptr(g_p)))


def transpose_values(ctx, ilu, val, val_t):
    """Values of A^T on the (symmetric) pattern of the ILU handle."""
    ctx.check(lib().cfa_csr_transpose_values(ctx.h, ilu.h, ptr(val), ptr(val_t)))


def apply_bc_momentum(ctx, m: DeviceMesh, A_val, rhs_u, rhs_v, u, v, u_max, H=1.0):
    bc = MomentumBc(u_max, H)
    ctx.check(lib().cfa_apply_bc_momentum(ctx.h, m.h, C.byref(bc), ptr(A_val), ptr(rhs_u), ptr(rhs_v), ptr(u), ptr(v)))


def lumped_mass(ctx, m: DeviceMesh, mass):
    ctx.check(lib().cfa_lumped_mass(ctx.h, m.h, ptr(mass)))


def oss_weights(ctx, m: DeviceMesh, u, v, dt, rho, nu, stab, elem_s):
    ctx.check(lib().cfa_oss_weights(ctx.h, m.h, ptr(u), ptr(v), C.c_double(dt), C.c_double(rho), C.c_double(nu),
                                    C.c_double(stab), ptr(elem_s)))


def scalar_gradient(ctx, m: DeviceMesh, f, elem_s, gx, gy):
    ctx.check(lib().cfa_scalar_gradient(ctx.h, m.h, ptr(f), ptr(elem_s), ptr(gx), ptr(gy)))


def assemble_ppe(ctx, m: DeviceMesh, u, v, p, gpx, gpy, mass, elem_s, dt, rho, stab, Kp, rhs, div, dp=None,
                 apply_bc=True):
    ctx.check(lib().cfa_assemble_ppe(ctx.h, m.h, ptr(u), ptr(v), ptr(p), ptr(gpx), ptr(gpy), ptr(mass), ptr(elem_s),
                                     C.c_double(dt), C.c_double(rho), C.c_double(stab), 1 if apply_bc else 0,
                                     ptr(Kp), ptr(rhs), ptr(div), ptr(dp)))


def apply_bc_pressure(ctx, m: DeviceMesh, Kp, rhs, dp, mass):
    ctx.check(lib().cfa_apply_bc_pressure(ctx.h, m.h, ptr(Kp), ptr(rhs), ptr(dp), ptr(mass)))


def assemble_oss(ctx, m: DeviceMesh, elem_s, mass, oss_val, inv_m):
    ctx.check(lib().cfa_assemble_oss(ctx.h, m.h, ptr(elem_s), ptr(mass), ptr(oss_val), ptr(inv_m)))


def assemble_pressure_system(ctx, m: DeviceMesh, u, v, p, gpx, gpy, mass, elem_s, dt, rho, stab, Kp, rhs, div, dp,
                             oss_val, inv_m):
    ctx.check(lib().cfa_assemble_pressure_system(ctx.h, m.h, ptr(u), ptr(v), ptr(p), ptr(gpx), ptr(gpy), ptr(mass),
                                                 ptr(elem_s), C.c_double(dt), C.c_double(rho), C.c_double(stab),
                                                 ptr(Kp), ptr(rhs), ptr(div), ptr(dp), ptr(oss_val), ptr(inv_m)))


def oss_apply(ctx, m: DeviceMesh, oss_val, inv_m, x, out):
    ctx.check(lib().cfa_oss_apply(ctx.h, m.h, ptr(oss_val), ptr(inv_m), ptr(x), ptr(out)))


def stiffness_apply(ctx, m: DeviceMesh, f, c, out):
    ctx.check(lib().cfa_stiffness_apply(ctx.h, m.h, ptr(f), C.c_double(c), ptr(out)))


def grad_dp_vorticity(ctx, m: DeviceMesh, dp, u, v, gdx, gdy, vort_num):
    ctx.check(lib().cfa_grad_dp_vorticity(ctx.h, m.h, ptr(dp), ptr(u), ptr(v), ptr(gdx), ptr(gdy), ptr(vort_num)))


def velocity_pressure_correction(ctx, m: DeviceMesh, dt, rho, p_update, rot_coeff, div_num, mass, gdx, gdy,
                                 vort_num, dp, u, v, p, vort=None):
    ctx.check(lib().cfa_velocity_pressure_correction(ctx.h, m.h, C.c_double(dt), C.c_double(rho),
                                                     C.c_double(p_update), C.c_double(rot_coeff), ptr(div_num),
                                                     ptr(mass), ptr(gdx), ptr(gdy), ptr(vort_num), ptr(dp), ptr(u),
                                                     ptr(v), ptr(p), ptr(vort)))


def project_step(ctx, m: DeviceMesh, dt_proj, rho, rot_coeff, rotational_from_dp, mass, dp, div_num, gdx, gdy,
                 vort_num, u, v, p, vort=None):
    ctx.check(lib().cfa_project_step(ctx.h, m.h, C.c_double(dt_proj), C.c_double(rho), C.c_double(rot_coeff),
                                     int(rotational_from_dp), ptr(mass), ptr(dp), ptr(div_num), ptr(gdx), ptr(gdy),
                                     ptr(vort_num), ptr(u), ptr(v), ptr(p), ptr(vort)))


def volume_forces(ctx, m: DeviceMesh, u, v, u_old, v_old, u_prev, v_prev, p, b0, b1, b2, nu, rho, out2):
    ctx.check(lib().cfa_volume_forces(ctx.h, m.h, ptr(u), ptr(v), ptr(u_old), ptr(v_old), ptr(u_prev), ptr(v_prev),
                                      ptr(p), C.c_double(b0), C.c_double(b1), C.c_double(b2), C.c_double(nu),
                                      C.c_double(rho), ptr(out2)))


def amr_indicators(ctx, m: DeviceMesh, u, v, u_max, H, mass, grad_rec, elem_error):
    """k_accumulate_recovered_gradient + k_compute_amr_error_indicator: grad_rec [4 n] and
    elem_error [2 ne] (device, overwritten)."""
    ctx.check(lib().cfa_recovered_gradient(ctx.h, m.h, ptr(u), ptr(v), C.c_double(u_max), C.c_double(H),
                                           ptr(grad_rec)))
    ctx.check(lib().cfa_amr_error_indicator(ctx.h, m.h, ptr(grad_rec), ptr(mass), ptr(elem_error)))


def spmv(ctx, rp, ci, val, x, y):
    ctx.check(lib().cfa_spmv(ctx.h, rp.numel() - 1, ptr(rp), ptr(ci), ptr(val), ptr(x), ptr(y)))


def spmv_multi(ctx, rp, ci, val, x, y, nrhs):
    ctx.check(lib().cfa_spmv_multi(ctx.h, rp.numel() - 1, nrhs, ptr(rp), ptr(ci), ptr(val), ptr(x), ptr(y)))


def pressure_operator_prepare(ctx, rp, ci, val, oss=None):
    ctx.check(lib().cfa_pressure_operator_prepare(ctx.h, rp.numel() - 1, ci.numel(), ptr(rp), ptr(ci), ptr(val),
                                                  C.byref(oss) if oss is not None else None))


def pressure_operator(ctx, rp, ci, val, x, y, oss=None):
    ctx.check(lib().cfa_pressure_operator(ctx.h, rp.numel() - 1, ci.numel(), ptr(rp), ptr(ci), ptr(val),
                                          C.byref(oss) if oss is not None else None, ptr(x), ptr(y)))


def pressure_operator_layout(ctx):
    """(passes, stored_nnz) of the prepared pressure operator."""
    passes, nz = C.c_int(), C.c_longlong()
    ctx.check(lib().cfa_pressure_operator_layout(ctx.h, C.byref(passes), C.byref(nz)))
    return passes.value, nz.value


def oss_operator(mesh: DeviceMesh, oss_val, inv_m) -> OssOperator:
    return OssOperator(mesh.h.value, oss_val.data_ptr(), inv_m.data_ptr())


# ---------------------------------------------------------------------------------------------
# solver classes mirroring src/cfa/linalg.cuh
# ---------------------------------------------------------------------------------------------
class MulticolourIlu0:
    """MulticolourIlu0 (src/cfa/linalg.cuh:435-568)."""

    def __init__(self, ctx: Context | None = None, precision: int = FP64):
        self.ctx = ctx or default_context()
        self.precision = precision
        self.h = None
        self.n = 0
        self.n_colours = 0
        self.colour_start = []

    def set_pattern(self, n, rp_host, ci_host, d_rp, d_ci):
        """A new pattern; the handle (and its device buffers) is kept across calls."""
        rp_h = np.ascontiguousarray(rp_host, dtype=np.int32)
        ci_h = np.ascontiguousarray(ci_host, dtype=np.int32)
        if self.h is None:
            h = C.c_void_p()
            self.ctx.check(lib().cfa_ilu_create(self.ctx.h, n, ptr(rp_h), ptr(ci_h), ptr(d_rp), ptr(d_ci),
                                                self.precision, C.byref(h)))
            self.h = h
        else:
            self.ctx.check(lib().cfa_ilu_set_pattern(self.ctx.h, self.h, n, ptr(rp_h), ptr(ci_h), ptr(d_rp),
                                                     ptr(d_ci)))
        self.n = n
        nc = C.c_int()
        lib().cfa_ilu_colours(self.h, C.byref(nc), None)
        cs = np.zeros(nc.value + 1, np.int32)
        lib().cfa_ilu_colours(self.h, C.byref(nc), ptr(cs))
        self.n_colours = nc.value
        self.colour_start = cs

    def factor(self, d_val):
        self.ctx.check(lib().cfa_ilu_factor(self.ctx.h, self.h, ptr(d_val)))

    def apply(self, r, z, nrhs=1):
        self.ctx.check(lib().cfa_ilu_apply(self.ctx.h, self.h, ptr(r), ptr(z), nrhs))

    def apply_interleaved(self, r, z):
        """Two right-hand sides interleaved per row (r[2i], r[2i + 1]): the momentum solve's sweeps."""
        self.ctx.check(lib().cfa_ilu_apply_interleaved(self.ctx.h, self.h, ptr(r), ptr(z)))

    def factor_transposed(self, d_val):
        """Factor A and keep (LU)^T: the handle then preconditions A^T."""
        self.ctx.check(lib().cfa_ilu_factor_transposed(self.ctx.h, self.h, ptr(d_val)))

    def device_arrays(self, nnz):
        import torch
        col, rows, lu = C.c_void_p(), C.c_void_p(), C.c_void_p()
        lib().cfa_ilu_device_arrays(self.h, C.byref(col), C.byref(rows), C.byref(lu))
        return _dev_view(col.value, self.n, torch.int32), _dev_view(rows.value, self.n, torch.int32), \
            _dev_view(lu.value, nnz, torch.float64)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().cfa_ilu_destroy(self.h)
                self.h = None
        except Exception:
            pass


class GpuBicgstab2:
    """GpuBicgstab2 (src/cfa/linalg.cuh:642-779): iters[2], converged[2], last_rel_residual[2]."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.iters = [0, 0]
        self.converged = [True, True]
        self.last_rel_residual = [0.0, 0.0]
        self.solve_ms = 0.0

    def solve(self, n, d_rp, d_ci, d_val, b_u, b_v, x_u, x_v, max_iter, tol, ilu: MulticolourIlu0):
        rep = SolveReport()
        opts = SolveOpts(max_iter, tol)
        self.ctx.check(lib().cfa_bicgstab2_solve(self.ctx.h, n, ptr(d_rp), ptr(d_ci), ptr(d_val), ptr(b_u), ptr(b_v),
                                                 ptr(x_u), ptr(x_v), ilu.h, C.byref(opts), C.byref(rep)),
                       allow=(CFA_OK, CFA_NOT_CONVERGED))
        self.iters = [rep.iterations[0], rep.iterations[1]]
        self.converged = [bool(rep.converged[0]), bool(rep.converged[1])]
        self.last_rel_residual = [rep.rel_residual[0], rep.rel_residual[1]]
        self.solve_ms = rep.solve_ms


class AmgPreconditioner:
    """AmgPreconditioner (src/cfa/linalg.cuh:939-1432); public knobs as members."""

    def __init__(self, ctx: Context | None = None, precision: int = FP64, theta=0.08, smooth_steps=2,
                 coarse_target=300, max_levels=15):
        self.ctx = ctx or default_context()
        self.theta, self.smooth_steps, self.coarse_target, self.max_levels = theta, smooth_steps, coarse_target, max_levels
        self.precision = precision
        self.h = None

    def _handle(self):
        if self.h is None:
            o = AmgOpts(self.theta, self.smooth_steps, self.coarse_target, self.max_levels, self.precision)
            h = C.c_void_p()
            self.ctx.check(lib().cfa_amg_create(self.ctx.h, C.byref(o), C.byref(h)))
            self.h = h
        return self.h

    def setup(self, n, nnz, d_rp, d_ci, d_val):
        self.ctx.check(lib().cfa_amg_setup(self.ctx.h, self._handle(), n, nnz, ptr(d_rp), ptr(d_ci), ptr(d_val)))

    def apply(self, r, z):
        self.ctx.check(lib().cfa_amg_apply(self.ctx.h, self.h, ptr(r), ptr(z)))

    def remap(self, n, nnz, d_rp, d_ci, d_val, h_rp, h_ci, new_to_old):
        """remap (src/cfa/linalg.cuh:1074-1157): host pattern and new_to_old as numpy int32."""
        h_rp = np.ascontiguousarray(h_rp, np.int32)
        h_ci = np.ascontiguousarray(h_ci, np.int32)
        n2o = np.ascontiguousarray(new_to_old, np.int32)
        self.ctx.check(lib().cfa_amg_remap(self.ctx.h, self._handle(), n, nnz, ptr(d_rp), ptr(d_ci), ptr(d_val),
                                           ptr(h_rp), ptr(h_ci), ptr(n2o)))

    @property
    def remaps(self) -> int:
        return int(lib().cfa_amg_remaps(self.h)) if self.h else 0

    def _info(self):
        nl, cn, ms = C.c_int(), C.c_int(), C.c_double()
        lib().cfa_amg_info(self.h, C.byref(nl), C.byref(cn), C.byref(ms))
        return nl.value, cn.value, ms.value

    def num_levels(self):
        return self._info()[0]

    @property
    def coarse_n(self):
        return self._info()[1]

    @property
    def setup_ms(self):
        return self._info()[2]

    def level(self, l):
        """Device views of level l: dict(rows, A, P, R (rp, ci, v), agg, omega)."""
        import torch
        info = np.zeros(5, np.int32)
        ps = [C.c_void_p() for _ in range(10)]
        om = C.c_double()
        s = lib().cfa_amg_level(self.h, l, ptr(info), *[C.byref(p) for p in ps], C.byref(om))
        if s != CFA_OK:
            raise CfaError(s, "cfa_amg_level")
        rows, annz, pcols, pnnz, rnnz = (int(v) for v in info)
        agg, arp, aci, av, prp, pci, pv, rrp, rci, rv = (p.value for p in ps)
        return dict(rows=rows, omega=om.value, pcols=pcols,
                    agg=_dev_view(agg, rows, torch.int32),
                    A=(_dev_view(arp, rows + 1, torch.int32), _dev_view(aci, annz, torch.int32), _dev_view(av, annz, torch.float64)),
                    P=(_dev_view(prp, rows + 1, torch.int32), _dev_view(pci, pnnz, torch.int32), _dev_view(pv, pnnz, torch.float64)),
                    R=(_dev_view(rrp, pcols + 1, torch.int32), _dev_view(rci, rnnz, torch.int32), _dev_view(rv, rnnz, torch.float64)))

    @property
    def phase_ms(self):
        out = np.zeros(8)
        lib().cfa_amg_phases(self.h, ptr(out))
        return dict(zip(("copy", "rho", "aggregation", "smoothing", "transpose", "galerkin", "tiles", "coarse"),
                        out.tolist()))

    def coarse_inverse(self):
        import torch
        p = C.c_void_p()
        lib().cfa_amg_coarse_inverse(self.h, C.byref(p))
        cn = self.coarse_n
        return _dev_view(p.value, cn * cn, torch.float64).reshape(cn, cn)

    def set_vcycle(self, composite_rows: int = -1, fuse_levels: int = -1, fold_rows: int = -1):
        """The V-cycle's forms for the setups that follow (-1 keeps the default): the composite
        coarse operator's largest level, the levels with the fused restriction, the largest level
        with the folded prolongation. (0, 0, 0) runs the plain level chain."""
        s = lib().cfa_amg_set_vcycle(self._handle(), composite_rows, fuse_levels, fold_rows)
        if s != CFA_OK:
            raise CfaError(s, "cfa_amg_set_vcycle")

    def set_fp64_phase(self, switch_rel: float = -1.0):
        """Mixed precision: the solves' V-cycles in FP64 until the relative residual falls below
        switch_rel, FP32 after (0: FP32 throughout; negative: the default), for the setups that
        follow."""
        s = lib().cfa_amg_set_fp64_phase(self._handle(), C.c_double(switch_rel))
        if s != CFA_OK:
            raise CfaError(s, "cfa_amg_set_fp64_phase")

    def set_aggregation(self, on_device: int = -1):
        """The setups' greedy aggregation on the device (1, the default) or the host (0); -1
        follows CFA_AGG_HOST. Both give the same aggregates."""
        s = lib().cfa_amg_set_aggregation(self._handle(), on_device)
        if s != CFA_OK:
            raise CfaError(s, "cfa_amg_set_aggregation")

    def composite(self):
        """(level, rows) of the composite coarse operator, level -1 when there is none."""
        lv, rows = C.c_int(), C.c_int()
        lib().cfa_amg_composite(self._handle(), C.byref(lv), C.byref(rows), None)
        return lv.value, rows.value

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().cfa_amg_destroy(self.h)
                self.h = None
        except Exception:
            pass


class GpuLinearSolver:
    """GpuLinearSolver (src/cfa/linalg.cuh:120-348): solve_pcg with the OSS term and the AMG passed
    as objects instead of std::function callbacks; converged, last_rel_residual."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.converged = True
        self.last_rel_residual = 0.0
        self.solve_ms = 0.0

    def solve_pcg(self, n, d_rp, d_ci, d_val, d_b, d_x, max_iter=400, tol=1e-7, oss: OssOperator | None = None,
                  amg: AmgPreconditioner | None = None) -> int:
        rep = SolveReport()
        opts = SolveOpts(max_iter, tol)
        self.ctx.check(lib().cfa_pcg_solve(self.ctx.h, n, ptr(d_rp), ptr(d_ci), ptr(d_val), ptr(d_b), ptr(d_x),
                                           C.byref(oss) if oss is not None else None, amg.h if amg is not None else None,
                                           C.byref(opts), C.byref(rep)),
                       allow=(CFA_OK, CFA_NOT_CONVERGED, CFA_BREAKDOWN))
        self.converged = bool(rep.converged[0])
        self.last_rel_residual = rep.rel_residual[0]
        self.solve_ms = rep.solve_ms
        return rep.iterations[0]

    def solve_pcg_host_ops(self, n, d_rp, d_ci, d_val, d_b, d_x, max_iter=400, tol=1e-7, extra_op=None,
                           amg: AmgPreconditioner | None = None, precond=None) -> int:
        """solve_pcg with the reference's std::function hooks as Python callables
        f(in_ptr, out_ptr) on device addresses: extra_op adds its operator into out, precond
        writes out = M^-1 in (cfa_pcg_solve_host_ops). They run on the host between the
        library's launches and must enqueue their work on this context's stream."""
        cb = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_void_p)
        hooks = [cb(lambda i, o, u, f=f: f(i, o)) if f is not None else None for f in (extra_op, precond)]
        rep = SolveReport()
        opts = SolveOpts(max_iter, tol)
        self.ctx.check(lib().cfa_pcg_solve_host_ops(self.ctx.h, n, ptr(d_rp), ptr(d_ci), ptr(d_val), ptr(d_b),
                                                    ptr(d_x), hooks[0], None, amg.h if amg is not None else None,
                                                    hooks[1], None, C.byref(opts), C.byref(rep)),
                       allow=(CFA_OK, CFA_NOT_CONVERGED, CFA_BREAKDOWN))
        self.converged = bool(rep.converged[0])
        self.last_rel_residual = rep.rel_residual[0]
        self.solve_ms = rep.solve_ms
        return rep.iterations[0]

    def solve_bicgstab(self, n, d_rp, d_ci, d_val, d_b, d_x, max_iter=200, tol=1e-7) -> int:
        rep = SolveReport()
        opts = SolveOpts(max_iter, tol)
        self.ctx.check(lib().cfa_bicgstab_solve(self.ctx.h, n, ptr(d_rp), ptr(d_ci), ptr(d_val), ptr(d_b), ptr(d_x),
                                                C.byref(opts), C.byref(rep)), allow=(CFA_OK, CFA_NOT_CONVERGED))
        self.converged = bool(rep.converged[0])
        self.last_rel_residual = rep.rel_residual[0]
        self.solve_ms = rep.solve_ms
        return rep.iterations[0]


def _dev_view(addr, count, dtype):
    """A torch tensor viewing `count` elements of library-owned device memory (valid while the
    owning handle keeps it; copy before the handle changes)."""
    import torch
    if count == 0 or not addr:
        return torch.empty(0, dtype=dtype, device="cuda")

    class _Holder:
        pass

    h = _Holder()
    h.__cuda_array_interface__ = {
        "shape": (count,), "typestr": {torch.int32: "<i4", torch.float64: "<f8", torch.float32: "<f4"}[dtype],
        "data": (addr, False), "version": 3,
    }
    return torch.as_tensor(h, device="cuda")
