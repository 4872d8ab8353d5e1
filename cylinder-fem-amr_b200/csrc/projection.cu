// Post-solve kernels of a time step (the driver's Steps C and D, src/cylinder_fem_amr.cu:462-513):
// the rotational term from the pressure increment, the nodal gradient of dp and the vorticity,
// the velocity projection / pressure update, and the volume-integral drag and lift.
//
// The reference scatters element contributions with FP64 atomics (an order that changes run to
// run). Here every node gathers its elements through the mesh's incidence list (ascending element
// order), and the forces are summed by a fixed-order two-stage reduction: deterministic results.
#include "internal.cuh"
#include "mesh.cuh"

namespace cfa {

struct ElemGrad {
    double area, dNdx[3], dNdy[3];
    bool ok;
};

__device__ __forceinline__ ElemGrad elem_grad(const int* nd, const double* __restrict__ x, const double* __restrict__ y) {
    ElemGrad g;
    const double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
    const double detJ = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
    g.area = 0.5 * fabs(detJ);
    g.ok = g.area >= 1.0e-14;
    const double inv2A = g.ok ? 1.0 / (2.0 * g.area) : 0.0;
    g.dNdx[0] = (y1 - y2) * inv2A; g.dNdx[1] = (y2 - y0) * inv2A; g.dNdx[2] = (y0 - y1) * inv2A;
    g.dNdy[0] = (x2 - x1) * inv2A; g.dNdy[1] = (x0 - x2) * inv2A; g.dNdy[2] = (x1 - x0) * inv2A;
    return g;
}

// Per node, over its elements:
//   stiff_i += c * area (dN_i . grad f)           (k_stiffness_apply, fem_kernels.cuh:618-637)
//   gdx_i, gdy_i = sum (area/3) grad dp;  vort_num_i = sum (area/3) (dv/dx - du/dy)
//                                                 (k_accumulate_grad_dp_and_vorticity, :536-575)
// stiff (nullable) is added to; gdx, gdy, vort_num (each nullable) are overwritten.
__global__ void __launch_bounds__(kThreads)
k_node_gradients(int n, const int* __restrict__ ev, const double* __restrict__ x, const double* __restrict__ y,
                 const int* __restrict__ inc_ptr, const int* __restrict__ inc, const double* __restrict__ f, double c,
                 double* __restrict__ stiff, const double* __restrict__ dp, const double* __restrict__ u,
                 const double* __restrict__ v, double* __restrict__ gdx, double* __restrict__ gdy,
                 double* __restrict__ vort_num) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0, sx = 0.0, sy = 0.0, sw = 0.0;
    for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        const int e = inc[k] >> 2, li = inc[k] & 3;
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        const ElemGrad g = elem_grad(nd, x, y);
        if (!g.ok) continue;
        if (stiff) {
            const double gx = f[nd[0]] * g.dNdx[0] + f[nd[1]] * g.dNdx[1] + f[nd[2]] * g.dNdx[2];
            const double gy = f[nd[0]] * g.dNdy[0] + f[nd[1]] * g.dNdy[1] + f[nd[2]] * g.dNdy[2];
            s += c * g.area * (g.dNdx[li] * gx + g.dNdy[li] * gy);
        }
        const double w = g.area / 3.0;
        if (gdx) {
            const double dpdx = dp[nd[0]] * g.dNdx[0] + dp[nd[1]] * g.dNdx[1] + dp[nd[2]] * g.dNdx[2];
            const double dpdy = dp[nd[0]] * g.dNdy[0] + dp[nd[1]] * g.dNdy[1] + dp[nd[2]] * g.dNdy[2];
            sx += w * dpdx;
            sy += w * dpdy;
        }
        if (vort_num) {
            const double dvdx = v[nd[0]] * g.dNdx[0] + v[nd[1]] * g.dNdx[1] + v[nd[2]] * g.dNdx[2];
            const double dudy = u[nd[0]] * g.dNdy[0] + u[nd[1]] * g.dNdy[1] + u[nd[2]] * g.dNdy[2];
            sw += w * (dvdx - dudy);
        }
    }
    if (stiff) stiff[i] += s;
    if (gdx) { gdx[i] = sx; gdy[i] = sy; }
    if (vort_num) vort_num[i] = sw;
}

// k_velocity_pressure_correction (fem_kernels.cuh:585-610):
//   vort = vort_num / m;  p += p_update (dp - rot_coeff div_num / m);
//   u -= (dt/rho) gdx / m, v likewise, on interior nodes and on the outlet when it is natural.
__global__ void k_correction(int n, const int* __restrict__ tag, OutletBc bc, double dt, double rho, double p_update,
                             double rot_coeff, const double* __restrict__ div_num, const double* __restrict__ mass,
                             const double* __restrict__ gdx, const double* __restrict__ gdy,
                             const double* __restrict__ vort_num, const double* __restrict__ dp, double* __restrict__ u,
                             double* __restrict__ v, double* __restrict__ p, double* __restrict__ vort) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double m_i = fmax(mass[i], 1.0e-14);
    if (vort) vort[i] = vort_num[i] / m_i;
    p[i] += p_update * (dp[i] - rot_coeff * div_num[i] / m_i);
    const int t = tag[i];
    if (t == BC_INTERIOR || (t == BC_OUTLET && !bc.outlet_dirichlet)) {
        u[i] -= (dt / rho) * (gdx[i] / m_i);
        v[i] -= (dt / rho) * (gdy[i] / m_i);
    }
}

// k_volume_forces (fem_kernels.cuh:1046-1123): the volume-integral drag and lift over the elements
// touching the cylinder (phi = 1 on cylinder nodes), edge-midpoint quadrature; out[0..1].
__global__ void __launch_bounds__(kThreads)
k_volume_forces(int ne, const int* __restrict__ ev, const int* __restrict__ tag, const double* __restrict__ x,
                const double* __restrict__ y, const double* __restrict__ u, const double* __restrict__ v,
                const double* __restrict__ u_old, const double* __restrict__ v_old, const double* __restrict__ u_prev,
                const double* __restrict__ v_prev, const double* __restrict__ p, double b0, double b1, double b2,
                double nu, double rho, double* __restrict__ part, unsigned int* __restrict__ counter,
                double* __restrict__ out) {
    CFA_GRID_DEP();
    __shared__ double sh[2 * kWarps];
    double acc[2] = {0.0, 0.0};
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        double phi[3];
        bool touches = false;
        for (int a = 0; a < 3; ++a) {
            phi[a] = tag[nd[a]] == BC_CYLINDER ? 1.0 : 0.0;
            touches = touches || phi[a] > 0.0;
        }
        if (!touches) continue;
        const ElemGrad g = elem_grad(nd, x, y);
        if (!g.ok) continue;
        double ue[3], ve[3], ute[3], vte[3];
        double dudx = 0.0, dudy = 0.0, dvdx = 0.0, dvdy = 0.0, dphidx = 0.0, dphidy = 0.0, p_bar = 0.0;
        for (int a = 0; a < 3; ++a) {
            ue[a] = u[nd[a]];
            ve[a] = v[nd[a]];
            ute[a] = b0 * ue[a] + b1 * u_old[nd[a]] + b2 * u_prev[nd[a]];
            vte[a] = b0 * ve[a] + b1 * v_old[nd[a]] + b2 * v_prev[nd[a]];
            dudx += ue[a] * g.dNdx[a];
            dudy += ue[a] * g.dNdy[a];
            dvdx += ve[a] * g.dNdx[a];
            dvdy += ve[a] * g.dNdy[a];
            dphidx += phi[a] * g.dNdx[a];
            dphidy += phi[a] * g.dNdy[a];
            p_bar += p[nd[a]] / 3.0;
        }
        double fx = 0.0, fy = 0.0;
        for (int a = 0; a < 3; ++a) {
            const int b = (a + 1) % 3;
            const double phi_m = 0.5 * (phi[a] + phi[b]);
            if (phi_m == 0.0) continue;
            const double um = 0.5 * (ue[a] + ue[b]), vm = 0.5 * (ve[a] + ve[b]);
            fx += (0.5 * (ute[a] + ute[b]) + (um * dudx + vm * dudy)) * phi_m;
            fy += (0.5 * (vte[a] + vte[b]) + (um * dvdx + vm * dvdy)) * phi_m;
        }
        fx *= g.area / 3.0;
        fy *= g.area / 3.0;
        fx += g.area * (nu * (dudx * dphidx + dudy * dphidy) - (p_bar / rho) * dphidx);
        fy += g.area * (nu * (dvdx * dphidx + dvdy * dphidy) - (p_bar / rho) * dphidy);
        acc[0] += fx;
        acc[1] += fy;
    }
    block_sum<2>(acc, sh);
    if (publish_partials<2>(acc, part, counter)) {
        reduce_partials<2>(acc, part, counter, sh);
        if (threadIdx.x == 0) { out[0] = acc[0]; out[1] = acc[1]; }
    }
}

// k_accumulate_recovered_gradient (fem_kernels.cuh:911-968) per node: the area-weighted P1
// gradient of the disturbance velocity u' = u - 4 U y (H - y) / H^2, v' = v;
// grad_rec = [du'/dx | du'/dy | dv/dx | dv/dy] (4 n, overwritten).
__global__ void __launch_bounds__(kThreads)
k_recovered_gradient(int n, const int* __restrict__ ev, const double* __restrict__ x, const double* __restrict__ y,
                     const int* __restrict__ inc_ptr, const int* __restrict__ inc, const double* __restrict__ u,
                     const double* __restrict__ v, double u_max, double H, double* __restrict__ grad_rec) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        const int e = inc[k] >> 2;
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        const ElemGrad g = elem_grad(nd, x, y);
        if (!g.ok) continue;
        double ud[3];
        for (int a = 0; a < 3; ++a) {
            const double ya = y[nd[a]];
            ud[a] = u[nd[a]] - 4.0 * u_max * ya * (H - ya) / (H * H);
        }
        const double w = g.area / 3.0;
        s[0] += w * (ud[0] * g.dNdx[0] + ud[1] * g.dNdx[1] + ud[2] * g.dNdx[2]);
        s[1] += w * (ud[0] * g.dNdy[0] + ud[1] * g.dNdy[1] + ud[2] * g.dNdy[2]);
        s[2] += w * (v[nd[0]] * g.dNdx[0] + v[nd[1]] * g.dNdx[1] + v[nd[2]] * g.dNdx[2]);
        s[3] += w * (v[nd[0]] * g.dNdy[0] + v[nd[1]] * g.dNdy[1] + v[nd[2]] * g.dNdy[2]);
    }
    for (int c = 0; c < 4; ++c) grad_rec[(size_t)c * n + i] = s[c];
}

// k_compute_amr_error_indicator (fem_kernels.cuh:995-1035): per element the disturbance
// vorticity times h_K and the P1 interpolation-error estimate from the recovered gradient.
__global__ void k_amr_indicator(int ne, int n, const int* __restrict__ ev, const double* __restrict__ x,
                                const double* __restrict__ y, const double* __restrict__ grad_rec,
                                const double* __restrict__ mass, double* __restrict__ elem_error) {
    CFA_GRID_DEP();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
    double G[3][4];
    for (int a = 0; a < 3; ++a) {
        const double inv_m = 1.0 / fmax(mass[nd[a]], 1.0e-14);
        for (int c = 0; c < 4; ++c) G[a][c] = grad_rec[(size_t)c * n + nd[a]] * inv_m;
    }
    const double x0 = x[nd[0]], y0 = y[nd[0]];
    const double area = 0.5 * fabs((x[nd[1]] - x0) * (y[nd[2]] - y0) - (x[nd[2]] - x0) * (y[nd[1]] - y0));
    double omega = 0.0, eta_i = 0.0;
    for (int a = 0; a < 3; ++a) {
        omega = fmax(omega, fabs(G[a][2] - G[a][1]));
        const int b = (a + 1) % 3;
        const double ex = x[nd[b]] - x[nd[a]], ey = y[nd[b]] - y[nd[a]];
        const double eu = (G[b][0] - G[a][0]) * ex + (G[b][1] - G[a][1]) * ey;
        const double evv = (G[b][2] - G[a][2]) * ex + (G[b][3] - G[a][3]) * ey;
        eta_i = fmax(eta_i, 0.125 * sqrt(eu * eu + evv * evv));
    }
    elem_error[e] = sqrt(2.0 * area) * omega;
    elem_error[ne + e] = eta_i;
}

}  // namespace cfa

using namespace cfa;

extern "C" {

cfa_status cfa_stiffness_apply(cfa_ctx* ctx, const cfa_mesh* m, const double* f, double c, double* out) {
    CFA_ENTER(ctx);
    CFA_ARG(m && f && out);
    CFA_LAUNCH(ctx, k_node_gradients, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->ev, m->x, m->y, m->inc_ptr.p,
               m->inc.p, f, c, out, (const double*)nullptr, (const double*)nullptr, (const double*)nullptr,
               (double*)nullptr, (double*)nullptr, (double*)nullptr);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_grad_dp_vorticity(cfa_ctx* ctx, const cfa_mesh* m, const double* dp, const double* u,
                                 const double* v, double* grad_dp_x, double* grad_dp_y, double* vort_num) {
    CFA_ENTER(ctx);
    CFA_ARG(m && dp && u && v && grad_dp_x && grad_dp_y && vort_num);
    CFA_LAUNCH(ctx, k_node_gradients, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->ev, m->x, m->y, m->inc_ptr.p,
               m->inc.p, (const double*)nullptr, 0.0, (double*)nullptr, dp, u, v, grad_dp_x, grad_dp_y, vort_num);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_velocity_pressure_correction(cfa_ctx* ctx, const cfa_mesh* m, double dt, double rho, double p_update,
                                            double rot_coeff, const double* div_num, const double* mass_lumped,
                                            const double* grad_dp_x, const double* grad_dp_y,
                                            const double* vort_num, const double* dp, double* u, double* v,
                                            double* p, double* vort) {
    CFA_ENTER(ctx);
    CFA_ARG(m && div_num && mass_lumped && grad_dp_x && grad_dp_y && dp && u && v && p && (!vort || vort_num));
    CFA_LAUNCH(ctx, k_correction, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->tag, m->bc, dt, rho, p_update,
               rot_coeff, div_num, mass_lumped, grad_dp_x, grad_dp_y, vort_num, dp, u, v, p, vort);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_project_step(cfa_ctx* ctx, const cfa_mesh* m, double dt_proj, double rho, double rot_coeff,
                            int rotational_from_dp, const double* mass_lumped, const double* dp, double* div_num,
                            double* grad_dp_x, double* grad_dp_y, double* vort_num, double* u, double* v, double* p,
                            double* vort) {
    CFA_ENTER(ctx);
    CFA_ARG(m && mass_lumped && dp && div_num && grad_dp_x && grad_dp_y && vort_num && u && v && p);
    if (rotational_from_dp) CFA_CUDA(cudaMemsetAsync(div_num, 0, (size_t)m->n * sizeof(double), ctx->stream));
    CFA_LAUNCH(ctx, k_node_gradients, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->ev, m->x, m->y, m->inc_ptr.p,
               m->inc.p, (const double*)dp, -dt_proj / rho, rotational_from_dp ? div_num : (double*)nullptr, dp,
               (const double*)u, (const double*)v, grad_dp_x, grad_dp_y, vort_num);
    CFA_LAUNCH(ctx, k_correction, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->tag, m->bc, dt_proj, rho, 1.0,
               rot_coeff, (const double*)div_num, mass_lumped, (const double*)grad_dp_x, (const double*)grad_dp_y,
               (const double*)vort_num, dp, u, v, p, vort);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_volume_forces(cfa_ctx* ctx, const cfa_mesh* m, const double* u, const double* v, const double* u_old,
                             const double* v_old, const double* u_prev, const double* v_prev, const double* p,
                             double b0, double b1, double b2, double nu, double rho, double* d_out2) {
    CFA_ENTER(ctx);
    CFA_ARG(m && u && v && u_old && v_old && u_prev && v_prev && p && d_out2);
    const int grid = std::min(ceil_div(m->ne, kThreads), 4 * ctx->num_sms);
    CFA_PROPAGATE(ensure_partials(ctx, 2 * (size_t)grid + 2));
    CFA_LAUNCH(ctx, k_volume_forces, grid, kThreads, 0, m->ne, m->ev, m->tag, m->x, m->y, u, v, u_old, v_old, u_prev,
               v_prev, p, b0, b1, b2, nu, rho, ctx->d_part, ctx->d_counters, d_out2);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_recovered_gradient(cfa_ctx* ctx, const cfa_mesh* m, const double* u, const double* v, double u_max,
                                  double H, double* grad_rec) {
    CFA_ENTER(ctx);
    CFA_ARG(m && u && v && grad_rec && H > 0.0);
    CFA_LAUNCH(ctx, k_recovered_gradient, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->ev, m->x, m->y,
               m->inc_ptr.p, m->inc.p, u, v, u_max, H, grad_rec);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_amr_error_indicator(cfa_ctx* ctx, const cfa_mesh* m, const double* grad_rec, const double* mass_lumped,
                                   double* elem_error) {
    CFA_ENTER(ctx);
    CFA_ARG(m && grad_rec && mass_lumped && elem_error);
    CFA_LAUNCH(ctx, k_amr_indicator, ceil_div(m->ne, kThreads), kThreads, 0, m->ne, m->n, m->ev, m->x, m->y, grad_rec,
               mass_lumped, elem_error);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

}  // extern "C"
