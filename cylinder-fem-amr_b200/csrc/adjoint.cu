// Adjoint of the momentum predictor (the driver's Step A, src/cylinder_fem_amr.cu:296-380).
//
// The step solves A(theta) x_c = b_c(theta), c in {u, v} (one matrix for both components), with
// theta = (u^n, v^n, u^{n-1}, v^{n-1}, p^n, nu, inflow amplitude U). Given the adjoint solution
// lambda_c of A^T lambda_c = dJ/dx_c, a scalar J(x) has
//     dJ/dtheta = sum_c lambda_c^T (db_c/dtheta - dA/dtheta x_c).
// Rows of Dirichlet nodes are identity rows whose right-hand side is the boundary value, so they
// depend on U only. Every other row is a sum of element contributions of
// k_assemble_momentum_fem (src/cfa/fem_kernels.cuh:40-181). Here that element computation is
// written once over a forward-mode dual number carrying the derivatives with respect to the 16
// element inputs (u^n, v^n, u^{n-1}, v^{n-1}, p^n at its three nodes and the element viscosity),
// and contracted with lambda and x per element; node gradients gather their elements in
// ascending order (deterministic, no atomics).
#include "internal.cuh"
#include "mesh.cuh"

namespace cfa {

constexpr int kAdjDirs = 16;   // momentum: u^n[3] v^n[3] u^{n-1}[3] v^{n-1}[3] p^n[3] nu_e
constexpr int kForceDirs = 21;  // forces: u[3] v[3] u_old[3] v_old[3] u_prev[3] v_prev[3] p[3]

template <int N>
struct DualN {
    double v;
    double d[N];
};
using Dual = DualN<kAdjDirs>;
using DualF = DualN<kForceDirs>;

template <int N>
__device__ __forceinline__ DualN<N> dconst_n(double a) {
    DualN<N> r;
    r.v = a;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = 0.0;
    return r;
}
template <int N>
__device__ __forceinline__ DualN<N> dvar_n(double a, int dir) {
    DualN<N> r = dconst_n<N>(a);
    r.d[dir] = 1.0;
    return r;
}
__device__ __forceinline__ Dual dconst(double a) { return dconst_n<kAdjDirs>(a); }
__device__ __forceinline__ Dual dvar(double a, int dir) { return dvar_n<kAdjDirs>(a, dir); }
template <int N>
__device__ __forceinline__ DualN<N> operator+(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ DualN<N> operator-(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ DualN<N> operator*(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ DualN<N> operator*(double s, const DualN<N>& a) {
    DualN<N> r;
    r.v = s * a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = s * a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ DualN<N> operator/(const DualN<N>& a, double s) { return (1.0 / s) * a; }
template <int N>
__device__ __forceinline__ DualN<N> operator+(const DualN<N>& a, double s) {
    DualN<N> r = a;
    r.v += s;
    return r;
}
template <int N>
__device__ __forceinline__ DualN<N> dsqrt(const DualN<N>& a) {
    DualN<N> r;
    r.v = sqrt(a.v);
    const double g = r.v > 0.0 ? 0.5 / r.v : 0.0;   // |w| at w = 0: the zero subgradient
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = g * a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ DualN<N> drecip(const DualN<N>& a) {
    DualN<N> r;
    r.v = 1.0 / a.v;
    const double g = -r.v * r.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = g * a.d[k];
    return r;
}

struct AdjParams {
    double nu, rho, a0, a1, a2, c1, c2, tau_time, skew_coef;
};

__device__ __forceinline__ bool adj_dirichlet(int tag, const OutletBc& bc) {
    return tag == BC_INLET || tag == BC_WALL || tag == BC_CYLINDER || (tag == BC_OUTLET && bc.outlet_dirichlet);
}

// Per element: g[k] = sum over its non-Dirichlet nodes a and c in {u, v} of
// lambda_c[a] (d f_ac / d theta_k - sum_j d A_aj / d theta_k x_c[j]).
__global__ void __launch_bounds__(128)
k_momentum_adjoint_elems(int ne, const int* __restrict__ ev, const double* __restrict__ x,
                         const double* __restrict__ y, const int* __restrict__ tag, OutletBc bc,
                         const double* __restrict__ u_old, const double* __restrict__ v_old,
                         const double* __restrict__ u_prev, const double* __restrict__ v_prev,
                         const double* __restrict__ p_old, const double* __restrict__ nu_node, AdjParams P,
                         const double* __restrict__ xu, const double* __restrict__ xv,
                         const double* __restrict__ lu, const double* __restrict__ lv, double* __restrict__ g_elem) {
    CFA_GRID_DEP();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
    double* g = g_elem + (size_t)e * kAdjDirs;
    const double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
    const double detJ = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
    const double area = 0.5 * fabs(detJ);
    bool any = false;
    for (int a = 0; a < 3; ++a) any = any || !adj_dirichlet(tag[nd[a]], bc);
    if (area < 1.0e-14 || !any) {
        for (int k = 0; k < kAdjDirs; ++k) g[k] = 0.0;
        return;
    }
    const double inv2A = 1.0 / (2.0 * area);
    const double dNdx[3] = {(y1 - y2) * inv2A, (y2 - y0) * inv2A, (y0 - y1) * inv2A};
    const double dNdy[3] = {(x2 - x1) * inv2A, (x0 - x2) * inv2A, (x1 - x0) * inv2A};
    // element inputs as dual numbers
    Dual u_h[3], v_h[3];
    Dual w_u = dconst(0.0), w_v = dconst(0.0), div_w = dconst(0.0), dpdx = dconst(0.0), dpdy = dconst(0.0);
    for (int k = 0; k < 3; ++k) {
        const Dual un = dvar(u_old[nd[k]], k), vn = dvar(v_old[nd[k]], 3 + k);
        const Dual um = dvar(u_prev[nd[k]], 6 + k), vm = dvar(v_prev[nd[k]], 9 + k);
        const Dual pk = dvar(p_old[nd[k]], 12 + k);
        u_h[k] = P.a1 * un + P.a2 * um;
        v_h[k] = P.a1 * vn + P.a2 * vm;
        const Dual wu = P.c1 * un + P.c2 * um, wv = P.c1 * vn + P.c2 * vm;
        w_u = w_u + wu / 3.0;
        w_v = w_v + wv / 3.0;
        div_w = div_w + (dNdx[k] * wu + dNdy[k] * wv);
        dpdx = dpdx + dNdx[k] * pk;
        dpdy = dpdy + dNdy[k] * pk;
    }
    dpdx = dpdx / P.rho;
    dpdy = dpdy / P.rho;
    const Dual nu = nu_node ? dvar((nu_node[nd[0]] + nu_node[nd[1]] + nu_node[nd[2]]) / 3.0, 15) : dvar(P.nu, 15);
    const Dual vel_mag = dsqrt(w_u * w_u + w_v * w_v) + 1.0e-12;
    const double h_K = sqrt(2.0 * area);
    const double term_t = 2.0 / P.tau_time;
    const Dual term_c = (2.0 / h_K) * vel_mag;
    const Dual term_d = (4.0 / (h_K * h_K)) * nu;
    const Dual tau = drecip(dsqrt(dconst(term_t * term_t) + term_c * term_c + 9.0 * (term_d * term_d)));
    Dual ugN[3];
    for (int k = 0; k < 3; ++k) ugN[k] = dNdx[k] * w_u + dNdy[k] * w_v;
    double acc[kAdjDirs];
    for (int k = 0; k < kAdjDirs; ++k) acc[k] = 0.0;
    for (int a = 0; a < 3; ++a) {
        if (adj_dirichlet(tag[nd[a]], bc)) continue;
        const double la_u = lu[nd[a]], la_v = lv[nd[a]];
        Dual fu = dconst(0.0), fv = dconst(0.0), ax_u = dconst(0.0), ax_v = dconst(0.0);
        for (int j = 0; j < 3; ++j) {
            const double M_ij = (a == j) ? (area / 6.0) : (area / 12.0);
            const double K_ij = area * (dNdx[a] * dNdx[j] + dNdy[a] * dNdy[j]);
            const Dual C_ij = (area / 3.0) * ugN[j] + (P.skew_coef * M_ij) * div_w;
            const Dual S_ij = area * (tau * (ugN[a] * ugN[j]));
            const Dual Ms_ij = (area / 3.0) * (tau * ugN[a]);
            const Dual A_ij = (P.a0 * (Ms_ij + M_ij)) + K_ij * nu + C_ij + S_ij;
            ax_u = ax_u + xu[nd[j]] * A_ij;
            ax_v = ax_v + xv[nd[j]] * A_ij;
            fu = fu + (Ms_ij + M_ij) * u_h[j];
            fv = fv + (Ms_ij + M_ij) * v_h[j];
        }
        const Dual tw = (area * (tau * ugN[a])) + area / 3.0;
        fu = fu - tw * dpdx;
        fv = fv - tw * dpdy;
        for (int k = 0; k < kAdjDirs; ++k) acc[k] += la_u * (fu.d[k] - ax_u.d[k]) + la_v * (fv.d[k] - ax_v.d[k]);
    }
    for (int k = 0; k < kAdjDirs; ++k) g[k] = acc[k];
}

// Node gradients from the element ones (incident elements in ascending order); g_nu gets a third
// of each element's viscosity derivative (nu_e = mean of the three nodal values).
__global__ void k_momentum_adjoint_nodes(int n, const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                                         const double* __restrict__ g_elem, double* __restrict__ g_u_old,
                                         double* __restrict__ g_v_old, double* __restrict__ g_u_prev,
                                         double* __restrict__ g_v_prev, double* __restrict__ g_p_old,
                                         double* __restrict__ g_nu) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        const int e = inc[k] >> 2, a = inc[k] & 3;
        const double* g = g_elem + (size_t)e * kAdjDirs;
        s[0] += g[a];
        s[1] += g[3 + a];
        s[2] += g[6 + a];
        s[3] += g[9 + a];
        s[4] += g[12 + a];
        s[5] += g[15] / 3.0;
    }
    g_u_old[i] = s[0];
    g_v_old[i] = s[1];
    g_u_prev[i] = s[2];
    g_v_prev[i] = s[3];
    g_p_old[i] = s[4];
    if (g_nu) g_nu[i] = s[5];
}

// dJ/dU = sum over Dirichlet rows of lambda_u db_u/dU (inflow parabola 4 y (H - y) / H^2 on the
// inlet, times outlet_scale on a Dirichlet outlet); the scalar viscosity derivative (nu_node
// NULL) = the sum of the element ones. Fixed-order two-stage sums into out[0..1].
__global__ void __launch_bounds__(kThreads)
k_momentum_adjoint_scalars(int n, int ne, const int* __restrict__ tag, const double* __restrict__ y, double H,
                           OutletBc bc, const double* __restrict__ lu, const double* __restrict__ g_elem,
                           double* __restrict__ part, unsigned int* __restrict__ counter, double* __restrict__ out) {
    CFA_GRID_DEP();
    __shared__ double sh[2 * kWarps];
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int t = tag[i];
        if (t == BC_INLET || (t == BC_OUTLET && bc.outlet_dirichlet))
            v[0] += lu[i] * 4.0 * y[i] * (H - y[i]) / (H * H) * (t == BC_OUTLET ? bc.outlet_scale : 1.0);
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x)
        v[1] += g_elem[(size_t)e * kAdjDirs + 15];
    block_sum<2>(v, sh);
    if (publish_partials<2>(v, part, counter)) {
        reduce_partials<2>(v, part, counter, sh);
        if (threadIdx.x == 0) { out[0] = v[0]; out[1] = v[1]; }
    }
}

// Pressure step without OSS (stab = 0): rhs_i = -(rho/dt') sum_e (|K|/3) div u*_e on rows that
// are not pressure-Dirichlet (k_assemble_pressure_poisson, fem_kernels.cuh:201-282, with
// apply_bc_pressure). Adds R^T lambda_p to g_u, g_v (per node, gathering its elements).
__global__ void k_ppe_rhs_adjoint(int n, const int* __restrict__ ev, const double* __restrict__ x,
                                  const double* __restrict__ y, const int* __restrict__ tag, OutletBc bc,
                                  const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                                  const double* __restrict__ lam_p, const double* __restrict__ mean2, double c,
                                  double* __restrict__ g_u, double* __restrict__ g_v) {
    CFA_GRID_DEP();
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    // with the pinned outlet every row's right-hand side enters the mean removal: the adjoint of
    // the raw right-hand side is l - (m.l / sum m) on every row, l = lambda zeroed at the pin
    const double shift = mean2 ? mean2[0] / mean2[1] : 0.0;
    double su = 0.0, sv = 0.0;
    for (int k = inc_ptr[j]; k < inc_ptr[j + 1]; ++k) {
        const int e = inc[k] >> 2, b = inc[k] & 3;
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        const double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
        const double area = 0.5 * fabs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
        if (area < 1.0e-14) continue;
        const double inv2A = 1.0 / (2.0 * area);
        const double dNdx[3] = {(y1 - y2) * inv2A, (y2 - y0) * inv2A, (y0 - y1) * inv2A};
        const double dNdy[3] = {(x2 - x1) * inv2A, (x0 - x2) * inv2A, (x1 - x0) * inv2A};
        double l = 0.0;
        for (int a = 0; a < 3; ++a) {
            const bool dir = pressure_dirichlet(nd[a], tag[nd[a]], bc);
            if (mean2) l += (dir ? 0.0 : lam_p[nd[a]]) - shift;
            else if (!dir) l += lam_p[nd[a]];
        }
        const double w = c * (area / 3.0) * l;
        su += w * dNdx[b];
        sv += w * dNdy[b];
    }
    g_u[j] += su;
    g_v[j] += sv;
}

// The pinned outlet's mean removal (k_sum / k_subtract_mean, src/cfa/fem_kernels.cuh:493-510)
// transposed: out[0] = sum_i m_i l_i with l = lambda zeroed at the pin, out[1] = sum_i m_i, both in
// a fixed order.
__global__ void __launch_bounds__(kThreads)
k_pin_mean(int n, int pin, const double* __restrict__ lam, const double* __restrict__ mass,
           double* __restrict__ part, unsigned int* __restrict__ counter, double* __restrict__ out) {
    CFA_GRID_DEP();
    __shared__ double sh[2 * kWarps];
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        v[0] += i == pin ? 0.0 : mass[i] * lam[i];
        v[1] += mass[i];
    }
    block_sum<2>(v, sh);
    if (publish_partials<2>(v, part, counter)) {
        reduce_partials<2>(v, part, counter, sh);
        if (threadIdx.x == 0) { out[0] = v[0]; out[1] = v[1]; }
    }
}

// Projection (k_velocity_pressure_correction with the rotational term from the increment):
// u' = u* - (dt'/rho) M^-1 G_x dp on interior nodes and a natural outlet, p' = p + dp + nu dt'
// M^-1 K dp. Given the adjoints of u', v', p': g_dp = p'bar + nu dt' K (p'bar / m)
// - (dt'/rho) (G_x^T (mask u'bar / m) + G_y^T (mask v'bar / m)) (overwritten).
__global__ void k_projection_adjoint(int n, const int* __restrict__ ev, const double* __restrict__ x,
                                     const double* __restrict__ y, const int* __restrict__ tag, OutletBc bc,
                                     const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                                     const double* __restrict__ mass, double dt, double rho, double nu,
                                     const double* __restrict__ gu, const double* __restrict__ gv,
                                     const double* __restrict__ gp, double* __restrict__ g_dp) {
    CFA_GRID_DEP();
    const int k0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (k0 >= n) return;
    double s = 0.0;
    for (int q = inc_ptr[k0]; q < inc_ptr[k0 + 1]; ++q) {
        const int e = inc[q] >> 2, b = inc[q] & 3;
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        const double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
        const double area = 0.5 * fabs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
        if (area < 1.0e-14) continue;
        const double inv2A = 1.0 / (2.0 * area);
        const double dNdx[3] = {(y1 - y2) * inv2A, (y2 - y0) * inv2A, (y0 - y1) * inv2A};
        const double dNdy[3] = {(x2 - x1) * inv2A, (x0 - x2) * inv2A, (x1 - x0) * inv2A};
        double psx = 0.0, psy = 0.0, au = 0.0, av = 0.0;
        for (int a = 0; a < 3; ++a) {
            const int i = nd[a];
            const double m_i = fmax(mass[i], 1.0e-14);
            const double psi = gp[i] / m_i;
            psx += psi * dNdx[a];
            psy += psi * dNdy[a];
            const int t = tag[i];
            if (t == BC_INTERIOR || (t == BC_OUTLET && !bc.outlet_dirichlet)) {
                au += gu[i] / m_i;
                av += gv[i] / m_i;
            }
        }
        s += nu * dt * area * (dNdx[b] * psx + dNdy[b] * psy);
        s -= (dt / rho) * (area / 3.0) * (dNdx[b] * au + dNdy[b] * av);
    }
    g_dp[k0] = gp[k0] + s;
}

// Volume forces (k_volume_forces, fem_kernels.cuh:1046-1123): per element the derivatives of
// wx F_x + wy F_y with respect to its 21 nodal inputs (dual numbers through the same formula).
__global__ void __launch_bounds__(128)
k_forces_adjoint_elems(int ne, const int* __restrict__ ev, const int* __restrict__ tag, const double* __restrict__ x,
                       const double* __restrict__ y, const double* __restrict__ u, const double* __restrict__ v,
                       const double* __restrict__ u_old, const double* __restrict__ v_old,
                       const double* __restrict__ u_prev, const double* __restrict__ v_prev,
                       const double* __restrict__ p, double b0, double b1, double b2, double nu, double rho, double wx,
                       double wy, double* __restrict__ g_elem) {
    CFA_GRID_DEP();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    double* g = g_elem + (size_t)e * kForceDirs;
    const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
    double phi[3];
    bool touches = false;
    for (int a = 0; a < 3; ++a) {
        phi[a] = tag[nd[a]] == BC_CYLINDER ? 1.0 : 0.0;
        touches = touches || phi[a] > 0.0;
    }
    const double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
    const double area = 0.5 * fabs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
    if (!touches || area < 1.0e-14) {
        for (int k = 0; k < kForceDirs; ++k) g[k] = 0.0;
        return;
    }
    const double inv2A = 1.0 / (2.0 * area);
    const double dNdx[3] = {(y1 - y2) * inv2A, (y2 - y0) * inv2A, (y0 - y1) * inv2A};
    const double dNdy[3] = {(x2 - x1) * inv2A, (x0 - x2) * inv2A, (x1 - x0) * inv2A};
    DualF ue[3], ve[3], ute[3], vte[3];
    DualF dudx = dconst_n<kForceDirs>(0.0), dudy = dudx, dvdx = dudx, dvdy = dudx, p_bar = dudx;
    double dphidx = 0.0, dphidy = 0.0;
    for (int a = 0; a < 3; ++a) {
        ue[a] = dvar_n<kForceDirs>(u[nd[a]], a);
        ve[a] = dvar_n<kForceDirs>(v[nd[a]], 3 + a);
        ute[a] = b0 * ue[a] + b1 * dvar_n<kForceDirs>(u_old[nd[a]], 6 + a) +
                 b2 * dvar_n<kForceDirs>(u_prev[nd[a]], 12 + a);
        vte[a] = b0 * ve[a] + b1 * dvar_n<kForceDirs>(v_old[nd[a]], 9 + a) +
                 b2 * dvar_n<kForceDirs>(v_prev[nd[a]], 15 + a);
        dudx = dudx + dNdx[a] * ue[a];
        dudy = dudy + dNdy[a] * ue[a];
        dvdx = dvdx + dNdx[a] * ve[a];
        dvdy = dvdy + dNdy[a] * ve[a];
        dphidx += phi[a] * dNdx[a];
        dphidy += phi[a] * dNdy[a];
        p_bar = p_bar + dvar_n<kForceDirs>(p[nd[a]], 18 + a) / 3.0;
    }
    DualF fx = dconst_n<kForceDirs>(0.0), fy = fx;
    for (int a = 0; a < 3; ++a) {
        const int b = (a + 1) % 3;
        const double phi_m = 0.5 * (phi[a] + phi[b]);
        if (phi_m == 0.0) continue;
        const DualF um = 0.5 * (ue[a] + ue[b]), vm = 0.5 * (ve[a] + ve[b]);
        fx = fx + phi_m * (0.5 * (ute[a] + ute[b]) + (um * dudx + vm * dudy));
        fy = fy + phi_m * (0.5 * (vte[a] + vte[b]) + (um * dvdx + vm * dvdy));
    }
    fx = (area / 3.0) * fx;
    fy = (area / 3.0) * fy;
    fx = fx + area * ((nu * dphidx) * dudx + (nu * dphidy) * dudy - (dphidx / rho) * p_bar);
    fy = fy + area * ((nu * dphidx) * dvdx + (nu * dphidy) * dvdy - (dphidy / rho) * p_bar);
    for (int k = 0; k < kForceDirs; ++k) g[k] = wx * fx.d[k] + wy * fy.d[k];
}

// Node sums of the element force derivatives into seven nodal gradients (added to).
__global__ void k_forces_adjoint_nodes(int n, const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                                       const double* __restrict__ g_elem, double* __restrict__ g_u,
                                       double* __restrict__ g_v, double* __restrict__ g_u_old,
                                       double* __restrict__ g_v_old, double* __restrict__ g_u_prev,
                                       double* __restrict__ g_v_prev, double* __restrict__ g_p) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        const int e = inc[k] >> 2, a = inc[k] & 3;
        const double* g = g_elem + (size_t)e * kForceDirs;
        for (int q = 0; q < 7; ++q) s[q] += g[3 * q + a];
    }
    g_u[i] += s[0]; g_v[i] += s[1]; g_u_old[i] += s[2]; g_v_old[i] += s[3];
    g_u_prev[i] += s[4]; g_v_prev[i] += s[5]; g_p[i] += s[6];
}

// ---- the OSS terms of the pressure step (stab > 0) ----
// With s_K the OSS weights of u* (k_compute_oss_weights, src/cfa/fem_kernels.cuh:697-719) and
// G(f)_k = sum_{K ∋ k} sqrt(s_K) |K|/3 grad f|K (k_accumulate_scalar_gradient, :726-757), the
// pressure step's matrix is (1 + s_K) K - [rows not Dirichlet] B^T M^-1 B and its right-hand side
// carries -[s_K |K| grad N_i . grad p^n - |K| grad N_i . sqrt(s_K)/3 sum_{k in K} G(p^n)_k / m_k]
// (k_assemble_pressure_poisson, :201-282; k_assemble_oss_operator). With the solution dp zero on
// Dirichlet rows and l the pressure adjoint with its Dirichlet entries zeroed, the s-dependent part
// of l^T (rhs_p - A dp) is -Phi(l, q), q = p^n + dp, where
//   Phi(l, q) = sum_K s_K |K| grad l|K . grad q|K - sum_k G(l)_k . G(q)_k / m_k.
// Per element: g_s = -dPhi/ds_K, mapped to u*, v* through ds_K/du*_j (the weight's formula,
// differentiated by hand; the zero subgradient where |u-bar| = 0); per vertex: -dPhi/dq_j, the
// p^n gradient. Five values per element: d/du and d/dv (equal for its three vertices), d/dp0..2.
// With the pinned outlet the right-hand side's mean removal adds c Phi(1, p^n) (c = m.l / sum m),
// which vanishes: the constant has no gradient, so Phi(1, .) = 0 and l zeroed at the pin suffices.
__global__ void __launch_bounds__(kThreads)
k_oss_adjoint_elems(int ne, const int* __restrict__ ev, const double* __restrict__ x, const double* __restrict__ y,
                    const double* __restrict__ us, const double* __restrict__ vs, const double* __restrict__ elem_s,
                    const double* __restrict__ mass, const double* __restrict__ lam, const double* __restrict__ q,
                    const double* __restrict__ glx, const double* __restrict__ gly, const double* __restrict__ gqx,
                    const double* __restrict__ gqy, double dt, double rho, double nu, double stab,
                    double* __restrict__ g_elem) {
    CFA_GRID_DEP();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    double* g = g_elem + (size_t)e * 5;
    const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
    const double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
    const double area = 0.5 * fabs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
    const double sK = elem_s[e];
    if (area < 1.0e-14 || !(sK > 0.0)) {
        for (int k = 0; k < 5; ++k) g[k] = 0.0;
        return;
    }
    const double inv2A = 1.0 / (2.0 * area);
    const double dNdx[3] = {(y1 - y2) * inv2A, (y2 - y0) * inv2A, (y0 - y1) * inv2A};
    const double dNdy[3] = {(x2 - x1) * inv2A, (x0 - x2) * inv2A, (x1 - x0) * inv2A};
    double lx = 0.0, ly = 0.0, qx = 0.0, qy = 0.0, slx = 0.0, sly = 0.0, sqx = 0.0, sqy = 0.0;
    for (int a = 0; a < 3; ++a) {
        const int k = nd[a];
        lx += lam[k] * dNdx[a];
        ly += lam[k] * dNdy[a];
        qx += q[k] * dNdx[a];
        qy += q[k] * dNdy[a];
        const double im = 1.0 / fmax(mass[k], 1.0e-14);
        slx += glx[k] * im;
        sly += gly[k] * im;
        sqx += gqx[k] * im;
        sqy += gqy[k] * im;
    }
    const double rs = sqrt(sK);
    // dPhi/ds_K: the s_K K term, and sqrt(s_K) in G(l)_k and G(q)_k of the element's vertices
    const double dphi = area * (lx * qx + ly * qy) - area / (6.0 * rs) * (lx * sqx + ly * sqy + slx * qx + sly * qy);
    const double gs = -dphi;
    // s_K = rho tau / dt, tau = stab / (rho (4 nu / h^2 + 2 |u-bar| / h) + 1e-300), h = sqrt(2 |K|)
    const double h = sqrt(2.0 * area);
    const double ub = (us[nd[0]] + us[nd[1]] + us[nd[2]]) / 3.0;
    const double vb = (vs[nd[0]] + vs[nd[1]] + vs[nd[2]]) / 3.0;
    const double nrm = sqrt(ub * ub + vb * vb);
    const double den = rho * (4.0 * nu / (h * h) + 2.0 * nrm / h) + 1.0e-300;
    const double ds_dnrm = (rho / dt) * (-stab / (den * den)) * (rho * 2.0 / h);
    const double c = nrm > 0.0 ? gs * ds_dnrm / (3.0 * nrm) : 0.0;
    g[0] = c * ub;
    g[1] = c * vb;
    // -dPhi/dq_j
    for (int j = 0; j < 3; ++j)
        g[2 + j] = -(sK * area * (lx * dNdx[j] + ly * dNdy[j]) - rs * (area / 3.0) * (dNdx[j] * slx + dNdy[j] * sly));
}

__global__ void k_oss_adjoint_nodes(int n, const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                                    const double* __restrict__ g_elem, double* __restrict__ g_u,
                                    double* __restrict__ g_v, double* __restrict__ g_p) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double su = 0.0, sv = 0.0, sp = 0.0;
    for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        const int e = inc[k] >> 2, a = inc[k] & 3;
        const double* g = g_elem + (size_t)e * 5;
        su += g[0];
        sv += g[1];
        sp += g[2 + a];
    }
    g_u[i] += su;
    g_v[i] += sv;
    g_p[i] += sp;
}

// l = lambda with its Dirichlet entries zeroed, q = p^n + dp
__global__ void k_oss_adjoint_inputs(int n, const int* __restrict__ tag, OutletBc bc, const double* __restrict__ lam,
                                     const double* __restrict__ p_old, const double* __restrict__ dp,
                                     double* __restrict__ l, double* __restrict__ q) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    l[i] = pressure_dirichlet(i, tag[i], bc) ? 0.0 : lam[i];
    q[i] = p_old[i] + dp[i];
}

}  // namespace cfa

using namespace cfa;

extern "C" {

cfa_status cfa_momentum_adjoint(cfa_ctx* ctx, const cfa_mesh* m, const double* u_old, const double* v_old,
                                const double* u_prev, const double* v_prev, const double* p_old,
                                const cfa_momentum_params* prm, const double* nu_node, const cfa_momentum_bc* bcp,
                                const double* x_u, const double* x_v, const double* lam_u, const double* lam_v,
                                double* g_u_old, double* g_v_old, double* g_u_prev, double* g_v_prev,
                                double* g_p_old, double* g_nu_node, double* d_scalars2) {
    CFA_ENTER(ctx);
    CFA_ARG(m && u_old && v_old && u_prev && v_prev && p_old && prm && bcp && x_u && x_v && lam_u && lam_v);
    CFA_ARG(g_u_old && g_v_old && g_u_prev && g_v_prev && g_p_old && d_scalars2 && (!g_nu_node || nu_node));
    AdjParams P{prm->nu, prm->rho, prm->a0, prm->a1, prm->a2, prm->c1, prm->c2, prm->tau_time, prm->skew_coef};
    DevBuf<double> g_elem;
    CFA_CUDA(g_elem.ensure((size_t)std::max(m->ne, 1) * kAdjDirs));
    CFA_LAUNCH(ctx, k_momentum_adjoint_elems, ceil_div(m->ne, 128), 128, 0, m->ne, m->ev, m->x, m->y, m->tag, m->bc,
               u_old, v_old, u_prev, v_prev, p_old, nu_node, P, x_u, x_v, lam_u, lam_v, g_elem.p);
    CFA_LAUNCH(ctx, k_momentum_adjoint_nodes, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->inc_ptr.p, m->inc.p,
               (const double*)g_elem.p, g_u_old, g_v_old, g_u_prev, g_v_prev, g_p_old, g_nu_node);
    const int grid = std::min(ceil_div(std::max(m->n, m->ne), kThreads), 4 * ctx->num_sms);
    CFA_PROPAGATE(ensure_partials(ctx, 2 * (size_t)grid + 2));
    CFA_LAUNCH(ctx, k_momentum_adjoint_scalars, grid, kThreads, 0, m->n, m->ne, m->tag, m->y, bcp->H, m->bc, lam_u,
               (const double*)g_elem.p, ctx->d_part, ctx->d_counters, d_scalars2);
    CFA_CHECK_LAUNCH();
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));   // g_elem is released on return
    return CFA_OK;
}

cfa_status cfa_ppe_rhs_adjoint(cfa_ctx* ctx, const cfa_mesh* m, const double* lam_p, double dt_proj, double rho,
                               double* g_u, double* g_v) {
    CFA_ENTER(ctx);
    CFA_ARG(m && lam_p && g_u && g_v && dt_proj > 0.0);
    const bool pinned = m->bc.outlet_dirichlet != 0;
    CFA_ARG(!pinned || (m->bc.pin >= 0 && m->bc.pin < m->n));
    DevBuf<double> buf;   // pinned outlet: lumped mass [n], the two sums
    const double* mean2 = nullptr;
    if (pinned) {
        CFA_CUDA(buf.ensure((size_t)m->n + 2));
        CFA_PROPAGATE(cfa_lumped_mass(ctx, m, buf.p));
        const int grid = row_grid(ctx, m->n, 1);
        CFA_PROPAGATE(ensure_partials(ctx, 2 * (size_t)grid + 2));
        CFA_LAUNCH(ctx, k_pin_mean, grid, kThreads, 0, m->n, m->bc.pin, lam_p, (const double*)buf.p, ctx->d_part,
                   ctx->d_counters, buf.p + m->n);
        mean2 = buf.p + m->n;
    }
    CFA_LAUNCH(ctx, k_ppe_rhs_adjoint, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->ev, m->x, m->y, m->tag, m->bc,
               m->inc_ptr.p, m->inc.p, lam_p, mean2, -(rho / dt_proj), g_u, g_v);
    CFA_CHECK_LAUNCH();
    if (pinned) CFA_CUDA(cudaStreamSynchronize(ctx->stream));   // buf is released on return
    return CFA_OK;
}

cfa_status cfa_oss_adjoint(cfa_ctx* ctx, const cfa_mesh* m, const double* u_star, const double* v_star, double dt_proj,
                           double rho, double nu, double stab, const double* elem_s, const double* mass_lumped,
                           const double* lam_p, const double* p_old, const double* dp, double* g_u, double* g_v,
                           double* g_p) {
    CFA_ENTER(ctx);
    CFA_ARG(m && u_star && v_star && elem_s && mass_lumped && lam_p && p_old && dp && g_u && g_v && g_p);
    CFA_ARG(dt_proj > 0.0 && stab > 0.0);
    const int n = m->n, ne = m->ne;
    DevBuf<double> buf;   // l, q, G(l) x/y, G(q) x/y, per-element values
    CFA_CUDA(buf.ensure(6 * (size_t)n + 5 * (size_t)ne));
    double *l = buf.p, *q = buf.p + n, *glx = buf.p + 2 * (size_t)n, *gly = buf.p + 3 * (size_t)n;
    double *gqx = buf.p + 4 * (size_t)n, *gqy = buf.p + 5 * (size_t)n, *ge = buf.p + 6 * (size_t)n;
    CFA_LAUNCH(ctx, k_oss_adjoint_inputs, ceil_div(n, kThreads), kThreads, 0, n, m->tag, m->bc, lam_p, p_old, dp, l, q);
    CFA_PROPAGATE(cfa_scalar_gradient(ctx, m, l, elem_s, glx, gly));
    CFA_PROPAGATE(cfa_scalar_gradient(ctx, m, q, elem_s, gqx, gqy));
    CFA_LAUNCH(ctx, k_oss_adjoint_elems, ceil_div(ne, kThreads), kThreads, 0, ne, m->ev, m->x, m->y, u_star, v_star,
               elem_s, mass_lumped, (const double*)l, (const double*)q, (const double*)glx, (const double*)gly,
               (const double*)gqx, (const double*)gqy, dt_proj, rho, nu, stab, ge);
    CFA_LAUNCH(ctx, k_oss_adjoint_nodes, ceil_div(n, kThreads), kThreads, 0, n, m->inc_ptr.p, m->inc.p,
               (const double*)ge, g_u, g_v, g_p);
    CFA_CHECK_LAUNCH();
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));   // buf is released on return
    return CFA_OK;
}

cfa_status cfa_projection_adjoint(cfa_ctx* ctx, const cfa_mesh* m, double dt_proj, double rho, double nu,
                                  const double* mass_lumped, const double* g_u_new, const double* g_v_new,
                                  const double* g_p_new, double* g_dp) {
    CFA_ENTER(ctx);
    CFA_ARG(m && mass_lumped && g_u_new && g_v_new && g_p_new && g_dp && g_dp != g_p_new);
    CFA_LAUNCH(ctx, k_projection_adjoint, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->ev, m->x, m->y, m->tag,
               m->bc, m->inc_ptr.p, m->inc.p, mass_lumped, dt_proj, rho, nu, g_u_new, g_v_new, g_p_new, g_dp);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_volume_forces_adjoint(cfa_ctx* ctx, const cfa_mesh* m, const double* u, const double* v,
                                     const double* u_old, const double* v_old, const double* u_prev,
                                     const double* v_prev, const double* p, double b0, double b1, double b2,
                                     double nu, double rho, double wx, double wy, double* g_u, double* g_v,
                                     double* g_u_old, double* g_v_old, double* g_u_prev, double* g_v_prev,
                                     double* g_p) {
    CFA_ENTER(ctx);
    CFA_ARG(m && u && v && u_old && v_old && u_prev && v_prev && p && g_u && g_v && g_u_old && g_v_old && g_u_prev &&
            g_v_prev && g_p);
    DevBuf<double> g_elem;
    CFA_CUDA(g_elem.ensure((size_t)std::max(m->ne, 1) * kForceDirs));
    CFA_LAUNCH(ctx, k_forces_adjoint_elems, ceil_div(m->ne, 128), 128, 0, m->ne, m->ev, m->tag, m->x, m->y, u, v,
               u_old, v_old, u_prev, v_prev, p, b0, b1, b2, nu, rho, wx, wy, g_elem.p);
    CFA_LAUNCH(ctx, k_forces_adjoint_nodes, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->inc_ptr.p, m->inc.p,
               (const double*)g_elem.p, g_u, g_v, g_u_old, g_v_old, g_u_prev, g_v_prev, g_p);
    CFA_CHECK_LAUNCH();
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));   // g_elem is released on return
    return CFA_OK;
}

}  // extern "C"
