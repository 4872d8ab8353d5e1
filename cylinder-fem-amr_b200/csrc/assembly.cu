// Atomic-free element assembly (a3-a9): one thread per matrix row gathers the contributions of
// the row's elements from the sorted node -> element incidence, in ascending element order, and
// writes every value once. Compared with the reference's one-thread-per-element kernels with FP64
// atomicAdd into a binary-searched CSR slot (src/cfa/fem_kernels.cuh:40-282, :697-909), there
// are no atomics and no searches, the result is deterministic, and each CSR value is written
// exactly once (coalesced along the row).
#include <mutex>

#include "internal.cuh"
#include "mesh.cuh"

namespace cfa {

struct Geom {
    double area, dNdx[3], dNdy[3];
    bool ok;
};

// Element geometry exactly as the reference kernels compute it (fem_kernels.cuh:77-87)
__device__ __forceinline__ Geom elem_geom(const int* nd, const double* __restrict__ x, const double* __restrict__ y) {
    Geom g;
    const double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
    const double detJ = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
    g.area = 0.5 * fabs(detJ);
    g.ok = !(g.area < 1.0e-14);
    const double inv2A = 1.0 / (2.0 * g.area);
    g.dNdx[0] = (y1 - y2) * inv2A; g.dNdx[1] = (y2 - y0) * inv2A; g.dNdx[2] = (y0 - y1) * inv2A;
    g.dNdy[0] = (x2 - x1) * inv2A; g.dNdy[1] = (x0 - x2) * inv2A; g.dNdy[2] = (x1 - x0) * inv2A;
    return g;
}

__device__ __forceinline__ void load_elem(const int* __restrict__ ev, int e, int* nd) {
    nd[0] = ev[3 * e]; nd[1] = ev[3 * e + 1]; nd[2] = ev[3 * e + 2];
}

struct MomParams {
    double dt, nu, rho, a0, a1, a2, c1, c2, tau_time, skew_coef;
};

// Dirichlet rows of the momentum system (k_apply_bc_momentum, fem_kernels.cuh:431-441)
__device__ __forceinline__ bool momentum_dirichlet(int tag, const OutletBc& bc) {
    return tag == BC_INLET || tag == BC_WALL || tag == BC_CYLINDER || (tag == BC_OUTLET && bc.outlet_dirichlet);
}
__device__ __forceinline__ double momentum_bc_u(int tag, double yi, double u_max, double H, const OutletBc& bc) {
    if (tag == BC_INLET || tag == BC_OUTLET)
        return 4.0 * u_max * yi * (H - yi) / (H * H) * (tag == BC_OUTLET ? bc.outlet_scale : 1.0);
    return 0.0;
}

// Momentum rows: k_assemble_momentum_fem (fem_kernels.cuh:40-181) gathered per row, lumped mass,
// and (with_bc) the Dirichlet rows of k_apply_bc_momentum (:411-453) on A and the RHS. A row of
// up to kMomCap entries accumulates in shared memory laid out [slot][thread] (conflict-free for
// any slot a thread adds to); longer rows in place in global memory. Same addition order.
constexpr int kMomCap = 16;
constexpr size_t kMomSmem = (size_t)kMomCap * kThreads * sizeof(double);

__global__ void __launch_bounds__(kThreads)
k_momentum_rows(int n, const int* __restrict__ ev, const double* __restrict__ x, const double* __restrict__ y,
                const int* __restrict__ tag, const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                const int* __restrict__ pos, const int* __restrict__ rp, const int* __restrict__ ci,
                const double* __restrict__ u_old, const double* __restrict__ v_old,
                const double* __restrict__ u_prev, const double* __restrict__ v_prev,
                const double* __restrict__ p_old, const double* __restrict__ nu_node, MomParams P, int with_bc,
                double u_max, double H, OutletBc bc, double* __restrict__ A_val, double* __restrict__ rhs_u,
                double* __restrict__ rhs_v, double* __restrict__ mass) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r0 = rp[i], len = rp[i + 1] - r0;
    const bool dir = with_bc && momentum_dirichlet(tag[i], bc);
    const bool local = len <= kMomCap;
    extern __shared__ double mom_sm[];   // [kMomCap][blockDim.x]
    const int T = blockDim.x;
    double* acc = mom_sm + threadIdx.x;  // acc[q * T]: entry q of this row
    if (!dir) {
        if (local) {
            for (int q = 0; q < len; ++q) acc[q * T] = 0.0;
        } else {
            for (int q = 0; q < len; ++q) A_val[r0 + q] = 0.0;
        }
    }
    double f_u_row = 0.0, f_v_row = 0.0, m_row = 0.0;
    // reciprocals of the constant and per-launch divisors, taken once (the products differ from
    // the quotients in the last bit at most; the element formula is division-bound in FP64)
    constexpr double kThird = 1.0 / 3.0, kSixth = 1.0 / 6.0, kTwelfth = 1.0 / 12.0;
    const double inv_rho = 1.0 / P.rho, term_t_p = 2.0 / P.tau_time;
    for (int s = inc_ptr[i]; s < inc_ptr[i + 1]; ++s) {
        const int e = inc[s] >> 2, a = inc[s] & 3;
        int nd[3];
        load_elem(ev, e, nd);
        const Geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        const double area = g.area;
        const double area3 = area * kThird;
        m_row += area3;
        if (dir) continue;
        double u_h[3], v_h[3], w_u = 0.0, w_v = 0.0, div_w = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double un = u_old[nd[k]], vn = v_old[nd[k]], um = u_prev[nd[k]], vm = v_prev[nd[k]];
            u_h[k] = P.a1 * un + P.a2 * um;
            v_h[k] = P.a1 * vn + P.a2 * vm;
            const double wu = P.c1 * un + P.c2 * um, wv = P.c1 * vn + P.c2 * vm;
            w_u += wu * kThird;
            w_v += wv * kThird;
            div_w += wu * g.dNdx[k] + wv * g.dNdy[k];
        }
        const double vel_mag = sqrt(w_u * w_u + w_v * w_v) + 1.0e-12;
        const double h_K = sqrt(2.0 * area);
        // element viscosity: the scalar nu, or the mean of a nodal field
        const double nu = nu_node ? (nu_node[nd[0]] + nu_node[nd[1]] + nu_node[nd[2]]) * kThird : P.nu;
        const double term_t = term_t_p;
        const double term_c = 2.0 * vel_mag / h_K;
        const double term_d = 4.0 * nu / (h_K * h_K);
        const double tau_supg = 1.0 / sqrt(term_t * term_t + term_c * term_c + 9.0 * term_d * term_d);
        const double p0 = p_old[nd[0]], p1 = p_old[nd[1]], p2 = p_old[nd[2]];
        const double dpdx = (p0 * g.dNdx[0] + p1 * g.dNdx[1] + p2 * g.dNdx[2]) * inv_rho;
        const double dpdy = (p0 * g.dNdy[0] + p1 * g.dNdy[1] + p2 * g.dNdy[2]) * inv_rho;
        double ugN[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) ugN[k] = w_u * g.dNdx[k] + w_v * g.dNdy[k];
        double f_u = 0.0, f_v = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double M_ij = (a == j) ? (area * kSixth) : (area * kTwelfth);
            const double K_ij = area * (g.dNdx[a] * g.dNdx[j] + g.dNdy[a] * g.dNdy[j]);
            const double C_ij = area3 * ugN[j] + P.skew_coef * div_w * M_ij;
            const double S_ij = area * tau_supg * ugN[a] * ugN[j];
            const double Ms_ij = area3 * tau_supg * ugN[a];
            const double A_ij = P.a0 * (M_ij + Ms_ij) + nu * K_ij + C_ij + S_ij;
            const int p = pos[3 * s + j];
            if (local) acc[(p - r0) * T] += A_ij; else A_val[p] += A_ij;
            f_u += (M_ij + Ms_ij) * u_h[j];
            f_v += (M_ij + Ms_ij) * v_h[j];
        }
        const double tw = area3 + area * tau_supg * ugN[a];
        f_u -= tw * dpdx;
        f_v -= tw * dpdy;
        f_u_row += f_u;
        f_v_row += f_v;
    }
    mass[i] = m_row;
    if (dir) {
        const int t = tag[i];
        const double ub = momentum_bc_u(t, y[i], u_max, H, bc);
        for (int q = 0; q < len; ++q) A_val[r0 + q] = (ci[r0 + q] == i) ? 1.0 : 0.0;
        rhs_u[i] = ub;
        rhs_v[i] = 0.0;
        return;
    }
    if (local)
        for (int q = 0; q < len; ++q) A_val[r0 + q] = acc[q * T];
    rhs_u[i] = f_u_row;
    rhs_v[i] = f_v_row;
}

// Dirichlet rows of the momentum system alone (k_apply_bc_momentum, fem_kernels.cuh:411-453);
// rows_too writes the A rows and RHS as well, otherwise only the solution values.
__global__ void k_momentum_bc(int n, const int* __restrict__ tag, const double* __restrict__ y,
                              const int* __restrict__ rp, const int* __restrict__ ci, double u_max, double H,
                              OutletBc bc, int rows_too, double* __restrict__ A_val, double* __restrict__ rhs_u,
                              double* __restrict__ rhs_v, double* __restrict__ u, double* __restrict__ v) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int t = tag[i];
    if (!momentum_dirichlet(t, bc)) return;
    const double ub = momentum_bc_u(t, y[i], u_max, H, bc);
    if (rows_too) {
        for (int q = rp[i]; q < rp[i + 1]; ++q) A_val[q] = (ci[q] == i) ? 1.0 : 0.0;
        rhs_u[i] = ub;
        rhs_v[i] = 0.0;
    }
    if (u) u[i] = ub;
    if (v) v[i] = 0.0;
}

// k_assemble_lumped_mass (fem_kernels.cuh:890-909), per row
__global__ void k_lumped_mass_rows(int n, const int* __restrict__ ev, const double* __restrict__ x,
                                   const double* __restrict__ y, const int* __restrict__ inc_ptr,
                                   const int* __restrict__ inc, double* __restrict__ m) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        int nd[3];
        load_elem(ev, inc[k] >> 2, nd);
        const double detJ = (x[nd[1]] - x[nd[0]]) * (y[nd[2]] - y[nd[0]]) - (x[nd[2]] - x[nd[0]]) * (y[nd[1]] - y[nd[0]]);
        s += fabs(detJ) / 6.0;
    }
    m[i] = s;
}

// k_compute_oss_weights (fem_kernels.cuh:697-719), one thread per element
__global__ void k_oss_weights(int ne, const int* __restrict__ ev, const double* __restrict__ x,
                              const double* __restrict__ y, const double* __restrict__ us,
                              const double* __restrict__ vs, double dt, double rho, double nu, double stab,
                              double* __restrict__ elem_s) {
    CFA_GRID_DEP();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int n0 = ev[3 * e], n1 = ev[3 * e + 1], n2 = ev[3 * e + 2];
    const double area = 0.5 * fabs((x[n1] - x[n0]) * (y[n2] - y[n0]) - (x[n2] - x[n0]) * (y[n1] - y[n0]));
    const double h = sqrt(2.0 * area);
    const double ub = (us[n0] + us[n1] + us[n2]) / 3.0;
    const double vb = (vs[n0] + vs[n1] + vs[n2]) / 3.0;
    const double tau = stab / (rho * (4.0 * nu / (h * h) + 2.0 * sqrt(ub * ub + vb * vb) / h) + 1.0e-300);
    elem_s[e] = rho * tau / dt;
}

// k_accumulate_scalar_gradient (fem_kernels.cuh:726-757), per row: G_i(f) numerators
__global__ void k_scalar_gradient_rows(int n, const int* __restrict__ ev, const double* __restrict__ x,
                                       const double* __restrict__ y, const int* __restrict__ inc_ptr,
                                       const int* __restrict__ inc, const double* __restrict__ f,
                                       const double* __restrict__ elem_s, double* __restrict__ gx_out,
                                       double* __restrict__ gy_out) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sx = 0.0, sy = 0.0;
    for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        const int e = inc[k] >> 2;
        int nd[3];
        load_elem(ev, e, nd);
        const double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
        const double detJ = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
        const double area = 0.5 * fabs(detJ);
        if (area < 1.0e-14) continue;
        const double inv2A = 1.0 / (2.0 * area);
        const double gx = (f[nd[0]] * (y1 - y2) + f[nd[1]] * (y2 - y0) + f[nd[2]] * (y0 - y1)) * inv2A;
        const double gy = (f[nd[0]] * (x2 - x1) + f[nd[1]] * (x0 - x2) + f[nd[2]] * (x1 - x0)) * inv2A;
        const double w = (elem_s ? sqrt(elem_s[e]) : 1.0) * area / 3.0;
        sx += w * gx;
        sy += w * gy;
    }
    gx_out[i] = sx;
    gy_out[i] = sy;
}

// Pressure rows: k_assemble_pressure_poisson (fem_kernels.cuh:201-282) gathered per row; with
// oss_val the rows of B and B^T of k_assemble_oss_operator (:807-847) and inv_m (:849-852) in
// the same pass; with with_bc the Dirichlet rows/columns of k_apply_bc_pressure (:460-490).
// A row of up to kPressCap entries accumulates K, Bx, By, B^T x, B^T y in shared memory laid out
// [array][slot][thread], so that threads adding to different slots of their rows hit different
// banks; longer rows accumulate in place in global memory. Every entry takes its terms in the
// element order of the incidence either way.
constexpr int kPressThreads = 128;
constexpr int kPressCap = 16;
constexpr size_t kPressSmem = (size_t)5 * kPressCap * kPressThreads * sizeof(double);

__global__ void __launch_bounds__(kPressThreads)
k_pressure_rows(int n, int nnz, const int* __restrict__ ev, const double* __restrict__ x,
                const double* __restrict__ y, const int* __restrict__ tag, const int* __restrict__ inc_ptr,
                const int* __restrict__ inc, const int* __restrict__ pos, const int* __restrict__ rp,
                const int* __restrict__ ci, const double* __restrict__ us, const double* __restrict__ vs,
                const double* __restrict__ p_old, const double* __restrict__ gpx, const double* __restrict__ gpy,
                const double* __restrict__ mass, const double* __restrict__ elem_s, double dt, double rho,
                double stab, int with_bc, OutletBc bc, double* __restrict__ Kp_val, double* __restrict__ rhs_p,
                double* __restrict__ div_num, double* __restrict__ dp, double* __restrict__ oss_val,
                double* __restrict__ inv_m) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r0 = rp[i], len = rp[i + 1] - r0;
    const bool local = len <= kPressCap;
    const bool want_oss = oss_val != nullptr;
    extern __shared__ double press_sm[];   // [5][kPressCap][blockDim.x]
    const int T = blockDim.x, tt = threadIdx.x;
    double* sK = press_sm + tt;                          // sK[q * T]: K entry q of this row
    double* sBx = press_sm + 1 * kPressCap * T + tt;
    double* sBy = press_sm + 2 * kPressCap * T + tt;
    double* sTx = press_sm + 3 * kPressCap * T + tt;
    double* sTy = press_sm + 4 * kPressCap * T + tt;
    double *Bx = oss_val, *By = oss_val + (size_t)nnz, *BTx = oss_val + 2 * (size_t)nnz, *BTy = oss_val + 3 * (size_t)nnz;
    if (local) {
        for (int q = 0; q < len; ++q) {
            sK[q * T] = 0.0;
            if (want_oss) { sBx[q * T] = 0.0; sBy[q * T] = 0.0; sTx[q * T] = 0.0; sTy[q * T] = 0.0; }
        }
    } else {
        for (int q = 0; q < len; ++q) Kp_val[r0 + q] = 0.0;
        if (want_oss)
            for (int q = 0; q < len; ++q) { Bx[r0 + q] = 0.0; By[r0 + q] = 0.0; BTx[r0 + q] = 0.0; BTy[r0 + q] = 0.0; }
    }
    double rhs_row = 0.0, div_row = 0.0;
    for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
        const int e = inc[k] >> 2, a = inc[k] & 3;
        int nd[3];
        load_elem(ev, e, nd);
        const Geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        const double area = g.area;
        const double div_u = us[nd[0]] * g.dNdx[0] + us[nd[1]] * g.dNdx[1] + us[nd[2]] * g.dNdx[2]
                           + vs[nd[0]] * g.dNdy[0] + vs[nd[1]] * g.dNdy[1] + vs[nd[2]] * g.dNdy[2];
        const double rhs_contrib = -(rho / dt) * (area / 3.0) * div_u;
        double s = 0.0, sx = 0.0, sy = 0.0, gx = 0.0, gy = 0.0;
        if (stab > 0.0) {
            s = elem_s[e];
            const double rs = sqrt(s);
            gx = p_old[nd[0]] * g.dNdx[0] + p_old[nd[1]] * g.dNdx[1] + p_old[nd[2]] * g.dNdx[2];
            gy = p_old[nd[0]] * g.dNdy[0] + p_old[nd[1]] * g.dNdy[1] + p_old[nd[2]] * g.dNdy[2];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const double im = 1.0 / fmax(mass[nd[q]], 1.0e-14);
                sx += gpx[nd[q]] * im;
                sy += gpy[nd[q]] * im;
            }
            sx *= rs / 3.0;
            sy *= rs / 3.0;
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double K_ij = area * (g.dNdx[a] * g.dNdx[j] + g.dNdy[a] * g.dNdy[j]);
            const int p = pos[3 * k + j];
            if (local) sK[(p - r0) * T] += (1.0 + s) * K_ij; else Kp_val[p] += (1.0 + s) * K_ij;
        }
        const double stab_i = s * area * (g.dNdx[a] * gx + g.dNdy[a] * gy) - area * (g.dNdx[a] * sx + g.dNdy[a] * sy);
        rhs_row += rhs_contrib - stab_i;
        div_row += (area / 3.0) * div_u;
        if (want_oss) {
            const double w = sqrt(elem_s[e]) * area / 3.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int p = pos[3 * k + j];
                // B_ij = sum_K w_K grad N_j|K (row i, column j); B^T_ij = B_ji = sum_K w_K grad N_i|K
                if (local) {
                    const int q = (p - r0) * T;
                    sBx[q] += w * g.dNdx[j];
                    sBy[q] += w * g.dNdy[j];
                    sTx[q] += w * g.dNdx[a];
                    sTy[q] += w * g.dNdy[a];
                } else {
                    Bx[p] += w * g.dNdx[j];
                    By[p] += w * g.dNdy[j];
                    BTx[p] += w * g.dNdx[a];
                    BTy[p] += w * g.dNdy[a];
                }
            }
        }
    }
    if (want_oss) {
        inv_m[i] = 1.0 / fmax(mass[i], 1.0e-14);
        if (local)
            for (int q = 0; q < len; ++q) {
                Bx[r0 + q] = sBx[q * T];
                By[r0 + q] = sBy[q * T];
                BTx[r0 + q] = sTx[q * T];
                BTy[r0 + q] = sTy[q * T];
            }
    }
    div_num[i] = div_row;
    if (with_bc && pressure_dirichlet(i, tag[i], bc)) {
        for (int q = 0; q < len; ++q) Kp_val[r0 + q] = (ci[r0 + q] == i) ? 1.0 : 0.0;
        rhs_p[i] = 0.0;
        if (dp) dp[i] = 0.0;
        return;
    }
    for (int q = 0; q < len; ++q) {
        double v = local ? sK[q * T] : Kp_val[r0 + q];
        if (with_bc) {
            const int c = ci[r0 + q];
            if (c != i && pressure_dirichlet(c, tag[c], bc)) v = 0.0;
        }
        Kp_val[r0 + q] = v;
    }
    rhs_p[i] = rhs_row;
}

// k_apply_bc_pressure (fem_kernels.cuh:460-490) alone; with mean removal first when pinned
// (k_sum / k_subtract_mean, :493-510, summed here in a fixed order).
__global__ void k_pressure_bc(int n, const int* __restrict__ tag, const int* __restrict__ rp,
                              const int* __restrict__ ci, OutletBc bc, const double* __restrict__ sums,
                              const double* __restrict__ mass, double* __restrict__ Kp_val,
                              double* __restrict__ rhs, double* __restrict__ dp) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (sums) rhs[i] -= sums[0] / sums[1] * mass[i];
    if (pressure_dirichlet(i, tag[i], bc)) {
        for (int q = rp[i]; q < rp[i + 1]; ++q) Kp_val[q] = (ci[q] == i) ? 1.0 : 0.0;
        rhs[i] = 0.0;
        if (dp) dp[i] = 0.0;
    } else {
        for (int q = rp[i]; q < rp[i + 1]; ++q) {
            const int c = ci[q];
            if (c != i && pressure_dirichlet(c, tag[c], bc)) Kp_val[q] = 0.0;
        }
    }
}

// Sums of rhs and mass in a fixed order (deterministic), into out[0], out[1]
__global__ void __launch_bounds__(kThreads)
k_sum2(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ part,
       unsigned int* __restrict__ counter, double* __restrict__ out) {
    CFA_GRID_DEP();
    __shared__ double sh[2 * kWarps];
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        v[0] += a[i];
        v[1] += b[i];
    }
    block_sum<2>(v, sh);
    if (publish_partials<2>(v, part, counter)) {
        reduce_partials<2>(v, part, counter, sh);
        if (threadIdx.x == 0) { out[0] = v[0]; out[1] = v[1]; }
    }
}

static cfa_status mean_removal_sums(cfa_ctx* ctx, int n, const double* rhs, const double* mass, double* out2) {
    const int grid = row_grid(ctx, n, 1);
    CFA_PROPAGATE(ensure_partials(ctx, 2 * (size_t)grid + 2));
    CFA_LAUNCH(ctx, k_sum2, grid, kThreads, 0, n, rhs, mass, ctx->d_part, ctx->d_counters, out2);
    return CFA_OK;
}

}  // namespace cfa

using namespace cfa;

extern "C" {

cfa_status cfa_assemble_momentum_nu(cfa_ctx* ctx, const cfa_mesh* m, const double* u_old, const double* v_old,
                                    const double* u_prev, const double* v_prev, const double* p_old,
                                    const cfa_momentum_params* prm, const double* nu_node,
                                    const cfa_momentum_bc* bcp, double* A_val, double* rhs_u, double* rhs_v,
                                    double* mass, double* u, double* v);

cfa_status cfa_assemble_momentum(cfa_ctx* ctx, const cfa_mesh* m, const double* u_old, const double* v_old,
                                 const double* u_prev, const double* v_prev, const double* p_old,
                                 const cfa_momentum_params* prm, const cfa_momentum_bc* bcp, double* A_val,
                                 double* rhs_u, double* rhs_v, double* mass, double* u, double* v) {
    return cfa_assemble_momentum_nu(ctx, m, u_old, v_old, u_prev, v_prev, p_old, prm, nullptr, bcp, A_val, rhs_u,
                                    rhs_v, mass, u, v);
}

cfa_status cfa_assemble_momentum_nu(cfa_ctx* ctx, const cfa_mesh* m, const double* u_old, const double* v_old,
                                    const double* u_prev, const double* v_prev, const double* p_old,
                                    const cfa_momentum_params* prm, const double* nu_node,
                                    const cfa_momentum_bc* bcp, double* A_val, double* rhs_u, double* rhs_v,
                                    double* mass, double* u, double* v) {
    CFA_ENTER(ctx);
    CFA_ARG(m && u_old && v_old && u_prev && v_prev && p_old && prm && A_val && rhs_u && rhs_v && mass);
    CFA_ARG(!bcp || (u && v));
    MomParams P{prm->dt, prm->nu, prm->rho, prm->a0, prm->a1, prm->a2, prm->c1, prm->c2, prm->tau_time, prm->skew_coef};
    const double u_max = bcp ? bcp->u_max : 0.0, H = bcp ? bcp->H : 1.0;
    CFA_LAUNCH(ctx, k_momentum_rows, ceil_div(m->n, kThreads), kThreads, kMomSmem, m->n, m->ev, m->x, m->y, m->tag,
               m->inc_ptr.p, m->inc.p, m->pos.p, m->rp, m->ci, u_old, v_old, u_prev, v_prev, p_old, nu_node, P,
               bcp ? 1 : 0, u_max, H, m->bc, A_val, rhs_u, rhs_v, mass);
    if (bcp)   // solution values on Dirichlet nodes after the rows (u may alias u_old)
        CFA_LAUNCH(ctx, k_momentum_bc, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->tag, m->y, m->rp, m->ci,
                   u_max, H, m->bc, 0, A_val, rhs_u, rhs_v, u, v);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_apply_bc_momentum(cfa_ctx* ctx, const cfa_mesh* m, const cfa_momentum_bc* bcp, double* A_val,
                                 double* rhs_u, double* rhs_v, double* u, double* v) {
    CFA_ENTER(ctx);
    CFA_ARG(m && bcp && A_val && rhs_u && rhs_v);
    CFA_LAUNCH(ctx, k_momentum_bc, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->tag, m->y, m->rp, m->ci,
               bcp->u_max, bcp->H, m->bc, 1, A_val, rhs_u, rhs_v, u, v);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_lumped_mass(cfa_ctx* ctx, const cfa_mesh* m, double* mass) {
    CFA_ENTER(ctx);
    CFA_ARG(m && mass);
    CFA_LAUNCH(ctx, k_lumped_mass_rows, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->ev, m->x, m->y,
               m->inc_ptr.p, m->inc.p, mass);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_oss_weights(cfa_ctx* ctx, const cfa_mesh* m, const double* us, const double* vs, double dt,
                           double rho, double nu, double stab, double* elem_s) {
    CFA_ENTER(ctx);
    CFA_ARG(m && us && vs && elem_s);
    CFA_LAUNCH(ctx, k_oss_weights, ceil_div(m->ne, kThreads), kThreads, 0, m->ne, m->ev, m->x, m->y, us, vs, dt,
               rho, nu, stab, elem_s);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_scalar_gradient(cfa_ctx* ctx, const cfa_mesh* m, const double* f, const double* elem_s, double* gx,
                               double* gy) {
    CFA_ENTER(ctx);
    CFA_ARG(m && f && gx && gy);
    CFA_LAUNCH(ctx, k_scalar_gradient_rows, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->ev, m->x, m->y,
               m->inc_ptr.p, m->inc.p, f, elem_s, gx, gy);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

static cfa_status assemble_pressure(cfa_ctx* ctx, const cfa_mesh* m, const double* us, const double* vs,
                                    const double* p_old, const double* gpx, const double* gpy, const double* mass,
                                    const double* elem_s, double dt, double rho, double stab, int apply_bc,
                                    double* Kp, double* rhs, double* div, double* dp, double* oss_val,
                                    double* inv_m) {
    // With the pinned outlet the RHS loses its mean before the BC rows (apply_bc_pressure,
    // fem_kernels.cuh:519-531): assemble without BC, then sums, then the BC kernel.
    const bool split = apply_bc && m->bc.outlet_dirichlet;
    static std::once_flag press_once;
    std::call_once(press_once, [] {
        cudaFuncSetAttribute(k_pressure_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPressSmem);
    });
    CFA_LAUNCH(ctx, k_pressure_rows, ceil_div(m->n, kPressThreads), kPressThreads, kPressSmem, m->n, m->nnz, m->ev,
               m->x, m->y, m->tag,
               m->inc_ptr.p, m->inc.p, m->pos.p, m->rp, m->ci, us, vs, p_old, gpx, gpy, mass, elem_s, dt, rho,
               stab, (apply_bc && !split) ? 1 : 0, m->bc, Kp, rhs, div, dp, oss_val, inv_m);
    if (split) {
        double* sums = ctx->d_part;   // after the partials region
        CFA_PROPAGATE(ensure_partials(ctx, 2 * (size_t)row_grid(ctx, m->n, 1) + 4));
        sums = ctx->d_part + ctx->part_cap - 2;
        CFA_PROPAGATE(mean_removal_sums(ctx, m->n, rhs, mass, sums));
        CFA_LAUNCH(ctx, k_pressure_bc, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->tag, m->rp, m->ci, m->bc,
                   (const double*)sums, mass, Kp, rhs, dp);
    }
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_assemble_ppe(cfa_ctx* ctx, const cfa_mesh* m, const double* us, const double* vs, const double* p_old,
                            const double* gpx, const double* gpy, const double* mass, const double* elem_s, double dt,
                            double rho, double stab, int apply_bc, double* Kp, double* rhs, double* div, double* dp) {
    CFA_ENTER(ctx);
    CFA_ARG(m && us && vs && Kp && rhs && div);
    CFA_ARG(!(stab > 0.0) || (p_old && gpx && gpy && mass && elem_s));
    return assemble_pressure(ctx, m, us, vs, p_old, gpx, gpy, mass, elem_s, dt, rho, stab, apply_bc, Kp, rhs, div,
                             dp, nullptr, nullptr);
}

cfa_status cfa_apply_bc_pressure(cfa_ctx* ctx, const cfa_mesh* m, double* Kp, double* rhs, double* dp,
                                 const double* mass) {
    CFA_ENTER(ctx);
    CFA_ARG(m && Kp && rhs);
    const double* sums = nullptr;
    if (m->bc.outlet_dirichlet) {
        CFA_ARG(mass);
        CFA_PROPAGATE(ensure_partials(ctx, 2 * (size_t)row_grid(ctx, m->n, 1) + 4));
        double* s = ctx->d_part + ctx->part_cap - 2;
        CFA_PROPAGATE(mean_removal_sums(ctx, m->n, rhs, mass, s));
        sums = s;
    }
    CFA_LAUNCH(ctx, k_pressure_bc, ceil_div(m->n, kThreads), kThreads, 0, m->n, m->tag, m->rp, m->ci, m->bc, sums,
               mass, Kp, rhs, dp);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_assemble_oss(cfa_ctx* ctx, const cfa_mesh* m, const double* elem_s, const double* mass,
                            double* oss_val, double* inv_m) {
    CFA_ENTER(ctx);
    CFA_ARG(m && elem_s && mass && oss_val && inv_m);
    // The B/B^T rows are produced by the pressure-row pass; K, RHS and div go to scratch here.
    DevBuf<double> scratch;
    CFA_CUDA(scratch.ensure((size_t)m->nnz + 2 * (size_t)m->n));
    double* K = scratch.p;
    double* rhs = K + m->nnz;
    double* div = rhs + m->n;
    CFA_PROPAGATE(assemble_pressure(ctx, m, m->x, m->y, m->x, m->x, m->y, mass, elem_s, 1.0, 1.0, 0.0, 0, K, rhs,
                                    div, nullptr, oss_val, inv_m));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));   // scratch is released on return
    return CFA_OK;
}

// Fused pressure system: PPE (+ BCs) and the OSS operator in one row pass.
cfa_status cfa_assemble_pressure_system(cfa_ctx* ctx, const cfa_mesh* m, const double* us, const double* vs,
                                        const double* p_old, const double* gpx, const double* gpy,
                                        const double* mass, const double* elem_s, double dt, double rho,
                                        double stab, double* Kp, double* rhs, double* div, double* dp,
                                        double* oss_val, double* inv_m) {
    CFA_ENTER(ctx);
    CFA_ARG(m && us && vs && Kp && rhs && div);
    CFA_ARG(!(stab > 0.0) || (p_old && gpx && gpy && mass && elem_s && oss_val && inv_m));
    return assemble_pressure(ctx, m, us, vs, p_old, gpx, gpy, mass, elem_s, dt, rho, stab, 1, Kp, rhs, div, dp,
                             stab > 0.0 ? oss_val : nullptr, inv_m);
}

}  // extern "C"
