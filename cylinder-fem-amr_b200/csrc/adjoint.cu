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

constexpr int kAdjDirs = 16;   // u^n[3] v^n[3] u^{n-1}[3] v^{n-1}[3] p^n[3] nu_e

struct Dual {
    double v;
    double d[kAdjDirs];
};

__device__ __forceinline__ Dual dconst(double a) {
    Dual r;
    r.v = a;
#pragma unroll
    for (int k = 0; k < kAdjDirs; ++k) r.d[k] = 0.0;
    return r;
}
__device__ __forceinline__ Dual dvar(double a, int dir) {
    Dual r = dconst(a);
    r.d[dir] = 1.0;
    return r;
}
__device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < kAdjDirs; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
__device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < kAdjDirs; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
__device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < kAdjDirs; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
__device__ __forceinline__ Dual operator*(double s, const Dual& a) {
    Dual r;
    r.v = s * a.v;
#pragma unroll
    for (int k = 0; k < kAdjDirs; ++k) r.d[k] = s * a.d[k];
    return r;
}
__device__ __forceinline__ Dual operator/(const Dual& a, double s) { return (1.0 / s) * a; }
__device__ __forceinline__ Dual operator+(const Dual& a, double s) {
    Dual r = a;
    r.v += s;
    return r;
}
__device__ __forceinline__ Dual dsqrt(const Dual& a) {
    Dual r;
    r.v = sqrt(a.v);
    const double g = r.v > 0.0 ? 0.5 / r.v : 0.0;   // |w| at w = 0: the zero subgradient
#pragma unroll
    for (int k = 0; k < kAdjDirs; ++k) r.d[k] = g * a.d[k];
    return r;
}
__device__ __forceinline__ Dual drecip(const Dual& a) {
    Dual r;
    r.v = 1.0 / a.v;
    const double g = -r.v * r.v;
#pragma unroll
    for (int k = 0; k < kAdjDirs; ++k) r.d[k] = g * a.d[k];
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

}  // namespace cfa

using namespace cfa;

extern "C" {

cfa_status cfa_momentum_adjoint(cfa_ctx* ctx, const cfa_mesh* m, const double* u_old, const double* v_old,
                                const double* u_prev, const double* v_prev, const double* p_old,
                                const cfa_momentum_params* prm, const double* nu_node, const cfa_momentum_bc* bcp,
                                const double* x_u, const double* x_v, const double* lam_u, const double* lam_v,
                                double* g_u_old, double* g_v_old, double* g_u_prev, double* g_v_prev,
                                double* g_p_old, double* g_nu_node, double* d_scalars2) {
    if (!ctx) return CFA_BAD_ARG;
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

}  // extern "C"
