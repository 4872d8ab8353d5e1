/*
 * CPU restatement of the reference solve path -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Used by tests/ as the checker and by bench.py's CPU-baseline leg; never linked or called by
 * the product library. FP64 throughout, plain C11 with OpenMP only where the result does not
 * depend on the thread count (row-parallel loops; dot products summed over fixed chunks).
 *
 * Each function cites the reference file:line it follows. Element assembly is restated as the
 * serial element loop of the reference kernels, which sums every matrix entry over its elements
 * in ascending element order (the reference itself uses atomics, i.e. some order).
 */
#include "cfa_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { BC_INTERIOR = 0, BC_INLET = 1, BC_OUTLET = 2, BC_WALL = 3, BC_CYLINDER = 4 };

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static void* xmalloc(size_t bytes) {
    void* p = malloc(bytes ? bytes : 1);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}
static void* xcalloc(size_t count, size_t size) {
    void* p = calloc(count ? count : 1, size ? size : 1);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

static int cmp_int(const void* a, const void* b) {
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* ============================================================================================
 * CSR pattern: rows sorted and unique, diagonal included (src/cfa/mesh.cuh:198-249)
 * ========================================================================================== */
static void build_rows(int n, int ne, const int* ev, int** out_ptr, int** out_rows, int** out_len) {
    int* inc_ptr = (int*)xcalloc((size_t)n + 1, sizeof(int));
    for (int e = 0; e < ne; ++e)
        for (int k = 0; k < 3; ++k) inc_ptr[ev[3 * e + k] + 1]++;
    for (int i = 0; i < n; ++i) inc_ptr[i + 1] += inc_ptr[i];
    int* inc = (int*)xmalloc(sizeof(int) * 3 * (size_t)ne);
    int* fill = (int*)xmalloc(sizeof(int) * (size_t)n);
    memcpy(fill, inc_ptr, sizeof(int) * (size_t)n);
    for (int e = 0; e < ne; ++e)
        for (int k = 0; k < 3; ++k) inc[fill[ev[3 * e + k]]++] = e;
    int* cap = (int*)xcalloc((size_t)n + 1, sizeof(int));
    for (int i = 0; i < n; ++i) cap[i + 1] = cap[i] + 1 + 2 * (inc_ptr[i + 1] - inc_ptr[i]);
    int* tmp = (int*)xmalloc(sizeof(int) * (size_t)cap[n]);
    int* len = (int*)xmalloc(sizeof(int) * (size_t)n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        int* row = tmp + cap[i];
        int m = 0;
        row[m++] = i;
        for (int s = inc_ptr[i]; s < inc_ptr[i + 1]; ++s) {
            const int* t = ev + 3 * inc[s];
            for (int k = 0; k < 3; ++k) if (t[k] != i) row[m++] = t[k];
        }
        qsort(row, (size_t)m, sizeof(int), cmp_int);
        int u = 0;
        for (int q = 0; q < m; ++q) if (u == 0 || row[u - 1] != row[q]) row[u++] = row[q];
        len[i] = u;
    }
    free(inc_ptr); free(inc); free(fill);
    *out_ptr = cap; *out_rows = tmp; *out_len = len;
}

int or_csr_count(int n, int ne, const int* elem_v, int* row_ptr) {
    int *cap, *tmp, *len;
    build_rows(n, ne, elem_v, &cap, &tmp, &len);
    row_ptr[0] = 0;
    for (int i = 0; i < n; ++i) row_ptr[i + 1] = row_ptr[i] + len[i];
    free(cap); free(tmp); free(len);
    return row_ptr[n];
}

void or_csr_fill(int n, int ne, const int* elem_v, const int* row_ptr, int* col_ind) {
    int *cap, *tmp, *len;
    build_rows(n, ne, elem_v, &cap, &tmp, &len);
    for (int i = 0; i < n; ++i) memcpy(col_ind + row_ptr[i], tmp + cap[i], sizeof(int) * (size_t)len[i]);
    free(cap); free(tmp); free(len);
}

/* find_csr_index (src/cfa/fem_kernels.cuh:12-28) */
static int find_csr_index(const int* ci, int lo, int hi_end, int col) {
    int hi = hi_end - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1, c = ci[mid];
        if (c == col) return mid;
        if (c < col) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

/* ============================================================================================
 * Assembly
 * ========================================================================================== */
typedef struct { double area, dNdx[3], dNdy[3]; int ok; } geom;

static geom elem_geom(const int* nd, const double* x, const double* y) {
    geom g;
    double x0 = x[nd[0]], y0 = y[nd[0]], x1 = x[nd[1]], y1 = y[nd[1]], x2 = x[nd[2]], y2 = y[nd[2]];
    double detJ = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
    g.area = 0.5 * fabs(detJ);
    g.ok = !(g.area < 1.0e-14);
    double inv2A = 1.0 / (2.0 * g.area);
    g.dNdx[0] = (y1 - y2) * inv2A; g.dNdx[1] = (y2 - y0) * inv2A; g.dNdx[2] = (y0 - y1) * inv2A;
    g.dNdy[0] = (x2 - x1) * inv2A; g.dNdy[1] = (x0 - x2) * inv2A; g.dNdy[2] = (x1 - x0) * inv2A;
    return g;
}

/* k_assemble_momentum_fem (src/cfa/fem_kernels.cuh:40-181), without the MMS body force */
void or_assemble_momentum(int n, int ne, const int* ev, const double* x, const double* y,
                          const double* u_old, const double* v_old, const double* u_prev,
                          const double* v_prev, const double* p_old, const or_mom_params* P,
                          const int* rp, const int* ci, double* A_val, double* rhs_u, double* rhs_v,
                          double* mass_lumped) {
    memset(A_val, 0, sizeof(double) * (size_t)rp[n]);
    memset(rhs_u, 0, sizeof(double) * (size_t)n);
    memset(rhs_v, 0, sizeof(double) * (size_t)n);
    memset(mass_lumped, 0, sizeof(double) * (size_t)n);
    for (int e = 0; e < ne; ++e) {
        const int* nd = ev + 3 * e;
        geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        double area = g.area;
        double u_h[3], v_h[3], w_u = 0.0, w_v = 0.0, div_w = 0.0;
        for (int k = 0; k < 3; ++k) {
            double un = u_old[nd[k]], vn = v_old[nd[k]], um = u_prev[nd[k]], vm = v_prev[nd[k]];
            u_h[k] = P->a1 * un + P->a2 * um;
            v_h[k] = P->a1 * vn + P->a2 * vm;
            double wu = P->c1 * un + P->c2 * um, wv = P->c1 * vn + P->c2 * vm;
            w_u += wu / 3.0;
            w_v += wv / 3.0;
            div_w += wu * g.dNdx[k] + wv * g.dNdy[k];
        }
        double p_e[3] = {p_old[nd[0]], p_old[nd[1]], p_old[nd[2]]};
        double u_bar = w_u, v_bar = w_v;
        double vel_mag = sqrt(u_bar * u_bar + v_bar * v_bar) + 1.0e-12;
        double h_K = sqrt(2.0 * area);
        double term_t = 2.0 / P->tau_time;
        double term_c = 2.0 * vel_mag / h_K;
        double term_d = 4.0 * P->nu / (h_K * h_K);
        double tau_supg = 1.0 / sqrt(term_t * term_t + term_c * term_c + 9.0 * term_d * term_d);
        double dpdx = (p_e[0] * g.dNdx[0] + p_e[1] * g.dNdx[1] + p_e[2] * g.dNdx[2]) / P->rho;
        double dpdy = (p_e[0] * g.dNdy[0] + p_e[1] * g.dNdy[1] + p_e[2] * g.dNdy[2]) / P->rho;
        double u_gradN[3];
        for (int i = 0; i < 3; ++i) u_gradN[i] = u_bar * g.dNdx[i] + v_bar * g.dNdy[i];
        double m_lump = area / 3.0;
        for (int i = 0; i < 3; ++i) {
            int row = nd[i];
            mass_lumped[row] += m_lump;
            double f_u = 0.0, f_v = 0.0;
            for (int j = 0; j < 3; ++j) {
                int col = nd[j];
                double M_ij = (i == j) ? (area / 6.0) : (area / 12.0);
                double K_ij = area * (g.dNdx[i] * g.dNdx[j] + g.dNdy[i] * g.dNdy[j]);
                double C_ij = (area / 3.0) * u_gradN[j] + P->skew_coef * div_w * M_ij;
                double S_ij = area * tau_supg * u_gradN[i] * u_gradN[j];
                double M_supg_ij = (area / 3.0) * tau_supg * u_gradN[i];
                double A_ij = P->a0 * (M_ij + M_supg_ij) + P->nu * K_ij + C_ij + S_ij;
                int idx = find_csr_index(ci, rp[row], rp[row + 1], col);
                if (idx >= 0) A_val[idx] += A_ij;
                f_u += (M_ij + M_supg_ij) * u_h[j];
                f_v += (M_ij + M_supg_ij) * v_h[j];
            }
            double test_weight = (area / 3.0) + area * tau_supg * u_gradN[i];
            f_u -= test_weight * dpdx;
            f_v -= test_weight * dpdy;
            rhs_u[row] += f_u;
            rhs_v[row] += f_v;
        }
    }
}

/* k_apply_bc_momentum (src/cfa/fem_kernels.cuh:411-453), without the MMS branch */
void or_apply_bc_momentum(int n, const int* bc_tag, const double* y, double u_max, double H,
                          int outlet_dirichlet, double outlet_scale, const int* rp, const int* ci,
                          double* A_val, double* rhs_u, double* rhs_v, double* u, double* v) {
    for (int i = 0; i < n; ++i) {
        int tag = bc_tag[i];
        if (tag == BC_INLET || tag == BC_WALL || tag == BC_CYLINDER || (tag == BC_OUTLET && outlet_dirichlet)) {
            double u_bc = 0.0, v_bc = 0.0;
            if (tag == BC_INLET || tag == BC_OUTLET) {
                double yi = y[i];
                u_bc = 4.0 * u_max * yi * (H - yi) / (H * H) * (tag == BC_OUTLET ? outlet_scale : 1.0);
            }
            for (int idx = rp[i]; idx < rp[i + 1]; ++idx) A_val[idx] = (ci[idx] == i) ? 1.0 : 0.0;
            rhs_u[i] = u_bc; rhs_v[i] = v_bc; u[i] = u_bc; v[i] = v_bc;
        }
    }
}

/* k_assemble_pressure_poisson (src/cfa/fem_kernels.cuh:201-282) */
void or_assemble_ppe(int n, int ne, const int* ev, const double* x, const double* y,
                     const double* u_star, const double* v_star, const double* p_old,
                     const double* gp_x, const double* gp_y, const double* mass_lumped,
                     const double* elem_s, double dt, double rho, double stab, const int* rp,
                     const int* ci, double* Kp_val, double* rhs_p, double* div_num) {
    memset(Kp_val, 0, sizeof(double) * (size_t)rp[n]);
    memset(rhs_p, 0, sizeof(double) * (size_t)n);
    memset(div_num, 0, sizeof(double) * (size_t)n);
    for (int e = 0; e < ne; ++e) {
        const int* nd = ev + 3 * e;
        geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        double area = g.area;
        double div_u = u_star[nd[0]] * g.dNdx[0] + u_star[nd[1]] * g.dNdx[1] + u_star[nd[2]] * g.dNdx[2]
                     + v_star[nd[0]] * g.dNdy[0] + v_star[nd[1]] * g.dNdy[1] + v_star[nd[2]] * g.dNdy[2];
        double rhs_contrib = -(rho / dt) * (area / 3.0) * div_u;
        double s = 0.0, sx = 0.0, sy = 0.0, gx = 0.0, gy = 0.0;
        if (stab > 0.0) {
            s = elem_s[e];
            double rs = sqrt(s);
            gx = p_old[nd[0]] * g.dNdx[0] + p_old[nd[1]] * g.dNdx[1] + p_old[nd[2]] * g.dNdx[2];
            gy = p_old[nd[0]] * g.dNdy[0] + p_old[nd[1]] * g.dNdy[1] + p_old[nd[2]] * g.dNdy[2];
            for (int k = 0; k < 3; ++k) {
                double inv_m = 1.0 / fmax(mass_lumped[nd[k]], 1.0e-14);
                sx += gp_x[nd[k]] * inv_m;
                sy += gp_y[nd[k]] * inv_m;
            }
            sx *= rs / 3.0;
            sy *= rs / 3.0;
        }
        for (int i = 0; i < 3; ++i) {
            int row = nd[i];
            for (int j = 0; j < 3; ++j) {
                double K_ij = area * (g.dNdx[i] * g.dNdx[j] + g.dNdy[i] * g.dNdy[j]);
                int idx = find_csr_index(ci, rp[row], rp[row + 1], nd[j]);
                if (idx >= 0) Kp_val[idx] += (1.0 + s) * K_ij;
            }
            double stab_i = s * area * (g.dNdx[i] * gx + g.dNdy[i] * gy) - area * (g.dNdx[i] * sx + g.dNdy[i] * sy);
            rhs_p[row] += rhs_contrib - stab_i;
            div_num[row] += (area / 3.0) * div_u;
        }
    }
}

/* pressure_dirichlet (src/cfa/common.cuh:87-89) */
static int pdir(int i, int tag, int outlet_dirichlet, int pin) {
    return outlet_dirichlet ? i == pin : tag == BC_OUTLET;
}

/* apply_bc_pressure + k_sum/k_subtract_mean + k_apply_bc_pressure (src/cfa/fem_kernels.cuh:460-531) */
void or_apply_bc_pressure(int n, const int* bc_tag, int outlet_dirichlet, int pin, const int* rp,
                          const int* ci, double* Kp_val, double* rhs_p, double* dp,
                          const double* mass_lumped) {
    if (outlet_dirichlet) {
        double sf = 0.0, sm = 0.0;
        for (int i = 0; i < n; ++i) { sf += rhs_p[i]; sm += mass_lumped[i]; }
        for (int i = 0; i < n; ++i) rhs_p[i] -= sf / sm * mass_lumped[i];
    }
    for (int i = 0; i < n; ++i) {
        if (pdir(i, bc_tag[i], outlet_dirichlet, pin)) {
            for (int idx = rp[i]; idx < rp[i + 1]; ++idx) Kp_val[idx] = (ci[idx] == i) ? 1.0 : 0.0;
            rhs_p[i] = 0.0;
            dp[i] = 0.0;
        } else {
            for (int idx = rp[i]; idx < rp[i + 1]; ++idx) {
                int col = ci[idx];
                if (col != i && pdir(col, bc_tag[col], outlet_dirichlet, pin)) Kp_val[idx] = 0.0;
            }
        }
    }
}

/* k_compute_oss_weights (src/cfa/fem_kernels.cuh:697-719) */
void or_oss_weights(int ne, const int* ev, const double* x, const double* y, const double* u_star,
                    const double* v_star, double dt, double rho, double nu, double stab, double* elem_s) {
    for (int e = 0; e < ne; ++e) {
        int n0 = ev[3 * e], n1 = ev[3 * e + 1], n2 = ev[3 * e + 2];
        double area = 0.5 * fabs((x[n1] - x[n0]) * (y[n2] - y[n0]) - (x[n2] - x[n0]) * (y[n1] - y[n0]));
        double h = sqrt(2.0 * area);
        double ub = (u_star[n0] + u_star[n1] + u_star[n2]) / 3.0;
        double vb = (v_star[n0] + v_star[n1] + v_star[n2]) / 3.0;
        double tau = stab / (rho * (4.0 * nu / (h * h) + 2.0 * sqrt(ub * ub + vb * vb) / h) + 1.0e-300);
        elem_s[e] = rho * tau / dt;
    }
}

/* k_accumulate_scalar_gradient (src/cfa/fem_kernels.cuh:726-757); gx, gy are accumulated */
void or_scalar_gradient(int ne, const int* ev, const double* x, const double* y, const double* f,
                        const double* elem_s, double* gx_num, double* gy_num) {
    for (int e = 0; e < ne; ++e) {
        int n0 = ev[3 * e], n1 = ev[3 * e + 1], n2 = ev[3 * e + 2];
        double x0 = x[n0], y0 = y[n0], x1 = x[n1], y1 = y[n1], x2 = x[n2], y2 = y[n2];
        double detJ = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0);
        double area = 0.5 * fabs(detJ);
        if (area < 1.0e-14) continue;
        double inv2A = 1.0 / (2.0 * area);
        double gx = (f[n0] * (y1 - y2) + f[n1] * (y2 - y0) + f[n2] * (y0 - y1)) * inv2A;
        double gy = (f[n0] * (x2 - x1) + f[n1] * (x0 - x2) + f[n2] * (x1 - x0)) * inv2A;
        double w = (elem_s ? sqrt(elem_s[e]) : 1.0) * area / 3.0;
        gx_num[n0] += w * gx; gy_num[n0] += w * gy;
        gx_num[n1] += w * gx; gy_num[n1] += w * gy;
        gx_num[n2] += w * gx; gy_num[n2] += w * gy;
    }
}

/* k_stiffness_apply (src/cfa/fem_kernels.cuh:618-637): out_i += c area (dN_i . grad f) */
void or_stiffness_apply(int ne, const int* ev, const double* x, const double* y, const double* f, double c,
                        double* out) {
    for (int e = 0; e < ne; ++e) {
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        double gx = f[nd[0]] * g.dNdx[0] + f[nd[1]] * g.dNdx[1] + f[nd[2]] * g.dNdx[2];
        double gy = f[nd[0]] * g.dNdy[0] + f[nd[1]] * g.dNdy[1] + f[nd[2]] * g.dNdy[2];
        for (int a = 0; a < 3; ++a) out[nd[a]] += c * g.area * (g.dNdx[a] * gx + g.dNdy[a] * gy);
    }
}

/* k_accumulate_grad_dp_and_vorticity (src/cfa/fem_kernels.cuh:536-575); accumulated */
void or_grad_dp_vorticity(int ne, const int* ev, const double* x, const double* y, const double* dp,
                          const double* u, const double* v, double* gdx, double* gdy, double* vort_num) {
    for (int e = 0; e < ne; ++e) {
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        double dpdx = dp[nd[0]] * g.dNdx[0] + dp[nd[1]] * g.dNdx[1] + dp[nd[2]] * g.dNdx[2];
        double dpdy = dp[nd[0]] * g.dNdy[0] + dp[nd[1]] * g.dNdy[1] + dp[nd[2]] * g.dNdy[2];
        double dvdx = v[nd[0]] * g.dNdx[0] + v[nd[1]] * g.dNdx[1] + v[nd[2]] * g.dNdx[2];
        double dudy = u[nd[0]] * g.dNdy[0] + u[nd[1]] * g.dNdy[1] + u[nd[2]] * g.dNdy[2];
        double w = g.area / 3.0;
        for (int a = 0; a < 3; ++a) {
            gdx[nd[a]] += w * dpdx;
            gdy[nd[a]] += w * dpdy;
            vort_num[nd[a]] += w * (dvdx - dudy);
        }
    }
}

/* k_velocity_pressure_correction (src/cfa/fem_kernels.cuh:585-610) */
void or_velocity_pressure_correction(int n, const int* tag, int outlet_dirichlet, double dt, double rho,
                                     double p_update, double rot_coeff, const double* div_num,
                                     const double* mass, const double* gdx, const double* gdy,
                                     const double* vort_num, const double* dp, double* u, double* v, double* p,
                                     double* vort) {
    for (int i = 0; i < n; ++i) {
        double m_i = fmax(mass[i], 1.0e-14);
        vort[i] = vort_num[i] / m_i;
        p[i] += p_update * (dp[i] - rot_coeff * div_num[i] / m_i);
        if (tag[i] == BC_INTERIOR || (tag[i] == BC_OUTLET && !outlet_dirichlet)) {
            u[i] -= (dt / rho) * (gdx[i] / m_i);
            v[i] -= (dt / rho) * (gdy[i] / m_i);
        }
    }
}

/* k_volume_forces (src/cfa/fem_kernels.cuh:1046-1123): out[0..1] accumulated */
void or_volume_forces(int ne, const int* ev, const int* tag, const double* x, const double* y, const double* u,
                      const double* v, const double* u_old, const double* v_old, const double* u_prev,
                      const double* v_prev, const double* p, double b0, double b1, double b2, double nu,
                      double rho, double* out) {
    for (int e = 0; e < ne; ++e) {
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        double phi[3];
        int touches = 0;
        for (int a = 0; a < 3; ++a) {
            phi[a] = tag[nd[a]] == BC_CYLINDER ? 1.0 : 0.0;
            touches = touches || phi[a] > 0.0;
        }
        if (!touches) continue;
        geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        double ue[3], ve[3], ute[3], vte[3];
        double dudx = 0.0, dudy = 0.0, dvdx = 0.0, dvdy = 0.0, dphidx = 0.0, dphidy = 0.0, p_bar = 0.0;
        for (int a = 0; a < 3; ++a) {
            ue[a] = u[nd[a]];
            ve[a] = v[nd[a]];
            ute[a] = b0 * ue[a] + b1 * u_old[nd[a]] + b2 * u_prev[nd[a]];
            vte[a] = b0 * ve[a] + b1 * v_old[nd[a]] + b2 * v_prev[nd[a]];
            dudx += ue[a] * g.dNdx[a]; dudy += ue[a] * g.dNdy[a];
            dvdx += ve[a] * g.dNdx[a]; dvdy += ve[a] * g.dNdy[a];
            dphidx += phi[a] * g.dNdx[a]; dphidy += phi[a] * g.dNdy[a];
            p_bar += p[nd[a]] / 3.0;
        }
        double fx = 0.0, fy = 0.0;
        for (int a = 0; a < 3; ++a) {
            int b = (a + 1) % 3;
            double phi_m = 0.5 * (phi[a] + phi[b]);
            if (phi_m == 0.0) continue;
            double um = 0.5 * (ue[a] + ue[b]), vm = 0.5 * (ve[a] + ve[b]);
            fx += (0.5 * (ute[a] + ute[b]) + (um * dudx + vm * dudy)) * phi_m;
            fy += (0.5 * (vte[a] + vte[b]) + (um * dvdx + vm * dvdy)) * phi_m;
        }
        fx *= g.area / 3.0;
        fy *= g.area / 3.0;
        fx += g.area * (nu * (dudx * dphidx + dudy * dphidy) - (p_bar / rho) * dphidx);
        fy += g.area * (nu * (dvdx * dphidx + dvdy * dphidy) - (p_bar / rho) * dphidy);
        out[0] += fx;
        out[1] += fy;
    }
}

/* k_accumulate_recovered_gradient (src/cfa/fem_kernels.cuh:911-968); grad_rec accumulated */
void or_recovered_gradient(int n, int ne, const int* ev, const double* x, const double* y, const double* u,
                           const double* v, double u_max, double H, double* grad_rec) {
    for (int e = 0; e < ne; ++e) {
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        double ud[3];
        for (int a = 0; a < 3; ++a) ud[a] = u[nd[a]] - 4.0 * u_max * y[nd[a]] * (H - y[nd[a]]) / (H * H);
        double gc[4] = {ud[0] * g.dNdx[0] + ud[1] * g.dNdx[1] + ud[2] * g.dNdx[2],
                        ud[0] * g.dNdy[0] + ud[1] * g.dNdy[1] + ud[2] * g.dNdy[2],
                        v[nd[0]] * g.dNdx[0] + v[nd[1]] * g.dNdx[1] + v[nd[2]] * g.dNdx[2],
                        v[nd[0]] * g.dNdy[0] + v[nd[1]] * g.dNdy[1] + v[nd[2]] * g.dNdy[2]};
        double w = g.area / 3.0;
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 4; ++c) grad_rec[(size_t)c * n + nd[a]] += w * gc[c];
    }
}

/* k_compute_amr_error_indicator (src/cfa/fem_kernels.cuh:995-1035) */
void or_amr_error_indicator(int n, int ne, const int* ev, const double* x, const double* y, const double* grad_rec,
                            const double* mass, double* elem_error) {
    for (int e = 0; e < ne; ++e) {
        const int nd[3] = {ev[3 * e], ev[3 * e + 1], ev[3 * e + 2]};
        double G[3][4];
        for (int a = 0; a < 3; ++a) {
            double inv_m = 1.0 / fmax(mass[nd[a]], 1.0e-14);
            for (int c = 0; c < 4; ++c) G[a][c] = grad_rec[(size_t)c * n + nd[a]] * inv_m;
        }
        double x0 = x[nd[0]], y0 = y[nd[0]];
        double area = 0.5 * fabs((x[nd[1]] - x0) * (y[nd[2]] - y0) - (x[nd[2]] - x0) * (y[nd[1]] - y0));
        double omega = 0.0, eta_i = 0.0;
        for (int a = 0; a < 3; ++a) {
            omega = fmax(omega, fabs(G[a][2] - G[a][1]));
            int b = (a + 1) % 3;
            double ex = x[nd[b]] - x[nd[a]], ey = y[nd[b]] - y[nd[a]];
            double eu = (G[b][0] - G[a][0]) * ex + (G[b][1] - G[a][1]) * ey;
            double evv = (G[b][2] - G[a][2]) * ex + (G[b][3] - G[a][3]) * ey;
            eta_i = fmax(eta_i, 0.125 * sqrt(eu * eu + evv * evv));
        }
        elem_error[e] = sqrt(2.0 * area) * omega;
        elem_error[ne + e] = eta_i;
    }
}

/* k_assemble_oss_operator + k_inverse_lumped_mass (src/cfa/fem_kernels.cuh:807-852),
 * assemble_oss_projection (src/cfa/device.cuh:304-314) */
void or_assemble_oss(int n, int ne, const int* ev, const double* x, const double* y,
                     const double* elem_s, const int* rp, const int* ci, const double* mass_lumped,
                     double* oss_val, double* inv_m) {
    const size_t nnz = (size_t)rp[n];
    memset(oss_val, 0, sizeof(double) * 4 * nnz);
    double *Bx = oss_val, *By = oss_val + nnz, *BTx = oss_val + 2 * nnz, *BTy = oss_val + 3 * nnz;
    for (int e = 0; e < ne; ++e) {
        const int* nd = ev + 3 * e;
        geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        double w = sqrt(elem_s[e]) * g.area / 3.0;
        for (int a = 0; a < 3; ++a) {
            int k = nd[a];
            for (int b = 0; b < 3; ++b) {
                int j = nd[b];
                int kj = find_csr_index(ci, rp[k], rp[k + 1], j);
                int jk = find_csr_index(ci, rp[j], rp[j + 1], k);
                if (kj < 0 || jk < 0) continue;
                Bx[kj] += w * g.dNdx[b];
                By[kj] += w * g.dNdy[b];
                BTx[jk] += w * g.dNdx[b];
                BTy[jk] += w * g.dNdy[b];
            }
        }
    }
    for (int i = 0; i < n; ++i) inv_m[i] = 1.0 / fmax(mass_lumped[i], 1.0e-14);
}

/* k_oss_apply_B + k_oss_apply_BT (src/cfa/fem_kernels.cuh:855-885): out -= B^T M^-1 B in */
void or_oss_apply(int n, const int* rp, const int* ci, const double* oss_val, const double* inv_m,
                  const int* bc_tag, int outlet_dirichlet, int pin, const double* in, double* out) {
    const size_t nnz = (size_t)rp[n];
    double* gx = (double*)xmalloc(sizeof(double) * (size_t)n);
    double* gy = (double*)xmalloc(sizeof(double) * (size_t)n);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; ++k) {
        double sx = 0.0, sy = 0.0;
        for (int a = rp[k]; a < rp[k + 1]; ++a) {
            double xj = in[ci[a]];
            sx += oss_val[a] * xj;
            sy += oss_val[nnz + a] * xj;
        }
        gx[k] = sx * inv_m[k];
        gy[k] = sy * inv_m[k];
    }
    const double *BTx = oss_val + 2 * nnz, *BTy = oss_val + 3 * nnz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (pdir(i, bc_tag[i], outlet_dirichlet, pin)) continue;
        double s = 0.0;
        for (int a = rp[i]; a < rp[i + 1]; ++a) {
            int k = ci[a];
            s += BTx[a] * gx[k] + BTy[a] * gy[k];
        }
        out[i] -= s;
    }
    free(gx); free(gy);
}

/* apply_oss_projection_matrix_free (src/cfa/device.cuh:287-298): k_accumulate_scalar_gradient
 * then k_oss_subtract_projection (src/cfa/fem_kernels.cuh:763-797) */
void or_oss_matrix_free(int n, int ne, const int* ev, const double* x, const double* y,
                        const int* bc_tag, int outlet_dirichlet, int pin, const double* elem_s,
                        const double* mass_lumped, const double* in, double* out) {
    double* gx = (double*)xcalloc((size_t)n, sizeof(double));
    double* gy = (double*)xcalloc((size_t)n, sizeof(double));
    or_scalar_gradient(ne, ev, x, y, in, elem_s, gx, gy);
    for (int e = 0; e < ne; ++e) {
        const int* nd = ev + 3 * e;
        geom g = elem_geom(nd, x, y);
        if (!g.ok) continue;
        double sx = 0.0, sy = 0.0;
        for (int k = 0; k < 3; ++k) {
            double inv = 1.0 / fmax(mass_lumped[nd[k]], 1.0e-14);
            sx += gx[nd[k]] * inv;
            sy += gy[nd[k]] * inv;
        }
        double w = sqrt(elem_s[e]) * g.area / 3.0;
        for (int i = 0; i < 3; ++i) {
            if (pdir(nd[i], bc_tag[nd[i]], outlet_dirichlet, pin)) continue;
            out[nd[i]] += -w * (g.dNdx[i] * sx + g.dNdy[i] * sy);
        }
    }
    free(gx); free(gy);
}

/* k_assemble_lumped_mass (src/cfa/fem_kernels.cuh:890-909) */
void or_lumped_mass(int n, int ne, const int* ev, const double* x, const double* y, double* m) {
    memset(m, 0, sizeof(double) * (size_t)n);
    for (int e = 0; e < ne; ++e) {
        int n0 = ev[3 * e], n1 = ev[3 * e + 1], n2 = ev[3 * e + 2];
        double detJ = (x[n1] - x[n0]) * (y[n2] - y[n0]) - (x[n2] - x[n0]) * (y[n1] - y[n0]);
        double w = fabs(detJ) / 6.0;
        m[n0] += w; m[n1] += w; m[n2] += w;
    }
}

/* ============================================================================================
 * Vector kernels
 * ========================================================================================== */
/* k_spmv_csr (src/cfa/linalg.cuh:8-26) */
void or_spmv(int n, const int* rp, const int* ci, const double* val, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) s += val[k] * x[ci[k]];
        y[i] = s;
    }
}

/* Deterministic dot: fixed 8192-element chunks summed in order (independent of threads) */
#define DOT_CHUNK 8192
double or_dot(int n, const double* a, const double* b) {
    int nch = (n + DOT_CHUNK - 1) / DOT_CHUNK;
    double stackpart[64];
    double* part = nch <= 64 ? stackpart : (double*)xmalloc(sizeof(double) * (size_t)nch);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nch; ++c) {
        double s = 0.0;
        int e = (c + 1) * DOT_CHUNK < n ? (c + 1) * DOT_CHUNK : n;
        for (int i = c * DOT_CHUNK; i < e; ++i) s += a[i] * b[i];
        part[c] = s;
    }
    double s = 0.0;
    for (int c = 0; c < nch; ++c) s += part[c];
    if (part != stackpart) free(part);
    return s;
}

/* ============================================================================================
 * Multicolour ILU(0) (src/cfa/linalg.cuh:350-568)
 * ========================================================================================== */
#define ILU_MAX_ROW 32
struct or_ilu {
    int n, nnz, nc, nl, nu;
    int *rp, *ci, *colour, *diag, *cstart, *rows, *lp, *up, *lc, *uc, *l_src, *u_src, *d_src;
    double *lu, *lv, *uv, *dinv;
};

/* MulticolourIlu0::set_pattern (src/cfa/linalg.cuh:456-528) */
or_ilu* or_ilu_create(int n, const int* rp, const int* ci) {
    for (int i = 0; i < n; ++i)
        if (rp[i + 1] - rp[i] > ILU_MAX_ROW) return NULL;
    or_ilu* h = (or_ilu*)xcalloc(1, sizeof(or_ilu));
    int nnz = rp[n];
    h->n = n; h->nnz = nnz;
    h->rp = (int*)xmalloc(sizeof(int) * ((size_t)n + 1)); memcpy(h->rp, rp, sizeof(int) * ((size_t)n + 1));
    h->ci = (int*)xmalloc(sizeof(int) * (size_t)nnz); memcpy(h->ci, ci, sizeof(int) * (size_t)nnz);
    h->colour = (int*)xmalloc(sizeof(int) * (size_t)n);
    h->diag = (int*)xmalloc(sizeof(int) * (size_t)n);
    int cap = 64, nc = 0;
    int* mark = (int*)xmalloc(sizeof(int) * (size_t)cap);
    for (int i = 0; i < n; ++i) { h->colour[i] = -1; h->diag[i] = -1; }
    for (int i = 0; i < n; ++i) {
        for (int a = rp[i]; a < rp[i + 1]; ++a) {
            int c = h->colour[ci[a]];
            if (c >= 0) mark[c] = i;
            if (ci[a] == i) h->diag[i] = a;
        }
        int c = 0;
        while (c < nc && mark[c] == i) ++c;
        if (c == nc) {
            if (nc == cap) { cap *= 2; mark = (int*)realloc(mark, sizeof(int) * (size_t)cap); }
            mark[nc++] = -1;
        }
        h->colour[i] = c;
    }
    free(mark);
    h->nc = nc;
    h->cstart = (int*)xcalloc((size_t)nc + 1, sizeof(int));
    for (int i = 0; i < n; ++i) h->cstart[h->colour[i] + 1]++;
    for (int c = 0; c < nc; ++c) h->cstart[c + 1] += h->cstart[c];
    h->rows = (int*)xmalloc(sizeof(int) * (size_t)n);
    int* fill = (int*)xmalloc(sizeof(int) * (size_t)nc);
    memcpy(fill, h->cstart, sizeof(int) * (size_t)nc);
    for (int i = 0; i < n; ++i) h->rows[fill[h->colour[i]]++] = i;
    free(fill);
    h->lp = (int*)xcalloc((size_t)n + 1, sizeof(int));
    h->up = (int*)xcalloc((size_t)n + 1, sizeof(int));
    for (int t = 0; t < n; ++t) {
        int i = h->rows[t], l = 0, u = 0;
        for (int a = rp[i]; a < rp[i + 1]; ++a) {
            if (ci[a] == i) continue;
            if (h->colour[ci[a]] < h->colour[i]) ++l; else ++u;
        }
        h->lp[t + 1] = l; h->up[t + 1] = u;
    }
    for (int t = 0; t < n; ++t) { h->lp[t + 1] += h->lp[t]; h->up[t + 1] += h->up[t]; }
    h->nl = h->lp[n]; h->nu = h->up[n];
    h->lc = (int*)xmalloc(sizeof(int) * (size_t)h->nl);
    h->uc = (int*)xmalloc(sizeof(int) * (size_t)h->nu);
    h->l_src = (int*)xmalloc(sizeof(int) * (size_t)h->nl);
    h->u_src = (int*)xmalloc(sizeof(int) * (size_t)h->nu);
    h->d_src = (int*)xmalloc(sizeof(int) * (size_t)n);
    for (int t = 0; t < n; ++t) {
        int i = h->rows[t], l = h->lp[t], u = h->up[t];
        for (int a = rp[i]; a < rp[i + 1]; ++a) {
            int j = ci[a];
            if (j == i) h->d_src[t] = a;
            else if (h->colour[j] < h->colour[i]) { h->lc[l] = j; h->l_src[l++] = a; }
            else { h->uc[u] = j; h->u_src[u++] = a; }
        }
    }
    h->lu = (double*)xmalloc(sizeof(double) * (size_t)nnz);
    h->lv = (double*)xmalloc(sizeof(double) * (size_t)h->nl);
    h->uv = (double*)xmalloc(sizeof(double) * (size_t)h->nu);
    h->dinv = (double*)xmalloc(sizeof(double) * (size_t)n);
    return h;
}

int or_ilu_colours(const or_ilu* h) { return h->nc; }

void or_ilu_export(const or_ilu* h, int* colour, int* colour_start, int* rows, int* lp, int* up,
                   int* lc, int* uc, int* l_src, int* u_src, int* d_src, int* nl_nu) {
    int n = h->n;
    if (colour) memcpy(colour, h->colour, sizeof(int) * (size_t)n);
    if (colour_start) memcpy(colour_start, h->cstart, sizeof(int) * ((size_t)h->nc + 1));
    if (rows) memcpy(rows, h->rows, sizeof(int) * (size_t)n);
    if (lp) memcpy(lp, h->lp, sizeof(int) * ((size_t)n + 1));
    if (up) memcpy(up, h->up, sizeof(int) * ((size_t)n + 1));
    if (lc) memcpy(lc, h->lc, sizeof(int) * (size_t)h->nl);
    if (uc) memcpy(uc, h->uc, sizeof(int) * (size_t)h->nu);
    if (l_src) memcpy(l_src, h->l_src, sizeof(int) * (size_t)h->nl);
    if (u_src) memcpy(u_src, h->u_src, sizeof(int) * (size_t)h->nu);
    if (d_src) memcpy(d_src, h->d_src, sizeof(int) * (size_t)n);
    if (nl_nu) { nl_nu[0] = h->nl; nl_nu[1] = h->nu; }
}

/* MulticolourIlu0::factor, k_ilu0_factor_colour, k_ilu0_gather (src/cfa/linalg.cuh:366-402, :531-541) */
void or_ilu_factor(or_ilu* h, const double* val, double* lu_out, double* lv, double* uv, double* dinv) {
    const int *rp = h->rp, *ci = h->ci, *colour = h->colour, *diag = h->diag;
    double* lu = h->lu;
    memcpy(lu, val, sizeof(double) * (size_t)h->nnz);
    for (int c = 1; c < h->nc; ++c) {
#pragma omp parallel for schedule(static)
        for (int t = h->cstart[c]; t < h->cstart[c + 1]; ++t) {
            const int i = h->rows[t];
            const int s = rp[i], len = rp[i + 1] - s, cii = colour[i];
            int cols[ILU_MAX_ROW], ccol[ILU_MAX_ROW];
            double a[ILU_MAX_ROW];
            for (int q = 0; q < len; ++q) { cols[q] = ci[s + q]; ccol[q] = colour[cols[q]]; a[q] = lu[s + q]; }
            for (int cc = 0; cc < cii; ++cc) {
                for (int q = 0; q < len; ++q) {
                    if (ccol[q] != cc) continue;
                    const int k = cols[q];
                    const double lik = a[q] / lu[diag[k]];
                    a[q] = lik;
                    for (int m = rp[k]; m < rp[k + 1]; ++m) {
                        const int j = ci[m];
                        for (int b = 0; b < len; ++b)
                            if (cols[b] == j) { if (ccol[b] > cc) a[b] -= lik * lu[m]; break; }
                    }
                }
            }
            for (int q = 0; q < len; ++q) lu[s + q] = a[q];
        }
    }
    for (int e = 0; e < h->nl; ++e) h->lv[e] = lu[h->l_src[e]];
    for (int e = 0; e < h->nu; ++e) h->uv[e] = lu[h->u_src[e]];
    for (int t = 0; t < h->n; ++t) h->dinv[t] = 1.0 / lu[h->d_src[t]];
    if (lu_out) memcpy(lu_out, lu, sizeof(double) * (size_t)h->nnz);
    if (lv) memcpy(lv, h->lv, sizeof(double) * (size_t)h->nl);
    if (uv) memcpy(uv, h->uv, sizeof(double) * (size_t)h->nu);
    if (dinv) memcpy(dinv, h->dinv, sizeof(double) * (size_t)h->n);
}

/* MulticolourIlu0::apply, k_ilu0_lower_colour, k_ilu0_upper_colour (src/cfa/linalg.cuh:406-433, :544-555) */
void or_ilu_apply(const or_ilu* h, const double* r, double* z, int nrhs) {
    const int n = h->n;
    for (int comp = 0; comp < nrhs; ++comp) {
        const size_t off = (size_t)comp * n;
        for (int c = 0; c < h->nc; ++c) {
            const int last = (c == h->nc - 1);
#pragma omp parallel for schedule(static)
            for (int t = h->cstart[c]; t < h->cstart[c + 1]; ++t) {
                const int i = h->rows[t];
                double acc = r[off + i];
                for (int e = h->lp[t]; e < h->lp[t + 1]; ++e) acc -= h->lv[e] * z[off + h->lc[e]];
                z[off + i] = last ? acc * h->dinv[t] : acc;
            }
        }
        for (int c = h->nc - 2; c >= 0; --c) {
#pragma omp parallel for schedule(static)
            for (int t = h->cstart[c]; t < h->cstart[c + 1]; ++t) {
                const int i = h->rows[t];
                double acc = z[off + i];
                for (int e = h->up[t]; e < h->up[t + 1]; ++e) acc -= h->uv[e] * z[off + h->uc[e]];
                z[off + i] = acc * h->dinv[t];
            }
        }
    }
}

void or_ilu_free(or_ilu* h) {
    if (!h) return;
    void* ps[] = {h->rp, h->ci, h->colour, h->diag, h->cstart, h->rows, h->lp, h->up, h->lc, h->uc,
                  h->l_src, h->u_src, h->d_src, h->lu, h->lv, h->uv, h->dinv};
    for (size_t k = 0; k < sizeof(ps) / sizeof(ps[0]); ++k) free(ps[k]);
    free(h);
}

/* ============================================================================================
 * Host CSR helpers (src/cfa/linalg.cuh:791-862)
 * ========================================================================================== */
typedef struct { int rows, cols; int *rp, *ci; double* v; } hcsr;

static void hcsr_free(hcsr* a) { free(a->rp); free(a->ci); free(a->v); memset(a, 0, sizeof(*a)); }

/* csr_multiply (src/cfa/linalg.cuh:799-845): rows summed in serial product order, sorted output */
static hcsr csr_mul(const hcsr* A, const hcsr* B) {
    hcsr C;
    C.rows = A->rows; C.cols = B->cols;
    C.rp = (int*)xcalloc((size_t)A->rows + 1, sizeof(int));
#pragma omp parallel
    {
        int* marker = (int*)xmalloc(sizeof(int) * (size_t)(B->cols > 0 ? B->cols : 1));
        for (int j = 0; j < B->cols; ++j) marker[j] = -1;
#pragma omp for schedule(static)
        for (int i = 0; i < A->rows; ++i) {
            int count = 0;
            for (int a = A->rp[i]; a < A->rp[i + 1]; ++a) {
                int k = A->ci[a];
                for (int b = B->rp[k]; b < B->rp[k + 1]; ++b) {
                    int j = B->ci[b];
                    if (marker[j] != i) { marker[j] = i; ++count; }
                }
            }
            C.rp[i + 1] = count;
        }
        free(marker);
    }
    for (int i = 0; i < A->rows; ++i) C.rp[i + 1] += C.rp[i];
    int nnz = C.rp[A->rows];
    C.ci = (int*)xmalloc(sizeof(int) * (size_t)nnz);
    C.v = (double*)xmalloc(sizeof(double) * (size_t)nnz);
#pragma omp parallel
    {
        int* marker = (int*)xmalloc(sizeof(int) * (size_t)(B->cols > 0 ? B->cols : 1));
        double* acc = (double*)xcalloc((size_t)(B->cols > 0 ? B->cols : 1), sizeof(double));
        int* cols = (int*)xmalloc(sizeof(int) * (size_t)(B->cols > 0 ? B->cols : 1));
        for (int j = 0; j < B->cols; ++j) marker[j] = -1;
#pragma omp for schedule(static)
        for (int i = 0; i < A->rows; ++i) {
            int nc = 0;
            for (int a = A->rp[i]; a < A->rp[i + 1]; ++a) {
                int k = A->ci[a];
                double av = A->v[a];
                for (int b = B->rp[k]; b < B->rp[k + 1]; ++b) {
                    int j = B->ci[b];
                    if (marker[j] != i) { marker[j] = i; acc[j] = 0.0; cols[nc++] = j; }
                    acc[j] += av * B->v[b];
                }
            }
            qsort(cols, (size_t)nc, sizeof(int), cmp_int);
            int out = C.rp[i];
            for (int q = 0; q < nc; ++q) { C.ci[out] = cols[q]; C.v[out] = acc[cols[q]]; ++out; }
        }
        free(marker); free(acc); free(cols);
    }
    return C;
}

/* csr_transpose (src/cfa/linalg.cuh:847-862) */
static hcsr csr_tr(const hcsr* A) {
    hcsr T;
    T.rows = A->cols; T.cols = A->rows;
    T.rp = (int*)xcalloc((size_t)A->cols + 1, sizeof(int));
    int nnz = A->rp[A->rows];
    for (int a = 0; a < nnz; ++a) T.rp[A->ci[a] + 1]++;
    for (int i = 0; i < A->cols; ++i) T.rp[i + 1] += T.rp[i];
    T.ci = (int*)xmalloc(sizeof(int) * (size_t)nnz);
    T.v = (double*)xmalloc(sizeof(double) * (size_t)nnz);
    int* fill = (int*)xmalloc(sizeof(int) * (size_t)(A->cols > 0 ? A->cols : 1));
    memcpy(fill, T.rp, sizeof(int) * (size_t)A->cols);
    for (int i = 0; i < A->rows; ++i)
        for (int a = A->rp[i]; a < A->rp[i + 1]; ++a) {
            int k = fill[A->ci[a]]++;
            T.ci[k] = i; T.v[k] = A->v[a];
        }
    free(fill);
    return T;
}

int or_csr_multiply(int ar, int ac, const int* arp, const int* aci, const double* av,
                    int bc, const int* brp, const int* bci, const double* bv,
                    int* crp, int* cci, double* cv) {
    hcsr A = {ar, ac, (int*)arp, (int*)aci, (double*)av};
    hcsr B = {ac, bc, (int*)brp, (int*)bci, (double*)bv};
    hcsr C = csr_mul(&A, &B);
    int nnz = C.rp[ar];
    memcpy(crp, C.rp, sizeof(int) * ((size_t)ar + 1));
    if (cci) memcpy(cci, C.ci, sizeof(int) * (size_t)nnz);
    if (cv) memcpy(cv, C.v, sizeof(double) * (size_t)nnz);
    hcsr_free(&C);
    return nnz;
}

void or_csr_transpose(int rows, int cols, const int* rp, const int* ci, const double* v,
                      int* trp, int* tci, double* tv) {
    hcsr A = {rows, cols, (int*)rp, (int*)ci, (double*)v};
    hcsr T = csr_tr(&A);
    int nnz = rp[rows];
    memcpy(trp, T.rp, sizeof(int) * ((size_t)cols + 1));
    memcpy(tci, T.ci, sizeof(int) * (size_t)nnz);
    memcpy(tv, T.v, sizeof(double) * (size_t)nnz);
    hcsr_free(&T);
}

/* ============================================================================================
 * SA-AMG (src/cfa/linalg.cuh:781-1432)
 * ========================================================================================== */
#define OR_MAX_LEVELS 32
typedef struct {
    hcsr A, P, R;
    double* dinv;
    double omega;
    int* agg;
    double *x, *b, *r, *Ax;
} or_level;

struct or_amg {
    int nlev, smooth_steps, coarse_n;
    or_level L[OR_MAX_LEVELS];
    double* coarse_A;    /* dense coarsest operator */
    double* coarse_inv;  /* its inverse */
    double *cx, *cb;
};

/* spectral_radius_DinvA (src/cfa/linalg.cuh:1276-1304) */
static double spectral_radius(const hcsr* A, const double* dinv) {
    const int n = A->rows, chunk = 4096, nch = (n + chunk - 1) / chunk;
    double* x = (double*)xmalloc(sizeof(double) * (size_t)n);
    double* y = (double*)xmalloc(sizeof(double) * (size_t)n);
    double* py = (double*)xmalloc(sizeof(double) * (size_t)nch);
    double* px = (double*)xmalloc(sizeof(double) * (size_t)nch);
    for (int i = 0; i < n; ++i) x[i] = 1.0 + 0.1 * sin(1.0 + i);
    double lambda = 1.0;
    for (int it = 0; it < 20; ++it) {
#pragma omp parallel for schedule(static)
        for (int c = 0; c < nch; ++c) {
            double sy = 0.0, sx = 0.0;
            int e = (c + 1) * chunk < n ? (c + 1) * chunk : n;
            for (int i = c * chunk; i < e; ++i) {
                double s = 0.0;
                for (int a = A->rp[i]; a < A->rp[i + 1]; ++a) s += A->v[a] * x[A->ci[a]];
                y[i] = dinv[i] * s;
                sy += y[i] * y[i];
                sx += x[i] * x[i];
            }
            py[c] = sy; px[c] = sx;
        }
        double nrm = 0.0, xn = 0.0;
        for (int c = 0; c < nch; ++c) { nrm += py[c]; xn += px[c]; }
        nrm = sqrt(nrm);
        lambda = nrm / sqrt(xn);
        for (int i = 0; i < n; ++i) x[i] = y[i] / nrm;
    }
    free(x); free(y); free(py); free(px);
    return (lambda > 1.0e-12 ? lambda : 1.0e-12) * 1.05;
}

/* smoothed_prolongator (src/cfa/linalg.cuh:1306-1392) */
static hcsr smoothed_prolongator(const hcsr* A, const double* dinv, double omega, double theta, int* agg) {
    const int n = A->rows;
    const int nnz = A->rp[n];
    double* diag = (double*)xmalloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) diag[i] = 1.0 / dinv[i];
    char* strong = (char*)xmalloc((size_t)(nnz > 0 ? nnz : 1));
    for (int i = 0; i < n; ++i)
        for (int a = A->rp[i]; a < A->rp[i + 1]; ++a) {
            int j = A->ci[a];
            strong[a] = j != i && fabs(A->v[a]) >= theta * sqrt(fabs(diag[i] * diag[j]));
        }
    for (int i = 0; i < n; ++i) agg[i] = -1;
    int na = 0;
    for (int i = 0; i < n; ++i) {                               /* phase 1 */
        if (agg[i] >= 0) continue;
        int free_nbhd = 1;
        for (int a = A->rp[i]; a < A->rp[i + 1] && free_nbhd; ++a)
            if (strong[a] && agg[A->ci[a]] >= 0) free_nbhd = 0;
        if (!free_nbhd) continue;
        agg[i] = na;
        for (int a = A->rp[i]; a < A->rp[i + 1]; ++a) if (strong[a]) agg[A->ci[a]] = na;
        ++na;
    }
    int* agg2 = (int*)xmalloc(sizeof(int) * (size_t)n);        /* phase 2 */
    memcpy(agg2, agg, sizeof(int) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        for (int a = A->rp[i]; a < A->rp[i + 1]; ++a)
            if (strong[a] && agg[A->ci[a]] >= 0) { agg2[i] = agg[A->ci[a]]; break; }
    }
    memcpy(agg, agg2, sizeof(int) * (size_t)n);
    free(agg2);
    for (int i = 0; i < n; ++i) {                               /* phase 3 */
        if (agg[i] >= 0) continue;
        agg[i] = na;
        for (int a = A->rp[i]; a < A->rp[i + 1]; ++a)
            if (strong[a] && agg[A->ci[a]] < 0) agg[A->ci[a]] = na;
        ++na;
    }
    int* size = (int*)xcalloc((size_t)(na > 0 ? na : 1), sizeof(int));
    for (int i = 0; i < n; ++i) size[agg[i]]++;
    hcsr P0;
    P0.rows = n; P0.cols = na;
    P0.rp = (int*)xmalloc(sizeof(int) * ((size_t)n + 1));
    P0.ci = (int*)xmalloc(sizeof(int) * (size_t)n);
    P0.v = (double*)xmalloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) { P0.rp[i] = i; P0.ci[i] = agg[i]; P0.v[i] = 1.0 / sqrt((double)size[agg[i]]); }
    P0.rp[n] = n;
    hcsr AP0 = csr_mul(A, &P0);
    hcsr P;
    P.rows = n; P.cols = na;
    P.rp = (int*)xcalloc((size_t)n + 1, sizeof(int));
    /* build_row: count pass then fill pass */
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            for (int i = 0; i < n; ++i) P.rp[i + 1] += P.rp[i];
            P.ci = (int*)xmalloc(sizeof(int) * (size_t)(P.rp[n] > 0 ? P.rp[n] : 1));
            P.v = (double*)xmalloc(sizeof(double) * (size_t)(P.rp[n] > 0 ? P.rp[n] : 1));
        }
        for (int i = 0; i < n; ++i) {
            int* cols = pass ? P.ci + P.rp[i] : NULL;
            double* vals = pass ? P.v + P.rp[i] : NULL;
            int out = 0, own = 0;
            const int own_col = agg[i];
            for (int a = AP0.rp[i]; a < AP0.rp[i + 1]; ++a) {
                int j = AP0.ci[a];
                if (!own && j > own_col) {
                    if (cols) { cols[out] = own_col; vals[out] = P0.v[i]; }
                    ++out; own = 1;
                }
                double val = -omega * dinv[i] * AP0.v[a];
                if (j == own_col) { val += P0.v[i]; own = 1; }
                if (val != 0.0) { if (cols) { cols[out] = j; vals[out] = val; } ++out; }
            }
            if (!own) { if (cols) { cols[out] = own_col; vals[out] = P0.v[i]; } ++out; }
            if (!pass) P.rp[i + 1] = out;
        }
    }
    hcsr_free(&AP0); hcsr_free(&P0);
    free(size); free(strong); free(diag);
    return P;
}

/* dense_spd_inverse (src/cfa/linalg.cuh:1394-1431); returns 0 if not SPD */
static int dense_spd_inverse(double* M, int n, double* inv) {
    for (int j = 0; j < n; ++j) {
        double d = M[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= M[(size_t)j * n + k] * M[(size_t)j * n + k];
        if (!(d > 0.0)) return 0;
        double ljj = sqrt(d);
        M[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            double s = M[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s -= M[(size_t)i * n + k] * M[(size_t)j * n + k];
            M[(size_t)i * n + j] = s / ljj;
        }
    }
#pragma omp parallel
    {
        double* col = (double*)xmalloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 8)
        for (int c = 0; c < n; ++c) {
            for (int i = 0; i < n; ++i) {
                double s = (i == c) ? 1.0 : 0.0;
                for (int k = 0; k < i; ++k) s -= M[(size_t)i * n + k] * col[k];
                col[i] = s / M[(size_t)i * n + i];
            }
            for (int i = n - 1; i >= 0; --i) {
                double s = col[i];
                for (int k = i + 1; k < n; ++k) s -= M[(size_t)k * n + i] * col[k];
                col[i] = s / M[(size_t)i * n + i];
            }
            for (int i = 0; i < n; ++i) inv[(size_t)i * n + c] = col[i];
        }
        free(col);
    }
    return 1;
}

static hcsr hcsr_copy(int n, const int* rp, const int* ci, const double* v) {
    hcsr A;
    A.rows = A.cols = n;
    int nnz = rp[n];
    A.rp = (int*)xmalloc(sizeof(int) * ((size_t)n + 1)); memcpy(A.rp, rp, sizeof(int) * ((size_t)n + 1));
    A.ci = (int*)xmalloc(sizeof(int) * (size_t)(nnz ? nnz : 1)); memcpy(A.ci, ci, sizeof(int) * (size_t)nnz);
    A.v = (double*)xmalloc(sizeof(double) * (size_t)(nnz ? nnz : 1)); memcpy(A.v, v, sizeof(double) * (size_t)nnz);
    return A;
}

/* AmgPreconditioner::setup (src/cfa/linalg.cuh:995-1060) */
or_amg* or_amg_setup(int n, const int* rp, const int* ci, const double* val, double theta,
                     int smooth_steps, int coarse_target, int max_levels) {
    or_amg* h = (or_amg*)xcalloc(1, sizeof(or_amg));
    h->smooth_steps = smooth_steps;
    hcsr A = hcsr_copy(n, rp, ci, val);
    if (max_levels > OR_MAX_LEVELS) max_levels = OR_MAX_LEVELS;
    while (A.rows > coarse_target && h->nlev < max_levels - 1) {
        double* dinv = (double*)xmalloc(sizeof(double) * (size_t)A.rows);
        for (int i = 0; i < A.rows; ++i) {
            double d = 0.0;
            for (int a = A.rp[i]; a < A.rp[i + 1]; ++a) if (A.ci[a] == i) d = A.v[a];
            dinv[i] = (fabs(d) > 1.0e-300) ? 1.0 / d : 1.0;
        }
        double omega = 4.0 / (3.0 * spectral_radius(&A, dinv));
        int* agg = (int*)xmalloc(sizeof(int) * (size_t)A.rows);
        hcsr P = smoothed_prolongator(&A, dinv, omega, theta, agg);
        if (P.cols >= (int)(0.85 * A.rows) || P.cols == 0) {
            hcsr_free(&P); free(dinv); free(agg);
            break;
        }
        hcsr R = csr_tr(&P);
        hcsr AP = csr_mul(&A, &P);
        hcsr Ac = csr_mul(&R, &AP);
        hcsr_free(&AP);
        or_level* L = &h->L[h->nlev++];
        L->A = A; L->P = P; L->R = R; L->dinv = dinv; L->omega = omega; L->agg = agg;
        int m = A.rows;
        L->x = (double*)xcalloc((size_t)m, sizeof(double));
        L->b = (double*)xcalloc((size_t)m, sizeof(double));
        L->r = (double*)xcalloc((size_t)m, sizeof(double));
        L->Ax = (double*)xcalloc((size_t)m, sizeof(double));
        A = Ac;
    }
    int cn = A.rows;
    h->coarse_n = cn;
    h->coarse_A = (double*)xcalloc((size_t)cn * cn + 1, sizeof(double));
    for (int i = 0; i < cn; ++i)
        for (int a = A.rp[i]; a < A.rp[i + 1]; ++a) h->coarse_A[(size_t)i * cn + A.ci[a]] = A.v[a];
    double* M = (double*)xmalloc(sizeof(double) * ((size_t)cn * cn + 1));
    memcpy(M, h->coarse_A, sizeof(double) * (size_t)cn * cn);
    h->coarse_inv = (double*)xcalloc((size_t)cn * cn + 1, sizeof(double));
    int ok = dense_spd_inverse(M, cn, h->coarse_inv);
    free(M);
    hcsr_free(&A);
    h->cx = (double*)xcalloc((size_t)cn + 1, sizeof(double));
    h->cb = (double*)xcalloc((size_t)cn + 1, sizeof(double));
    if (!ok) { or_amg_free(h); return NULL; }
    return h;
}

int or_amg_num_levels(const or_amg* h) { return h->nlev; }

void or_amg_level_info(const or_amg* h, int l, int* info, double* omega) {
    const or_level* L = &h->L[l];
    info[0] = L->A.rows; info[1] = L->A.rp[L->A.rows]; info[2] = L->P.cols; info[3] = L->P.rp[L->P.rows];
    if (omega) *omega = L->omega;
}

void or_amg_level_agg(const or_amg* h, int l, int* agg) {
    memcpy(agg, h->L[l].agg, sizeof(int) * (size_t)h->L[l].A.rows);
}

void or_amg_level_csr(const or_amg* h, int l, int which, int* rp, int* ci, double* v) {
    const hcsr* M = which == 0 ? &h->L[l].A : which == 1 ? &h->L[l].P : &h->L[l].R;
    int nnz = M->rp[M->rows];
    if (rp) memcpy(rp, M->rp, sizeof(int) * ((size_t)M->rows + 1));
    if (ci) memcpy(ci, M->ci, sizeof(int) * (size_t)nnz);
    if (v) memcpy(v, M->v, sizeof(double) * (size_t)nnz);
}

void or_amg_level_dinv(const or_amg* h, int l, double* dinv) {
    memcpy(dinv, h->L[l].dinv, sizeof(double) * (size_t)h->L[l].A.rows);
}

int or_amg_coarse_n(const or_amg* h) { return h->coarse_n; }

void or_amg_coarse(const or_amg* h, double* Ac_dense, double* inv) {
    size_t sz = (size_t)h->coarse_n * h->coarse_n;
    if (Ac_dense) memcpy(Ac_dense, h->coarse_A, sizeof(double) * sz);
    if (inv) memcpy(inv, h->coarse_inv, sizeof(double) * sz);
}

/* k_csr_op semantics (src/cfa/linalg.cuh:884-901), sequential row sums */
static void csr_op(const hcsr* M, int op, const double* x, const double* b, const double* dinv,
                   double omega, double* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < M->rows; ++i) {
        double s = 0.0;
        for (int k = M->rp[i]; k < M->rp[i + 1]; ++k) s += M->v[k] * x[M->ci[k]];
        if (op == 0) y[i] = s;
        else if (op == 1) y[i] += s;
        else if (op == 2) y[i] = b[i] - s;
        else y[i] = x[i] + omega * dinv[i] * (b[i] - s);
    }
}

static void dense_matvec(int n, const double* A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += A[(size_t)i * n + j] * x[j];
        y[i] = s;
    }
}

/* vcycle (src/cfa/linalg.cuh:1184-1206) */
static void vcycle(const or_amg* h, int l, const double* b) {
    or_level* L = (or_level*)&h->L[l];
    const int n = L->A.rows;
    for (int i = 0; i < n; ++i) L->x[i] = L->omega * L->dinv[i] * b[i];
    for (int s = 1; s < h->smooth_steps; ++s) {
        csr_op(&L->A, 3, L->x, b, L->dinv, L->omega, L->Ax);
        double* t = L->x; L->x = L->Ax; L->Ax = t;
    }
    csr_op(&L->A, 2, L->x, b, NULL, 0.0, L->r);
    double* cb = (l + 1 < h->nlev) ? h->L[l + 1].b : h->cb;
    csr_op(&L->R, 0, L->r, NULL, NULL, 0.0, cb);
    const double* cx;
    if (l + 1 < h->nlev) {
        vcycle(h, l + 1, h->L[l + 1].b);
        cx = h->L[l + 1].x;
    } else {
        dense_matvec(h->coarse_n, h->coarse_inv, h->cb, h->cx);
        cx = h->cx;
    }
    csr_op(&L->P, 1, cx, NULL, NULL, 0.0, L->x);
    for (int s = 0; s < h->smooth_steps; ++s) {
        csr_op(&L->A, 3, L->x, b, L->dinv, L->omega, L->Ax);
        double* t = L->x; L->x = L->Ax; L->Ax = t;
    }
}

/* AmgPreconditioner::apply (src/cfa/linalg.cuh:1161-1168) */
void or_amg_apply(const or_amg* h, const double* r, double* z) {
    if (h->nlev == 0) { dense_matvec(h->coarse_n, h->coarse_inv, r, z); return; }
    vcycle(h, 0, r);
    memcpy(z, h->L[0].x, sizeof(double) * (size_t)h->L[0].A.rows);
}

void or_amg_free(or_amg* h) {
    if (!h) return;
    for (int l = 0; l < h->nlev; ++l) {
        or_level* L = &h->L[l];
        hcsr_free(&L->A); hcsr_free(&L->P); hcsr_free(&L->R);
        free(L->dinv); free(L->agg); free(L->x); free(L->b); free(L->r); free(L->Ax);
    }
    free(h->coarse_A); free(h->coarse_inv); free(h->cx); free(h->cb);
    free(h);
}

/* AmgPreconditioner::remap (src/cfa/linalg.cuh:1074-1157): level 0 takes the new operator, its
 * inverse diagonal and a prolongator whose rows come from the old one (kept node: its old row;
 * new node: the mean of the rows of its graph neighbours that already have one, pass by pass
 * outwards); levels >= 1, omega and the coarse inverse stay. Rows of new nodes are summed in
 * column order with equal columns in accumulation order (a stable sort; the reference's
 * std::sort leaves the order of equal columns unspecified, so its sums may differ in the last
 * bit). Returns 1, or 0 when there is nothing to reuse (no levels, or new nodes without any
 * neighbour that has a row): the caller then sets the hierarchy up anew. */
typedef struct { int c; double v; } cv_pair;

static void pair_msort(cv_pair* a, cv_pair* tmp, int n) {
    if (n < 2) return;
    int h = n / 2;
    pair_msort(a, tmp, h);
    pair_msort(a + h, tmp, n - h);
    int i = 0, j = h, k = 0;
    while (i < h && j < n) tmp[k++] = (a[j].c < a[i].c) ? a[j++] : a[i++];
    while (i < h) tmp[k++] = a[i++];
    while (j < n) tmp[k++] = a[j++];
    memcpy(a, tmp, sizeof(cv_pair) * (size_t)n);
}

int or_amg_remap(or_amg* h, int n, const int* rp, const int* ci, const double* val, const int* new_to_old) {
    if (h->nlev == 0) return 0;
    const hcsr* Po = &h->L[0].P;
    int* extra_of = (int*)xmalloc(sizeof(int) * (size_t)(n + 1));
    char* has_row = (char*)xmalloc((size_t)n + 1);
    int* pending = (int*)xmalloc(sizeof(int) * (size_t)(n + 1));
    int* still = (int*)xmalloc(sizeof(int) * (size_t)(n + 1));
    int* set_now = (int*)xmalloc(sizeof(int) * (size_t)(n + 1));
    int np = 0;
    for (int i = 0; i < n; ++i) {
        extra_of[i] = -1;
        has_row[i] = new_to_old[i] >= 0;
        if (new_to_old[i] < 0) pending[np++] = i;
    }
    /* rows of new nodes: ex_rp[r] .. ex_rp[r + 1] in ex (grown geometrically) */
    int nex = 0, ex_cap = 1024, rp_cap = 256;
    cv_pair* ex = (cv_pair*)xmalloc(sizeof(cv_pair) * (size_t)ex_cap);
    int* ex_rp = (int*)xmalloc(sizeof(int) * (size_t)rp_cap);
    ex_rp[0] = 0;
    int acc_cap = 256;
    cv_pair* acc = (cv_pair*)xmalloc(sizeof(cv_pair) * (size_t)acc_cap);
    cv_pair* tmp = (cv_pair*)xmalloc(sizeof(cv_pair) * (size_t)acc_cap);
    int ok = 1;
    while (np > 0) {
        int ns = 0, nset = 0;
        for (int q = 0; q < np; ++q) {
            const int i = pending[q];
            int na = 0, cnt = 0;
            for (int a = rp[i]; a < rp[i + 1]; ++a) {
                const int k = ci[a];
                if (k == i || !has_row[k]) continue;
                ++cnt;
                const cv_pair* src;
                cv_pair one;
                int len;
                int j = new_to_old[k];
                int b0, b1;
                if (j >= 0) { b0 = Po->rp[j]; b1 = Po->rp[j + 1]; len = b1 - b0; }
                else { b0 = ex_rp[extra_of[k]]; b1 = ex_rp[extra_of[k] + 1]; len = b1 - b0; }
                if (na + len > acc_cap) {
                    while (na + len > acc_cap) acc_cap *= 2;
                    acc = (cv_pair*)realloc(acc, sizeof(cv_pair) * (size_t)acc_cap);
                    tmp = (cv_pair*)realloc(tmp, sizeof(cv_pair) * (size_t)acc_cap);
                }
                for (int b = b0; b < b1; ++b) {
                    if (j >= 0) { one.c = Po->ci[b]; one.v = Po->v[b]; src = &one; }
                    else src = &ex[b];
                    acc[na++] = *src;
                }
            }
            if (cnt == 0) { still[ns++] = i; continue; }
            pair_msort(acc, tmp, na);
            int nr = 0;
            for (int e = 0; e < na; ++e) {
                if (nr > 0 && acc[nr - 1].c == acc[e].c) acc[nr - 1].v += acc[e].v;
                else acc[nr++] = acc[e];
            }
            for (int e = 0; e < nr; ++e) acc[e].v /= cnt;
            if (nex + 2 > rp_cap) { rp_cap *= 2; ex_rp = (int*)realloc(ex_rp, sizeof(int) * (size_t)rp_cap); }
            if (ex_rp[nex] + nr > ex_cap) {
                while (ex_rp[nex] + nr > ex_cap) ex_cap *= 2;
                ex = (cv_pair*)realloc(ex, sizeof(cv_pair) * (size_t)ex_cap);
            }
            memcpy(ex + ex_rp[nex], acc, sizeof(cv_pair) * (size_t)nr);
            ex_rp[nex + 1] = ex_rp[nex] + nr;
            extra_of[i] = nex++;
            set_now[nset++] = i;
        }
        if (nset == 0) { ok = 0; break; }
        for (int q = 0; q < nset; ++q) has_row[set_now[q]] = 1;
        memcpy(pending, still, sizeof(int) * (size_t)ns);
        np = ns;
    }
    if (ok) {
        hcsr P;
        P.rows = n; P.cols = Po->cols;
        P.rp = (int*)xcalloc((size_t)n + 1, sizeof(int));
        for (int i = 0; i < n; ++i) {
            const int j = new_to_old[i];
            P.rp[i + 1] = P.rp[i] + (j >= 0 ? Po->rp[j + 1] - Po->rp[j] : ex_rp[extra_of[i] + 1] - ex_rp[extra_of[i]]);
        }
        P.ci = (int*)xmalloc(sizeof(int) * (size_t)(P.rp[n] + 1));
        P.v = (double*)xmalloc(sizeof(double) * (size_t)(P.rp[n] + 1));
        for (int i = 0; i < n; ++i) {
            const int j = new_to_old[i];
            int o = P.rp[i];
            if (j >= 0) {
                for (int b = Po->rp[j]; b < Po->rp[j + 1]; ++b, ++o) { P.ci[o] = Po->ci[b]; P.v[o] = Po->v[b]; }
            } else {
                for (int b = ex_rp[extra_of[i]]; b < ex_rp[extra_of[i] + 1]; ++b, ++o) { P.ci[o] = ex[b].c; P.v[o] = ex[b].v; }
            }
        }
        or_level* L = &h->L[0];
        hcsr R = csr_tr(&P);
        hcsr_free(&L->A); hcsr_free(&L->P); hcsr_free(&L->R);
        L->A = hcsr_copy(n, rp, ci, val);
        L->P = P;
        L->R = R;
        free(L->dinv); free(L->agg); free(L->x); free(L->b); free(L->r); free(L->Ax);
        L->dinv = (double*)xmalloc(sizeof(double) * (size_t)(n + 1));
        for (int i = 0; i < n; ++i) {
            double d = 0.0;
            for (int a = rp[i]; a < rp[i + 1]; ++a) if (ci[a] == i) d = val[a];
            L->dinv[i] = (fabs(d) > 1.0e-300) ? 1.0 / d : 1.0;
        }
        L->agg = (int*)xmalloc(sizeof(int) * (size_t)(n + 1));
        for (int i = 0; i < n; ++i) L->agg[i] = -1;
        L->x = (double*)xcalloc((size_t)n + 1, sizeof(double));
        L->b = (double*)xcalloc((size_t)n + 1, sizeof(double));
        L->r = (double*)xcalloc((size_t)n + 1, sizeof(double));
        L->Ax = (double*)xcalloc((size_t)n + 1, sizeof(double));
    }
    free(extra_of); free(has_row); free(pending); free(still); free(set_now);
    free(ex); free(ex_rp); free(acc); free(tmp);
    return ok;
}

/* ============================================================================================
 * Krylov solvers
 * ========================================================================================== */
static double* dvec(int n) { return (double*)xcalloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* GpuLinearSolver::solve_pcg (src/cfa/linalg.cuh:183-256) */
void or_pcg(int n, const int* rp, const int* ci, const double* val, const double* b, double* x,
            int max_iter, double tol, const double* oss_val, const double* inv_m,
            const int* bc_tag, int outlet_dirichlet, int pin, const or_amg* amg, or_report* rep) {
    rep->iterations = 0; rep->converged = 1; rep->rel_residual = 0.0;
    double *r = dvec(n), *z = dvec(n), *p = dvec(n), *q = dvec(n), *inv_diag = dvec(n);
#define APPLY(in, out) do { or_spmv(n, rp, ci, val, in, out); \
        if (oss_val) or_oss_apply(n, rp, ci, oss_val, inv_m, bc_tag, outlet_dirichlet, pin, in, out); } while (0)
    double b_norm = sqrt(or_dot(n, b, b));
    if (b_norm < 1.0e-14) {
        memset(x, 0, sizeof(double) * (size_t)n);
        goto done;
    }
    for (int i = 0; i < n; ++i) {
        double d = 1.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) if (ci[k] == i) { d = val[k]; break; }
        inv_diag[i] = (fabs(d) > 1.0e-14) ? (1.0 / d) : 1.0;
    }
    APPLY(x, q);
    for (int i = 0; i < n; ++i) r[i] = b[i] - q[i];
    {
        double r_norm = sqrt(or_dot(n, r, r));
        if (r_norm < tol * b_norm) goto done;
        if (amg) or_amg_apply(amg, r, z); else for (int i = 0; i < n; ++i) z[i] = inv_diag[i] * r[i];
        memcpy(p, z, sizeof(double) * (size_t)n);
        double rz_old = or_dot(n, r, z);
        int iter = 0, fin = 0;
        for (; iter < max_iter; ++iter) {
            APPLY(p, q);
            double pq = or_dot(n, p, q);
            if (fabs(pq) < 1.0e-30) break;
            double alpha = rz_old / pq;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] += -alpha * q[i]; }
            r_norm = sqrt(or_dot(n, r, r));
            rep->rel_residual = r_norm / b_norm;
            if (r_norm < tol * b_norm) { ++iter; fin = 1; break; }
            if (amg) or_amg_apply(amg, r, z); else for (int i = 0; i < n; ++i) z[i] = inv_diag[i] * r[i];
            double rz_new = or_dot(n, r, z);
            double beta = rz_new / (rz_old + 1.0e-30);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
            rz_old = rz_new;
        }
        rep->converged = fin;
        rep->iterations = iter;
    }
#undef APPLY
done:
    free(r); free(z); free(p); free(q); free(inv_diag);
}

/* GpuLinearSolver::solve_bicgstab (src/cfa/linalg.cuh:261-347) */
void or_bicgstab(int n, const int* rp, const int* ci, const double* val, const double* b,
                 double* x, int max_iter, double tol, or_report* rep) {
    rep->iterations = 0; rep->converged = 1; rep->rel_residual = 0.0;
    double *r = dvec(n), *r0 = dvec(n), *p = dvec(n), *v = dvec(n), *s = dvec(n), *t = dvec(n);
    double *phat = dvec(n), *shat = dvec(n), *inv_diag = dvec(n);
    for (int i = 0; i < n; ++i) {
        double d = 1.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) if (ci[k] == i) { d = val[k]; break; }
        inv_diag[i] = (fabs(d) > 1.0e-14) ? (1.0 / d) : 1.0;
    }
    or_spmv(n, rp, ci, val, x, v);
    for (int i = 0; i < n; ++i) { r[i] = b[i] - v[i]; r0[i] = r[i]; p[i] = r[i]; v[i] = 0.0; }
    double r_norm0 = sqrt(or_dot(n, r, r));
    if (r_norm0 < 1.0e-13) goto done;
    {
        double rho_old = 1.0, alpha = 1.0, omega = 1.0;
        const double breakdown = 1.0e-30 * r_norm0 * r_norm0 + 1.0e-300;
        int iter = 0, fin = 0;
        for (; iter < max_iter; ++iter) {
            double rho_new = or_dot(n, r0, r);
            if (fabs(rho_new) < breakdown) break;
            if (iter > 0) {
                double beta = (rho_new / rho_old) * (alpha / (omega + 1.0e-30));
                for (int i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
            }
            for (int i = 0; i < n; ++i) phat[i] = inv_diag[i] * p[i];
            or_spmv(n, rp, ci, val, phat, v);
            double r0_v = or_dot(n, r0, v);
            if (fabs(r0_v) < breakdown) break;
            alpha = rho_new / r0_v;
            for (int i = 0; i < n; ++i) s[i] = r[i] + -alpha * v[i];
            double s_norm = sqrt(or_dot(n, s, s));
            if (s_norm < tol * r_norm0 || s_norm < 1.0e-11) {
                for (int i = 0; i < n; ++i) x[i] += alpha * phat[i];
                ++iter; fin = 1; break;
            }
            for (int i = 0; i < n; ++i) shat[i] = inv_diag[i] * s[i];
            or_spmv(n, rp, ci, val, shat, t);
            double tt = or_dot(n, t, t);
            omega = (tt > breakdown) ? (or_dot(n, t, s) / tt) : 0.0;
            for (int i = 0; i < n; ++i) { x[i] += alpha * phat[i]; x[i] += omega * shat[i]; }
            for (int i = 0; i < n; ++i) r[i] = s[i] + -omega * t[i];
            double r_norm = sqrt(or_dot(n, r, r));
            rep->rel_residual = r_norm / r_norm0;
            if (r_norm < tol * r_norm0 || r_norm < 1.0e-11) { ++iter; fin = 1; break; }
            rho_old = rho_new;
        }
        rep->converged = fin;
        rep->iterations = iter;
    }
done:
    free(r); free(r0); free(p); free(v); free(s); free(t); free(phat); free(shat); free(inv_diag);
}

/* GpuBicgstab2::solve (src/cfa/linalg.cuh:660-754), both components, MC-ILU(0) right preconditioner */
void or_bicgstab2(int n, const int* rp, const int* ci, const double* val, const double* b_u,
                  const double* b_v, double* x_u, double* x_v, int max_iter, double tol,
                  const or_ilu* ilu, or_report* rep) {
    const int n2 = 2 * n;
    double *X = dvec(n2), *B = dvec(n2), *r = dvec(n2), *r0 = dvec(n2), *p = dvec(n2), *v = dvec(n2);
    double *s = dvec(n2), *t = dvec(n2), *phat = dvec(n2), *shat = dvec(n2);
    memcpy(X, x_u, sizeof(double) * (size_t)n); memcpy(X + n, x_v, sizeof(double) * (size_t)n);
    memcpy(B, b_u, sizeof(double) * (size_t)n); memcpy(B + n, b_v, sizeof(double) * (size_t)n);
#define SPMV2(in, out) do { or_spmv(n, rp, ci, val, in, out); or_spmv(n, rp, ci, val, (in) + n, (out) + n); } while (0)
#define DOT2(a, b, o) do { (o)[0] = or_dot(n, a, b); (o)[1] = or_dot(n, (a) + n, (b) + n); } while (0)
    SPMV2(X, v);
    for (int i = 0; i < n2; ++i) r[i] = B[i] - 1.0 * v[i];
    memcpy(r0, r, sizeof(double) * (size_t)n2);
    memcpy(p, r, sizeof(double) * (size_t)n2);
    memset(v, 0, sizeof(double) * (size_t)n2);
    double o[6];
    DOT2(r, r, o);
    double rn0[2], bd[2], rho[2], rho_old[2] = {1.0, 1.0}, alpha[2] = {1.0, 1.0}, omega[2] = {1.0, 1.0};
    int active[2];
    for (int c = 0; c < 2; ++c) {
        rn0[c] = sqrt(o[c]);
        rho[c] = o[c];
        bd[c] = 1.0e-30 * rn0[c] * rn0[c] + 1.0e-300;
        rep[c].iterations = 0; rep[c].converged = 1; rep[c].rel_residual = 0.0;
        active[c] = rn0[c] >= 1.0e-13;
    }
#define STOP(c, it, ok) do { active[c] = 0; rep[c].iterations = (it); rep[c].converged = (ok); } while (0)
    for (int iter = 0; iter < max_iter && (active[0] || active[1]); ++iter) {
        double cb[2] = {0, 0}, co[2] = {0, 0};
        for (int c = 0; c < 2; ++c) {
            if (active[c] && fabs(rho[c]) < bd[c]) STOP(c, iter, 0);
            if (active[c] && iter > 0) {
                cb[c] = (rho[c] / rho_old[c]) * (alpha[c] / (omega[c] + 1.0e-30));
                co[c] = omega[c];
            }
        }
        if (!(active[0] || active[1])) break;
        if (iter > 0)
            for (int i = 0; i < n2; ++i) { int c = i >= n; p[i] = r[i] + cb[c] * (p[i] - co[c] * v[i]); }
        or_ilu_apply(ilu, p, phat, 2);
        SPMV2(phat, v);
        DOT2(r0, v, o);
        double ca[2] = {0, 0};
        for (int c = 0; c < 2; ++c) {
            if (active[c] && fabs(o[c]) < bd[c]) STOP(c, iter, 0);
            if (active[c]) { alpha[c] = rho[c] / o[c]; ca[c] = alpha[c]; }
        }
        if (!(active[0] || active[1])) break;
        for (int i = 0; i < n2; ++i) s[i] = r[i] - ca[i >= n] * v[i];
        or_ilu_apply(ilu, s, shat, 2);
        SPMV2(shat, t);
        double oss[2], ott[2], ots[2];
        DOT2(s, s, oss); DOT2(t, t, ott); DOT2(t, s, ots);
        double a1[2] = {0, 0}, a2[2] = {0, 0}, cw[2] = {0, 0};
        int s_done[2] = {0, 0};
        for (int c = 0; c < 2; ++c) {
            if (!active[c]) continue;
            a1[c] = alpha[c];
            const double s_norm = sqrt(oss[c]);
            if (s_norm < tol * rn0[c] || s_norm < 1.0e-11) { s_done[c] = 1; continue; }
            const double tt = ott[c];
            omega[c] = (tt > bd[c]) ? (ots[c] / tt) : 0.0;
            a2[c] = omega[c]; cw[c] = omega[c];
        }
        for (int i = 0; i < n2; ++i) {
            int c = i >= n;
            X[i] += a1[c] * phat[i] + a2[c] * shat[i];
            r[i] = s[i] - cw[c] * t[i];
        }
        for (int c = 0; c < 2; ++c) if (s_done[c]) STOP(c, iter + 1, 1);
        if (!(active[0] || active[1])) break;
        double orr[2], or0r[2];
        DOT2(r, r, orr); DOT2(r0, r, or0r);
        for (int c = 0; c < 2; ++c) {
            if (!active[c]) continue;
            const double r_norm = sqrt(orr[c]);
            rep[c].rel_residual = r_norm / rn0[c];
            if (r_norm < tol * rn0[c] || r_norm < 1.0e-11) { STOP(c, iter + 1, 1); continue; }
            rho_old[c] = rho[c];
            rho[c] = or0r[c];
            if (iter + 1 == max_iter) STOP(c, max_iter, 0);
        }
    }
#undef STOP
#undef SPMV2
#undef DOT2
    memcpy(x_u, X, sizeof(double) * (size_t)n); memcpy(x_v, X + n, sizeof(double) * (size_t)n);
    free(X); free(B); free(r); free(r0); free(p); free(v); free(s); free(t); free(phat); free(shat);
}
