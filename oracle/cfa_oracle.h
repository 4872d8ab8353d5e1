/*
 * CPU restatement of the reference solve path (TEST INFRASTRUCTURE ONLY).
 *
 * This is the oracle: a plain-C, FP64 statement of the reference's algorithms, used by the
 * tests as the checker, by the CPU-baseline leg of the benchmark, and nowhere else. The product
 * (the CUDA library) never links or calls it.
 *
 * Every function cites the reference file:line it restates (paths inside the reference project).
 */
#ifndef CFA_ORACLE_H
#define CFA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- CSR pattern: build_csr_and_boundary_topology (src/cfa/mesh.cuh:198-249) ---- */
int  or_csr_count(int n, int ne, const int* elem_v, int* row_ptr);           /* returns nnz */
void or_csr_fill(int n, int ne, const int* elem_v, const int* row_ptr, int* col_ind);

/* ---- assembly (src/cfa/fem_kernels.cuh) ---- */
typedef struct {
    double dt, nu, rho, a0, a1, a2, c1, c2, tau_time, skew_coef;
} or_mom_params;
void or_assemble_momentum(int n, int ne, const int* elem_v, const double* x, const double* y,
                          const double* u_old, const double* v_old, const double* u_prev,
                          const double* v_prev, const double* p_old, const or_mom_params* prm,
                          const int* rp, const int* ci, double* A_val, double* rhs_u, double* rhs_v,
                          double* mass_lumped);
void or_apply_bc_momentum(int n, const int* bc_tag, const double* y, double u_max, double H,
                          int outlet_dirichlet, double outlet_scale, const int* rp, const int* ci,
                          double* A_val, double* rhs_u, double* rhs_v, double* u, double* v);
void or_assemble_ppe(int n, int ne, const int* elem_v, const double* x, const double* y,
                     const double* u_star, const double* v_star, const double* p_old,
                     const double* gp_x, const double* gp_y, const double* mass_lumped,
                     const double* elem_s, double dt, double rho, double stab, const int* rp,
                     const int* ci, double* Kp_val, double* rhs_p, double* div_num);
void or_apply_bc_pressure(int n, const int* bc_tag, int outlet_dirichlet, int pin, const int* rp,
                          const int* ci, double* Kp_val, double* rhs_p, double* dp,
                          const double* mass_lumped);
void or_oss_weights(int ne, const int* elem_v, const double* x, const double* y,
                    const double* u_star, const double* v_star, double dt, double rho, double nu,
                    double stab, double* elem_s);
void or_scalar_gradient(int ne, const int* elem_v, const double* x, const double* y,
                        const double* f, const double* elem_s, double* gx, double* gy);
void or_assemble_oss(int n, int ne, const int* elem_v, const double* x, const double* y,
                     const double* elem_s, const int* rp, const int* ci, const double* mass_lumped,
                     double* oss_val, double* inv_m);
void or_oss_apply(int n, const int* rp, const int* ci, const double* oss_val, const double* inv_m,
                  const int* bc_tag, int outlet_dirichlet, int pin, const double* in, double* out);
void or_oss_matrix_free(int n, int ne, const int* elem_v, const double* x, const double* y,
                        const int* bc_tag, int outlet_dirichlet, int pin, const double* elem_s,
                        const double* mass_lumped, const double* in, double* out);
void or_lumped_mass(int n, int ne, const int* elem_v, const double* x, const double* y, double* m);

/* ---- linear algebra (src/cfa/linalg.cuh) ---- */
void or_spmv(int n, const int* rp, const int* ci, const double* val, const double* x, double* y);
double or_dot(int n, const double* a, const double* b);

/* after the solves (src/cfa/fem_kernels.cuh:536-637, :1046-1123); outputs accumulated */
void or_stiffness_apply(int ne, const int* ev, const double* x, const double* y, const double* f, double c,
                        double* out);
void or_grad_dp_vorticity(int ne, const int* ev, const double* x, const double* y, const double* dp,
                          const double* u, const double* v, double* gdx, double* gdy, double* vort_num);
void or_velocity_pressure_correction(int n, const int* tag, int outlet_dirichlet, double dt, double rho,
                                     double p_update, double rot_coeff, const double* div_num,
                                     const double* mass, const double* gdx, const double* gdy,
                                     const double* vort_num, const double* dp, double* u, double* v, double* p,
                                     double* vort);
void or_volume_forces(int ne, const int* ev, const int* tag, const double* x, const double* y, const double* u,
                      const double* v, const double* u_old, const double* v_old, const double* u_prev,
                      const double* v_prev, const double* p, double b0, double b1, double b2, double nu,
                      double rho, double* out);

/* AMR indicators (src/cfa/fem_kernels.cuh:911-1035); grad_rec accumulated */
void or_recovered_gradient(int n, int ne, const int* ev, const double* x, const double* y, const double* u,
                           const double* v, double u_max, double H, double* grad_rec);
void or_amr_error_indicator(int n, int ne, const int* ev, const double* x, const double* y, const double* grad_rec,
                            const double* mass, double* elem_error);

typedef struct or_ilu or_ilu;
or_ilu* or_ilu_create(int n, const int* rp, const int* ci);        /* NULL: row longer than 32 */
int  or_ilu_colours(const or_ilu* h);
void or_ilu_export(const or_ilu* h, int* colour, int* colour_start, int* rows, int* lp, int* up,
                   int* lc, int* uc, int* l_src, int* u_src, int* d_src, int* nl_nu);
void or_ilu_factor(or_ilu* h, const double* val, double* lu_out, double* lv, double* uv, double* dinv);
void or_ilu_apply(const or_ilu* h, const double* r, double* z, int nrhs);
void or_ilu_free(or_ilu* h);

typedef struct or_amg or_amg;
/* returns NULL on a non-SPD coarse operator (the reference exits) */
or_amg* or_amg_setup(int n, const int* rp, const int* ci, const double* val, double theta,
                     int smooth_steps, int coarse_target, int max_levels);
int  or_amg_num_levels(const or_amg* h);               /* levels with P (reference: levels.size()) */
/* info[0..3] = rows, A nnz, P cols, P nnz; omega out */
void or_amg_level_info(const or_amg* h, int l, int* info, double* omega);
void or_amg_level_agg(const or_amg* h, int l, int* agg);
void or_amg_level_csr(const or_amg* h, int l, int which /*0 A 1 P 2 R*/, int* rp, int* ci, double* v);
void or_amg_level_dinv(const or_amg* h, int l, double* dinv);
int  or_amg_coarse_n(const or_amg* h);
void or_amg_coarse(const or_amg* h, double* Ac_dense, double* inv);
void or_amg_apply(const or_amg* h, const double* r, double* z);
/* remap (src/cfa/linalg.cuh:1074-1157) onto a new operator; 0: set the hierarchy up anew */
int  or_amg_remap(or_amg* h, int n, const int* rp, const int* ci, const double* val, const int* new_to_old);
void or_amg_free(or_amg* h);

/* Reference host SpGEMM and transpose (src/cfa/linalg.cuh:799-862) on plain CSR arrays.
 * Two calls: with C_ci == NULL only C_rp is filled and nnz returned. */
int or_csr_multiply(int ar, int ac, const int* arp, const int* aci, const double* av,
                    int bc, const int* brp, const int* bci, const double* bv,
                    int* crp, int* cci, double* cv);
void or_csr_transpose(int rows, int cols, const int* rp, const int* ci, const double* v,
                      int* trp, int* tci, double* tv);

typedef struct {
    int iterations, converged;
    double rel_residual;
} or_report;

/* PCG (src/cfa/linalg.cuh:183-256). oss_val may be NULL; amg may be NULL (Jacobi). */
void or_pcg(int n, const int* rp, const int* ci, const double* val, const double* b, double* x,
            int max_iter, double tol, const double* oss_val, const double* inv_m,
            const int* bc_tag, int outlet_dirichlet, int pin, const or_amg* amg, or_report* rep);
/* Jacobi BiCGSTAB (src/cfa/linalg.cuh:261-347) */
void or_bicgstab(int n, const int* rp, const int* ci, const double* val, const double* b,
                 double* x, int max_iter, double tol, or_report* rep);
/* Two-component BiCGSTAB with MC-ILU(0) (src/cfa/linalg.cuh:660-754); rep[2] */
void or_bicgstab2(int n, const int* rp, const int* ci, const double* val, const double* b_u,
                  const double* b_v, double* x_u, double* x_v, int max_iter, double tol,
                  const or_ilu* ilu, or_report* rep);

int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
