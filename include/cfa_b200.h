/*
 * cfa_b200 -- B200 (sm_100a) implementation of the per-timestep solve path of the P1-P1
 * projection solver: element assembly of the momentum and pressure (PPE + OSS) systems, the
 * multicolour-ILU(0) two-component BiCGSTAB for momentum and the SA-AMG-preconditioned CG for
 * the pressure.
 *
 * C ABI: plain pointers and sizes. Every pointer named d_* (or documented as device memory) is
 * device memory owned by the caller, exactly as in the reference driver, which cudaMallocs the
 * mesh, CSR and solution arrays itself (src/cfa/device.cuh:21-115). Solver handles own their
 * workspaces. Every call is asynchronous on the context's CUDA stream unless it says it
 * synchronises; calls returning a report synchronise.
 *
 * Layouts are the reference's: int32 CSR (row_ptr[n+1], sorted unique col_ind[nnz], diagonal
 * present), one value array per matrix, u and v sharing the momentum matrix, the OSS operator as
 * [Bx | By | BTx | BTy] (4 nnz doubles, src/cfa/fem_kernels.cuh:799-806), multicolour ILU rows in
 * colour order with split L/U (src/cfa/linalg.cuh:435-447), triangles as 3 ints per element.
 *
 * Errors are returned as cfa_status (the reference exits the process instead,
 * src/cfa/common.cuh:33-41); cfa_ctx_last_error() holds the message.
 */
#ifndef CFA_B200_H
#define CFA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CFA_OK = 0,
    CFA_NOT_CONVERGED = 1,  /* solve stopped at max_iter (reference: converged = false)        */
    CFA_BREAKDOWN = 2,      /* Krylov breakdown guard hit (reference: converged = false)       */
    CFA_ROW_TOO_LONG = 3,   /* ILU row above 32 entries (reference exits, linalg.cuh:464-467)  */
    CFA_COARSE_NOT_SPD = 4, /* AMG coarsest operator not SPD (reference exits, :1399-1402)     */
    CFA_CUDA_ERROR = 5,
    CFA_TIMEOUT = 6,        /* a bounded device wait gave up                                   */
    CFA_BAD_ARG = 7,
    CFA_NO_MEMORY = 8
} cfa_status;

typedef enum {
    CFA_FP64 = 0,   /* preconditioner stored and applied in FP64 (the reference)              */
    CFA_MIXED = 1   /* preconditioner stored and applied in FP32 inside FP64 Krylov iterations */
} cfa_precision;

typedef struct cfa_ctx cfa_ctx;
typedef struct cfa_mesh cfa_mesh;
typedef struct cfa_ilu cfa_ilu;
typedef struct cfa_amg cfa_amg;

/* ---------------------------------------------------------------------------------------------
 * context: one per CUDA stream (cudaStream_t passed as void*, NULL = legacy default stream)
 * ------------------------------------------------------------------------------------------- */
cfa_status cfa_ctx_create(void* cuda_stream, cfa_ctx** out);
cfa_status cfa_ctx_destroy(cfa_ctx* ctx);
const char* cfa_ctx_last_error(const cfa_ctx* ctx);
const char* cfa_status_string(cfa_status s);
/* Kernels launched through this context since creation (all of them are this library's). */
long long cfa_ctx_kernel_launches(const cfa_ctx* ctx);
/* Synchronises the context's stream. */
cfa_status cfa_ctx_sync(cfa_ctx* ctx);

/* Device memory of the library's buffers comes from a block cache. A block that a resized or
 * destroyed buffer lets go is reused, in stream order, by later allocations of the context that
 * allocated it, and becomes free for any context of the device once that context is destroyed
 * (the reference calls cudaMalloc/cudaFree at every resize, src/cfa/linalg.cuh:131-151, and
 * cudaFree waits for the whole device). A handle (mesh, ILU, AMG, OSS operator) used from a second
 * context needs that context ordered after the first (cfa_ctx_sync).
 * cfa_mem_trim synchronises ctx (may be NULL) and returns the blocks cached for ctx's stream and
 * the idle ones to the device; cfa_mem_cached reports the device and pinned host bytes held. */
cfa_status cfa_mem_trim(cfa_ctx* ctx);
cfa_status cfa_mem_cached(size_t* device_bytes, size_t* pinned_bytes);

/* Autotuner of the V-cycle's tile heights (replaces, where it is on, the fixed shapes of the
 * reference's csr_threads_per_row rule, src/cfa/linalg.cuh:918-927, for the matrices it tunes).
 * Off by default; cfa_autotune_set(1) or CFA_AUTOTUNE=1 turns it on for the AMG setups that
 * follow. For each tile-streamed matrix of the hierarchy whose kernel carries no reduction (every
 * matrix of the levels >= 1, and level 0's transfers), it times tiles of 1/4, 1/2, 1 and 2 times
 * the default height on that kernel and keeps the fastest; lanes per row are not changed, so
 * every result is bit for bit the one of the default shapes. Choices are cached per pattern
 * class for the life of the process. cfa_autotune_log copies the log (one JSON object per line:
 * class, rows, nnz, chosen row_shift, the microseconds per candidate) into buf (cap bytes,
 * NUL-terminated) and its full length into *len. */
cfa_status cfa_autotune_set(int enabled);
cfa_status cfa_autotune_log(char* buf, size_t cap, size_t* len);

/* ---------------------------------------------------------------------------------------------
 * CSR pattern of the P1 mesh graph: node i's row holds i and the vertices of its elements,
 * sorted and unique. Replaces build_csr_and_boundary_topology (src/cfa/mesh.cuh:198-249).
 * cfa_csr_count fills d_row_ptr and returns nnz (synchronises); cfa_csr_fill fills d_col_ind.
 * ------------------------------------------------------------------------------------------- */
cfa_status cfa_csr_count(cfa_ctx* ctx, int n_nodes, int n_elems, const int* d_elem_v, int* d_row_ptr,
                         int* nnz_out);
cfa_status cfa_csr_fill(cfa_ctx* ctx, int n_nodes, int n_elems, const int* d_elem_v,
                        const int* d_row_ptr, int* d_col_ind);

/* ---------------------------------------------------------------------------------------------
 * mesh: the device mesh and pattern of DeviceMeshBuffers (src/cfa/device.cuh:21-59) plus the
 * assembly plan built from them (node-to-element incidence and CSR scatter positions, which
 * replace find_csr_index, src/cfa/fem_kernels.cuh:12-28). The arrays stay owned by the caller
 * and must outlive the handle. Synchronises.
 * ------------------------------------------------------------------------------------------- */
cfa_status cfa_mesh_create(cfa_ctx* ctx, int n_nodes, int n_elems, const int* d_elem_v,
                           const double* d_x, const double* d_y, const int* d_bc_tag,
                           const int* d_row_ptr, const int* d_col_ind, cfa_mesh** out);
cfa_status cfa_mesh_destroy(cfa_mesh* mesh);
/* Outlet condition of src/cfa/common.cuh:76-89 (c_outlet_dirichlet, c_pressure_pin,
 * c_outlet_scale). Default: p = 0 Dirichlet on BC_OUTLET nodes. */
cfa_status cfa_mesh_set_outlet(cfa_mesh* mesh, int outlet_dirichlet, int pressure_pin, double outlet_scale);

/* ---------------------------------------------------------------------------------------------
 * assembly (atomic-free, deterministic: every entry is summed over its elements in ascending
 * element order). Outputs are overwritten (the reference memsets them and accumulates).
 * ------------------------------------------------------------------------------------------- */
typedef struct {
    double dt, nu, rho;
    double a0, a1, a2;      /* du/dt ~ a0 u* - (a1 u^n + a2 u^{n-1})           */
    double c1, c2;          /* advecting velocity w = c1 u^n + c2 u^{n-1}        */
    double tau_time;        /* SUPG tau time scale T                             */
    double skew_coef;       /* 0.5 skew-symmetric convection, 0 convective form  */
} cfa_momentum_params;

typedef struct {
    double u_max;           /* inflow peak: u = 4 u_max y (H - y) / H^2 on BC_INLET */
    double H;               /* channel height                                        */
} cfa_momentum_bc;

/* k_assemble_momentum_fem (src/cfa/fem_kernels.cuh:40-181) with the lumped mass. If bc is not
 * NULL, k_apply_bc_momentum (:411-453) is applied in the same pass (then d_u, d_v receive the
 * Dirichlet values; otherwise they are not touched and may be NULL). */
cfa_status cfa_assemble_momentum(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u_old,
                                 const double* d_v_old, const double* d_u_prev, const double* d_v_prev,
                                 const double* d_p_old, const cfa_momentum_params* prm,
                                 const cfa_momentum_bc* bc, double* d_A_val, double* d_rhs_u,
                                 double* d_rhs_v, double* d_mass_lumped, double* d_u, double* d_v);
/* cfa_assemble_momentum with a per-node viscosity field (d_nu_node, n values; the element uses
 * their mean). The reference has a scalar nu; with d_nu_node NULL this is cfa_assemble_momentum. */
cfa_status cfa_assemble_momentum_nu(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u_old,
                                    const double* d_v_old, const double* d_u_prev, const double* d_v_prev,
                                    const double* d_p_old, const cfa_momentum_params* prm,
                                    const double* d_nu_node, const cfa_momentum_bc* bc, double* d_A_val,
                                    double* d_rhs_u, double* d_rhs_v, double* d_mass_lumped, double* d_u,
                                    double* d_v);
/* Adjoint of the momentum predictor (no counterpart in the reference). With x = (u*, v*) the
 * solution of the system cfa_assemble_momentum_nu built (bc required) and lambda the solution of
 * A^T lambda_c = dJ/dx_c (cfa_ilu_factor_transposed + cfa_csr_transpose_values +
 * cfa_bicgstab2_solve), writes dJ/dtheta = sum_c lambda_c^T (db_c/dtheta - dA/dtheta x_c) for
 * the nodal inputs u_old, v_old, u_prev, v_prev, p_old and, when d_nu_node is given, the nodal
 * viscosity (each n values, overwritten); d_scalars2[0] = dJ/du_max (the inflow amplitude),
 * d_scalars2[1] = dJ/dnu for the scalar viscosity. The element derivatives are exact (forward-mode
 * dual numbers through the element assembly). Synchronises. */
cfa_status cfa_momentum_adjoint(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u_old, const double* d_v_old,
                                const double* d_u_prev, const double* d_v_prev, const double* d_p_old,
                                const cfa_momentum_params* prm, const double* d_nu_node,
                                const cfa_momentum_bc* bc, const double* d_x_u, const double* d_x_v,
                                const double* d_lambda_u, const double* d_lambda_v, double* d_g_u_old,
                                double* d_g_v_old, double* d_g_u_prev, double* d_g_v_prev, double* d_g_p_old,
                                double* d_g_nu_node, double* d_scalars2);
/* Adjoint pieces of the rest of a step (no counterpart in the reference). cfa_ppe_rhs_adjoint adds
 * R^T lambda_p to d_g_u, d_g_v, where rhs_p = R (u*, v*) is the PPE right-hand side
 * -(rho/dt') (N_i, div u*) after the pressure boundary conditions of the mesh's outlet rule: with
 * the default p = 0 outlet the Dirichlet rows' multipliers are ignored; with the pinned outlet
 * (cfa_mesh_set_outlet) the right-hand side's mean removal is transposed as well (l - (m.l/sum m)
 * on every row, l = lambda_p zeroed at the pin; synchronises in that case). lambda_p is the
 * pressure solve's adjoint. */
cfa_status cfa_ppe_rhs_adjoint(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_lambda_p, double dt_proj,
                               double rho, double* d_g_u, double* d_g_v);
/* Adjoint of the OSS terms of the pressure step (stab > 0, either outlet rule; no counterpart in
 * the reference). Given the pressure adjoint lambda (the solution of A lambda = g
 * with g zeroed on Dirichlet rows, A the step's operator (1 + s) K - B^T M^-1 B), the step's u*,
 * its OSS weights d_elem_s (cfa_oss_weights), p^n and the solution dp, adds the derivatives of
 * lambda^T (rhs_p - A dp) through the weights to d_g_u, d_g_v (u*, v*) and through the OSS
 * right-hand side to d_g_p (p^n). Synchronises. */
cfa_status cfa_oss_adjoint(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u_star, const double* d_v_star,
                           double dt_proj, double rho, double nu, double stab, const double* d_elem_s,
                           const double* d_mass_lumped, const double* d_lambda_p, const double* d_p_old,
                           const double* d_dp, double* d_g_u, double* d_g_v, double* d_g_p);
/* Adjoint of cfa_project_step with the rotational term from the increment: given the adjoints of
 * the corrected u, v, p, writes the adjoint of dp (overwritten); those of u* and p^n are the
 * corrected ones unchanged (the caller passes them through). */
cfa_status cfa_projection_adjoint(cfa_ctx* ctx, const cfa_mesh* mesh, double dt_proj, double rho, double nu,
                                  const double* d_mass_lumped, const double* d_g_u_new, const double* d_g_v_new,
                                  const double* d_g_p_new, double* d_g_dp);
/* Adds the derivatives of wx F_x + wy F_y (cfa_volume_forces) with respect to its seven nodal
 * inputs to the seven gradients. Synchronises. */
cfa_status cfa_volume_forces_adjoint(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u, const double* d_v,
                                     const double* d_u_old, const double* d_v_old, const double* d_u_prev,
                                     const double* d_v_prev, const double* d_p, double b0, double b1, double b2,
                                     double nu, double rho, double wx, double wy, double* d_g_u, double* d_g_v,
                                     double* d_g_u_old, double* d_g_v_old, double* d_g_u_prev,
                                     double* d_g_v_prev, double* d_g_p);
/* k_apply_bc_momentum (src/cfa/fem_kernels.cuh:411-453) alone. */
cfa_status cfa_apply_bc_momentum(cfa_ctx* ctx, const cfa_mesh* mesh, const cfa_momentum_bc* bc,
                                 double* d_A_val, double* d_rhs_u, double* d_rhs_v, double* d_u,
                                 double* d_v);
/* k_assemble_lumped_mass (src/cfa/fem_kernels.cuh:890-909). */
cfa_status cfa_lumped_mass(cfa_ctx* ctx, const cfa_mesh* mesh, double* d_mass_lumped);
/* k_compute_oss_weights (src/cfa/fem_kernels.cuh:697-719): s_K per element. */
cfa_status cfa_oss_weights(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u_star,
                           const double* d_v_star, double dt, double rho, double nu, double stab,
                           double* d_elem_s);
/* k_accumulate_scalar_gradient (src/cfa/fem_kernels.cuh:726-757): G(f) numerators, weights
 * sqrt(s_K) (d_elem_s NULL: weight 1). Overwrites d_gx, d_gy. */
cfa_status cfa_scalar_gradient(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_f,
                               const double* d_elem_s, double* d_gx, double* d_gy);
/* k_assemble_pressure_poisson (src/cfa/fem_kernels.cuh:201-282); with apply_bc != 0 also
 * apply_bc_pressure (:519-531) in the same pass, which then writes d_dp on Dirichlet rows.
 * With the pinned outlet (cfa_mesh_set_outlet) the RHS mean removal needs apply_bc != 0. */
cfa_status cfa_assemble_ppe(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u_star,
                            const double* d_v_star, const double* d_p_old, const double* d_gp_x,
                            const double* d_gp_y, const double* d_mass_lumped, const double* d_elem_s,
                            double dt, double rho, double stab, int apply_bc, double* d_Kp_val,
                            double* d_rhs_p, double* d_div_num, double* d_dp);
/* apply_bc_pressure (src/cfa/fem_kernels.cuh:460-531) alone. */
cfa_status cfa_apply_bc_pressure(cfa_ctx* ctx, const cfa_mesh* mesh, double* d_Kp_val,
                                 double* d_rhs_p, double* d_dp, const double* d_mass_lumped);
/* assemble_oss_projection (src/cfa/device.cuh:304-314): B, B^T into d_oss_val (4 nnz) and
 * 1/max(m, 1e-14) into d_inv_m. */
cfa_status cfa_assemble_oss(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_elem_s,
                            const double* d_mass_lumped, double* d_oss_val, double* d_inv_m);
/* The pressure system of one step in one row pass: k_assemble_pressure_poisson +
 * apply_bc_pressure + assemble_oss_projection (the driver's sequence at
 * src/cylinder_fem_amr.cu:412-441). With stab = 0 the OSS outputs are not written. */
cfa_status cfa_assemble_pressure_system(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u_star,
                                        const double* d_v_star, const double* d_p_old,
                                        const double* d_gp_x, const double* d_gp_y,
                                        const double* d_mass_lumped, const double* d_elem_s, double dt,
                                        double rho, double stab, double* d_Kp_val, double* d_rhs_p,
                                        double* d_div_num, double* d_dp, double* d_oss_val,
                                        double* d_inv_m);
/* apply_oss_projection (src/cfa/device.cuh:316-323): d_out -= B^T M^-1 B d_in, Dirichlet rows
 * untouched. */
cfa_status cfa_oss_apply(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_oss_val,
                         const double* d_inv_m, const double* d_in, double* d_out);
/* cfa_oss_apply without any device allocation. This entry point has no counterpart in the
 * reference. It is for callers that must not allocate device memory while they run: for example,
 * a time-step loop whose device memory is all handed to another allocator, or one that cannot
 * afford the device-wide synchronisation that cudaFree (and cudaMalloc, at times) implies.
 * cfa_oss_apply grows a workspace on first use; this entry point keeps the intermediate vector
 * g = M^-1 B d_in in a fixed static device array instead, and it does not synchronise.
 * Limit: mesh->n <= 524288 nodes (the array is 8 MiB); larger meshes get CFA_BAD_ARG.
 * Nothing needs to start at zero: every call writes each scratch entry it reads.
 * Setup: the call makes the context's device current for its duration (and restores the
 * caller's device). The first call on each device looks up the array's address and must come
 * before any stream capture on that device; the address is kept for the life of the process,
 * so the entry point must not be called on a device after cudaDeviceReset there.
 * There is one array per device and process: calls in flight at the same time on one device (two
 * streams, contexts or threads) race on it. Order such calls, e.g. on one stream or with events.
 * Result: the same d_out as cfa_oss_apply (same per-row summation order). Asynchronous on the
 * context's stream. */
cfa_status cfa_oss_apply_noalloc(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_oss_val,
                                 const double* d_inv_m, const double* d_in, double* d_out);

/* ---------------------------------------------------------------------------------------------
 * after the solves (the driver's Steps C and D, src/cylinder_fem_amr.cu:462-513); node sums are
 * gathered over each node's elements in ascending element order (the reference scatters them
 * with atomics), so results are deterministic.
 * ------------------------------------------------------------------------------------------- */
/* k_stiffness_apply (src/cfa/fem_kernels.cuh:618-637): d_out[i] += c (grad N_i, grad f). */
cfa_status cfa_stiffness_apply(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_f, double c,
                               double* d_out);
/* k_accumulate_grad_dp_and_vorticity (src/cfa/fem_kernels.cuh:536-575): the lumped-mass
 * numerators of grad dp and of the vorticity dv/dx - du/dy. Overwrites the three outputs (the
 * reference accumulates into zeroed arrays). */
cfa_status cfa_grad_dp_vorticity(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_dp,
                                 const double* d_u, const double* d_v, double* d_grad_dp_x,
                                 double* d_grad_dp_y, double* d_vort_num);
/* k_velocity_pressure_correction (src/cfa/fem_kernels.cuh:585-610): vort = vort_num / m,
 * p += p_update (dp - rot_coeff div_num / m), u -= (dt/rho) grad_dp_x / m and likewise v on
 * interior nodes and on a natural outlet. d_vort may be NULL. */
cfa_status cfa_velocity_pressure_correction(cfa_ctx* ctx, const cfa_mesh* mesh, double dt, double rho,
                                            double p_update, double rot_coeff, const double* d_div_num,
                                            const double* d_mass_lumped, const double* d_grad_dp_x,
                                            const double* d_grad_dp_y, const double* d_vort_num,
                                            const double* d_dp, double* d_u, double* d_v, double* d_p,
                                            double* d_vort);
/* Step C in two passes: with rotational_from_dp, div_num = -(dt_proj/rho) K dp (the driver's
 * k_stiffness_apply on a zeroed div_num, src/cylinder_fem_amr.cu:467-472; otherwise div_num is
 * used as the PPE assembly left it), then grad dp and vorticity, then the correction with
 * p_update = 1. */
cfa_status cfa_project_step(cfa_ctx* ctx, const cfa_mesh* mesh, double dt_proj, double rho,
                            double rot_coeff, int rotational_from_dp, const double* d_mass_lumped,
                            const double* d_dp, double* d_div_num, double* d_grad_dp_x,
                            double* d_grad_dp_y, double* d_vort_num, double* d_u, double* d_v,
                            double* d_p, double* d_vort);
/* k_volume_forces (src/cfa/fem_kernels.cuh:1046-1123): volume-integral drag and lift into
 * d_out2[0..1] (device; overwritten), du/dt = b0 u + b1 u_old + b2 u_prev. */
cfa_status cfa_volume_forces(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u, const double* d_v,
                             const double* d_u_old, const double* d_v_old, const double* d_u_prev,
                             const double* d_v_prev, const double* d_p, double b0, double b1, double b2,
                             double nu, double rho, double* d_out2);

/* AMR refinement indicators (the remesh side of the path). k_accumulate_recovered_gradient
 * (src/cfa/fem_kernels.cuh:911-968): d_grad_rec[4 n] = [du'/dx | du'/dy | dv/dx | dv/dy]
 * numerators of the disturbance velocity u' = u - 4 U y (H - y) / H^2 (overwritten). */
cfa_status cfa_recovered_gradient(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_u, const double* d_v,
                                  double u_max, double H, double* d_grad_rec);
/* k_compute_amr_error_indicator (src/cfa/fem_kernels.cuh:995-1035): d_elem_error[2 ne] =
 * [h_K max |omega - omega_P| | P1 interpolation-error estimate]. */
cfa_status cfa_amr_error_indicator(cfa_ctx* ctx, const cfa_mesh* mesh, const double* d_grad_rec,
                                   const double* d_mass_lumped, double* d_elem_error);

/* ---------------------------------------------------------------------------------------------
 * sparse kernels
 * ------------------------------------------------------------------------------------------- */
/* k_spmv_csr (src/cfa/linalg.cuh:8-26): y = A x, FP64. */
cfa_status cfa_spmv(cfa_ctx* ctx, int n, const int* d_row_ptr, const int* d_col_ind,
                    const double* d_val, const double* d_x, double* d_y);
/* k_spmv_csr_multi (src/cfa/linalg.cuh:572-581): nrhs vectors of stride n, A read once. */
cfa_status cfa_spmv_multi(cfa_ctx* ctx, int n, int nrhs, const int* d_row_ptr, const int* d_col_ind,
                          const double* d_val, const double* d_x, double* d_y);

/* ---------------------------------------------------------------------------------------------
 * multicolour ILU(0): MulticolourIlu0 (src/cfa/linalg.cuh:435-568)
 * ------------------------------------------------------------------------------------------- */
/* set_pattern (:456-528): greedy colouring in node order (bit-exact with the reference) from the
 * host copy of the pattern; d_row_ptr/d_col_ind are the same pattern on the device (kept for the
 * reference's signature: the handle uploads its own copy from the host arrays, so nothing of the
 * caller's needs to outlive the call). Synchronises. CFA_ROW_TOO_LONG above 32 entries per row. */
cfa_status cfa_ilu_create(cfa_ctx* ctx, int n, const int* h_row_ptr, const int* h_col_ind,
                          const int* d_row_ptr, const int* d_col_ind, cfa_precision precision,
                          cfa_ilu** out);
cfa_status cfa_ilu_destroy(cfa_ilu* ilu);
/* set_pattern (:456-528) on an existing handle (a new mesh after a remesh): as cfa_ilu_create,
 * keeping the handle's precision and reusing its device buffers. On failure the handle holds no
 * usable pattern until a successful call. */
cfa_status cfa_ilu_set_pattern(cfa_ctx* ctx, cfa_ilu* ilu, int n, const int* h_row_ptr, const int* h_col_ind,
                               const int* d_row_ptr, const int* d_col_ind);
/* factor (:531-541): ILU(0) of d_val in colour order, in FP64; the split factors are then kept in
 * the handle's precision. */
cfa_status cfa_ilu_factor(cfa_ctx* ctx, cfa_ilu* ilu, const double* d_val);
/* apply (:544-555): z = (LU)^-1 r for nrhs vectors of stride n. */
cfa_status cfa_ilu_apply(cfa_ctx* ctx, const cfa_ilu* ilu, const double* d_r, double* d_z, int nrhs);
/* z = (LU)^-1 r for two right-hand sides stored interleaved per row: d_r[2i] and d_r[2i + 1] are
 * the first and second right-hand side's entries of row i (d_r, d_z: 2n doubles, 16-byte
 * aligned, distinct). No counterpart in the reference, whose apply takes the two with stride n
 * (MulticolourIlu0::apply, src/cfa/linalg.cuh:544-555); this is the layout this library's
 * BiCGSTAB2 keeps its vectors in, and these are the sweeps it runs. FP64 handles sweep in FP64
 * (the same operations as cfa_ilu_apply with nrhs = 2); mixed-precision handles sweep in FP32
 * arithmetic on an FP32 work vector held by the handle (d_r rounded to FP32 once, d_z the FP32
 * result widened). Calls on one handle must not overlap on the GPU (the work vector). */
cfa_status cfa_ilu_apply_interleaved(cfa_ctx* ctx, const cfa_ilu* ilu, const double* d_r, double* d_z);
/* Adjoint support (no counterpart in the reference): factors d_val as cfa_ilu_factor does and
 * keeps (LU)^T in the handle, so that cfa_ilu_apply gives z = (LU)^-T r and the handle
 * preconditions A^T (in the same colour order: (LU)^T = (U^T D^-1)(D L^T)). Needs a structurally
 * symmetric pattern (CFA_BAD_ARG otherwise; synchronises the first time). cfa_ilu_factor
 * switches the handle back. */
cfa_status cfa_ilu_factor_transposed(cfa_ctx* ctx, cfa_ilu* ilu, const double* d_val);
/* d_val_t = the values of A^T on the same (structurally symmetric) pattern as the handle's. */
cfa_status cfa_csr_transpose_values(cfa_ctx* ctx, cfa_ilu* ilu, const double* d_val, double* d_val_t);
/* n_colours and colour_start (host, n_colours + 1 entries, may be NULL). */
cfa_status cfa_ilu_colours(const cfa_ilu* ilu, int* n_colours, int* colour_start);
/* Device arrays of the handle (public members d_colour, d_rows, d_lu of the reference class):
 * colour[n], rows[n] (colour order), lu[nnz] (FP64 factor on the CSR pattern). */
cfa_status cfa_ilu_device_arrays(const cfa_ilu* ilu, const int** d_colour, const int** d_rows,
                                 const double** d_lu);

/* ---------------------------------------------------------------------------------------------
 * solvers
 * ------------------------------------------------------------------------------------------- */
typedef struct {
    int max_iter;
    double tol;             /* relative tolerance, the reference's stopping rules */
} cfa_solve_opts;

typedef struct {
    int iterations[2];      /* [0] = the (u) system, [1] = v for the two-component solve */
    int converged[2];
    double rel_residual[2]; /* the reference's last_rel_residual */
    double solve_ms;        /* device time of the solve (CUDA events) */
} cfa_solve_report;

/* Two-component BiCGSTAB, right MC-ILU(0): GpuBicgstab2::solve (src/cfa/linalg.cuh:656-754).
 * Per-component stop |r| < tol |r0| or |r| < 1e-11, breakdown 1e-30 r0^2 + 1e-300. x_u, x_v are
 * the initial guesses and receive the solutions. Synchronises (report). Returns CFA_OK when both
 * components converged, else CFA_NOT_CONVERGED (details in the report). */
cfa_status cfa_bicgstab2_solve(cfa_ctx* ctx, int n, const int* d_row_ptr, const int* d_col_ind,
                               const double* d_val, const double* d_b_u, const double* d_b_v,
                               double* d_x_u, double* d_x_v, const cfa_ilu* ilu,
                               const cfa_solve_opts* opts, cfa_solve_report* report);
/* Jacobi BiCGSTAB: GpuLinearSolver::solve_bicgstab (src/cfa/linalg.cuh:261-347). */
cfa_status cfa_bicgstab_solve(cfa_ctx* ctx, int n, const int* d_row_ptr, const int* d_col_ind,
                              const double* d_val, const double* d_b, double* d_x,
                              const cfa_solve_opts* opts, cfa_solve_report* report);

/* SA-AMG: AmgPreconditioner (src/cfa/linalg.cuh:939-1432) */
typedef struct {
    double theta;           /* strength threshold (0.08)          */
    int smooth_steps;       /* Jacobi sweeps per side (2)         */
    int coarse_target;      /* dense solve below this size (300)  */
    int max_levels;         /* (15)                               */
    cfa_precision precision;
} cfa_amg_opts;
void cfa_amg_default_opts(cfa_amg_opts* opts);
cfa_status cfa_amg_create(cfa_ctx* ctx, const cfa_amg_opts* opts, cfa_amg** out);
cfa_status cfa_amg_destroy(cfa_amg* amg);
/* setup (:995-1060): hierarchy of the device matrix; FP64 setup arithmetic in the reference's
 * order (aggregates, P, R and Galerkin operators bit-exact with the reference's host setup).
 * Synchronises. CFA_COARSE_NOT_SPD if the coarsest operator is not SPD. */
cfa_status cfa_amg_setup(cfa_ctx* ctx, cfa_amg* amg, int n, int nnz, const int* d_row_ptr,
                         const int* d_col_ind, const double* d_val);
/* remap (:1074-1157): carries the hierarchy over to a new mesh. Level 0 takes the new operator,
 * its inverse diagonal and a prolongator built from the old one: a kept node (h_new_to_old[i] =
 * its old row) keeps its row, a new node (-1) gets the mean of the rows of its graph neighbours
 * that already have one, pass by pass outwards. Levels >= 1, omega and the coarse inverse stay.
 * h_rp/h_ci: host copy of the new operator's pattern. Sets the hierarchy up anew (as setup) when
 * nothing can be reused: no levels, or new nodes none of whose neighbours has a row.
 * Synchronises. */
cfa_status cfa_amg_remap(cfa_ctx* ctx, cfa_amg* amg, int n, int nnz, const int* d_row_ptr,
                         const int* d_col_ind, const double* d_val, const int* h_row_ptr,
                         const int* h_col_ind, const int* h_new_to_old);
/* remaps: remap() calls that reused the hierarchy (the reference's `remaps`). */
int cfa_amg_remaps(const cfa_amg* amg);
/* apply (:1161-1168): one symmetric V-cycle, z = M^-1 r. */
cfa_status cfa_amg_apply(cfa_ctx* ctx, cfa_amg* amg, const double* d_r, double* d_z);
/* num_levels() (reference: levels with P + the coarsest), coarse_n, setup time [ms] */
cfa_status cfa_amg_info(const cfa_amg* amg, int* num_levels, int* coarse_n, double* setup_ms);
/* Level l (0 <= l < num_levels - 1): info = {rows, A nnz, P cols, P nnz, R nnz}; FP64 device
 * arrays of A, P, R (any pointer argument may be NULL), the aggregate of every row, omega. */
cfa_status cfa_amg_level(const cfa_amg* amg, int l, int* info, const int** d_agg,
                         const int** d_A_rp, const int** d_A_ci, const double** d_A_v,
                         const int** d_P_rp, const int** d_P_ci, const double** d_P_v,
                         const int** d_R_rp, const int** d_R_ci, const double** d_R_v, double* omega);
/* Accumulated setup phase times [ms] over all setups (the reference's phase_ms[],
 * src/cfa/linalg.cuh:970-982): copy, D^-1 + rho, strength + aggregation, P smoothing, transpose,
 * Galerkin products, tile packing, coarse inverse. */
cfa_status cfa_amg_phases(const cfa_amg* amg, double* ms8);
/* dense inverse of the coarsest operator (device, coarse_n^2 FP64, row-major) */
cfa_status cfa_amg_coarse_inverse(const cfa_amg* amg, const double** d_inv);
/* The composite coarse operator (no counterpart in the reference): the V-cycle below a small
 * level (the first level l >= 1 with at most 2048 rows; CFA_COMPOSITE_ROWS overrides, 0 turns it
 * off) is one linear map of that level's right-hand side, formed at setup as a dense row-major
 * FP64 matrix (rows x rows) and applied as one matrix-vector product. *level = -1 when none.
 * d_m may be NULL. */
cfa_status cfa_amg_composite(const cfa_amg* amg, int* level, int* rows, const double** d_m);
/* The V-cycle's forms for the setups that follow on this handle (no counterpart in the reference;
 * -1 keeps the default or the environment's): composite_rows, the largest level replaced by the
 * composite operator (0: none; default 2048, CFA_COMPOSITE_ROWS); fuse_levels, the levels whose
 * restriction runs fused, R b - (R A) x in one pass (0 none, 1 levels >= 1, the default, 2 all;
 * CFA_VC_FUSE); fold_rows, the largest fused level whose prolongation is folded into the first
 * post-smoothing sweep (default 16384, CFA_VC_ADDJAC_ROWS). Every form is the same preconditioner
 * up to rounding; each costs setup time that only repeated solves with one hierarchy (a time loop
 * between rebuilds) earn back, so a caller that solves once per setup turns them off (0, 0, 0). */
cfa_status cfa_amg_set_vcycle(cfa_amg* amg, int composite_rows, int fuse_levels, int fold_rows);
/* Mixed-precision handles (no counterpart in the reference): the Krylov solves preconditioned by
 * this handle run their V-cycles in FP64 until the relative residual falls below switch_rel and
 * in FP32 after that, for the setups that follow (0: FP32 throughout; negative: the default 1e-1
 * or CFA_FP64_PHASE). The FP32 V-cycle's rounding, about 1e-7 of the residual it is applied to,
 * enters the CG's search directions and costs iterations near a tight tolerance only when it is
 * made while the residual is still large; the FP64 copy of the level tiles costs setup time and
 * memory. CFA_BAD_ARG for switch_rel >= 1. */
cfa_status cfa_amg_set_fp64_phase(cfa_amg* amg, double switch_rel);
/* Where the setups that follow run the greedy aggregation (the reference's host loop,
 * src/cfa/linalg.cuh:1321-1348): on the device (1, the default), on the host (0), or as
 * CFA_AGG_HOST says (-1; CFA_AGG_HOST=1 selects the host). Both give the same aggregates. The
 * device form decides each phase in one launch whose blocks wait on one another's decisions; it
 * is the faster one for a single solve stream, while callers that overlap many small setups on
 * several streams (the batch path) keep the SMs free with the host loop. CFA_BAD_ARG for
 * on_device > 1. */
cfa_status cfa_amg_set_aggregation(cfa_amg* amg, int on_device);

/* The assembled OSS term of the pressure operator (apply_oss_projection,
 * src/cfa/device.cuh:316-323): A x = K x - B^T M^-1 B x on non-Dirichlet rows. */
typedef struct {
    const cfa_mesh* mesh;   /* boundary tags and outlet rule */
    const double* d_oss_val;
    const double* d_inv_m;
} cfa_oss_operator;

/* PCG: GpuLinearSolver::solve_pcg (src/cfa/linalg.cuh:183-256). The OSS term and the AMG are
 * handles instead of std::function callbacks (oss / amg NULL: plain CSR operator / Jacobi).
 * Warm start from d_x; stop when |r| < tol |b|; x = 0 and 0 iterations when |b| < 1e-14.
 * Synchronises (report). CFA_NOT_CONVERGED / CFA_BREAKDOWN as the reference's converged flag. */
cfa_status cfa_pcg_solve(cfa_ctx* ctx, int n, const int* d_row_ptr, const int* d_col_ind,
                         const double* d_val, const double* d_b, double* d_x,
                         const cfa_oss_operator* oss, cfa_amg* amg, const cfa_solve_opts* opts,
                         cfa_solve_report* report);

/* Host-side operator hook: a preconditioner writes d_out = M^-1 d_in; an extra operator adds its
 * part into d_out. Called on the host between this library's launches; the work it enqueues must
 * run after the context stream's earlier work and before its later work (true for the legacy
 * default stream when the context owns its stream, cfa_ctx_create(NULL, ...), and for the
 * context stream itself). */
typedef void (*cfa_host_op)(const double* d_in, double* d_out, void* user);

/* PCG with the reference's std::function hooks kept as host callbacks (GpuLinearSolver::solve_pcg,
 * src/cfa/linalg.cuh:183-256, extra_op and precond): A p = K p, then extra_op(p, A p) adds the
 * matrix-free part; precond, when set, replaces the AMG / Jacobi preconditioner (amg and precond
 * are exclusive). The kernels of cfa_pcg_solve without the CUDA graph (callbacks cannot be
 * captured); the stopping test stays on the device, polled every 8 iterations. No counterpart
 * as a separate entry point in the reference: it is solve_pcg with arbitrary closures. */
cfa_status cfa_pcg_solve_host_ops(cfa_ctx* ctx, int n, const int* d_row_ptr, const int* d_col_ind,
                                  const double* d_val, const double* d_b, double* d_x,
                                  cfa_host_op extra_op, void* extra_user, cfa_amg* amg,
                                  cfa_host_op precond, void* precond_user, const cfa_solve_opts* opts,
                                  cfa_solve_report* report);

/* Snapshots the pressure operator's current values into the context's tile-streamed layout
 * (the layout cfa_pcg_solve streams each iteration; one synchronisation when the pattern is
 * new). Call again after the values change. */
cfa_status cfa_pressure_operator_prepare(cfa_ctx* ctx, int n, int nnz, const int* d_row_ptr,
                                         const int* d_col_ind, const double* d_val,
                                         const cfa_oss_operator* oss);
/* Layout of the prepared pressure operator (diagnostic of this library; no counterpart in the
 * reference): passes = 1 when K - B^T M^-1 B is stored as one matrix on the two-ring pattern (or
 * there is no OSS term), 2 for the two-pass apply; stored_nnz = entries of the matrix streamed in
 * the (last) pass. CFA_BAD_ARG before cfa_pressure_operator_prepare. */
cfa_status cfa_pressure_operator_layout(const cfa_ctx* ctx, int* passes, long long* stored_nnz);
/* The pressure operator alone (operator of cfa_pcg_solve): y = K x (- B^T M^-1 B x).
 * Asynchronous (nnz passed by the caller). Uses the tile-streamed kernels when the same operator
 * was prepared, the row kernels otherwise. */
cfa_status cfa_pressure_operator(cfa_ctx* ctx, int n, int nnz, const int* d_row_ptr,
                                 const int* d_col_ind, const double* d_val,
                                 const cfa_oss_operator* oss, const double* d_x, double* d_y);

#ifdef __cplusplus
}
#endif
#endif
