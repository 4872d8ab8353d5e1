// Reference harness -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference solver's own translation unit (the file `cylinder_fem_amr.cu` of the
// reference project, found through the include path given by oracle/build.py; nothing of it is
// copied here) with CFA_NO_MAIN, the same mechanism as the reference's tests/test_cfa.cu:10-11,
// and exposes its functions and classes behind extern "C" entry points taking host arrays:
//   * host-only reference code (runs without a GPU): the CSR build, csr_multiply/csr_transpose,
//     the AMG setup primitives (spectral radius, smoothed prolongator, dense SPD inverse) and the
//     setup loop of AmgPreconditioner::setup restated over them;
//   * the reference's GPU code (assembly kernels, MulticolourIlu0, GpuBicgstab2, GpuLinearSolver,
//     AmgPreconditioner), for golden vectors on a GPU and for the benchmark's reference arm.
// Used by tests/golden/make_golden.py and bench.py --impl reference only.

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <future>
#include <iomanip>
#include <iostream>
#include <memory>
#include <numeric>
#include <sstream>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#include <parallel/algorithm>
#endif

// The AMG setup primitives are private members of AmgPreconditioner; they are host-only code.
#define CFA_NO_MAIN
#define private public
#include "cylinder_fem_amr.cu"
#undef private

namespace {

Mesh2D to_mesh(int n, int ne, const int* ev, const double* x, const double* y, const int* tag) {
    Mesh2D m;
    m.x.assign(x, x + n);
    m.y.assign(y, y + n);
    if (tag) m.bc_tag.assign(tag, tag + n); else m.bc_tag.assign(n, BC_INTERIOR);
    m.elems.resize(ne);
    for (int e = 0; e < ne; ++e) {
        for (int k = 0; k < 3; ++k) m.elems[e].v[k] = ev[3 * e + k];
        m.elems[e].level = 0;
        m.elems[e].gen = 0;
    }
    m.num_nodes = n;
    m.num_elems = ne;
    build_csr_and_boundary_topology(m);
    return m;
}

HostCsr to_host(int rows, int cols, const int* rp, const int* ci, const double* v) {
    HostCsr A;
    A.rows = rows;
    A.cols = cols;
    A.rp.assign(rp, rp + rows + 1);
    A.ci.assign(ci, ci + rp[rows]);
    A.v.assign(v, v + rp[rows]);
    return A;
}

void from_host(const HostCsr& A, int* rp, int* ci, double* v) {
    if (rp) std::copy(A.rp.begin(), A.rp.end(), rp);
    if (ci) std::copy(A.ci.begin(), A.ci.end(), ci);
    if (v) std::copy(A.v.begin(), A.v.end(), v);
}

struct HostHierarchy {
    std::vector<HostCsr> A, P, R;
    std::vector<double> omega;
    HostCsr coarse;
    std::vector<double> coarse_inv;
    bool spd = true;
};

template <class T>
T* dev_upload(const T* h, size_t count) {
    T* d = nullptr;
    CUDA_CHECK(cudaMalloc(&d, std::max<size_t>(count, 1) * sizeof(T)));
    if (count) CUDA_CHECK(cudaMemcpy(d, h, count * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}
template <class T>
void dev_download(T* h, const T* d, size_t count) {
    if (count) CUDA_CHECK(cudaMemcpy(h, d, count * sizeof(T), cudaMemcpyDeviceToHost));
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------------------------------
// host-only reference code
// ------------------------------------------------------------------------------------------
int ref_csr_build(int n, int ne, const int* ev, const double* x, const double* y, const int* tag,
                  int* rp, int* ci) {
    Mesh2D m = to_mesh(n, ne, ev, x, y, tag);
    std::copy(m.csr_row_ptr.begin(), m.csr_row_ptr.end(), rp);
    if (ci) std::copy(m.csr_col_ind.begin(), m.csr_col_ind.end(), ci);
    return m.nnz;
}

int ref_csr_multiply(int ar, int ac, const int* arp, const int* aci, const double* av, int bc,
                     const int* brp, const int* bci, const double* bv, int* crp, int* cci, double* cv) {
    HostCsr A = to_host(ar, ac, arp, aci, av), B = to_host(ac, bc, brp, bci, bv);
    HostCsr C = csr_multiply(A, B);
    from_host(C, crp, cci, cv);
    return (int)C.ci.size();
}

void ref_csr_transpose(int rows, int cols, const int* rp, const int* ci, const double* v,
                       int* trp, int* tci, double* tv) {
    HostCsr A = to_host(rows, cols, rp, ci, v);
    from_host(csr_transpose(A), trp, tci, tv);
}

double ref_spectral_radius(int n, const int* rp, const int* ci, const double* v, const double* dinv) {
    HostCsr A = to_host(n, n, rp, ci, v);
    std::vector<double> d(dinv, dinv + n);
    return AmgPreconditioner::spectral_radius_DinvA(A, d);
}

// Runs the setup loop of AmgPreconditioner::setup (src/cfa/linalg.cuh:1007-1058) on the host with
// the reference's own primitives; the result is kept in a handle.
void* ref_amg_host_setup(int n, const int* rp, const int* ci, const double* v) {
    AmgPreconditioner amg;
    auto* H = new HostHierarchy();
    HostCsr A = to_host(n, n, rp, ci, v);
    while (A.rows > amg.coarse_target && (int)H->A.size() < amg.max_levels - 1) {
        std::vector<double> dinv(A.rows);
        for (int i = 0; i < A.rows; ++i) {
            double d = 0.0;
            for (int a = A.rp[i]; a < A.rp[i + 1]; ++a) if (A.ci[a] == i) d = A.v[a];
            dinv[i] = (std::fabs(d) > 1.0e-300) ? 1.0 / d : 1.0;
        }
        double omega = 4.0 / (3.0 * AmgPreconditioner::spectral_radius_DinvA(A, dinv));
        HostCsr P = amg.smoothed_prolongator(A, dinv, omega);
        if (P.cols >= (int)(0.85 * A.rows) || P.cols == 0) break;
        HostCsr R = csr_transpose(P);
        HostCsr Ac = csr_multiply(R, csr_multiply(A, P));
        H->A.push_back(A);
        H->P.push_back(P);
        H->R.push_back(R);
        H->omega.push_back(omega);
        A = std::move(Ac);
    }
    const int cn = A.rows;
    std::vector<double> D((size_t)cn * cn, 0.0);
    for (int i = 0; i < cn; ++i)
        for (int a = A.rp[i]; a < A.rp[i + 1]; ++a) D[(size_t)i * cn + A.ci[a]] = A.v[a];
    // The reference exits on a non-SPD coarse operator; check the pivots first (same arithmetic).
    std::vector<double> M = D;
    for (int j = 0; j < cn && H->spd; ++j) {
        double d = M[(size_t)j * cn + j];
        for (int k = 0; k < j; ++k) d -= M[(size_t)j * cn + k] * M[(size_t)j * cn + k];
        if (!(d > 0.0)) { H->spd = false; break; }
        double ljj = std::sqrt(d);
        M[(size_t)j * cn + j] = ljj;
        for (int i = j + 1; i < cn; ++i) {
            double s = M[(size_t)i * cn + j];
            for (int k = 0; k < j; ++k) s -= M[(size_t)i * cn + k] * M[(size_t)j * cn + k];
            M[(size_t)i * cn + j] = s / ljj;
        }
    }
    if (H->spd) H->coarse_inv = AmgPreconditioner::dense_spd_inverse(D, cn);
    H->coarse = std::move(A);
    return H;
}

int ref_amg_host_levels(void* h) { return (int)static_cast<HostHierarchy*>(h)->A.size(); }

// which: 0 A, 1 P, 2 R, 3 coarsest operator (l ignored). info = {rows, cols, nnz}
void ref_amg_host_level(void* h, int l, int which, int* info, int* rp, int* ci, double* v) {
    auto* H = static_cast<HostHierarchy*>(h);
    const HostCsr& M = which == 0 ? H->A[l] : which == 1 ? H->P[l] : which == 2 ? H->R[l] : H->coarse;
    if (info) { info[0] = M.rows; info[1] = M.cols; info[2] = (int)M.ci.size(); }
    from_host(M, rp, ci, v);
}

double ref_amg_host_omega(void* h, int l) { return static_cast<HostHierarchy*>(h)->omega[l]; }

int ref_amg_host_coarse_inv(void* h, double* inv) {
    auto* H = static_cast<HostHierarchy*>(h);
    if (!H->spd) return 0;
    if (inv) std::copy(H->coarse_inv.begin(), H->coarse_inv.end(), inv);
    return 1;
}

void ref_amg_host_free(void* h) { delete static_cast<HostHierarchy*>(h); }

// ------------------------------------------------------------------------------------------
// the reference's GPU code
// ------------------------------------------------------------------------------------------
int ref_gpu_available(void) {
    int count = 0;
    return cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
}

// MulticolourIlu0: set_pattern, factor, then one apply of r (nrhs vectors). Outputs may be NULL.
int ref_ilu(int n, const int* rp, const int* ci, const double* val, int* colour, int* colour_start,
            int* rows, double* lu, const double* r, double* z, int nrhs) {
    const int nnz = rp[n];
    int* d_rp = dev_upload(rp, n + 1);
    int* d_ci = dev_upload(ci, nnz);
    double* d_val = dev_upload(val, nnz);
    std::vector<int> hrp(rp, rp + n + 1), hci(ci, ci + nnz);
    int nc = 0;
    {
        MulticolourIlu0 ilu;
        ilu.set_pattern(n, hrp, hci, d_rp, d_ci);
        ilu.factor(d_val);
        nc = ilu.n_colours;
        if (colour) dev_download(colour, ilu.d_colour, n);
        if (rows) dev_download(rows, ilu.d_rows, n);
        if (lu) dev_download(lu, ilu.d_lu, nnz);
        if (colour_start) std::copy(ilu.colour_start.begin(), ilu.colour_start.end(), colour_start);
        if (r && z) {
            double* d_r = dev_upload(r, (size_t)nrhs * n);
            double* d_z = nullptr;
            CUDA_CHECK(cudaMalloc(&d_z, (size_t)nrhs * n * sizeof(double)));
            ilu.apply(d_r, d_z, nrhs);
            CUDA_CHECK(cudaDeviceSynchronize());
            dev_download(z, d_z, (size_t)nrhs * n);
            cudaFree(d_r);
            cudaFree(d_z);
        }
    }
    cudaFree(d_rp); cudaFree(d_ci); cudaFree(d_val);
    return nc;
}

// GpuBicgstab2::solve with MulticolourIlu0. info[c] = {iters, converged}; rel[c]
void ref_bicgstab2(int n, const int* rp, const int* ci, const double* val, const double* bu,
                   const double* bv, double* xu, double* xv, int max_iter, double tol, int* info,
                   double* rel) {
    const int nnz = rp[n];
    int* d_rp = dev_upload(rp, n + 1);
    int* d_ci = dev_upload(ci, nnz);
    double* d_val = dev_upload(val, nnz);
    double* d_bu = dev_upload(bu, n);
    double* d_bv = dev_upload(bv, n);
    double* d_xu = dev_upload(xu, n);
    double* d_xv = dev_upload(xv, n);
    std::vector<int> hrp(rp, rp + n + 1), hci(ci, ci + nnz);
    {
        MulticolourIlu0 ilu;
        ilu.set_pattern(n, hrp, hci, d_rp, d_ci);
        ilu.factor(d_val);
        GpuBicgstab2 s;
        s.solve(n, d_rp, d_ci, d_val, d_bu, d_bv, d_xu, d_xv, max_iter, tol, ilu);
        for (int c = 0; c < 2; ++c) { info[2 * c] = s.iters[c]; info[2 * c + 1] = s.converged[c]; rel[c] = s.last_rel_residual[c]; }
    }
    dev_download(xu, d_xu, n);
    dev_download(xv, d_xv, n);
    for (void* p : {(void*)d_rp, (void*)d_ci, (void*)d_val, (void*)d_bu, (void*)d_bv, (void*)d_xu, (void*)d_xv}) cudaFree(p);
}

// GpuLinearSolver::solve_bicgstab (Jacobi)
int ref_bicgstab(int n, const int* rp, const int* ci, const double* val, const double* b, double* x,
                 int max_iter, double tol, int* converged, double* rel) {
    const int nnz = rp[n];
    int* d_rp = dev_upload(rp, n + 1);
    int* d_ci = dev_upload(ci, nnz);
    double* d_val = dev_upload(val, nnz);
    double* d_b = dev_upload(b, n);
    double* d_x = dev_upload(x, n);
    int it = 0;
    {
        GpuLinearSolver s;
        it = s.solve_bicgstab(n, d_rp, d_ci, d_val, d_b, d_x, max_iter, tol);
        *converged = s.converged;
        *rel = s.last_rel_residual;
    }
    dev_download(x, d_x, n);
    for (void* p : {(void*)d_rp, (void*)d_ci, (void*)d_val, (void*)d_b, (void*)d_x}) cudaFree(p);
    return it;
}

// GpuLinearSolver::solve_pcg with the assembled OSS term (oss_val/inv_m/bc_tag may be NULL) and
// AmgPreconditioner (use_amg). Also returns one V-cycle of amg_r (if given) in amg_z.
int ref_pcg(int n, const int* rp, const int* ci, const double* val, const double* b, double* x,
            int max_iter, double tol, const double* oss_val, const double* inv_m, const int* bc_tag,
            int use_amg, int* converged, double* rel, int* levels, const double* amg_r, double* amg_z) {
    const int nnz = rp[n];
    int* d_rp = dev_upload(rp, n + 1);
    int* d_ci = dev_upload(ci, nnz);
    double* d_val = dev_upload(val, nnz);
    double* d_b = dev_upload(b, n);
    double* d_x = dev_upload(x, n);
    double *d_oss = nullptr, *d_inv = nullptr, *d_gx = nullptr, *d_gy = nullptr;
    int* d_tag = nullptr;
    if (oss_val) {
        d_oss = dev_upload(oss_val, 4 * (size_t)nnz);
        d_inv = dev_upload(inv_m, n);
        d_tag = dev_upload(bc_tag, n);
        CUDA_CHECK(cudaMalloc(&d_gx, n * sizeof(double)));
        CUDA_CHECK(cudaMalloc(&d_gy, n * sizeof(double)));
    }
    int it = 0;
    {
        AmgPreconditioner amg;
        std::function<void(const double*, double*)> prec = [&amg](const double* r, double* z) { amg.apply(r, z); };
        std::function<void(const double*, double*)> oss = [&](const double* in, double* out) {
            const int blocks = (n + 255) / 256;
            k_oss_apply_B<<<blocks, 256>>>(n, d_rp, d_ci, nnz, d_oss, d_inv, in, d_gx, d_gy);
            k_oss_apply_BT<<<blocks, 256>>>(n, d_rp, d_ci, nnz, d_oss, d_tag, d_gx, d_gy, out);
        };
        if (use_amg) {
            amg.setup(n, nnz, d_rp, d_ci, d_val);
            if (levels) *levels = amg.num_levels();
            if (amg_r && amg_z) {
                double* d_r = dev_upload(amg_r, n);
                double* d_z = nullptr;
                CUDA_CHECK(cudaMalloc(&d_z, n * sizeof(double)));
                amg.apply(d_r, d_z);
                CUDA_CHECK(cudaDeviceSynchronize());
                dev_download(amg_z, d_z, n);
                cudaFree(d_r);
                cudaFree(d_z);
            }
        }
        GpuLinearSolver s;
        it = s.solve_pcg(n, d_rp, d_ci, d_val, d_b, d_x, max_iter, tol, oss_val ? &oss : nullptr,
                         use_amg ? &prec : nullptr);
        *converged = s.converged;
        *rel = s.last_rel_residual;
    }
    dev_download(x, d_x, n);
    for (void* p : {(void*)d_rp, (void*)d_ci, (void*)d_val, (void*)d_b, (void*)d_x, (void*)d_oss,
                    (void*)d_inv, (void*)d_tag, (void*)d_gx, (void*)d_gy})
        if (p) cudaFree(p);
    return it;
}

// ------------------------------------------------------------------------------------------
// One time step's solve path, as the reference driver runs it (src/cylinder_fem_amr.cu:300-475):
// Step A (momentum assembly + BCs, ILU factor, BiCGSTAB2) and Step B (OSS weights, G(p^n), PPE
// assembly + BCs, assembled OSS projection, PCG with OSS and SA-AMG). Every run_step starts from
// the same state (u = u^n, dp = 0), so repeated steps do identical work.
// ------------------------------------------------------------------------------------------
struct RefStep {
    Mesh2D mesh;
    DeviceMeshBuffers g;
    MulticolourIlu0 ilu;
    GpuBicgstab2 mom;
    GpuLinearSolver solver;
    AmgPreconditioner amg;
    std::vector<double> u0, v0, p0;
    double dt, nu, rho, u_max, H, tau_time, stab, tol;
    int max_it_mom, max_it_p;
};

void* ref_step_create(int n, int ne, const int* ev, const double* x, const double* y, const int* tag,
                      const double* u, const double* v, const double* p, double dt, double nu,
                      double rho, double u_max, double H, double tau_time, double stab, double tol,
                      int max_it_mom, int max_it_p) {
#ifdef _OPENMP
    // The reference application's host-thread rule (src/cylinder_fem_amr.cu:134-138), which
    // CFA_NO_MAIN skips with the rest of main(): unless OMP_NUM_THREADS is set, half the logical
    // CPUs, at most 8. Without it the AMG setup's OpenMP loops oversubscribe the host and run
    // several times slower than in the reference's own program.
    if (!std::getenv("OMP_NUM_THREADS")) omp_set_num_threads(std::max(1, std::min(8, omp_get_num_procs() / 2)));
#endif
    auto* S = new RefStep();
    S->mesh = to_mesh(n, ne, ev, x, y, tag);
    S->u0.assign(u, u + n);
    S->v0.assign(v, v + n);
    S->p0.assign(p, p + n);
    S->dt = dt; S->nu = nu; S->rho = rho; S->u_max = u_max; S->H = H; S->tau_time = tau_time;
    S->stab = stab; S->tol = tol; S->max_it_mom = max_it_mom; S->max_it_p = max_it_p;
    S->g.sync_from_host(S->mesh, S->u0, S->v0, S->p0, S->u0, S->v0);
    S->ilu.set_pattern(n, S->mesh.csr_row_ptr, S->mesh.csr_col_ind, S->g.d_row_ptr, S->g.d_col_ind);
    CUDA_CHECK(cudaDeviceSynchronize());
    return S;
}

static void ref_reset(RefStep* S) {
    DeviceMeshBuffers& g = S->g;
    const size_t nb = (size_t)g.n_nodes * sizeof(double);
    CUDA_CHECK(cudaMemcpy(g.d_u, S->u0.data(), nb, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(g.d_v, S->v0.data(), nb, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(g.d_u_prev, S->u0.data(), nb, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(g.d_v_prev, S->v0.data(), nb, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(g.d_p, S->p0.data(), nb, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(g.d_dp, 0, nb));
    CUDA_CHECK(cudaDeviceSynchronize());
}

// Step A (src/cylinder_fem_amr.cu:300-384): momentum assembly + BCs, ILU factor, BiCGSTAB2.
static void ref_step_momentum(RefStep* S) {
    DeviceMeshBuffers& g = S->g;
    const int n = g.n_nodes, ne = g.n_elems, nnz = g.nnz, tb = 256;
    const int bn = (n + tb - 1) / tb, be = (ne + tb - 1) / tb;
    const double dt = S->dt;
    const double a0 = 1.5 / dt, a1 = 2.0 / dt, a2 = -0.5 / dt, c1 = 2.0, c2 = -1.0;
    CUDA_CHECK(cudaMemset(g.d_A_val, 0, nnz * sizeof(double)));
    CUDA_CHECK(cudaMemset(g.d_rhs_u, 0, n * sizeof(double)));
    CUDA_CHECK(cudaMemset(g.d_rhs_v, 0, n * sizeof(double)));
    CUDA_CHECK(cudaMemset(g.d_mass_lumped, 0, n * sizeof(double)));
    k_assemble_momentum_fem<<<be, tb>>>(ne, g.d_elem_v, g.d_x, g.d_y, g.d_u, g.d_v, g.d_u_prev, g.d_v_prev,
                                        g.d_p, dt, S->nu, S->rho, a0, a1, a2, c1, c2, S->tau_time, 0.5,
                                        g.d_row_ptr, g.d_col_ind, g.d_A_val, g.d_rhs_u, g.d_rhs_v,
                                        g.d_mass_lumped, nullptr, nullptr);
    k_apply_bc_momentum<<<bn, tb>>>(n, g.d_bc_tag, g.d_y, S->u_max, S->H, g.d_row_ptr, g.d_col_ind,
                                    g.d_A_val, g.d_rhs_u, g.d_rhs_v, g.d_u, g.d_v, g.d_x, -1.0);
    S->ilu.factor(g.d_A_val);
    S->mom.solve(n, g.d_row_ptr, g.d_col_ind, g.d_A_val, g.d_rhs_u, g.d_rhs_v, g.d_u, g.d_v,
                 S->max_it_mom, S->tol, S->ilu);
    CUDA_CHECK(cudaDeviceSynchronize());
}

// Step B assembly (src/cylinder_fem_amr.cu:387-441): OSS weights, G(p^n), PPE + BCs, OSS operator.
static void ref_step_pressure_assembly(RefStep* S) {
    DeviceMeshBuffers& g = S->g;
    const int n = g.n_nodes, ne = g.n_elems, nnz = g.nnz, tb = 256;
    const int be = (ne + tb - 1) / tb;
    const double dt_proj = (2.0 / 3.0) * S->dt;
    CUDA_CHECK(cudaMemset(g.d_Kp_val, 0, nnz * sizeof(double)));
    CUDA_CHECK(cudaMemset(g.d_rhs_p, 0, n * sizeof(double)));
    CUDA_CHECK(cudaMemset(g.d_div_num, 0, n * sizeof(double)));
    CUDA_CHECK(cudaMemset(g.d_grad_dp_x, 0, n * sizeof(double)));
    CUDA_CHECK(cudaMemset(g.d_grad_dp_y, 0, n * sizeof(double)));
    const bool oss = S->stab > 0.0;
    if (oss) {
        k_compute_oss_weights<<<be, tb>>>(ne, g.d_elem_v, g.d_x, g.d_y, g.d_u, g.d_v, dt_proj, S->rho,
                                          S->nu, S->stab, g.d_elem_s);
        k_accumulate_scalar_gradient<<<be, tb>>>(ne, g.d_elem_v, g.d_x, g.d_y, g.d_p, g.d_elem_s,
                                                 g.d_grad_dp_x, g.d_grad_dp_y);
    }
    k_assemble_pressure_poisson<<<be, tb>>>(ne, g.d_elem_v, g.d_x, g.d_y, g.d_u, g.d_v, g.d_p,
                                            g.d_grad_dp_x, g.d_grad_dp_y, g.d_mass_lumped, g.d_elem_s,
                                            dt_proj, S->rho, S->stab, g.d_row_ptr, g.d_col_ind,
                                            g.d_Kp_val, g.d_rhs_p, g.d_div_num);
    apply_bc_pressure(n, g.d_bc_tag, g.d_row_ptr, g.d_col_ind, g.d_Kp_val, g.d_rhs_p, g.d_dp, g.d_mass_lumped);
    if (oss) assemble_oss_projection(g);
}

// Builds the AMG hierarchy as the driver does every amg_rebuild steps: from this step's pressure
// operator, i.e. after the momentum solve (src/cylinder_fem_amr.cu:445-452). Returns setup ms.
double ref_step_amg_setup(void* h) {
    auto* S = static_cast<RefStep*>(h);
    DeviceMeshBuffers& g = S->g;
    ref_reset(S);
    ref_step_momentum(S);
    ref_step_pressure_assembly(S);
    CUDA_CHECK(cudaDeviceSynchronize());
    S->amg.setup(g.n_nodes, g.nnz, g.d_row_ptr, g.d_col_ind, g.d_Kp_val);
    CUDA_CHECK(cudaDeviceSynchronize());
    return S->amg.setup_ms;
}

// Runs one step; returns its wall time [ms] (host clock with device syncs, as the reference times
// its phases). it[0..2] = momentum u, v and pressure iterations; conv[0..2] converged flags.
// If out_u/out_v/out_dp are given, the solved u*, v* and dp are returned.
double ref_step_run(void* h, int* it, int* conv, double* rel, double* out_u, double* out_v, double* out_dp) {
    auto* S = static_cast<RefStep*>(h);
    DeviceMeshBuffers& g = S->g;
    ref_reset(S);
    const int n = g.n_nodes;
    auto t0 = std::chrono::steady_clock::now();
    ref_step_momentum(S);
    ref_step_pressure_assembly(S);
    std::function<void(const double*, double*)> oss_op = [&g](const double* in, double* out) {
        apply_oss_projection(g, in, out);
    };
    std::function<void(const double*, double*)> prec = [S](const double* r, double* z) { S->amg.apply(r, z); };
    const bool use_amg = !S->amg.levels.empty() || S->amg.coarse_n > 0;
    int it_p = S->solver.solve_pcg(n, g.d_row_ptr, g.d_col_ind, g.d_Kp_val, g.d_rhs_p, g.d_dp, S->max_it_p,
                                   S->tol, S->stab > 0.0 ? &oss_op : nullptr, use_amg ? &prec : nullptr);
    CUDA_CHECK(cudaDeviceSynchronize());
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (it) { it[0] = S->mom.iters[0]; it[1] = S->mom.iters[1]; it[2] = it_p; }
    if (conv) { conv[0] = S->mom.converged[0]; conv[1] = S->mom.converged[1]; conv[2] = S->solver.converged; }
    if (rel) { rel[0] = S->mom.last_rel_residual[0]; rel[1] = S->mom.last_rel_residual[1]; rel[2] = S->solver.last_rel_residual; }
    if (out_u) dev_download(out_u, g.d_u, n);
    if (out_v) dev_download(out_v, g.d_v, n);
    if (out_dp) dev_download(out_dp, g.d_dp, n);
    return ms;
}

// Assembled systems of the step (after the momentum solve for the pressure part), for parity.
void ref_step_systems(void* h, double* A_val, double* rhs_u, double* rhs_v, double* mass, double* Kp_val,
                      double* rhs_p, double* div_num, double* elem_s, double* gpx, double* gpy,
                      double* oss_val, double* inv_m) {
    auto* S = static_cast<RefStep*>(h);
    DeviceMeshBuffers& g = S->g;
    const int n = g.n_nodes, ne = g.n_elems, nnz = g.nnz;
    if (A_val) dev_download(A_val, g.d_A_val, nnz);
    if (rhs_u) dev_download(rhs_u, g.d_rhs_u, n);
    if (rhs_v) dev_download(rhs_v, g.d_rhs_v, n);
    if (mass) dev_download(mass, g.d_mass_lumped, n);
    if (Kp_val) dev_download(Kp_val, g.d_Kp_val, nnz);
    if (rhs_p) dev_download(rhs_p, g.d_rhs_p, n);
    if (div_num) dev_download(div_num, g.d_div_num, n);
    if (elem_s) dev_download(elem_s, g.d_elem_s, ne);
    if (gpx) dev_download(gpx, g.d_grad_dp_x, n);
    if (gpy) dev_download(gpy, g.d_grad_dp_y, n);
    if (oss_val) dev_download(oss_val, g.d_oss_val, 4 * (size_t)nnz);
    if (inv_m) dev_download(inv_m, g.d_inv_m, n);
}

void ref_step_free(void* h) { delete static_cast<RefStep*>(h); }

// Stored entries of the step's CSR pattern.
int ref_step_nnz(void* h) { return static_cast<RefStep*>(h)->g.nnz; }

// Host threads the reference's OpenMP loops (AMG setup) run with.
int ref_omp_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
