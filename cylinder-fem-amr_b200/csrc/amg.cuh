// SA-AMG handle (AmgPreconditioner, src/cfa/linalg.cuh:939-1432).
#pragma once

#include <vector>

#include "internal.cuh"
#include "tiled.cuh"

namespace cfa {

struct DCsr {
    int rows = 0, cols = 0, nnz = 0;
    int tpr = 1;                   // threads per row of the V-cycle kernels
    DevBuf<int> rp, ci;
    DevBuf<double> v;              // FP64 values (setup arithmetic)
    DevBuf<float> v32;             // FP32 copy (mixed precision)
};

struct AmgLevel {
    DCsr A, P, R;
    TiledCsr tA, tP, tR;           // tile-streamed copies in the hierarchy precision
    // fused transfers: tQ (fusedQ), the restricted residual R b - (R A) x in one pass over the
    // next level's rows; tW (fusedW), the prolongation-add folded into the first post-smoothing
    // sweep (values [A | A P] and [I | P] on one pattern); columns with the top bit set read the
    // second vector (x, resp. the coarse correction)
    TiledCsr tQ, tW;
    // FP64 copies of tA, tP, tR, tQ, tW in a mixed-precision hierarchy, for the FP64 V-cycles that
    // a solve runs first (amg_fp64_phase); empty otherwise
    TiledCsr tA64, tP64, tR64, tQ64, tW64;
    bool fusedQ = false, fusedW = false;
    bool ra_spgemm = false;        // R A formed by SpGEMM (A not symmetric) rather than as (A P)^T
    DCsr AP;                       // A P of the Galerkin product (rows 0 after a remap changed P)
    DevBuf<double> dinv;
    DevBuf<float> dinv32;
    double omega = 0.0;
    DevBuf<int> agg;
    // V-cycle vectors in the hierarchy precision: x, t (Jacobi ping-pong), b, r
    DevBuf<double> x64, t64, b64, r64;
    DevBuf<float> x32, t32, b32, r32;
};

// Pinned, grow-only host buffer (blocks from the pinned cache, pool.cu)
template <class T>
struct HostBuf {
    T* p = nullptr;
    size_t cap = 0;
    size_t bytes = 0;
    cudaStream_t owner = nullptr;
    cudaError_t ensure(size_t count) {
        if (count <= cap && p) return cudaSuccess;
        if (p) pinned_release(p, bytes, owner);
        p = nullptr;
        cap = bytes = 0;
        size_t b = (count + count / 2 + 64) * sizeof(T);
        void* q = nullptr;
        cudaError_t e = pinned_alloc(&q, &b);
        if (e != cudaSuccess) return e;
        p = static_cast<T*>(q);
        bytes = b;
        cap = b / sizeof(T);
        owner = scope_stream();
        return cudaSuccess;
    }
    ~HostBuf() { if (p) pinned_release(p, bytes, owner); }
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
};

// Setup temporaries, kept across setups (grow-only): no allocation in a repeated setup.
struct SetupScratch {
    DevBuf<int> sg_ub, sg_cnt, sg_scol, sg_big, tr_keys, tr_idx, tr_perm, tr_row_of, cnt, p0rp, ierr;
    DevBuf<long long> sg_off;
    DevBuf<double> sg_sval, pow_x, pow_y, pow_py, pow_px, pow_st, p0v, M, colbuf;
    DevBuf<unsigned char> strong;
    DevBuf<int> ag_trp, ag_tci, ag_fill, ag_rank, ag_agg1, ag_agg2, ag_size, ag_flag, ag_cptr, ag_conf;   // device aggregation
    DevBuf<unsigned char> ag_state;
    HostBuf<int> h_ag;                  // flag / totals read back by the aggregation rounds
    DevBuf<char> cub_tmp;
    HostBuf<int> h_rp, h_ci, h_cnt, h_ub, h_agg, h_p0rp;
    HostBuf<long long> h_off;
    HostBuf<unsigned char> h_strong;
    HostBuf<double> h_p0v, h_st;
    DCsr AP0, AP;
    DCsr fRA, fAP, fQ, fW, fAt;         // fused transfers: R A, A P, the merged operators, A^T
    DevBuf<double> fW1;                 // second value array of fW
    DevBuf<int> fcnt;
};

}  // namespace cfa

struct cfa_amg {
    cfa::SetupScratch scratch;
    cfa_amg_opts opts{};
    std::vector<cfa::AmgLevel> levels;   // levels with a prolongator (reference: levels)
    int coarse_n = 0;
    cfa::DevBuf<double> coarse_inv;      // dense inverse of the coarsest operator, row-major
    cfa::DevBuf<double> cb64, cx64;      // coarsest right-hand side / solution (FP64)
    cfa::DevBuf<float> cb32, cx32;
    double setup_ms = 0.0;
    int remaps = 0;                      // remap() calls that reused the hierarchy
    long long version = 0;               // process-unique, renewed by every setup (graph caches key on it)
    std::vector<double> host_x0;         // 1 + 0.1 sin(1 + i), the power-iteration start vector
    cfa::DevBuf<double> x0;
    bool tiled = false;                  // V-cycle on the tile-streamed kernels
    // accumulated setup phases [ms] (the reference's phase_ms[], src/cfa/linalg.cuh:970-982):
    // 0 copy, 1 D^-1 + rho, 2 strength + aggregation, 3 P smoothing, 4 transpose, 5 Galerkin,
    // 6 tile packing, 7 coarse inverse
    double phase_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // coarse tail: levels >= tail_level run inside one kernel launched as one thread-block cluster
    int tail_level = -1;
    int tail_grid = 0;
    cfa::AmgLevel coarse_holder;         // the coarsest operator (its buffers recycled by the next setup)
    cfa::DevBuf<int> err;                // tile pipeline error word
    // composite: the V-cycle from level comp_level down (its smoothing, transfers and coarse
    // solve) is one linear map of that level's right-hand side, kept as a dense row-major FP64
    // matrix (comp_n x comp_n) and applied as one matrix-vector product; -1: none
    int comp_level = -1;
    int comp_n = 0;
    cfa::DevBuf<double> comp;
    // V-cycle forms chosen for this handle (cfa_amg_set_vcycle); -1: the default / environment
    int vc_composite_rows = -1, vc_fuse = -1, vc_fold_rows = -1;
    // mixed precision: relative residual below which a solve's V-cycles switch from FP64 to FP32
    // (0: FP32 throughout); the FP64 level tiles exist when it is positive. vc_fp64_phase is the
    // value asked for by cfa_amg_set_fp64_phase (-1: CFA_FP64_PHASE or the default)
    double phase_switch = 0.0;
    double vc_fp64_phase = -1.0;
    // aggregation on the device (1) or the host (0); -1: CFA_AGG_HOST or the device
    int vc_agg_device = -1;
};

namespace cfa {
// The condition of a solve graph's WHILE node (use = 0 outside a graph)
struct CondArg {
    cudaGraphConditionalHandle handle;
    int use;
};

__device__ __forceinline__ void set_cond(CondArg c, unsigned v) {
    if (c.use) cudaGraphSetConditional(c.handle, v);
}

// Device-resident state of a CG solve
struct CgState {
    double bnorm, tol, rz, alpha, beta, rel, zero;
    int iter, max_iter, done, converged, status, nullb;
};

// One symmetric V-cycle z = M^-1 r (FP64 in/out). Kernels return at once while *done != 0
// (done nullable).
cfa_status amg_vcycle(cfa_ctx* ctx, cfa_amg* amg, const double* r, double* z, const int* done, bool fp64 = false);

// Mixed precision by phases: a Krylov solve runs its first V-cycles in FP64 on the hierarchy's
// FP64 tiles and switches to the FP32 V-cycle once its relative residual falls below the
// returned threshold (0: no FP64 phase). The FP32 V-cycle's rounding, about 1e-7 of the
// residual it is applied to, enters the CG's search directions; while the residual is large
// those errors are large against the final 1e-10 and cost iterations at the end (67 instead of
// 59 on a 402k-vertex pressure system), but made below about 1e-1 of the initial residual they
// stay below it.
double amg_fp64_phase(const cfa_amg* amg);

// The CG's dots after the preconditioner (r.z, and z.q for the flexible beta) folded into the
// V-cycle's last sweep, which already reads r and writes z; its last block finishes them as the
// CG's own kernel would: beta = flexible ? -alpha (z.q) / rz_old : (r.z) / rz_old, rz = r.z.
struct RzFuse {
    const double* q;
    int flexible;
    double* rz;
    double* beta;
    const double* alpha;
    double* part;
    unsigned int* counter;
};
// The CG's update before the preconditioner (x += alpha pn, r -= alpha q, p = pn, |r| and the
// stopping test) folded into the V-cycle's level-0 kernels: the pre-smoothing sweep gathers
// r - alpha q for its right-hand side, the residual pass (which reads only its own rows) writes
// the new r, x and p and finishes |r| as the CG's update kernel would.
struct CgFuse {
    double* r;
    const double* q;
    const double* pn;
    double* x;
    double* p;
    CgState* st;
    double* part;
    unsigned int* counter;
    CondArg cond;
};
// Whether amg_vcycle_rz takes the CG's update (CFA_CG_FUSE_UPDATE=1, a tile-streamed hierarchy
// with two smoothing steps and level 0's residual pass unfused).
bool amg_can_fuse_update(const cfa_amg* amg);
// The level-0 pre-smoothing's scaling: its first iterate is c = omega0 D0^-1 r in the V-cycle's
// level-0 vector type (fp32: float), which a caller that writes r anyway can form (dinv, omega)
// so that the pre-smoothing gathers c alone. False where the V-cycle does not take c (not
// tile-streamed, fewer than two smoothing steps, or CFA_PRESCALE=0).
struct PreScale {
    const void* dinv;
    double omega;
    int fp32;
};
bool amg_prescale(const cfa_amg* amg, PreScale* out, bool fp64 = false);
// amg_vcycle with the dots fused when the hierarchy runs tile-streamed (*fused = true); otherwise
// the plain V-cycle (*fused = false) and the caller computes the dots. cg (nullable; only where
// amg_can_fuse_update) folds the CG's update into level 0; c (nullable; only where amg_prescale)
// is omega0 D0^-1 r, formed by the caller.
cfa_status amg_vcycle_rz(cfa_ctx* ctx, cfa_amg* amg, const double* r, double* z, const int* done, const RzFuse& f,
                         bool* fused, const CgFuse* cg = nullptr, const void* c = nullptr, bool fp64 = false);
}  // namespace cfa
