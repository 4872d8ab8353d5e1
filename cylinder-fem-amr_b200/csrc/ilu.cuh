// Multicolour ILU(0) handle (MulticolourIlu0, src/cfa/linalg.cuh:435-568).
#pragma once

#include <vector>

#include "internal.cuh"

struct cfa_ilu {
    int n = 0, nnz = 0, nc = 0, nl = 0, nu = 0;
    long long uid = 0;
    cfa_precision precision = CFA_FP64;
    const int* rp = nullptr;          // device pattern (the handle's copy below)
    const int* ci = nullptr;
    cfa::DevBuf<int> own_rp, own_ci;
    std::vector<int> colour_start;    // host, nc + 1
    cfa::DevBuf<int> rows, colour, diag, lp, up, lc, uc, l_src, u_src, d_src;
    cfa::DevBuf<double> lu;           // FP64 factor on the CSR pattern
    cfa::DevBuf<double> lv64, uv64, dinv64;
    cfa::DevBuf<float> lv32, uv32, dinv32;
    cfa::DevBuf<float> work32;        // FP32 sweep work vector of the interleaved pair (mixed), 2 n
    cfa::DevBuf<double> work64;       // FP64 work vector of the colour-order pair sweeps, 2 n
    cfa::DevBuf<int> pos, lcp, ucp;   // colour position of each row; lc / uc as colour positions
    // symbolic factorization (elimination program), rows in colour order:
    // elim[ep[t] .. ep[t+1]) = {local index q of l_ik in row i, CSR position of u_kk, first update},
    // upd[elim.ub .. next.ub) = {local index b in row i, CSR position m in row k}: a_ib -= l_ik lu_m
    cfa::DevBuf<int> ep;              // [n + 1]
    cfa::DevBuf<int4> elim;           // {q, dk, ub, 0}
    cfa::DevBuf<int2> upd;            // {b, m}
    int n_elim = 0, n_upd = 0;
    cfa::DevBuf<int> tpos;            // CSR position of the mirrored entry (j, i) of every (i, j)
    bool mirror = false;              // tpos holds the current pattern's mirror positions
    bool transposed = false;          // the split factor holds (LU)^T (cfa_ilu_factor_transposed)
};

namespace cfa {
// z = (LU)^-1 r, nrhs in {1, 2} vectors of stride n. FP64 in/out; internal precision of the
// handle. `done` (nullable): device flag, the sweep kernels return at once when it is set and
// `active` (nullable, 2 ints) masks components (inactive: z left unchanged).
cfa_status ilu_apply(cfa_ctx* ctx, const cfa_ilu* ilu, const double* r, double* z, int nrhs, const int* done);
// z = (LU)^-1 r for the two components of the momentum solve stored interleaved per row
// (r[2i], r[2i + 1] = u_i, v_i; 16-byte aligned): FP64 handles sweep in FP64 in place in z, mixed
// handles sweep in FP32 on the handle's FP32 work vector. FP64 in and out.
// staged: the apply's first pass (the right-hand side into the colour-order work vector) was done
// by the kernel that produced r, as ilu_pair_staging describes.
cfa_status ilu_apply_pair(cfa_ctx* ctx, const cfa_ilu* ilu, const double* r, double* z, const int* done,
                          bool staged = false);
// The colour-order work vector of the pair apply, for a kernel that produces the apply's
// right-hand side and can also write it there: w[pos[i]] = row i's pair in the work precision
// (fp32: float2, else double2). False where the apply has no such pass (natural row order, one
// colour) or CFA_ILU_STAGED=0.
struct IluStaging {
    const int* pos;
    void* w;
    int fp32;
};
bool ilu_pair_staging(const cfa_ilu* ilu, IluStaging* out);
}  // namespace cfa
