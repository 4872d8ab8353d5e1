// SA-AMG on the GPU.
//
// Setup (AmgPreconditioner::setup, src/cfa/linalg.cuh:995-1060): every FP64 operation of the
// reference's host setup is reproduced in the same order with explicitly rounded multiplies and
// adds (no fused multiply-add), so the hierarchy -- aggregates, P, R, Galerkin operators, omega,
// coarse inverse -- is bit-identical to the reference's:
//   * D^-1, strength of connection, P smoothing, transposes: one thread per row on the GPU;
//   * the power iteration for rho(D^-1 A) with the reference's fixed 4096-row chunk sums;
//   * the Galerkin products with an exact-order row SpGEMM (csr_multiply, :797-845): per row,
//     products are accumulated in A's row order then B's row order into a sorted list;
//   * the coarsest dense Cholesky inverse in one CTA / one thread per column (:1394-1431);
//   * the greedy aggregation (:1321-1348), whose phases 1 and 3 are sequential in node order,
//     runs on the host over the strength flags computed on the GPU.
// V-cycle (vcycle, :1184-1206): symmetric V(s,s) with damped Jacobi, thread groups of TPR lanes
// per row; the first pre-smoothing step is fused with the x = omega D^-1 b initialisation; FP64
// or FP32 hierarchy (mixed precision: FP32 values and vectors, FP64 coarsest solve).
#include <cub/cub.cuh>

#include <algorithm>
#include <functional>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <type_traits>

#include "amg.cuh"

namespace cfa {

// =============================================================================================
// setup kernels (FP64, reference operation order)
// =============================================================================================
__global__ void k_amg_dinv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                           double* __restrict__ dinv) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    for (int a = rp[i]; a < rp[i + 1]; ++a) if (ci[a] == i) d = v[a];
    dinv[i] = (fabs(d) > 1.0e-300) ? __ddiv_rn(1.0, d) : 1.0;
}

// power iteration pieces (spectral_radius_DinvA, :1276-1304)
__global__ void k_pow_y(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                        const double* __restrict__ dinv, const double* __restrict__ x, double* __restrict__ y) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int a = rp[i]; a < rp[i + 1]; ++a) s = __dadd_rn(s, __dmul_rn(v[a], x[ci[a]]));
    y[i] = __dmul_rn(dinv[i], s);
}

// One block per chunk of kPowChunk rows: the chunk's x and y are staged in shared memory by the
// whole block (coalesced), then two threads of different warps run the two sums, each strictly
// in row order as the reference's per-chunk loop does.
constexpr int kPowChunk = 4096;
constexpr int kPowThreads = 256;

__global__ void __launch_bounds__(kPowThreads)
k_pow_chunks(int n, int nch, const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ py,
             double* __restrict__ px) {
    CFA_GRID_DEP();
    extern __shared__ double pow_sm[];   // [2 * kPowChunk]: y then x
    const int c = blockIdx.x;
    if (c >= nch) return;
    const int b = c * kPowChunk, m = min(n, b + kPowChunk) - b;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        pow_sm[i] = y[b + i];
        pow_sm[kPowChunk + i] = x[b + i];
    }
    __syncthreads();
    if (threadIdx.x == 0 || threadIdx.x == 32) {
        const double* v = pow_sm + (threadIdx.x == 0 ? 0 : kPowChunk);
        double acc = 0.0;
#pragma unroll 8
        for (int i = 0; i < m; ++i) acc = __dadd_rn(acc, __dmul_rn(v[i], v[i]));
        if (threadIdx.x == 0) py[c] = acc;
        else px[c] = acc;
    }
}

__global__ void k_pow_finish(int nch, const double* __restrict__ py, const double* __restrict__ px, double* __restrict__ st) {
    CFA_GRID_DEP();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double nrm = 0.0, xn = 0.0;
    for (int c = 0; c < nch; ++c) { nrm = __dadd_rn(nrm, py[c]); xn = __dadd_rn(xn, px[c]); }
    nrm = __dsqrt_rn(nrm);
    st[0] = nrm;
    st[1] = __ddiv_rn(nrm, __dsqrt_rn(xn));
}

__global__ void k_pow_scale(int n, const double* __restrict__ y, const double* __restrict__ st, double* __restrict__ x) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = __ddiv_rn(y[i], st[0]);
}

// strong connections (smoothed_prolongator, :1310-1319)
__global__ void k_strength(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                           const double* __restrict__ dinv, double theta, unsigned char* __restrict__ strong) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double di = __ddiv_rn(1.0, dinv[i]);
    for (int a = rp[i]; a < rp[i + 1]; ++a) {
        const int j = ci[a];
        const double dj = __ddiv_rn(1.0, dinv[j]);
        strong[a] = (j != i) && fabs(v[a]) >= __dmul_rn(theta, __dsqrt_rn(fabs(__dmul_rn(di, dj))));
    }
}

// exact-order SpGEMM (csr_multiply): upper bounds, sorted accumulation, copy
__global__ void k_sg_ub(int rows, const int* __restrict__ arp, const int* __restrict__ aci, const int* __restrict__ brp,
                        int* __restrict__ ub) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    int s = 0;
    for (int a = arp[i]; a < arp[i + 1]; ++a) s += brp[aci[a] + 1] - brp[aci[a]];
    ub[i] = s;
}

// Accumulation of C = A B, a warp per row of C: the row's products are generated in order
// (a-major, b-minor) into shared memory, the first occurrence of every column is marked, each lane
// then sums one column's products in product order (first touch 0.0 + prod, then += prod: per entry
// the operations and their order of csr_multiply's dense accumulator), and the columns are written
// sorted into the row's slice of the scratch. Rows with more than kSgCap products are left to
// k_sg_accum_big.
constexpr int kSgWarps = 8;
constexpr int kSgCap = 512;

__global__ void __launch_bounds__(kSgWarps * 32)
k_sg_accum_warp(int rows, const int* __restrict__ arp, const int* __restrict__ aci, const double* __restrict__ av,
                const int* __restrict__ brp, const int* __restrict__ bci, const double* __restrict__ bv,
                const long long* __restrict__ off, const int* __restrict__ ub, int* __restrict__ scol,
                double* __restrict__ sval, int* __restrict__ cnt) {
    CFA_GRID_DEP();
    extern __shared__ __align__(16) unsigned char sg_sm[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* pv = reinterpret_cast<double*>(sg_sm) + (size_t)w * kSgCap;
    int* pc = reinterpret_cast<int*>(sg_sm + sizeof(double) * kSgWarps * kSgCap) + (size_t)w * kSgCap;
    int* uq = reinterpret_cast<int*>(sg_sm + (sizeof(double) + sizeof(int)) * kSgWarps * kSgCap) + (size_t)w * kSgCap;
    const int i = blockIdx.x * kSgWarps + w;
    if (i >= rows) return;   // warp-uniform
    int* gcols = scol + off[i];
    double* gvals = sval + off[i];
    const int np = ub[i];
    if (np > kSgCap) return;   // k_sg_accum_big takes the row
    // 1. the products in order
    int base = 0;
    for (int a = arp[i]; a < arp[i + 1]; ++a) {
        const int k = aci[a];
        const double x = av[a];
        const int b0 = brp[k], len = brp[k + 1] - b0;
        for (int q = lane; q < len; q += 32) {
            pc[base + q] = bci[b0 + q];
            pv[base + q] = __dmul_rn(x, bv[b0 + q]);
        }
        base += len;
    }
    __syncwarp();
    // 2. first occurrences, compacted in product order
    int u = 0;
    for (int p0 = 0; p0 < np; p0 += 32) {
        const int p = p0 + lane;
        bool first = false;
        if (p < np) {
            const int c = pc[p];
            first = true;
            for (int q = 0; q < p; ++q)
                if (pc[q] == c) { first = false; break; }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, first);
        if (first) uq[u + __popc(mask & ((1u << lane) - 1u))] = p;
        u += __popc(mask);
    }
    __syncwarp();
    // 3. one column per lane: its products summed in product order; 4. written at its rank
    for (int k0 = 0; k0 < u; k0 += 32) {
        const int k = k0 + lane;
        const bool has = k < u;
        const int p1 = has ? uq[k] : np;
        const int c = has ? pc[p1] : 0;
        double acc = 0.0;
        if (has) {
            acc = __dadd_rn(0.0, pv[p1]);
            for (int p = p1 + 1; p < np; ++p)
                if (pc[p] == c) acc = __dadd_rn(acc, pv[p]);
            int rank = 0;
            for (int q = 0; q < u; ++q) rank += pc[uq[q]] < c;
            gcols[rank] = c;
            gvals[rank] = acc;
        }
    }
    if (lane == 0) cnt[i] = u;
}

// The rows of C with more than kSgCap products, a block per row. With C's columns below
// kSgDenseCols: the products are staged in order, kSgChunk at a time, and thread t accumulates the
// columns c with c % blockDim.x == t into a dense accumulator, visiting the products in order (so
// per entry: first touch 0.0 + prod, then += prod in product order); the touched columns are
// written in ascending order. Wider C: thread 0 runs the same arithmetic as a sorted insertion
// into the row's slice.
constexpr int kSgBigThreads = 1024;
constexpr int kSgChunk = 4096;
constexpr int kSgDenseCols = 16384;

__global__ void __launch_bounds__(kSgBigThreads)
k_sg_accum_big(const int* __restrict__ big, int bc, const int* __restrict__ arp, const int* __restrict__ aci,
               const double* __restrict__ av, const int* __restrict__ brp, const int* __restrict__ bci,
               const double* __restrict__ bv, const long long* __restrict__ off, int* __restrict__ scol,
               double* __restrict__ sval, int* __restrict__ cnt) {
    CFA_GRID_DEP();
    extern __shared__ __align__(16) unsigned char sgb_sm[];
    double* acc = reinterpret_cast<double*>(sgb_sm);                                   // [kSgDenseCols]
    double* pv = acc + kSgDenseCols;                                                   // [kSgChunk]
    int* pc = reinterpret_cast<int*>(pv + kSgChunk);                                   // [kSgChunk]
    unsigned* bits = reinterpret_cast<unsigned*>(pc + kSgChunk);                       // [kSgDenseCols / 32]
    int* wpre = reinterpret_cast<int*>(bits + kSgDenseCols / 32);                      // [kSgDenseCols / 32 + 1]
    const int i = big[blockIdx.x];
    int* gcols = scol + off[i];
    double* gvals = sval + off[i];
    if (bc > kSgDenseCols) {
        if (threadIdx.x == 0) {
            int m = 0;
            for (int a = arp[i]; a < arp[i + 1]; ++a) {
                const int k = aci[a];
                const double x = av[a];
                for (int b = brp[k]; b < brp[k + 1]; ++b) {
                    const int j = bci[b];
                    const double prod = __dmul_rn(x, bv[b]);
                    int lo = 0, hi = m;
                    while (lo < hi) { const int mid = (lo + hi) >> 1; if (gcols[mid] < j) lo = mid + 1; else hi = mid; }
                    if (lo < m && gcols[lo] == j) {
                        gvals[lo] = __dadd_rn(gvals[lo], prod);
                    } else {
                        for (int q = m; q > lo; --q) { gcols[q] = gcols[q - 1]; gvals[q] = gvals[q - 1]; }
                        gcols[lo] = j;
                        gvals[lo] = __dadd_rn(0.0, prod);
                        ++m;
                    }
                }
            }
            cnt[i] = m;
        }
        return;
    }
    const int nw = (bc + 31) / 32;
    for (int w = threadIdx.x; w < nw; w += blockDim.x) bits[w] = 0u;
    __syncthreads();
    // this thread's columns, accumulated over one staged chunk of products
    auto process = [&](int np) {
        for (int p = 0; p < np; ++p) {
            const int c = pc[p];
            if (c % kSgBigThreads != (int)threadIdx.x) continue;
            const unsigned bit = 1u << (c & 31);
            if (bits[c >> 5] & bit) {
                acc[c] = __dadd_rn(acc[c], pv[p]);
            } else {
                acc[c] = __dadd_rn(0.0, pv[p]);
                atomicOr(&bits[c >> 5], bit);
            }
        }
    };
    int fill = 0;
    for (int a = arp[i]; a < arp[i + 1]; ++a) {
        const int k = aci[a];
        const double x = av[a];
        int b0 = brp[k];
        const int b1 = brp[k + 1];
        while (b0 < b1) {
            const int take = min(b1 - b0, kSgChunk - fill);
            for (int q = threadIdx.x; q < take; q += blockDim.x) {
                pc[fill + q] = bci[b0 + q];
                pv[fill + q] = __dmul_rn(x, bv[b0 + q]);
            }
            fill += take;
            b0 += take;
            if (fill == kSgChunk) {
                __syncthreads();
                process(fill);
                __syncthreads();
                fill = 0;
            }
        }
    }
    __syncthreads();
    process(fill);
    __syncthreads();
    // touched columns in ascending order: per-word counts, an exclusive scan, then the writes
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < nw; ++w) {
            wpre[w] = run;
            run += __popc(bits[w]);
        }
        wpre[nw] = run;
        cnt[i] = run;
    }
    __syncthreads();
    for (int w = threadIdx.x; w < nw; w += blockDim.x) {
        unsigned m = bits[w];
        int r = wpre[w];
        while (m) {
            const int bpos = __ffs(m) - 1;
            const int c = w * 32 + bpos;
            gcols[r] = c;
            gvals[r] = acc[c];
            ++r;
            m &= m - 1u;
        }
    }
}

__global__ void k_sg_copy(int rows, const long long* __restrict__ off, const int* __restrict__ scol,
                          const double* __restrict__ sval, const int* __restrict__ crp, int* __restrict__ cci,
                          double* __restrict__ cv) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const long long o = off[i];
    const int c0 = crp[i], m = crp[i + 1] - c0;
    for (int q = 0; q < m; ++q) { cci[c0 + q] = scol[o + q]; cv[c0 + q] = sval[o + q]; }
}

// P = P0 - omega D^-1 A P0 from the rows of AP0 (build_row, :1367-1383)
__global__ void k_p_rows(int n, const int* __restrict__ aprp, const int* __restrict__ apci, const double* __restrict__ apv,
                         const int* __restrict__ agg, const double* __restrict__ p0v, const double* __restrict__ dinv,
                         double omega, const int* __restrict__ prp, int* __restrict__ pci, double* __restrict__ pv,
                         int* __restrict__ cnt) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool fill = pci != nullptr;
    int out = 0;
    const int base = fill ? prp[i] : 0;
    bool own = false;
    const int own_col = agg[i];
    const double coef = __dmul_rn(-omega, dinv[i]);
    for (int a = aprp[i]; a < aprp[i + 1]; ++a) {
        const int j = apci[a];
        if (!own && j > own_col) {
            if (fill) { pci[base + out] = own_col; pv[base + out] = p0v[i]; }
            ++out;
            own = true;
        }
        double val = __dmul_rn(coef, apv[a]);
        if (j == own_col) { val = __dadd_rn(val, p0v[i]); own = true; }
        if (val != 0.0) { if (fill) { pci[base + out] = j; pv[base + out] = val; } ++out; }
    }
    if (!own) { if (fill) { pci[base + out] = own_col; pv[base + out] = p0v[i]; } ++out; }
    if (!fill) cnt[i] = out;
}

__global__ void k_entry_rows(int rows, const int* __restrict__ rp, int* __restrict__ row_of) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    for (int a = rp[i]; a < rp[i + 1]; ++a) row_of[a] = i;
}

__global__ void k_iota(int n, int* __restrict__ v) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__global__ void k_ptr_from_sorted(int rows, int m, const int* __restrict__ keys, int* __restrict__ ptr) {
    CFA_GRID_DEP();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > m) return;
    const int cur = t < m ? keys[t] : rows;
    const int prev = t > 0 ? keys[t - 1] : -1;
    for (int i = prev + 1; i <= cur && i <= rows; ++i) ptr[i] = t;
}

__global__ void k_transpose_fill(int m, const int* __restrict__ perm, const int* __restrict__ row_of,
                                 const double* __restrict__ v, int* __restrict__ tci, double* __restrict__ tv) {
    CFA_GRID_DEP();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int e = perm[t];
    tci[t] = row_of[e];
    tv[t] = v[e];
}

__global__ void k_dense_build(int cn, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                              double* __restrict__ D) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cn) return;
    for (int q = 0; q < cn; ++q) D[(size_t)i * cn + q] = 0.0;
    for (int a = rp[i]; a < rp[i + 1]; ++a) D[(size_t)i * cn + ci[a]] = v[a];
}

// Cholesky M = L L^T in place, one CTA (dense_spd_inverse, :1396-1410); err = 1 if not SPD
__global__ void k_cholesky(int cn, double* __restrict__ M, int* __restrict__ err) {
    CFA_GRID_DEP();
    __shared__ double ljj_s;
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int j = 0; j < cn; ++j) {
        if (threadIdx.x == 0) {
            double d = M[(size_t)j * cn + j];
            for (int k = 0; k < j; ++k) d = __dsub_rn(d, __dmul_rn(M[(size_t)j * cn + k], M[(size_t)j * cn + k]));
            if (!(d > 0.0)) { bad = 1; d = 1.0; }
            const double l = __dsqrt_rn(d);
            M[(size_t)j * cn + j] = l;
            ljj_s = l;
        }
        __syncthreads();
        if (bad) break;
        const double ljj = ljj_s;
        for (int i = j + 1 + threadIdx.x; i < cn; i += blockDim.x) {
            double s = M[(size_t)i * cn + j];
            for (int k = 0; k < j; ++k) s = __dsub_rn(s, __dmul_rn(M[(size_t)i * cn + k], M[(size_t)j * cn + k]));
            M[(size_t)i * cn + j] = __ddiv_rn(s, ljj);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *err = bad;
}

// Column c of the inverse from L (:1411-1429)
__global__ void k_chol_inverse(int cn, const double* __restrict__ M, double* __restrict__ inv, double* __restrict__ colbuf) {
    CFA_GRID_DEP();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cn) return;
    double* col = colbuf + (size_t)c * cn;
    for (int i = 0; i < cn; ++i) {
        double s = (i == c) ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k) s = __dsub_rn(s, __dmul_rn(M[(size_t)i * cn + k], col[k]));
        col[i] = __ddiv_rn(s, M[(size_t)i * cn + i]);
    }
    for (int i = cn - 1; i >= 0; --i) {
        double s = col[i];
        for (int k = i + 1; k < cn; ++k) s = __dsub_rn(s, __dmul_rn(M[(size_t)k * cn + i], col[k]));
        col[i] = __ddiv_rn(s, M[(size_t)i * cn + i]);
    }
    for (int i = 0; i < cn; ++i) inv[(size_t)i * cn + c] = col[i];
}

// Blocked form of the same Cholesky (dense_spd_inverse, :1396-1410), one CTA. Every entry still
// receives its terms one at a time in ascending k: s_ij -= L_ik L_jk for k = 0, 1, ..., j-1, then
// L_ij = s_ij / L_jj (the reference sums the same terms in the same order, left-looking); only
// the moment each term is applied changes. Panels of kCholPanel columns are factored in shared
// memory (rows p0.., stride kCholStride); the entries right of a panel then take the panel's terms
// in ascending k, 4x4 entries per thread. L is written to M (row-major) and to Lt (Lt[k cn + i] =
// L_ik, both triangles' roles swapped) for the inverse.
constexpr int kCholPanel = 32;
constexpr int kCholStride = 33;        // padded row stride of the panel (conflict-free columns)
constexpr int kCholThreads = 512;
constexpr int kInvCols = 32;           // columns of the inverse per CTA (one thread each)
constexpr size_t kCoarseSmemMax = 200 * 1024;

inline size_t chol_smem(int cn) { return (size_t)(cn + 4) * kCholStride * sizeof(double); }
// x vectors (cn x kInvCols), two staged rows of Lt and the diagonal of L
inline size_t inv_smem(int cn) { return (size_t)cn * (kInvCols + 3) * sizeof(double); }
inline bool coarse_blocked(int cn) { return chol_smem(cn) <= kCoarseSmemMax && inv_smem(cn) <= kCoarseSmemMax; }

__global__ void __launch_bounds__(kCholThreads) k_coarse_cholesky(int cn, double* __restrict__ M, double* __restrict__ Lt,
                                                                   int* __restrict__ err) {
    CFA_GRID_DEP();
    extern __shared__ double P[];      // (cn + 4) x kCholStride
    __shared__ double piv[kCholPanel];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    int bad = 0;
    for (int p0 = 0; p0 < cn && !bad; p0 += kCholPanel) {
        const int pw = min(kCholPanel, cn - p0);
        const int R = cn - p0;
        // the panel: rows p0..cn-1 of columns p0..p0+pw-1 (+4 zero rows read by the edge tiles)
        for (int r = warp; r < R + 4; r += nwarps)
            if (lane < kCholStride) P[r * kCholStride + lane] = (r < R && lane < pw) ? M[(size_t)(p0 + r) * cn + p0 + lane] : 0.0;
        if (lane == 0)
            for (int r = warp; r < R + 4; r += nwarps) P[r * kCholStride + 32] = 0.0;
        __syncthreads();
        for (int kk = 0; kk < pw; ++kk) {
            // every thread takes the pivot itself (same value, same rounding): no broadcast step;
            // the diagonal entry is not read again, the factor goes to piv[] for the write-back
            const double d = P[kk * kCholStride + kk];
            if (!(d > 0.0)) { bad = 1; break; }
            const double l = __dsqrt_rn(d);
            if (tid == 0) piv[kk] = l;
            for (int r = kk + 1 + tid; r < R; r += blockDim.x)
                P[r * kCholStride + kk] = __ddiv_rn(P[r * kCholStride + kk], l);
            __syncthreads();
            // term k = p0 + kk for the panel's later columns: lane = column, warps stride the rows,
            // four rows loaded before any is stored
            const int c2 = kk + 1 + lane;
            if (c2 < pw) {
                const double lc = P[c2 * kCholStride + kk];
                int r = c2 + warp;
                for (; r + 3 * nwarps < R; r += 4 * nwarps) {
                    double a[4], b[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        a[u] = P[(r + u * nwarps) * kCholStride + c2];
                        b[u] = P[(r + u * nwarps) * kCholStride + kk];
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) P[(r + u * nwarps) * kCholStride + c2] = __dsub_rn(a[u], __dmul_rn(b[u], lc));
                }
                for (; r < R; r += nwarps)
                    P[r * kCholStride + c2] = __dsub_rn(P[r * kCholStride + c2], __dmul_rn(P[r * kCholStride + kk], lc));
            }
            __syncthreads();
        }
        if (bad) break;
        for (int r = warp; r < R; r += nwarps) {
            if (lane < pw && r >= lane) {
                const double v = r == lane ? piv[lane] : P[r * kCholStride + lane];
                M[(size_t)(p0 + r) * cn + p0 + lane] = v;
                Lt[(size_t)(p0 + lane) * cn + p0 + r] = v;
            }
        }
        // the panel's terms for the entries (i, j), i >= j >= q0, in ascending k, 4x4 per thread
        const int q0 = p0 + pw, R2 = cn - q0;
        if (R2 > 0) {
            const int nb = (R2 + 3) / 4;
            const long long T = (long long)nb * (nb + 1) / 2;
            for (long long tt = tid; tt < T; tt += blockDim.x) {
                int bi = (int)((sqrt(8.0 * (double)tt + 1.0) - 1.0) * 0.5);
                while ((long long)bi * (bi + 1) / 2 > tt) --bi;
                while ((long long)(bi + 1) * (bi + 2) / 2 <= tt) ++bi;
                const int bj = (int)(tt - (long long)bi * (bi + 1) / 2);
                const int i0 = q0 + 4 * bi, j0 = q0 + 4 * bj;
                double acc[4][4];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int i = i0 + a, j = j0 + b;
                        acc[a][b] = (i < cn && j <= i) ? M[(size_t)i * cn + j] : 0.0;
                    }
                const double* pi = P + (size_t)(i0 - p0) * kCholStride;
                const double* pj = P + (size_t)(j0 - p0) * kCholStride;
                for (int kk = 0; kk < pw; ++kk) {
                    double li[4], lj[4];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        li[a] = pi[a * kCholStride + kk];
                        lj[a] = pj[a * kCholStride + kk];
                    }
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int b = 0; b < 4; ++b) acc[a][b] = __dsub_rn(acc[a][b], __dmul_rn(li[a], lj[b]));
                }
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int i = i0 + a, j = j0 + b;
                        if (i < cn && j <= i) M[(size_t)i * cn + j] = acc[a][b];
                    }
            }
        }
        __syncthreads();
    }
    if (tid == 0) *err = bad;
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Columns of the inverse from L (:1411-1429), one thread per column c, its vector in shared memory
// (xs[i kInvCols + lane]). L y = e_c column-oriented: y_k = s_k / L_kk, then s_i -= L_ik y_k for
// i > k, so every s_i still takes its terms in ascending k (rows i < c are +0.0 in the reference,
// whose terms with k < c subtract products with +0.0 and change nothing). L^T x = y row-oriented
// with ascending k, as the reference. The row of Lt each step reads is staged in shared memory by
// the warp one step ahead (cp.async), so the per-column chains wait only on shared memory.
__global__ void __launch_bounds__(kInvCols) k_coarse_inverse(int cn, const double* __restrict__ L,
                                                              const double* __restrict__ Lt, double* __restrict__ inv) {
    CFA_GRID_DEP();
    extern __shared__ double sm[];
    double* xs = sm;                                   // cn x kInvCols
    double* rows = sm + (size_t)cn * kInvCols;         // 2 x cn
    double* dg = rows + 2 * (size_t)cn;                // cn
    const int lane = threadIdx.x;
    const int c0 = blockIdx.x * kInvCols;
    const int c = c0 + lane;
    const bool valid = c < cn;
    for (int i = lane; i < cn; i += kInvCols) dg[i] = L[(size_t)i * cn + i];
    for (int i = 0; i < cn; ++i) xs[i * kInvCols + lane] = (i == c) ? 1.0 : 0.0;
    // forward: step k reads Lt[k][k+1 .. cn-1] (= L_ik, i > k)
    auto stage_fwd = [&](int k, int buf) {
        const double* src = Lt + (size_t)k * cn + k + 1;
        double* dst = rows + (size_t)buf * cn;
        for (int j = lane; j < cn - k - 1; j += kInvCols) cp_async8(dst + j, src + j);
        cp_async_commit();
    };
    if (c0 < cn) stage_fwd(c0, 0);
    for (int k = c0; k < cn; ++k) {
        const int buf = (k - c0) & 1;
        cp_async_wait_all();
        __syncwarp();
        if (k + 1 < cn) stage_fwd(k + 1, buf ^ 1);
        if (valid && k >= c) {
            const double y = __ddiv_rn(xs[k * kInvCols + lane], dg[k]);
            xs[k * kInvCols + lane] = y;
            const double* lk = rows + (size_t)buf * cn;   // lk[j] = L_ik, i = k + 1 + j
            int i = k + 1;
            for (; i + 8 <= cn; i += 8) {   // eight rows loaded before any is stored
                double xv[8], lv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    xv[u] = xs[(i + u) * kInvCols + lane];
                    lv[u] = lk[i + u - k - 1];
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) xs[(i + u) * kInvCols + lane] = __dsub_rn(xv[u], __dmul_rn(lv[u], y));
            }
            for (; i < cn; ++i)
                xs[i * kInvCols + lane] = __dsub_rn(xs[i * kInvCols + lane], __dmul_rn(lk[i - k - 1], y));
        }
        __syncwarp();
    }
    cp_async_wait_all();
    __syncwarp();
    // backward: row i reads Lt[i][i+1 .. cn-1] (= L_ki, k > i)
    stage_fwd(cn - 1, 0);
    for (int i = cn - 1; i >= 0; --i) {
        const int buf = (cn - 1 - i) & 1;
        cp_async_wait_all();
        __syncwarp();
        if (i > 0) stage_fwd(i - 1, buf ^ 1);
        const double* li = rows + (size_t)buf * cn;       // li[j] = L_ki, k = i + 1 + j
        double s = xs[i * kInvCols + lane];
        // the products do not depend on s: those of the next eight terms are formed while the
        // chain of subtractions runs through the current eight (a +0.0 pad leaves s unchanged)
        double cur[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int k = i + 1 + u;
            cur[u] = k < cn ? __dmul_rn(li[k - i - 1], xs[k * kInvCols + lane]) : 0.0;
        }
        for (int k0 = i + 1; k0 < cn; k0 += 8) {
            double nxt[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int k = k0 + 8 + u;
                nxt[u] = k < cn ? __dmul_rn(li[k - i - 1], xs[k * kInvCols + lane]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) s = __dsub_rn(s, cur[u]);
#pragma unroll
            for (int u = 0; u < 8; ++u) cur[u] = nxt[u];
        }
        xs[i * kInvCols + lane] = __ddiv_rn(s, dg[i]);
        __syncwarp();
    }
    if (valid)
        for (int i = 0; i < cn; ++i) inv[(size_t)i * cn + c] = xs[i * kInvCols + lane];
}

__global__ void k_to_float(long long n, const double* __restrict__ a, float* __restrict__ b) {
    CFA_GRID_DEP();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// =============================================================================================
// V-cycle kernels. Thread groups of TPR lanes per row, warp-uniform loops, the lane-strided
// sum and shuffle tree of the reference's k_csr_op (:885-901).
// =============================================================================================
template <int TPR, class T, class X>
__device__ __forceinline__ T group_row_sum(const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                                           const X* __restrict__ x, int row, bool valid, int lane) {
    T s = (T)0;
    if (valid)
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) s += val[k] * (T)x[ci[k]];
#pragma unroll
    for (int o = TPR / 2; o > 0; o /= 2) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    return s;
}

#define ROW_LOOP_BEGIN(TPR, n)                                                                    \
    const int lane_ = threadIdx.x % (TPR);                                                        \
    const int gw_ = (blockIdx.x * blockDim.x + threadIdx.x) / 32;                                 \
    const int nw_ = gridDim.x * blockDim.x / 32;                                                  \
    constexpr int rpw_ = 32 / (TPR);                                                              \
    for (int base_ = gw_ * rpw_; base_ < (n); base_ += nw_ * rpw_) {                              \
        const int row = base_ + (threadIdx.x & 31) / (TPR);                                       \
        const bool valid = row < (n);                                                             \
        const int lane = lane_;

#define ROW_LOOP_END }

// x = omega D^-1 b, then (fused) one Jacobi step x <- x + omega D^-1 (b - A x) when `jac`
template <int TPR, class T, class B>
__global__ void k_vc_pre(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                         const T* __restrict__ dinv, T omega, const B* __restrict__ b, int jac, T* __restrict__ xo,
                         const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    ROW_LOOP_BEGIN(TPR, n)
    if (!jac) {
        if (valid && lane == 0) xo[row] = omega * dinv[row] * (T)b[row];
        continue;
    }
    T s = (T)0;
    if (valid)
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
            const int j = ci[k];
            s += val[k] * (omega * dinv[j] * (T)b[j]);
        }
#pragma unroll
    for (int o = TPR / 2; o > 0; o /= 2) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (valid && lane == 0) {
        const T x0 = omega * dinv[row] * (T)b[row];
        xo[row] = x0 + omega * dinv[row] * ((T)b[row] - s);
    }
    ROW_LOOP_END
}

// y = x + omega D^-1 (b - A x); O = output type (FP64 z at the end of level 0)
template <int TPR, class T, class B, class O>
__global__ void k_vc_jacobi(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                            const T* __restrict__ dinv, T omega, const B* __restrict__ b, const T* __restrict__ x,
                            O* __restrict__ y, const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    ROW_LOOP_BEGIN(TPR, n)
    const T s = group_row_sum<TPR, T, T>(rp, ci, val, x, row, valid, lane);
    if (valid && lane == 0) y[row] = (O)(x[row] + omega * dinv[row] * ((T)b[row] - s));
    ROW_LOOP_END
}

// r = b - A x
template <int TPR, class T, class B>
__global__ void k_vc_resid(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                           const B* __restrict__ b, const T* __restrict__ x, T* __restrict__ r, const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    ROW_LOOP_BEGIN(TPR, n)
    const T s = group_row_sum<TPR, T, T>(rp, ci, val, x, row, valid, lane);
    if (valid && lane == 0) r[row] = (T)b[row] - s;
    ROW_LOOP_END
}

// y = M x (add = 0) or y += M x (add = 1); Y output type
template <int TPR, class T, class Y>
__global__ void k_vc_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                          const T* __restrict__ x, int add, Y* __restrict__ y, const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    ROW_LOOP_BEGIN(TPR, n)
    const T s = group_row_sum<TPR, T, T>(rp, ci, val, x, row, valid, lane);
    if (valid && lane == 0) y[row] = add ? (Y)((T)y[row] + s) : (Y)s;
    ROW_LOOP_END
}

// x = M b with a dense row-major FP64 matrix (the coarsest inverse, k_dense_matvec, :929-937, or
// the composite operator): one block of kDenseWarps warps per row, warp w taking the columns
// [w cn / kDenseWarps, (w + 1) cn / kDenseWarps) with eight loads of each lane issued before they
// are summed; the warps' partial sums are added in warp order. Four warps per row put four
// times the loads in flight that one warp per row would (a 1069-row matrix is 1069 rows of
// 8.5 KB: one warp per row leaves each SM eight warps).
constexpr int kDenseWarps = 4;

template <class B, class X>
__global__ void __launch_bounds__(32 * kDenseWarps)
k_vc_dense(int cn, const double* __restrict__ inv, const B* __restrict__ b, X* __restrict__ x,
           const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    __shared__ double part[kDenseWarps];
    const int i = blockIdx.x, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (i >= cn) return;
    const double* m = inv + (size_t)i * cn;
    const int c0 = (int)((long long)cn * w / kDenseWarps), c1 = (int)((long long)cn * (w + 1) / kDenseWarps);
    constexpr int U = 8;
    double acc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) acc[u] = 0.0;
    int j = c0 + lane;
    for (; j + 32 * (U - 1) < c1; j += 32 * U) {
        double a[U], g[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            a[u] = __ldg(m + j + 32 * u);
            g[u] = (double)b[j + 32 * u];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) acc[u] += a[u] * g[u];
    }
    for (; j < c1; j += 32) acc[0] += m[j] * (double)b[j];
    double s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    s = warp_sum(s);
    if (lane == 0) part[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = part[0];
        for (int k = 1; k < kDenseWarps; ++k) t += part[k];
        x[i] = (X)t;
    }
}

// ---------------------------------------------------------------------------------------------
// Composite coarse operator. The V-cycle below a small level is linear in that level's
// right-hand side (damped Jacobi from a zero start, residual, restriction, the coarse solve,
// prolongation), so it is one dense matrix M with M b = V-cycle(b). Setup forms M by running the
// V-cycle's row operations on a block of right-hand sides (the identity); the V-cycle then applies
// it with k_vc_dense, one launch in place of the levels' chain of dependent launches (about
// seven per level). M equals the chain up to rounding (the products are summed in another order).
// Blocks are row-major m x nb (row i, column c at [i * nb + c]), one thread per entry.
// ---------------------------------------------------------------------------------------------
enum BmOp { BM_PRE = 0, BM_JAC = 1, BM_RES = 2, BM_SPMV = 3, BM_ADD = 4 };

template <int OP>
__global__ void k_bm(int m, int nb, const int* __restrict__ rp, const int* __restrict__ ci,
                     const double* __restrict__ val, const double* __restrict__ dinv, double omega, int jac,
                     const double* __restrict__ B, const double* __restrict__ X, double* __restrict__ Y) {
    CFA_GRID_DEP();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)m * nb) return;
    const int i = (int)(idx / nb), c = (int)(idx % nb);
    double s = 0.0;
    if (OP != BM_PRE || jac)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            s += val[k] * (OP == BM_PRE ? omega * dinv[j] * B[(size_t)j * nb + c] : X[(size_t)j * nb + c]);
        }
    const size_t o = (size_t)i * nb + c;
    if (OP == BM_PRE) {
        const double x0 = omega * dinv[i] * B[o];
        Y[o] = jac ? x0 + omega * dinv[i] * (B[o] - s) : x0;
    } else if (OP == BM_JAC) {
        Y[o] = X[o] + omega * dinv[i] * (B[o] - s);
    } else if (OP == BM_RES) {
        Y[o] = B[o] - s;
    } else if (OP == BM_SPMV) {
        Y[o] = s;
    } else {
        Y[o] += s;
    }
}

// X = inv B with the dense coarse inverse (cn x cn), blocks cn x nb
__global__ void k_bm_dense(int cn, int nb, const double* __restrict__ inv, const double* __restrict__ B,
                           double* __restrict__ X) {
    CFA_GRID_DEP();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)cn * nb) return;
    const int i = (int)(idx / nb), c = (int)(idx % nb);
    double s = 0.0;
    for (int j = 0; j < cn; ++j) s += inv[(size_t)i * cn + j] * B[(size_t)j * nb + c];
    X[(size_t)i * nb + c] = s;
}

// B = identity (nb x nb)
__global__ void k_bm_eye(int nb, double* __restrict__ B) {
    CFA_GRID_DEP();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nb * nb) return;
    B[idx] = (idx / nb == idx % nb) ? 1.0 : 0.0;
}

// ---------------------------------------------------------------------------------------------
// tile-streamed V-cycle kernel (tiled.cuh): one kernel for the five row operations
// ---------------------------------------------------------------------------------------------
// VC_RESTRICT (fused transfers): y = [R | -R A] [b ; x] over the next level's rows;
// VC_ADDJAC: with x' = x + P xc, y = x' + omega D^-1 (b - A x'), x' never stored: sums of
// [A | A P] and [I | P] over [x ; xc]. A column with the top bit set reads the second vector.
// Explicitly rounded product and fused multiply-add, so that two kernels which form the same
// value in different places round it the same way whatever the compiler contracts.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// VC_PREC: VC_PRE with its first iterate c = omega D^-1 b given (x = c, formed by the caller).
enum VcOp { VC_PRE = 0, VC_JAC = 1, VC_RES = 2, VC_SPMV = 3, VC_ADD = 4, VC_RESTRICT = 5, VC_ADDJAC = 6, VC_PREC = 7 };
constexpr int kSecondVec = (int)0x80000000u;

template <int TPR, int OP, class V, class T, class B, class O, bool RZ = false, bool CGU = false>
__global__ void __launch_bounds__(kTileThreads)
k_vct(TileView tv, const T* __restrict__ dinv, T omega, const B* __restrict__ b, const T* __restrict__ x,
      O* __restrict__ y, const int* __restrict__ done, RzFuse rzf, const T* __restrict__ xc, CgFuse cgf) {
    extern __shared__ __align__(128) unsigned char tsmem[];
    double dots[2] = {0.0, 0.0};   // RZ: this thread's rows of r.z and z.q; CGU (residual): of |r|^2
    // gathers issued together per lane: with four or more lanes the Galerkin levels' rows carry
    // five or six entries per lane, so a batch of eight issues a third of its slots predicated
    // off; the entries are summed in the same order whatever the batch
    constexpr int kVcBatch = TPR >= 4 ? 6 : kGatherBatch;
    // the level's tiles are packed at setup: their first copies go out before the wait
    const bool go = tile_loop_dep(tv, tsmem, [&] { return !(done && *done); },
                                  [&](int, int r0, int nr, const unsigned char* ch) {
        const int* rr = reinterpret_cast<const int*>(ch);
        const int ne = rr[nr];
        const int* cs = reinterpret_cast<const int*>(ch + tile_ci_off(nr));
        const V* vv = reinterpret_cast<const V*>(ch + tile_val_off(nr, ne, (int)sizeof(V), 0));
        const V* vv1 = reinterpret_cast<const V*>(ch + tile_val_off(nr, ne, (int)sizeof(V), 1));
        for (int base = 0; base < nr; base += kTileThreads / TPR) {
            const int lr = base + (int)threadIdx.x / TPR, lane = threadIdx.x % TPR;
            const bool valid = lr < nr;
            const int row = r0 + lr;
            // the row's own operands, loaded before the gathers so both round trips overlap
            T di = (T)0, bi = (T)0, xi = (T)0;
            // CGU: the right-hand side is the CG residual after this iteration's update,
            // r - alpha q, formed here as the CG's update kernel forms it
            const double alpha = CGU ? cgf.st->alpha : 0.0;
            double rn = 0.0;
            if (valid && lane == 0) {
                if (OP == VC_PRE || OP == VC_PREC || OP == VC_JAC || OP == VC_ADDJAC) di = dinv[row];
                if (OP == VC_PREC) xi = x[row];
                if (CGU) {
                    rn = (double)b[row] + -alpha * cgf.q[row];
                    bi = (T)rn;
                } else if (OP == VC_PRE || OP == VC_PREC || OP == VC_JAC || OP == VC_RES || OP == VC_ADDJAC) {
                    bi = (T)b[row];
                }
                if (OP == VC_JAC) xi = x[row];
                if (OP == VC_ADD) xi = (T)y[row];
            }
            T s = (T)0, s1 = (T)0;
            if (valid) {
                const int end = rr[lr + 1];
                for (int e0 = rr[lr] + lane; e0 < end; e0 += kVcBatch * TPR) {
                    // all loads of the batch first, then the sums in entry order
                    V a[kVcBatch], a1[kVcBatch];
                    T g0[kVcBatch];
                    B g1[kVcBatch];
#pragma unroll
                    for (int u = 0; u < kVcBatch; ++u) {
                        const int e = e0 + u * TPR;
                        if (e < end) {
                            const int j = cs[e];
                            a[u] = vv[e];
                            if (OP == VC_PRE) {
                                g0[u] = dinv[j];
                                if (CGU) g1[u] = (B)((double)b[j] + -alpha * cgf.q[j]);
                                else g1[u] = b[j];
                            }
                            else if (OP == VC_RESTRICT) g0[u] = j < 0 ? x[j & ~kSecondVec] : (T)b[j];
                            else if (OP == VC_ADDJAC) { g0[u] = j < 0 ? xc[j & ~kSecondVec] : x[j]; a1[u] = vv1[e]; }
                            else g0[u] = x[j];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kVcBatch; ++u)
                        if (e0 + u * TPR < end) {
                            if (OP == VC_PRE) s += (T)a[u] * mul_rn(omega * g0[u], (T)g1[u]);
                            else s += (T)a[u] * g0[u];
                            if (OP == VC_ADDJAC) s1 += (T)a1[u] * g0[u];
                        }
                }
            }
#pragma unroll
            for (int o = TPR / 2; o > 0; o /= 2) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
            if (OP == VC_ADDJAC) {
#pragma unroll
                for (int o = TPR / 2; o > 0; o /= 2) s1 += __shfl_down_sync(0xffffffffu, s1, o, TPR);
            }
            if (valid && lane == 0) {
                if (OP == VC_PRE) {
                    // rounded product, then one fused multiply-add: the same operations as the
                    // pre-scaled form, whose first iterate the caller stored
                    const T od = omega * di;
                    y[row] = (O)fma_rn(od, bi - s, mul_rn(od, bi));
                } else if (OP == VC_PREC) {
                    y[row] = (O)fma_rn(omega * di, bi - s, xi);
                } else if (OP == VC_JAC) {
                    const O out = (O)(xi + omega * di * (bi - s));
                    y[row] = out;
                    if constexpr (RZ) {
                        const double zr = (double)out;
                        dots[0] += (double)b[row] * zr;
                        if (rzf.flexible) dots[1] += zr * rzf.q[row];
                    }
                } else if (OP == VC_RES) {
                    y[row] = (O)(bi - s);
                    if constexpr (CGU) {   // the CG's update of this row (k_cg_update)
                        const double pi = cgf.pn[row];
                        cgf.x[row] += alpha * pi;
                        cgf.r[row] = rn;
                        cgf.p[row] = pi;
                        dots[0] += rn * rn;
                    }
                } else if (OP == VC_SPMV || OP == VC_RESTRICT) {
                    y[row] = (O)s;
                } else if (OP == VC_ADDJAC) {
                    y[row] = (O)(s1 + omega * di * (bi - s));
                } else {
                    y[row] = (O)(xi + s);
                }
            }
        }
    });
    if (!go) return;
    if constexpr (CGU && OP == VC_RES) {
        // |r| and the stopping test of the CG's update kernel (solve_pcg, src/cfa/linalg.cuh:239-246)
        __shared__ double sh[2 * kWarps];
        block_sum<2>(dots, sh);
        if (publish_partials<2>(dots, cgf.part, cgf.counter)) {
            reduce_partials<2>(dots, cgf.part, cgf.counter, sh);
            if (threadIdx.x == 0) {
                CgState* st = cgf.st;
                const double rnorm = sqrt(dots[0]);
                st->rel = rnorm / st->bnorm;
                const int it = st->iter + 1;
                st->iter = it;
                if (rnorm < st->tol * st->bnorm) {
                    st->done = 1;
                    st->converged = 1;
                    set_cond(cgf.cond, 0);
                } else if (it >= st->max_iter) {
                    st->done = 1;
                    st->converged = 0;
                    st->status = CFA_NOT_CONVERGED;
                    set_cond(cgf.cond, 0);
                }
            }
        }
    }
    if constexpr (RZ) {
        __shared__ double sh[2 * kWarps];
        block_sum<2>(dots, sh);
        if (publish_partials<2>(dots, rzf.part, rzf.counter)) {
            reduce_partials<2>(dots, rzf.part, rzf.counter, sh);
            if (threadIdx.x == 0) {
                const double rz_old = *rzf.rz;
                *rzf.beta = rzf.flexible ? -(*rzf.alpha) * dots[1] / (rz_old + 1.0e-30) : dots[0] / (rz_old + 1.0e-30);
                *rzf.rz = dots[0];
            }
        }
    }
}

// Launches (or, dry, only prepares) one tiled V-cycle operation; values of type V in the tiles.
// rz: fold the CG's dots into this launch (the level-0 last sweep only).
template <int OP, class V, class T, class B, class O>
static void vct(cfa_ctx* ctx, bool dry, const TiledCsr& M, int* err, const T* dinv, T omega, const B* b, const T* x,
                O* y, const int* done, const RzFuse* rz = nullptr, const T* xc = nullptr, const CgFuse* cg = nullptr) {
    constexpr bool kRz = OP == VC_JAC && std::is_same<O, double>::value && std::is_same<B, double>::value;
    constexpr bool kCgu = (OP == VC_PRE || OP == VC_RES) && std::is_same<B, double>::value;
    const int tpr = M.tpr;
    TileView tv = M.view(err);
    tv.l2hint = l2_hint_vcycle();
    const RzFuse none{};
    const CgFuse nocg{};
    switch (tpr) {
#define VCT_CASE(N)                                                                                     \
    case N:                                                                                             \
        if (dry) {                                                                                      \
            allow_tile_kernel((const void*)k_vct<N, OP, V, T, B, O>);                                   \
            if (kRz) allow_tile_kernel((const void*)k_vct<N, OP, V, T, B, O, kRz>);                     \
            if (kCgu) allow_tile_kernel((const void*)k_vct<N, OP, V, T, B, O, false, kCgu>);            \
        } else if (kRz && rz) {                                                                         \
            const TileLaunch L = tile_launch(ctx, M, (const void*)k_vct<N, OP, V, T, B, O, kRz>);       \
            CFA_LAUNCH(ctx, (k_vct<N, OP, V, T, B, O, kRz>), L.grid, kTileThreads, L.smem, tv, dinv, omega, b, x, y, \
                       done, *rz, xc, nocg);                                                            \
        } else if (kCgu && cg) {                                                                        \
            const TileLaunch L = tile_launch(ctx, M, (const void*)k_vct<N, OP, V, T, B, O, false, kCgu>); \
            CFA_LAUNCH(ctx, (k_vct<N, OP, V, T, B, O, false, kCgu>), L.grid, kTileThreads, L.smem, tv, dinv, omega, \
                       b, x, y, done, none, xc, *cg);                                                   \
        } else {                                                                                        \
            const TileLaunch L = tile_launch(ctx, M, (const void*)k_vct<N, OP, V, T, B, O>);            \
            CFA_LAUNCH(ctx, (k_vct<N, OP, V, T, B, O>), L.grid, kTileThreads, L.smem, tv, dinv, omega, b, x, y, done, \
                       none, xc, nocg);                                                                 \
        }                                                                                               \
        break;
        VCT_CASE(1) VCT_CASE(2) VCT_CASE(4) VCT_CASE(8) VCT_CASE(16)
        default:
        VCT_CASE(32)
#undef VCT_CASE
    }
}

// ---------------------------------------------------------------------------------------------
// launch helpers with the TPR dispatch
// ---------------------------------------------------------------------------------------------
#define CFA_TPR_SWITCH(tpr, ...)                                                               \
    do {                                                                                       \
        switch (tpr) {                                                                         \
            case 1: { constexpr int TPR = 1; __VA_ARGS__; } break;                              \
            case 2: { constexpr int TPR = 2; __VA_ARGS__; } break;                              \
            case 4: { constexpr int TPR = 4; __VA_ARGS__; } break;                              \
            case 8: { constexpr int TPR = 8; __VA_ARGS__; } break;                              \
            case 16: { constexpr int TPR = 16; __VA_ARGS__; } break;                            \
            default: { constexpr int TPR = 32; __VA_ARGS__; } break;                            \
        }                                                                                      \
    } while (0)

template <class T>
struct LevelView {
    const int *Arp, *Aci, *Prp, *Pci, *Rrp, *Rci;
    const T *Av, *Pv, *Rv, *dinv;
    T *x, *t, *b, *r;
    T omega;
};

template <class T>
static LevelView<T> view(AmgLevel& L);
template <>
LevelView<double> view<double>(AmgLevel& L) {
    return {L.A.rp.p, L.A.ci.p, L.P.rp.p, L.P.ci.p, L.R.rp.p, L.R.ci.p, L.A.v.p, L.P.v.p, L.R.v.p, L.dinv.p,
            L.x64.p, L.t64.p, L.b64.p, L.r64.p, L.omega};
}
template <>
LevelView<float> view<float>(AmgLevel& L) {
    return {L.A.rp.p, L.A.ci.p, L.P.rp.p, L.P.ci.p, L.R.rp.p, L.R.ci.p, L.A.v32.p, L.P.v32.p, L.R.v32.p, L.dinv32.p,
            L.x32.p, L.t32.p, L.b32.p, L.r32.p, (float)L.omega};
}

// V-cycle on level l; b is the level's right-hand side (level 0: caller's FP64 r), the result
// ends in the level's x (level 0: in z).
template <class T, class B>
static void vcycle_level(cfa_ctx* ctx, cfa_amg* amg, int l, const B* b, double* z, const int* done) {
    AmgLevel& L = amg->levels[l];
    LevelView<T> V = view<T>(L);
    const int n = L.A.rows, s = amg->opts.smooth_steps;
    const int tA = L.A.tpr, tP = L.P.tpr, tR = L.R.tpr;
    const int gA = row_grid(ctx, n, tA);
    // pre-smoothing from x = 0
    CFA_TPR_SWITCH(tA, CFA_LAUNCH(ctx, (k_vc_pre<TPR, T, B>), gA, kThreads, 0, n, V.Arp, V.Aci, V.Av, V.dinv, V.omega,
                                  b, s >= 2 ? 1 : 0, V.x, done));
    T* x = V.x;
    T* t = V.t;
    for (int k = 2; k < s; ++k) {
        CFA_TPR_SWITCH(tA, CFA_LAUNCH(ctx, (k_vc_jacobi<TPR, T, B, T>), gA, kThreads, 0, n, V.Arp, V.Aci, V.Av, V.dinv,
                                      V.omega, b, x, t, done));
        std::swap(x, t);
    }
    // restricted residual
    CFA_TPR_SWITCH(tA, CFA_LAUNCH(ctx, (k_vc_resid<TPR, T, B>), gA, kThreads, 0, n, V.Arp, V.Aci, V.Av, b, x, V.r, done));
    const bool last = l + 1 == (int)amg->levels.size();
    const int nc = L.P.cols;
    T* cb = last ? (std::is_same<T, double>::value ? (T*)amg->cb64.p : (T*)amg->cb32.p)
                 : view<T>(amg->levels[l + 1]).b;
    CFA_TPR_SWITCH(tR, CFA_LAUNCH(ctx, (k_vc_spmv<TPR, T, T>), row_grid(ctx, nc, tR), kThreads, 0, nc, V.Rrp, V.Rci,
                                  V.Rv, V.r, 0, cb, done));
    const T* cx;
    if (!last && l + 1 == amg->comp_level) {
        cx = view<T>(amg->levels[l + 1]).x;
        CFA_LAUNCH(ctx, (k_vc_dense<T, T>), amg->comp_n, 32 * kDenseWarps, 0,
                   amg->comp_n, amg->comp.p, (const T*)cb, view<T>(amg->levels[l + 1]).x, done);
    } else if (!last) {
        vcycle_level<T, T>(ctx, amg, l + 1, cb, nullptr, done);
        cx = view<T>(amg->levels[l + 1]).x;
    } else {
        T* dst = std::is_same<T, double>::value ? (T*)amg->cx64.p : (T*)amg->cx32.p;
        CFA_LAUNCH(ctx, (k_vc_dense<T, T>), amg->coarse_n, 32 * kDenseWarps, 0,
                   amg->coarse_n, amg->coarse_inv.p, (const T*)cb, dst, done);
        cx = dst;
    }
    // coarse correction x += P x_c
    CFA_TPR_SWITCH(tP, CFA_LAUNCH(ctx, (k_vc_spmv<TPR, T, T>), row_grid(ctx, n, tP), kThreads, 0, n, V.Prp, V.Pci, V.Pv,
                                  cx, 1, x, done));
    // post-smoothing; the last step of level 0 writes z
    for (int k = 0; k < s; ++k) {
        if (l == 0 && k == s - 1) {
            CFA_TPR_SWITCH(tA, CFA_LAUNCH(ctx, (k_vc_jacobi<TPR, T, B, double>), gA, kThreads, 0, n, V.Arp, V.Aci, V.Av,
                                          V.dinv, V.omega, b, x, z, done));
        } else {
            CFA_TPR_SWITCH(tA, CFA_LAUNCH(ctx, (k_vc_jacobi<TPR, T, B, T>), gA, kThreads, 0, n, V.Arp, V.Aci, V.Av,
                                          V.dinv, V.omega, b, x, t, done));
            std::swap(x, t);
        }
    }
    // the level's result must be in L.x for the caller's prolongation
    if (l > 0 && x != V.x) {
        // odd number of swaps: copy back (only for odd smoothing counts)
        cudaMemcpyAsync(V.x, x, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream);
    }
}

// ---------------------------------------------------------------------------------------------
// coarse tail: the V-cycle below level l0 in ONE kernel launched as a single thread-block
// cluster (16 CTAs x 1024 threads, one CTA per SM). Each phase is a cluster-stride row
// operation; phases are separated by the hardware cluster barrier (barrier.cluster with
// release/acquire semantics), so no software spin is involved. Mutable vectors are read through
// L2 (__ldcg) since other CTAs of the cluster wrote them earlier in the same kernel.
// ---------------------------------------------------------------------------------------------
constexpr int kTailMaxLevels = 16;
constexpr int kTailThreads = 1024;
constexpr int kTailTpr = 8;

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <class V>
struct TailLevel {
    int n, nc;
    const int *Arp, *Aci, *Prp, *Pci, *Rrp, *Rci;
    const V *Av, *Pv, *Rv;
    const double* dinv;
    double omega;
    double *x, *t, *b, *r;
};

template <class V>
struct TailArgs {
    TailLevel<V> lv[kTailMaxLevels];
    int nlev, s, cn;
    const double* cinv;
    double *cb, *cx;
    int* err;
    const int* done;
};

enum TailOp { T_PRE, T_JAC, T_RES, T_SPMV, T_ADD };

// One row operation over all rows of a matrix (grid-stride warps, kTailTpr lanes per row).
template <int OP, class V>
__device__ __forceinline__ void tail_rows(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                          const V* __restrict__ val, const double* __restrict__ dinv, double omega,
                                          const double* b, const double* x, double* y) {
    constexpr int TPR = kTailTpr;
    const int lane = threadIdx.x % TPR;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int nw = gridDim.x * blockDim.x / 32;
    constexpr int rpw = 32 / TPR;
    for (int base = gw * rpw; base < n; base += nw * rpw) {
        const int row = base + (threadIdx.x & 31) / TPR;
        const bool valid = row < n;
        double s = 0.0;
        if (valid)
            for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
                const int j = ci[k];
                if (OP == T_PRE) s += (double)val[k] * (omega * dinv[j] * __ldcg(b + j));
                else s += (double)val[k] * __ldcg(x + j);
            }
#pragma unroll
        for (int o = TPR / 2; o > 0; o /= 2) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
        if (valid && lane == 0) {
            if (OP == T_PRE) {
                const double bi = __ldcg(b + row);
                const double x0 = omega * dinv[row] * bi;
                y[row] = x0 + omega * dinv[row] * (bi - s);
            } else if (OP == T_JAC) {
                y[row] = __ldcg(x + row) + omega * dinv[row] * (__ldcg(b + row) - s);
            } else if (OP == T_RES) {
                y[row] = __ldcg(b + row) - s;
            } else if (OP == T_SPMV) {
                y[row] = s;
            } else {
                y[row] = __ldcg(y + row) + s;
            }
        }
    }
}

template <class V>
__global__ void __launch_bounds__(kTailThreads, 1) k_vc_tail(TailArgs<V> a) {
    CFA_GRID_DEP();
    if (a.done && *a.done) return;
    const int L = a.nlev, s = a.s;
    // down
    for (int l = 0; l < L; ++l) {
        const TailLevel<V>& v = a.lv[l];
        double* x = v.x;
        double* t = v.t;
        if (s >= 2) tail_rows<T_PRE, V>(v.n, v.Arp, v.Aci, v.Av, v.dinv, v.omega, v.b, nullptr, x);
        else {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.n; i += gridDim.x * blockDim.x)
                x[i] = v.omega * v.dinv[i] * __ldcg(v.b + i);
        }
        cluster_sync_all();
        for (int k = 2; k < s; ++k) {
            tail_rows<T_JAC, V>(v.n, v.Arp, v.Aci, v.Av, v.dinv, v.omega, v.b, x, t);
            double* tmp = x; x = t; t = tmp;
            cluster_sync_all();
        }
        if (x != v.x) {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.n; i += gridDim.x * blockDim.x) v.x[i] = __ldcg(x + i);
            cluster_sync_all();
        }
        tail_rows<T_RES, V>(v.n, v.Arp, v.Aci, v.Av, v.dinv, v.omega, v.b, v.x, v.r);
        cluster_sync_all();
        double* cb = (l + 1 < L) ? a.lv[l + 1].b : a.cb;
        tail_rows<T_SPMV, V>(v.nc, v.Rrp, v.Rci, v.Rv, nullptr, 0.0, nullptr, v.r, cb);
        cluster_sync_all();
    }
    // coarsest: dense inverse, one warp per row
    {
        const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, nw = gridDim.x * blockDim.x / 32;
        const int lane = threadIdx.x & 31;
        for (int i = warp; i < a.cn; i += nw) {
            double acc = 0.0;
            for (int j = lane; j < a.cn; j += 32) acc += a.cinv[(size_t)i * a.cn + j] * __ldcg(a.cb + j);
            acc = warp_sum(acc);
            if (lane == 0) a.cx[i] = acc;
        }
        cluster_sync_all();
    }
    // up
    for (int l = L - 1; l >= 0; --l) {
        const TailLevel<V>& v = a.lv[l];
        const double* cx = (l + 1 < L) ? a.lv[l + 1].x : a.cx;
        tail_rows<T_ADD, V>(v.n, v.Prp, v.Pci, v.Pv, nullptr, 0.0, nullptr, cx, v.x);
        cluster_sync_all();
        double* x = v.x;
        double* t = v.t;
        for (int k = 0; k < s; ++k) {
            tail_rows<T_JAC, V>(v.n, v.Arp, v.Aci, v.Av, v.dinv, v.omega, v.b, x, t);
            double* tmp = x; x = t; t = tmp;
            cluster_sync_all();
        }
        if (x != v.x) {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.n; i += gridDim.x * blockDim.x) v.x[i] = __ldcg(x + i);
            cluster_sync_all();
        }
    }
}

template <class V>
static void launch_tail(cfa_ctx* ctx, cfa_amg* amg, int l0, const int* done) {
    TailArgs<V> a{};
    const int L = (int)amg->levels.size() - l0;
    a.nlev = L;
    a.s = amg->opts.smooth_steps;
    a.cn = amg->coarse_n;
    a.cinv = amg->coarse_inv.p;
    a.cb = amg->cb64.p;
    a.cx = amg->cx64.p;
    a.err = amg->err.p;
    a.done = done;
    for (int k = 0; k < L; ++k) {
        AmgLevel& Lv = amg->levels[l0 + k];
        TailLevel<V>& t = a.lv[k];
        t.n = Lv.A.rows;
        t.nc = Lv.P.cols;
        t.Arp = Lv.A.rp.p; t.Aci = Lv.A.ci.p;
        t.Prp = Lv.P.rp.p; t.Pci = Lv.P.ci.p;
        t.Rrp = Lv.R.rp.p; t.Rci = Lv.R.ci.p;
        if constexpr (std::is_same<V, float>::value) { t.Av = Lv.A.v32.p; t.Pv = Lv.P.v32.p; t.Rv = Lv.R.v32.p; }
        else { t.Av = Lv.A.v.p; t.Pv = Lv.P.v.p; t.Rv = Lv.R.v.p; }
        t.dinv = Lv.dinv.p;
        t.omega = Lv.omega;
        t.x = Lv.x64.p; t.t = Lv.t64.p; t.b = Lv.b64.p; t.r = Lv.r64.p;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(amg->tail_grid, 1, 1);
    cfg.blockDim = dim3(kTailThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = amg->tail_grid;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ctx->launches++;
    cudaLaunchKernelEx(&cfg, k_vc_tail<V>, a);
}

// The coarse tail is opt-in (CFA_TAIL_ROWS = largest level, in rows, that it takes over): on the
// P1 pressure hierarchies measured (400k nodes: levels of 67k, 8.2k, 1.1k rows and a 230-row
// coarse solve), one 16-SM cluster is no faster than the grid-wide kernels per level, whose
// launches the solve graph already pipelines. Picks the cluster size (16 CTAs where the GPU
// allows a non-portable cluster of 16, else 8).
static cfa_status plan_tail(cfa_ctx* ctx, cfa_amg* amg) {
    amg->tail_level = -1;
    const char* e = std::getenv("CFA_TAIL_ROWS");
    const int tail_rows = e ? std::atoi(e) : 0;
    if (tail_rows <= 0) return CFA_OK;
    const void* k = amg->opts.precision == CFA_MIXED ? (const void*)k_vc_tail<float> : (const void*)k_vc_tail<double>;
    int csize = 0;
    for (int c : {16, 8}) {
        if (c == 16) cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c, 1, 1);
        cfg.blockDim = dim3(kTailThreads, 1, 1);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, k, &cfg) == cudaSuccess && nclusters > 0) { csize = c; break; }
        cudaGetLastError();
    }
    if (csize == 0) return CFA_OK;
    for (int l = 1; l < (int)amg->levels.size(); ++l)
        if (amg->levels[l].A.rows <= tail_rows) { amg->tail_level = l; break; }
    if (amg->tail_level < 0 || (int)amg->levels.size() - amg->tail_level > kTailMaxLevels) {
        amg->tail_level = -1;
        return CFA_OK;
    }
    amg->tail_grid = csize;
    return CFA_OK;
}

// Level vectors of the tiled V-cycle in the vector type T
template <class T>
struct TVec;
template <>
struct TVec<double> {
    static double* x(AmgLevel& L) { return L.x64.p; }
    static double* t(AmgLevel& L) { return L.t64.p; }
    static double* b(AmgLevel& L) { return L.b64.p; }
    static double* r(AmgLevel& L) { return L.r64.p; }
    static const double* dinv(AmgLevel& L) { return L.dinv.p; }
    static double* cb(cfa_amg* a) { return a->cb64.p; }
    static double* cx(cfa_amg* a) { return a->cx64.p; }
};
template <>
struct TVec<float> {
    static float* x(AmgLevel& L) { return L.x32.p; }
    static float* t(AmgLevel& L) { return L.t32.p; }
    static float* b(AmgLevel& L) { return L.b32.p; }
    static float* r(AmgLevel& L) { return L.r32.p; }
    static const float* dinv(AmgLevel& L) { return L.dinv32.p; }
    static float* cb(cfa_amg* a) { return a->cb32.p; }
    static float* cx(cfa_amg* a) { return a->cx32.p; }
};

// V-cycle on the tile-streamed kernels: values V in the tiles (FP32 in mixed precision), vectors
// and arithmetic in T (FP64; FP32 too in mixed precision unless CFA_VCYCLE_FP64 is set), the
// right-hand side of the level in B (level 0: the caller's FP64 r) (dry: prepare the kernels
// only, no launches)
template <class V, class T, class B>
static void vcycle_tiled(cfa_ctx* ctx, cfa_amg* amg, int l, const B* b, double* z, const int* done, bool dry,
                         const RzFuse* rz = nullptr, const CgFuse* cg = nullptr, const T* c0 = nullptr) {
    AmgLevel& L = amg->levels[l];
    const int s = amg->opts.smooth_steps;
    int* err = amg->err.p;
    // FP64 values on a mixed hierarchy: its FP64 tile copies
    const bool t64 = std::is_same<V, double>::value && amg->opts.precision == CFA_MIXED;
    const TiledCsr& tA = t64 ? L.tA64 : L.tA;
    const TiledCsr& tP = t64 ? L.tP64 : L.tP;
    const TiledCsr& tR = t64 ? L.tR64 : L.tR;
    const TiledCsr& tQ = t64 ? L.tQ64 : L.tQ;
    const TiledCsr& tW = t64 ? L.tW64 : L.tW;
    const T omega = (T)L.omega;
    const T* dinv = TVec<T>::dinv(L);
    T* x = TVec<T>::x(L);
    T* t = TVec<T>::t(L);
    if (s >= 2 && c0 && !cg) {   // the first iterate formed by the caller
        vct<VC_PREC, V, T, B, T>(ctx, dry, tA, err, dinv, omega, b, c0, x, done);
    } else if (s >= 2) {
        if (dry) vct<VC_PREC, V, T, B, T>(ctx, dry, tA, err, dinv, omega, b, (const T*)nullptr, x, done);
        vct<VC_PRE, V, T, B, T>(ctx, dry, tA, err, dinv, omega, b, (const T*)nullptr, x, done, nullptr, nullptr, cg);
    } else if (!dry) {
        CFA_TPR_SWITCH(L.A.tpr, CFA_LAUNCH(ctx, (k_vc_pre<TPR, T, B>), row_grid(ctx, L.A.rows, L.A.tpr), kThreads, 0,
                                           L.A.rows, L.A.rp.p, L.A.ci.p,
                                           (const T*)(std::is_same<T, float>::value ? (const void*)L.A.v32.p
                                                                                    : (const void*)L.A.v.p),
                                           dinv, omega, b, 0, x, done));
    }
    for (int k = 2; k < s; ++k) {
        vct<VC_JAC, V, T, B, T>(ctx, dry, tA, err, dinv, omega, b, (const T*)x, t, done);
        std::swap(x, t);
    }
    const bool last = l + 1 == (int)amg->levels.size();
    T* cb = last ? TVec<T>::cb(amg) : TVec<T>::b(amg->levels[l + 1]);
    if (L.fusedQ) {   // cb = R b - (R A) x in one pass
        vct<VC_RESTRICT, V, T, B, T>(ctx, dry, tQ, err, dinv, omega, b, (const T*)x, cb, done);
    } else {
        vct<VC_RES, V, T, B, T>(ctx, dry, tA, err, dinv, omega, b, (const T*)x, TVec<T>::r(L), done, nullptr,
                                nullptr, cg);
        vct<VC_SPMV, V, T, T, T>(ctx, dry, tR, err, dinv, omega, (const T*)nullptr, (const T*)TVec<T>::r(L), cb,
                                 done);
    }
    const T* cx;
    if (!last && l + 1 == amg->comp_level) {
        if (!dry)
            CFA_LAUNCH(ctx, (k_vc_dense<T, T>), amg->comp_n, 32 * kDenseWarps, 0,
                       amg->comp_n, amg->comp.p, (const T*)cb, TVec<T>::x(amg->levels[l + 1]), done);
        cx = TVec<T>::x(amg->levels[l + 1]);
    } else if (!last && l + 1 == amg->tail_level && std::is_same<T, double>::value) {
        if (!dry) launch_tail<V>(ctx, amg, l + 1, done);
        cx = TVec<T>::x(amg->levels[l + 1]);
    } else if (!last) {
        vcycle_tiled<V, T, T>(ctx, amg, l + 1, cb, nullptr, done, dry);
        cx = TVec<T>::x(amg->levels[l + 1]);
    } else {
        if (!dry)
            CFA_LAUNCH(ctx, (k_vc_dense<T, T>), amg->coarse_n, 32 * kDenseWarps, 0,
                       amg->coarse_n, amg->coarse_inv.p, (const T*)cb, TVec<T>::cx(amg), done);
        cx = TVec<T>::cx(amg);
    }
    int k0 = 0;
    if (L.fusedW) {   // the first post-smoothing sweep from x + P cx
        vct<VC_ADDJAC, V, T, B, T>(ctx, dry, tW, err, dinv, omega, b, (const T*)x, t, done, nullptr, cx);
        std::swap(x, t);
        k0 = 1;
    } else {
        vct<VC_ADD, V, T, T, T>(ctx, dry, tP, err, dinv, omega, (const T*)nullptr, cx, x, done);
    }
    for (int k = k0; k < s; ++k) {
        if (l == 0 && k == s - 1) {
            vct<VC_JAC, V, T, B, double>(ctx, dry, tA, err, dinv, omega, b, (const T*)x, z, done, rz);
        } else {
            vct<VC_JAC, V, T, B, T>(ctx, dry, tA, err, dinv, omega, b, (const T*)x, t, done);
            std::swap(x, t);
        }
    }
    if (l > 0 && x != TVec<T>::x(L) && !dry)
        cudaMemcpyAsync(TVec<T>::x(L), x, (size_t)L.A.rows * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream);
}

// mixed precision: the whole V-cycle in FP32 (CFA_VCYCLE_FP64=1 keeps FP64 vectors)
static bool vcycle_fp32(const cfa_amg* amg) {
    if (amg->opts.precision != CFA_MIXED) return false;
    const char* e = std::getenv("CFA_VCYCLE_FP64");
    return !(e && e[0] == '1');
}

static void vcycle_tiled_top(cfa_ctx* ctx, cfa_amg* amg, const double* r, double* z, const int* done, bool dry,
                             const RzFuse* rz = nullptr, const CgFuse* cg = nullptr, const void* c0 = nullptr,
                             bool fp64 = false) {
    if (amg->opts.precision != CFA_MIXED || (fp64 && amg->phase_switch > 0.0))
        vcycle_tiled<double, double, double>(ctx, amg, 0, r, z, done, dry, rz, cg, (const double*)c0);
    else if (vcycle_fp32(amg))
        vcycle_tiled<float, float, double>(ctx, amg, 0, r, z, done, dry, rz, cg, (const float*)c0);
    else
        vcycle_tiled<float, double, double>(ctx, amg, 0, r, z, done, dry, rz, cg, (const double*)c0);
}

double amg_fp64_phase(const cfa_amg* amg) {
    return amg && amg->tiled && !amg->levels.empty() ? amg->phase_switch : 0.0;
}

bool amg_prescale(const cfa_amg* amg, PreScale* out, bool fp64) {
    const char* e = std::getenv("CFA_PRESCALE");
    if ((e && e[0] == '0') || !amg || amg->levels.empty() || !amg->tiled || amg->opts.smooth_steps < 2) return false;
    const AmgLevel& L = amg->levels[0];
    const bool f32 = vcycle_fp32(amg) && !(fp64 && amg->phase_switch > 0.0);
    out->dinv = f32 ? (const void*)L.dinv32.p : (const void*)L.dinv.p;
    out->omega = L.omega;
    out->fp32 = f32 ? 1 : 0;
    return true;
}

// Off unless CFA_CG_FUSE_UPDATE=1: measured on the 402k-vertex step the folded form was not
// faster (13.78 against 13.60 ms without setup): the pre-smoothing pass gathers q beside r for every entry and the
// residual pass takes the grid reduction, which cost what the update kernel's launch saved.
bool amg_can_fuse_update(const cfa_amg* amg) {
    const char* e = std::getenv("CFA_CG_FUSE_UPDATE");
    const bool on = e && e[0] == '1';
    return on && amg && !amg->levels.empty() && amg->tiled && amg->opts.smooth_steps == 2 &&
           !amg->levels[0].fusedQ;
}

cfa_status amg_vcycle(cfa_ctx* ctx, cfa_amg* amg, const double* r, double* z, const int* done, bool fp64) {
    if (amg->levels.empty()) {
        CFA_LAUNCH(ctx, (k_vc_dense<double, double>), amg->coarse_n, 32 * kDenseWarps, 0,
                   amg->coarse_n, amg->coarse_inv.p, r, z, done);
    } else if (amg->tiled) {
        vcycle_tiled_top(ctx, amg, r, z, done, false, nullptr, nullptr, nullptr, fp64);
    } else if (amg->opts.precision == CFA_MIXED) {
        vcycle_level<float, double>(ctx, amg, 0, r, z, done);
    } else {
        vcycle_level<double, double>(ctx, amg, 0, r, z, done);
    }
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status amg_vcycle_rz(cfa_ctx* ctx, cfa_amg* amg, const double* r, double* z, const int* done, const RzFuse& f,
                         bool* fused, const CgFuse* cg, const void* c, bool fp64) {
    *fused = false;
    if (cg && !amg_can_fuse_update(amg))
        return set_error(ctx, CFA_BAD_ARG, "the CG update cannot be folded into this hierarchy", __FILE__, __LINE__);
    if (amg->levels.empty() || !amg->tiled || amg->opts.smooth_steps < 1) return amg_vcycle(ctx, amg, r, z, done, fp64);
    if (c && cg) return set_error(ctx, CFA_BAD_ARG, "prescaled residual with the folded update", __FILE__, __LINE__);
    vcycle_tiled_top(ctx, amg, r, z, done, false, &f, cg, c, fp64);
    CFA_CHECK_LAUNCH();
    *fused = true;
    return CFA_OK;
}

// =============================================================================================
// setup driver
// =============================================================================================
// Exact-order SpGEMM C = A B into C (device CSR), temporaries from the setup scratch.
static cfa_status spgemm(cfa_ctx* ctx, SetupScratch& S, int ar, int bc, const int* arp, const int* aci, const double* av,
                         const int* brp, const int* bci, const double* bv, DCsr& C) {
    CFA_CUDA(S.sg_ub.ensure(ar + 1));
    CFA_CUDA(S.sg_off.ensure(ar + 1));
    CFA_CUDA(S.sg_cnt.ensure(ar + 1));
    CFA_CUDA(S.h_ub.ensure(ar + 1));
    CFA_CUDA(S.h_off.ensure(ar + 1));
    CFA_CUDA(S.h_cnt.ensure(ar + 1));
    CFA_LAUNCH(ctx, k_sg_ub, ceil_div(ar, kThreads), kThreads, 0, ar, arp, aci, brp, S.sg_ub.p);
    CFA_CUDA(cudaMemcpyAsync(S.h_ub.p, S.sg_ub.p, ar * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    long long* h_off = S.h_off.p;
    h_off[0] = 0;
    for (int i = 0; i < ar; ++i) h_off[i + 1] = h_off[i] + S.h_ub.p[i];
    const long long total = h_off[ar];
    CFA_CUDA(cudaMemcpyAsync(S.sg_off.p, h_off, (ar + 1) * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    CFA_CUDA(S.sg_scol.ensure(std::max<long long>(total, 1)));
    CFA_CUDA(S.sg_sval.ensure(std::max<long long>(total, 1)));
    constexpr int sg_smem = kSgWarps * kSgCap * (int)(sizeof(double) + 2 * sizeof(int));
    static std::once_flag sg_once;
    std::call_once(sg_once, [] {
        cudaFuncSetAttribute(k_sg_accum_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, sg_smem);
    });
    CFA_LAUNCH(ctx, k_sg_accum_warp, ceil_div(ar, kSgWarps), kSgWarps * 32, sg_smem, ar, arp, aci, av, brp, bci, bv,
               (const long long*)S.sg_off.p, (const int*)S.sg_ub.p, S.sg_scol.p, S.sg_sval.p, S.sg_cnt.p);
    // the rows with more products than the warp kernel stages
    std::vector<int> big;
    for (int i = 0; i < ar; ++i)
        if (S.h_ub.p[i] > kSgCap) big.push_back(i);
    if (!big.empty()) {
        constexpr int big_smem = (kSgDenseCols + kSgChunk) * (int)sizeof(double) + kSgChunk * (int)sizeof(int) +
                                 (kSgDenseCols / 32) * (int)sizeof(unsigned) + (kSgDenseCols / 32 + 1) * (int)sizeof(int);
        static std::once_flag big_once;
        std::call_once(big_once, [] {
            cudaFuncSetAttribute(k_sg_accum_big, cudaFuncAttributeMaxDynamicSharedMemorySize, big_smem);
        });
        CFA_CUDA(S.sg_big.ensure(big.size()));
        CFA_CUDA(cudaMemcpyAsync(S.sg_big.p, big.data(), big.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        CFA_LAUNCH(ctx, k_sg_accum_big, (int)big.size(), kSgBigThreads, big_smem, (const int*)S.sg_big.p, bc, arp, aci,
                   av, brp, bci, bv, (const long long*)S.sg_off.p, S.sg_scol.p, S.sg_sval.p, S.sg_cnt.p);
    }
    CFA_CUDA(cudaMemcpyAsync(S.h_cnt.p, S.sg_cnt.p, ar * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    int* h_rp = S.h_ub.p;   // reuse: C row pointer
    h_rp[0] = 0;
    for (int i = 0; i < ar; ++i) h_rp[i + 1] = h_rp[i] + S.h_cnt.p[i];
    C.rows = ar;
    C.cols = bc;
    C.nnz = h_rp[ar];
    CFA_CUDA(C.rp.ensure(ar + 1));
    CFA_CUDA(C.ci.ensure(std::max(C.nnz, 1)));
    CFA_CUDA(C.v.ensure(std::max(C.nnz, 1)));
    CFA_CUDA(cudaMemcpyAsync(C.rp.p, h_rp, (ar + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CFA_LAUNCH(ctx, k_sg_copy, ceil_div(ar, kThreads), kThreads, 0, ar, (const long long*)S.sg_off.p,
               (const int*)S.sg_scol.p, (const double*)S.sg_sval.p, (const int*)C.rp.p, C.ci.p, C.v.p);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

// T = A^T (csr_transpose, :847-862): entries of each column in ascending row order
static cfa_status transpose(cfa_ctx* ctx, SetupScratch& S, const DCsr& A, DCsr& T) {
    const int m = A.nnz;
    CFA_CUDA(S.tr_keys.ensure(std::max(m, 1)));
    CFA_CUDA(S.tr_idx.ensure(std::max(m, 1)));
    CFA_CUDA(S.tr_perm.ensure(std::max(m, 1)));
    CFA_CUDA(S.tr_row_of.ensure(std::max(m, 1)));
    T.rows = A.cols;
    T.cols = A.rows;
    T.nnz = m;
    CFA_CUDA(T.rp.ensure(A.cols + 1));
    CFA_CUDA(T.ci.ensure(std::max(m, 1)));
    CFA_CUDA(T.v.ensure(std::max(m, 1)));
    if (m > 0) {
        CFA_LAUNCH(ctx, k_iota, ceil_div(m, kThreads), kThreads, 0, m, S.tr_idx.p);
        CFA_LAUNCH(ctx, k_entry_rows, ceil_div(A.rows, kThreads), kThreads, 0, A.rows, (const int*)A.rp.p, S.tr_row_of.p);
        int bits = 1;
        while ((1LL << bits) <= A.cols) ++bits;
        size_t tmp_bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, A.ci.p, S.tr_keys.p, S.tr_idx.p, S.tr_perm.p, m, 0, bits,
                                        ctx->stream);
        CFA_CUDA(S.cub_tmp.ensure(tmp_bytes + 16));
        CFA_CUDA(cub::DeviceRadixSort::SortPairs(S.cub_tmp.p, tmp_bytes, A.ci.p, S.tr_keys.p, S.tr_idx.p, S.tr_perm.p, m,
                                                 0, bits, ctx->stream));
        ctx->launches += 4;
        CFA_LAUNCH(ctx, k_transpose_fill, ceil_div(m, kThreads), kThreads, 0, m, (const int*)S.tr_perm.p,
                   (const int*)S.tr_row_of.p, (const double*)A.v.p, T.ci.p, T.v.p);
    }
    CFA_LAUNCH(ctx, k_ptr_from_sorted, ceil_div(m + 1, kThreads), kThreads, 0, A.cols, m, (const int*)S.tr_keys.p, T.rp.p);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

// ---------------------------------------------------------------------------------------------
// The greedy 3-phase aggregation (smoothed_prolongator, src/cfa/linalg.cuh:1321-1348) on the
// device, giving the aggregates of the sequential loop bit for bit.
//
// Phase 1 visits nodes in index order; node i becomes a root (a new aggregate with its strong
// neighbours) iff, when it is visited, neither i nor any strong neighbour j of i is aggregated.
// "Aggregated when i is visited" only involves roots k < i: i is aggregated iff some root k < i
// has i as a strong neighbour (k -> i); j is iff j is a root below i, or some root k < i has
// k -> j. So root(i) depends only on the root status of lower-numbered nodes within two strong
// hops -- the lexicographically first independent set of that conflict relation: an undecided
// node becomes a non-root as soon as one lower conflict is a root, and a root once all of its
// lower conflicts are decided non-roots. States only move from undecided to final, so a node may
// read the others' states at any time. The decisions form chains (about 1800 dependent steps on
// the ~400k-node pressure matrix), which rule out one launch per step: one launch per phase
// decides all nodes as a dataflow (k_agg_flow). Aggregate ids follow root order (a prefix sum); a
// non-root takes the id of the root that has it as a strong neighbour (at most one can).
// Phase 2 (parallel in the reference too) gives an unaggregated node the aggregate of its first
// aggregated strong neighbour. Phase 3 visits the rest in index order: an unaggregated node
// starts a new aggregate and claims its unaggregated strong neighbours (all of higher index), so
// it is a root iff no lower root claims it, and a claimed node belongs to the lowest root that
// claims it. The strong relation is read as directed (row i's entries), as in the reference:
// coarse Galerkin operators need not be symmetric to the last bit.
// ---------------------------------------------------------------------------------------------
enum : unsigned char { AGG_UNDECIDED = 0, AGG_ROOT = 1, AGG_MEMBER = 2 };

// in-degree of the strong graph (k -> j counted at j)
__global__ void k_strong_indeg(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                               const unsigned char* __restrict__ strong, int* __restrict__ cnt) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int a = rp[i]; a < rp[i + 1]; ++a)
        if (strong[a]) atomicAdd(cnt + ci[a], 1);
}

// in-neighbour lists (their order within a list does not matter to the rounds below)
__global__ void k_strong_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                              const unsigned char* __restrict__ strong, const int* __restrict__ trp,
                              int* __restrict__ fill, int* __restrict__ tci) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int a = rp[i]; a < rp[i + 1]; ++a)
        if (strong[a]) {
            const int j = ci[a];
            tci[trp[j] + atomicAdd(fill + j, 1)] = i;
        }
}

__device__ __forceinline__ unsigned char agg_state(const unsigned char* st, int k) {
    return *reinterpret_cast<const volatile unsigned char*>(st + k);
}

// Phase 1 ids: a root's from the prefix sum of roots; a member's from the root that has it as a
// strong neighbour; -1 for the rest.
__global__ void k_agg_p1_ids(int n, const int* __restrict__ trp, const int* __restrict__ tci,
                             const unsigned char* __restrict__ st, const int* __restrict__ rank, int* __restrict__ agg) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = -1;
    if (st[i] == AGG_ROOT) {
        a = rank[i];
    } else {
        for (int q = trp[i]; q < trp[i + 1]; ++q) {
            const int k = tci[q];
            if (st[k] == AGG_ROOT) { a = rank[k]; break; }
        }
    }
    agg[i] = a;
}

// Phase 2: the first aggregated strong neighbour (row order) of an unaggregated node; also marks
// the nodes left for phase 3 (undecided) and the others (member).
__global__ void k_agg_p2(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                         const unsigned char* __restrict__ strong, const int* __restrict__ agg1, int* __restrict__ agg2,
                         unsigned char* __restrict__ st3) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = agg1[i];
    if (a < 0)
        for (int e = rp[i]; e < rp[i + 1]; ++e)
            if (strong[e] && agg1[ci[e]] >= 0) { a = agg1[ci[e]]; break; }
    agg2[i] = a;
    st3[i] = a < 0 ? AGG_UNDECIDED : AGG_MEMBER;
}

// Both sequential phases as one dataflow launch each. Chunks of kAggChunk consecutive nodes go
// to CTAs in ticket order (a CTA takes the next chunk when it starts), one node per thread; a
// thread re-evaluates its node until it is decided. A chunk's states live in shared memory as well
// as in global memory, so the many decisions that wait on a node of the same chunk (the mesh
// numbering keeps conflicts close in index) take a shared-memory round trip rather than an L2 one.
// Each evaluation reads the states of the node's lower conflicts from a precomputed list
// (k_agg_conf_*), kAggBatch loads issued together, so one poll costs about one L2 round trip.
// Progress: the lowest undecided node has all its lower conflicts decided, and its chunk has
// started, because every CTA with an earlier ticket holds only lower nodes, all decided, and
// retires. Every wait is bounded: a thread that polls kAggPollLimit times, or sees another thread
// give up, records CFA_TIMEOUT in *err and leaves its node undecided.
constexpr int kAggChunk = 1024;
constexpr int kAggBatch = 16;
constexpr unsigned kAggPollLimit = 1u << 20;

struct AggView {
    const unsigned char* g;     // global states
    volatile unsigned char* s;  // this chunk's states
    int base;
    __device__ __forceinline__ unsigned char operator()(int k) const {
        const unsigned kk = (unsigned)(k - base);
        return kk < (unsigned)kAggChunk ? s[kk] : agg_state(g, k);
    }
};

// Phase 1's lower conflicts of node i (repeats allowed): its in-neighbours k < i (k -> i), its
// strong neighbours j < i, and the in-neighbours k < i of each strong neighbour j (k -> j). FILL:
// write them at conf[cptr[i]..]; else count them into cnt[i].
template <bool FILL>
__global__ void k_agg_conf(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const unsigned char* __restrict__ strong, const int* __restrict__ trp,
                           const int* __restrict__ tci, int* __restrict__ cnt, const int* __restrict__ cptr,
                           int* __restrict__ conf) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int o = FILL ? cptr[i] : 0;
    for (int q = trp[i]; q < trp[i + 1]; ++q) {
        const int k = tci[q];
        if (k < i) { if (FILL) conf[o] = k; ++o; }
    }
    for (int a = rp[i]; a < rp[i + 1]; ++a) {
        if (!strong[a]) continue;
        const int j = ci[a];
        if (j < i) { if (FILL) conf[o] = j; ++o; }
        for (int q = trp[j]; q < trp[j + 1]; ++q) {
            const int k = tci[q];
            if (k < i) { if (FILL) conf[o] = k; ++o; }
        }
    }
    if (!FILL) cnt[i] = o;
}

// The state node i can take from what its lower conflicts have decided so far (UNDECIDED: not
// yet): a non-root as soon as one is a root, a root once all are decided non-roots. Phase 1: the
// conflict list of k_agg_conf. Phase 3 (nodes that phases 1 and 2 left unaggregated; the others
// hold the non-root state): the in-neighbours k < i (k -> i).
__device__ __forceinline__ unsigned char agg_decide(int i, const int* __restrict__ list, int beg, int end,
                                                    bool lower_only, const AggView& st) {
    bool pending = false;
    for (int q = beg; q < end; q += kAggBatch) {
        unsigned char sv[kAggBatch];
#pragma unroll
        for (int u = 0; u < kAggBatch; ++u) {
            sv[u] = AGG_MEMBER;
            if (q + u < end) {
                const int k = list[q + u];
                if (!lower_only || k < i) sv[u] = st(k);
            }
        }
#pragma unroll
        for (int u = 0; u < kAggBatch; ++u) {
            if (sv[u] == AGG_ROOT) return AGG_MEMBER;
            pending |= sv[u] == AGG_UNDECIDED;
        }
    }
    return pending ? AGG_UNDECIDED : AGG_ROOT;
}

// P3 = false: phase 1 on the conflict lists (lptr, list); P3 = true: phase 3 on the in-neighbour
// lists (lptr = trp, list = tci).
template <bool P3>
__global__ void __launch_bounds__(kAggChunk)
k_agg_flow(int n, const int* __restrict__ lptr, const int* __restrict__ list, unsigned char* st,
           int* __restrict__ ticket, int* err) {
    CFA_GRID_DEP();
    __shared__ int s_chunk;
    __shared__ unsigned char s_st[kAggChunk];
    if (threadIdx.x == 0) s_chunk = atomicAdd(ticket, 1);
    __syncthreads();
    const int base = s_chunk * kAggChunk;
    const int i = base + threadIdx.x;
    unsigned char mine = i < n ? agg_state(st, i) : AGG_MEMBER;
    s_st[threadIdx.x] = mine;
    __syncthreads();
    const AggView view{st, s_st, base};
    volatile int* verr = err;
    const int beg = i < n ? lptr[i] : 0, end = i < n ? lptr[i + 1] : 0;
    for (unsigned it = 0; mine == AGG_UNDECIDED; ++it) {
        mine = agg_decide(i, list, beg, end, P3, view);
        if (mine != AGG_UNDECIDED) {
            s_st[threadIdx.x] = mine;
            *reinterpret_cast<volatile unsigned char*>(st + i) = mine;
        } else if (it >= kAggPollLimit || *verr != 0) {
            atomicCAS(err, 0, (int)CFA_TIMEOUT);
            break;
        }
    }
}

// Phase 3 ids (after na1 phase-1 aggregates): roots in order; a claimed node takes its lowest
// claiming root's id. Also counts the aggregate sizes.
__global__ void k_agg_p3_ids(int n, int na1, const int* __restrict__ trp, const int* __restrict__ tci,
                             const unsigned char* __restrict__ st, const int* __restrict__ rank,
                             const int* __restrict__ agg2, int* __restrict__ agg, int* __restrict__ size) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = agg2[i];
    if (a < 0) {
        if (st[i] == AGG_ROOT) {
            a = na1 + rank[i];
        } else {
            int kmin = n;
            for (int q = trp[i]; q < trp[i + 1]; ++q) {
                const int k = tci[q];
                if (k < kmin && agg2[k] < 0 && st[k] == AGG_ROOT) kmin = k;
            }
            a = na1 + rank[kmin];
        }
    }
    agg[i] = a;
    atomicAdd(size + a, 1);
}

// Tentative prolongator: P0 row i holds 1 / sqrt(|aggregate of i|) in column agg[i].
__global__ void k_agg_p0(int n, const int* __restrict__ agg, const int* __restrict__ size, int* __restrict__ p0rp,
                         double* __restrict__ p0v) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    p0rp[i] = i;
    if (i < n) p0v[i] = 1.0 / sqrt((double)size[agg[i]]);
}


// exclusive prefix sum of n ints (n + 1 outputs: the total at out[n])
static cfa_status exclusive_sum(cfa_ctx* ctx, SetupScratch& S, const int* in, int* out, int n) {
    size_t bytes = 0;
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n + 1, ctx->stream));
    CFA_CUDA(S.cub_tmp.ensure(bytes + 16));
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(S.cub_tmp.p, bytes, in, out, n + 1, ctx->stream));
    ctx->launches += 2;
    return CFA_OK;
}

__global__ void k_agg_is_root(int n, const unsigned char* __restrict__ st, int* __restrict__ flag) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) flag[i] = (i < n && st[i] == AGG_ROOT) ? 1 : 0;
}

// The aggregates of A's strong graph (S.strong) into agg[m]; na = their count; the tentative
// prolongator's row offsets and values into S.p0rp / S.p0v.
static cfa_status aggregate_device(cfa_ctx* ctx, SetupScratch& S, const DCsr& A, int* agg, int* na_out) {
    const int n = A.rows;
    const int g = ceil_div(n, kThreads), g1 = ceil_div(n + 1, kThreads);
    for (DevBuf<int>* b : {&S.ag_trp, &S.ag_fill, &S.ag_rank, &S.ag_agg1, &S.ag_agg2, &S.ag_size})
        CFA_CUDA(b->ensure(n + 1));
    CFA_CUDA(S.ag_tci.ensure(std::max(A.nnz, 1)));
    CFA_CUDA(S.ag_state.ensure(n));
    CFA_CUDA(S.ag_flag.ensure(2));
    CFA_CUDA(S.h_ag.ensure(3));
    CFA_CUDA(S.p0v.ensure(n));
    CFA_CUDA(S.p0rp.ensure(n + 1));
    // in-neighbour lists of the strong graph
    CFA_CUDA(cudaMemsetAsync(S.ag_fill.p, 0, (n + 1) * sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_strong_indeg, g, kThreads, 0, n, A.rp.p, A.ci.p, (const unsigned char*)S.strong.p, S.ag_fill.p);
    CFA_PROPAGATE(exclusive_sum(ctx, S, S.ag_fill.p, S.ag_trp.p, n));
    CFA_CUDA(cudaMemsetAsync(S.ag_fill.p, 0, (n + 1) * sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_strong_fill, g, kThreads, 0, n, A.rp.p, A.ci.p, (const unsigned char*)S.strong.p,
               (const int*)S.ag_trp.p, S.ag_fill.p, S.ag_tci.p);
    // phase 1's conflict lists
    CFA_CUDA(S.ag_cptr.ensure(n + 1));
    CFA_LAUNCH(ctx, k_agg_conf<false>, g, kThreads, 0, n, A.rp.p, A.ci.p, (const unsigned char*)S.strong.p,
               (const int*)S.ag_trp.p, (const int*)S.ag_tci.p, S.ag_fill.p, (const int*)nullptr, (int*)nullptr);
    CFA_CUDA(cudaMemsetAsync(S.ag_fill.p + n, 0, sizeof(int), ctx->stream));
    CFA_PROPAGATE(exclusive_sum(ctx, S, S.ag_fill.p, S.ag_cptr.p, n));
    int nconf = 0;
    CFA_CUDA(cudaMemcpyAsync(&nconf, S.ag_cptr.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    CFA_CUDA(S.ag_conf.ensure(std::max(nconf, 1)));
    CFA_LAUNCH(ctx, k_agg_conf<true>, g, kThreads, 0, n, A.rp.p, A.ci.p, (const unsigned char*)S.strong.p,
               (const int*)S.ag_trp.p, (const int*)S.ag_tci.p, (int*)nullptr, (const int*)S.ag_cptr.p, S.ag_conf.p);
    // phase 1 (ag_flag: [0] chunk tickets, [1] error status)
    const int chunks = ceil_div(n, kAggChunk);
    CFA_CUDA(cudaMemsetAsync(S.ag_state.p, AGG_UNDECIDED, n, ctx->stream));
    CFA_CUDA(cudaMemsetAsync(S.ag_flag.p, 0, 2 * sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_agg_flow<false>, chunks, kAggChunk, 0, n, (const int*)S.ag_cptr.p, (const int*)S.ag_conf.p,
               S.ag_state.p, S.ag_flag.p, S.ag_flag.p + 1);
    CFA_LAUNCH(ctx, k_agg_is_root, g1, kThreads, 0, n, (const unsigned char*)S.ag_state.p, S.ag_fill.p);
    CFA_PROPAGATE(exclusive_sum(ctx, S, S.ag_fill.p, S.ag_rank.p, n));
    CFA_LAUNCH(ctx, k_agg_p1_ids, g, kThreads, 0, n, (const int*)S.ag_trp.p, (const int*)S.ag_tci.p,
               (const unsigned char*)S.ag_state.p, (const int*)S.ag_rank.p, S.ag_agg1.p);
    // phase 2
    CFA_LAUNCH(ctx, k_agg_p2, g, kThreads, 0, n, A.rp.p, A.ci.p, (const unsigned char*)S.strong.p,
               (const int*)S.ag_agg1.p, S.ag_agg2.p, S.ag_state.p);
    // phase 3 (the number of phase-1 aggregates first: the ids continue from it)
    CFA_CUDA(cudaMemcpyAsync(S.h_ag.p + 1, S.ag_rank.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaMemsetAsync(S.ag_flag.p, 0, sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_agg_flow<true>, chunks, kAggChunk, 0, n, (const int*)S.ag_trp.p, (const int*)S.ag_tci.p,
               S.ag_state.p, S.ag_flag.p, S.ag_flag.p + 1);
    CFA_CUDA(cudaMemcpyAsync(S.h_ag.p + 2, S.ag_flag.p + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    if (S.h_ag.p[2] != 0)
        return set_error(ctx, CFA_TIMEOUT, "aggregation: a node's decision waited past its poll limit", __FILE__,
                         __LINE__);
    const int na1 = S.h_ag.p[1];
    CFA_LAUNCH(ctx, k_agg_is_root, g1, kThreads, 0, n, (const unsigned char*)S.ag_state.p, S.ag_fill.p);
    CFA_PROPAGATE(exclusive_sum(ctx, S, S.ag_fill.p, S.ag_rank.p, n));
    CFA_CUDA(cudaMemsetAsync(S.ag_size.p, 0, (n + 1) * sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_agg_p3_ids, g, kThreads, 0, n, na1, (const int*)S.ag_trp.p, (const int*)S.ag_tci.p,
               (const unsigned char*)S.ag_state.p, (const int*)S.ag_rank.p, (const int*)S.ag_agg2.p, agg,
               S.ag_size.p);
    CFA_CUDA(cudaMemcpyAsync(S.h_ag.p, S.ag_rank.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_LAUNCH(ctx, k_agg_p0, g1, kThreads, 0, n, (const int*)agg, (const int*)S.ag_size.p, S.p0rp.p, S.p0v.p);
    CFA_CHECK_LAUNCH();
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    *na_out = na1 + S.h_ag.p[0];
    return CFA_OK;
}


// Greedy 3-phase aggregation of smoothed_prolongator (:1321-1348) on the host strength flags
// (aggregate_host, the reference's sequential loop) or in the device rounds (aggregate_device).
// The greedy aggregation on the host (the reference's loop) or on the device (the same
// aggregates): the handle's choice (cfa_amg_set_aggregation), else CFA_AGG_HOST, else the device.
static bool agg_on_host(const cfa_amg* amg) {
    if (amg->vc_agg_device >= 0) return amg->vc_agg_device == 0;
    const char* e = std::getenv("CFA_AGG_HOST");
    return e && e[0] == '1';
}

static int aggregate_host(int n, const int* rp, const int* ci, const unsigned char* strong, int* agg) {
    for (int i = 0; i < n; ++i) agg[i] = -1;
    int na = 0;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        bool free_nbhd = true;
        for (int a = rp[i]; a < rp[i + 1] && free_nbhd; ++a)
            if (strong[a] && agg[ci[a]] >= 0) free_nbhd = false;
        if (!free_nbhd) continue;
        agg[i] = na;
        for (int a = rp[i]; a < rp[i + 1]; ++a) if (strong[a]) agg[ci[a]] = na;
        ++na;
    }
    std::vector<int> agg2(agg, agg + n);
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        for (int a = rp[i]; a < rp[i + 1]; ++a)
            if (strong[a] && agg[ci[a]] >= 0) { agg2[i] = agg[ci[a]]; break; }
    }
    std::copy(agg2.begin(), agg2.end(), agg);
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        agg[i] = na;
        for (int a = rp[i]; a < rp[i + 1]; ++a)
            if (strong[a] && agg[ci[a]] < 0) agg[ci[a]] = na;
        ++na;
    }
    return na;
}

static cfa_status copy_csr(cfa_ctx* ctx, int rows, int nnz, const int* rp, const int* ci, const double* v, DCsr& D) {
    D.rows = rows;
    D.cols = rows;
    D.nnz = nnz;
    CFA_CUDA(D.rp.ensure(rows + 1));
    CFA_CUDA(D.ci.ensure(std::max(nnz, 1)));
    CFA_CUDA(D.v.ensure(std::max(nnz, 1)));
    CFA_CUDA(cudaMemcpyAsync(D.rp.p, rp, (rows + 1) * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(D.ci.p, ci, (size_t)nnz * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(D.v.p, v, (size_t)nnz * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    return CFA_OK;
}

static cfa_status to_float(cfa_ctx* ctx, DCsr& M) {
    CFA_CUDA(M.v32.ensure(std::max(M.nnz, 1)));
    if (M.nnz) CFA_LAUNCH(ctx, k_to_float, std::min(ceil_div(M.nnz, kThreads), 8 * ctx->num_sms), kThreads, 0,
                          (long long)M.nnz, M.v.p, M.v32.p);
    return CFA_OK;
}

// 1 + 0.1 sin(1 + i) for i < n: the power-iteration start vector (host libm, as the reference),
// computed once per process (shared by the threads of all contexts).
static std::vector<double> start_vector(int n) {
    static std::mutex mu;
    static std::vector<double> x0;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)x0.size() < n) {
        const size_t old = x0.size();
        x0.resize(n);
        for (size_t i = old; i < (size_t)n; ++i) x0[i] = 1.0 + 0.1 * std::sin(1.0 + (double)i);
    }
    return std::vector<double>(x0.begin(), x0.begin() + n);
}

// rho(D^-1 A) by 20 power iterations (spectral_radius_DinvA, :1276-1304), on the device.
static cfa_status spectral_radius(cfa_ctx* ctx, cfa_amg* amg, const DCsr& A, const double* dinv, double* rho) {
    SetupScratch& S = amg->scratch;
    const int n = A.rows, nch = (n + kPowChunk - 1) / kPowChunk;
    static std::once_flag smem_once;
    std::call_once(smem_once, [] {
        cudaFuncSetAttribute(k_pow_chunks, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * kPowChunk * sizeof(double)));
    });
    if (!amg->x0.p || amg->x0.cap < (size_t)n) {
        const std::vector<double> h = start_vector(n);
        CFA_CUDA(amg->x0.ensure(n));
        // pageable source: the call returns once `h` has been staged
        CFA_CUDA(cudaMemcpyAsync(amg->x0.p, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    }
    CFA_CUDA(S.pow_x.ensure(n));
    CFA_CUDA(S.pow_y.ensure(n));
    CFA_CUDA(S.pow_py.ensure(nch));
    CFA_CUDA(S.pow_px.ensure(nch));
    CFA_CUDA(S.pow_st.ensure(2));
    CFA_CUDA(S.h_st.ensure(2));
    CFA_CUDA(cudaMemcpyAsync(S.pow_x.p, amg->x0.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    for (int it = 0; it < 20; ++it) {
        CFA_LAUNCH(ctx, k_pow_y, ceil_div(n, kThreads), kThreads, 0, n, (const int*)A.rp.p, (const int*)A.ci.p,
                   (const double*)A.v.p, dinv, (const double*)S.pow_x.p, S.pow_y.p);
        CFA_LAUNCH(ctx, k_pow_chunks, nch, kPowThreads, 2 * kPowChunk * sizeof(double), n, nch,
                   (const double*)S.pow_x.p, (const double*)S.pow_y.p, S.pow_py.p, S.pow_px.p);
        CFA_LAUNCH(ctx, k_pow_finish, 1, 32, 0, nch, (const double*)S.pow_py.p, (const double*)S.pow_px.p, S.pow_st.p);
        CFA_LAUNCH(ctx, k_pow_scale, ceil_div(n, kThreads), kThreads, 0, n, (const double*)S.pow_y.p,
                   (const double*)S.pow_st.p, S.pow_x.p);
    }
    CFA_CUDA(cudaMemcpyAsync(S.h_st.p, S.pow_st.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    *rho = std::max(S.h_st.p[1], 1.0e-12) * 1.05;
    return CFA_OK;
}

static cfa_status level_vectors(cfa_ctx* ctx, cfa_amg* amg, AmgLevel& L, int n) {
    if (amg->opts.precision == CFA_MIXED) {
        CFA_CUDA(L.x32.ensure(n)); CFA_CUDA(L.t32.ensure(n)); CFA_CUDA(L.b32.ensure(n)); CFA_CUDA(L.r32.ensure(n));
    } else {
        CFA_CUDA(L.x64.ensure(n)); CFA_CUDA(L.t64.ensure(n)); CFA_CUDA(L.b64.ensure(n)); CFA_CUDA(L.r64.ensure(n));
    }
    return CFA_OK;
}

static cfa_status level_vectors64(cfa_ctx* ctx, AmgLevel& L, int n) {
    CFA_CUDA(L.x64.ensure(n)); CFA_CUDA(L.t64.ensure(n)); CFA_CUDA(L.b64.ensure(n)); CFA_CUDA(L.r64.ensure(n));
    return CFA_OK;
}

// ---- fused transfers (AmgLevel::tQ, tW) ----
// Q = [R | -R A] row by row: R's entries (columns of b), then R A's with the second-vector bit
// (columns of x) and negated values. Qrp = Rrp + RArp.
__global__ void k_fuse_q_rp(int nc, const int* __restrict__ a, const int* __restrict__ b, int* __restrict__ out) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= nc) out[i] = a[i] + b[i];
}

__global__ void k_fuse_q_fill(int nc, const int* __restrict__ Rrp, const int* __restrict__ Rci,
                              const double* __restrict__ Rv, const int* __restrict__ Crp, const int* __restrict__ Cci,
                              const double* __restrict__ Cv, const int* __restrict__ Qrp, int* __restrict__ Qci,
                              double* __restrict__ Qv) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    int o = Qrp[i];
    for (int k = Rrp[i]; k < Rrp[i + 1]; ++k, ++o) { Qci[o] = Rci[k]; Qv[o] = Rv[k]; }
    for (int k = Crp[i]; k < Crp[i + 1]; ++k, ++o) { Qci[o] = Cci[k] | kSecondVec; Qv[o] = -Cv[k]; }
}

// W row i = A's entries (columns of x; v0 = A, v1 = 1 on the diagonal), then A P's (columns of
// the coarse correction; v0 = A P, v1 = P where P has the column), then P's columns that A P
// lacks (v0 = 0). count: entries per row into cnt; fill: the rows at Wrp.
template <bool FILL>
__global__ void k_fuse_w(int n, const int* __restrict__ Arp, const int* __restrict__ Aci, const double* __restrict__ Av,
                         const int* __restrict__ Brp, const int* __restrict__ Bci, const double* __restrict__ Bv,
                         const int* __restrict__ Prp, const int* __restrict__ Pci, const double* __restrict__ Pv,
                         int* __restrict__ cnt, const int* __restrict__ Wrp, int* __restrict__ Wci,
                         double* __restrict__ W0, double* __restrict__ W1) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int o = FILL ? Wrp[i] : 0;
    for (int k = Arp[i]; k < Arp[i + 1]; ++k, ++o)
        if (FILL) { Wci[o] = Aci[k]; W0[o] = Av[k]; W1[o] = Aci[k] == i ? 1.0 : 0.0; }
    for (int k = Brp[i]; k < Brp[i + 1]; ++k, ++o) {
        if (!FILL) continue;
        double pv = 0.0;
        for (int q = Prp[i]; q < Prp[i + 1]; ++q)
            if (Pci[q] == Bci[k]) pv = Pv[q];
        Wci[o] = Bci[k] | kSecondVec; W0[o] = Bv[k]; W1[o] = pv;
    }
    for (int q = Prp[i]; q < Prp[i + 1]; ++q) {
        bool in = false;
        for (int k = Brp[i]; k < Brp[i + 1] && !in; ++k) in = Bci[k] == Pci[q];
        if (in) continue;
        if (FILL) { Wci[o] = Pci[q] | kSecondVec; W0[o] = 0.0; W1[o] = Pv[q]; }
        ++o;
    }
    if (!FILL) cnt[i] = o;
}

// Levels whose transfers run fused: CFA_VC_FUSE=0 none, 1 levels >= 1 (the default: there the
// V-cycle is a chain of short launches), 2 every level. Needs at least two smoothing steps (the
// first post-smoothing sweep carries the prolongation). The restriction (VC_RESTRICT) is fused on
// every such level; the prolongation (VC_ADDJAC) only on levels of at most CFA_VC_ADDJAC_ROWS rows
// (default 16384): [A | A P] holds about twice A's and P's entries together, which costs more than
// the launch it saves once a level's sweeps are no longer latency-bound.
static bool fuse_level(const cfa_amg* amg, const AmgLevel& L) {
    const char* e = std::getenv("CFA_VC_FUSE");
    const int mode = amg->vc_fuse >= 0 ? amg->vc_fuse : e ? std::atoi(e) : 1;
    if (mode <= 0 || amg->opts.smooth_steps < 2) return false;
    return mode >= 2 || &L != &amg->levels[0];
}

static bool fuse_prolongation(const cfa_amg* amg, const AmgLevel& L) {
    const char* e = std::getenv("CFA_VC_ADDJAC_ROWS");
    const int rows = amg->vc_fold_rows >= 0 ? amg->vc_fold_rows : e ? std::atoi(e) : 16384;
    return L.A.rows <= rows;
}

// a_ij == a_ji on every entry of A (T = A^T, the same pattern), to 1e-10 of the entries or 1e-12
// of sqrt(|a_ii a_jj|) (entries left by cancellation in the Galerkin sums differ in their last
// bits relative to themselves, not to the row's scale)
__global__ void k_sym_check(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                            const double* __restrict__ av, const int* __restrict__ trp, const int* __restrict__ tci,
                            const double* __restrict__ tv, const double* __restrict__ dinv, int* __restrict__ asym) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (arp[i + 1] - arp[i] != trp[i + 1] - trp[i]) { *asym = 1; return; }
    for (int k = arp[i], q = trp[i]; k < arp[i + 1]; ++k, ++q) {
        const int j = aci[k];
        if (j != tci[q]) { *asym = 1; return; }
        const double d = fabs(av[k] - tv[q]);
        const double scale = sqrt(fabs(1.0 / (dinv[i] * dinv[j])));
        if (!(d <= 1e-10 * (fabs(av[k]) + fabs(tv[q])) || d <= 1e-12 * scale)) { *asym = 1; return; }
    }
}

// Pipeline depth of the level tiles (CFA_VC_STAGES, default 2). Two stages leave room for more
// CTAs per SM (six instead of four on the finest level's 256-row FP32 tiles) and more rows'
// gathers in flight, while two waves of tiles in flight still cover the DRAM latency: the
// 4.2M-row V-cycle 692 -> 620 us, the 402k-row one unchanged. The pressure operator keeps three.
static int level_tile_stages() {
    static const int s = [] {
        const char* e = std::getenv("CFA_VC_STAGES");
        const int v = e ? std::atoi(e) : 2;
        return v >= 2 && v <= kTileStages ? v : 2;
    }();
    return s;
}

static cfa_status pack_from_device(cfa_ctx* ctx, cfa_amg* amg, const DCsr& M, const double* v0, const double* v1,
                                   int vb, TiledCsr& T) {
    HostBuf<int>& hr = amg->scratch.h_rp;
    CFA_CUDA(hr.ensure(M.rows + 1));
    CFA_CUDA(cudaMemcpyAsync(hr.p, M.rp.p, (M.rows + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    T.stages = level_tile_stages();
    CFA_PROPAGATE(plan_tiled(ctx, hr.p, M.rows, v1 ? 2 : 1, vb, T));
    return pack_tiled(ctx, M.rp.p, M.ci.p, v0, v1, nullptr, T);
}

// The fused transfer operators of a level: Q = [R | -R A] and, with_w, W = ([A | A P], [I | P]),
// packed as tiles in the hierarchy precision. A P is the Galerkin product's (recomputed after a
// remap changed P). R A = P^T A is (A P)^T when A is symmetric (checked entry by entry; the
// Galerkin operators are, to rounding); otherwise the exact-order SpGEMM forms it.
static cfa_status build_fused(cfa_ctx* ctx, cfa_amg* amg, AmgLevel& L, int vb, bool with_w) {
    SetupScratch& S = amg->scratch;
    const int n = L.A.rows, nc = L.R.rows;
    const bool keep_ap = L.AP.rows == n && L.AP.cols == L.P.cols && L.AP.nnz > 0;
    if (!keep_ap)
        CFA_PROPAGATE(spgemm(ctx, S, n, L.P.cols, L.A.rp.p, L.A.ci.p, L.A.v.p, L.P.rp.p, L.P.ci.p, L.P.v.p, S.fAP));
    const DCsr& AP = keep_ap ? L.AP : S.fAP;
    CFA_PROPAGATE(transpose(ctx, S, L.A, S.fAt));
    CFA_CUDA(S.ierr.ensure(1));
    CFA_CUDA(cudaMemsetAsync(S.ierr.p, 0, sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_sym_check, ceil_div(n, kThreads), kThreads, 0, n, (const int*)L.A.rp.p, (const int*)L.A.ci.p,
               (const double*)L.A.v.p, (const int*)S.fAt.rp.p, (const int*)S.fAt.ci.p, (const double*)S.fAt.v.p,
               (const double*)L.dinv.p, S.ierr.p);
    int asym = 0;
    CFA_CUDA(cudaMemcpyAsync(&asym, S.ierr.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    if (asym) CFA_PROPAGATE(spgemm(ctx, S, nc, n, L.R.rp.p, L.R.ci.p, L.R.v.p, L.A.rp.p, L.A.ci.p, L.A.v.p, S.fRA));
    else CFA_PROPAGATE(transpose(ctx, S, AP, S.fRA));
    L.ra_spgemm = asym != 0;
    // Q
    DCsr& Q = S.fQ;
    Q.rows = nc;
    Q.cols = n;
    Q.nnz = L.R.nnz + S.fRA.nnz;
    CFA_CUDA(Q.rp.ensure(nc + 1));
    CFA_CUDA(Q.ci.ensure(std::max(Q.nnz, 1)));
    CFA_CUDA(Q.v.ensure(std::max(Q.nnz, 1)));
    CFA_LAUNCH(ctx, k_fuse_q_rp, ceil_div(nc + 1, kThreads), kThreads, 0, nc, (const int*)L.R.rp.p,
               (const int*)S.fRA.rp.p, Q.rp.p);
    CFA_LAUNCH(ctx, k_fuse_q_fill, ceil_div(nc, kThreads), kThreads, 0, nc, (const int*)L.R.rp.p,
               (const int*)L.R.ci.p, (const double*)L.R.v.p, (const int*)S.fRA.rp.p, (const int*)S.fRA.ci.p,
               (const double*)S.fRA.v.p, (const int*)Q.rp.p, Q.ci.p, Q.v.p);
    CFA_PROPAGATE(pack_from_device(ctx, amg, Q, Q.v.p, nullptr, vb, L.tQ));
    if (amg->phase_switch > 0.0 && vb != 8) CFA_PROPAGATE(pack_from_device(ctx, amg, Q, Q.v.p, nullptr, 8, L.tQ64));
    L.fusedQ = true;
    if (!with_w) {
        CFA_CHECK_LAUNCH();
        return CFA_OK;
    }
    // W: count, offsets, fill
    DCsr& W = S.fW;
    CFA_CUDA(S.fcnt.ensure(n + 1));
    CFA_CUDA(W.rp.ensure(n + 1));
    CFA_LAUNCH(ctx, k_fuse_w<false>, ceil_div(n, kThreads), kThreads, 0, n, (const int*)L.A.rp.p, (const int*)L.A.ci.p,
               (const double*)L.A.v.p, (const int*)AP.rp.p, (const int*)AP.ci.p, (const double*)AP.v.p,
               (const int*)L.P.rp.p, (const int*)L.P.ci.p, (const double*)L.P.v.p, S.fcnt.p, (const int*)nullptr,
               (int*)nullptr, (double*)nullptr, (double*)nullptr);
    CFA_CUDA(cudaMemsetAsync(S.fcnt.p + n, 0, sizeof(int), ctx->stream));
    CFA_PROPAGATE(exclusive_sum(ctx, S, S.fcnt.p, W.rp.p, n));
    int total = 0;
    CFA_CUDA(cudaMemcpyAsync(&total, W.rp.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    W.rows = n;
    W.cols = n;
    W.nnz = total;
    CFA_CUDA(W.ci.ensure(std::max(total, 1)));
    CFA_CUDA(W.v.ensure(std::max(total, 1)));
    CFA_CUDA(S.fW1.ensure(std::max(total, 1)));
    CFA_LAUNCH(ctx, k_fuse_w<true>, ceil_div(n, kThreads), kThreads, 0, n, (const int*)L.A.rp.p, (const int*)L.A.ci.p,
               (const double*)L.A.v.p, (const int*)AP.rp.p, (const int*)AP.ci.p, (const double*)AP.v.p,
               (const int*)L.P.rp.p, (const int*)L.P.ci.p, (const double*)L.P.v.p, (int*)nullptr,
               (const int*)W.rp.p, W.ci.p, W.v.p, S.fW1.p);
    CFA_PROPAGATE(pack_from_device(ctx, amg, W, W.v.p, S.fW1.p, vb, L.tW));
    if (amg->phase_switch > 0.0 && vb != 8) CFA_PROPAGATE(pack_from_device(ctx, amg, W, W.v.p, S.fW1.p, 8, L.tW64));
    CFA_CHECK_LAUNCH();
    L.fusedW = true;
    return CFA_OK;
}

// ---- autotuner for the tile heights of the V-cycle's matrices (tiled.cuh) ----
// Mean time of one launch of operation OP on the tiles M (3 untimed launches first), in us.
template <int OP, class V, class T>
static double time_tile_op(cfa_ctx* ctx, const TiledCsr& M, int* err, const T* dinv, const T* b, const T* x, T* y,
                           const T* xc) {
    constexpr int kReps = 10;
    vct<OP, V, T, T, T>(ctx, true, M, err, dinv, (T)0.5, b, x, y, nullptr, nullptr, xc);
    for (int k = 0; k < 3; ++k) vct<OP, V, T, T, T>(ctx, false, M, err, dinv, (T)0.5, b, x, y, nullptr, nullptr, xc);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    for (int k = 0; k < kReps; ++k) vct<OP, V, T, T, T>(ctx, false, M, err, dinv, (T)0.5, b, x, y, nullptr, nullptr, xc);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 1e3 * ms / kReps;
}

// One matrix: the cached choice of its pattern class, or the candidates timed and the fastest
// kept; T is re-planned and re-packed when the choice is not the default height.
template <class V, class T>
static cfa_status tune_one(cfa_ctx* ctx, cfa_amg* amg, const char* kind, int op, const DCsr& M, const double* v0,
                           const double* v1, int vb, TiledCsr& tiles, const T* dinv, T* const* vec) {
    const int nvals = v1 ? 2 : 1;
    HostBuf<int>& hr = amg->scratch.h_rp;
    auto replan = [&](TiledCsr& dst, int shift) -> cfa_status {
        CFA_CUDA(hr.ensure(M.rows + 1));
        CFA_CUDA(cudaMemcpyAsync(hr.p, M.rp.p, (M.rows + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CFA_CUDA(cudaStreamSynchronize(ctx->stream));
        dst.stages = level_tile_stages();
        const cfa_status st = plan_tiled(ctx, hr.p, M.rows, nvals, vb, dst, shift);
        if (st != CFA_OK) return st;
        return pack_tiled(ctx, M.rp.p, M.ci.p, v0, v1, nullptr, dst);
    };
    int best = 0;
    if (!autotune_lookup(kind, vb, nvals, M.rows, M.nnz, &best)) {
        int* err = amg->err.p;
        const int cand[4] = {-2, -1, 0, 1};
        double us[4];
        int shifts[4], nc = 0;
        double best_us = 0.0;
        for (int c : cand) {
            TiledCsr trial;
            const TiledCsr* use = &tiles;
            if (c != 0) {
                if (replan(trial, c) != CFA_OK) continue;
                use = &trial;
            }
            double t = 0.0;
            switch (op) {
                case VC_JAC: t = time_tile_op<VC_JAC, V, T>(ctx, *use, err, dinv, vec[0], vec[1], vec[2], nullptr); break;
                case VC_ADD: t = time_tile_op<VC_ADD, V, T>(ctx, *use, err, dinv, nullptr, vec[3], vec[2], nullptr); break;
                case VC_SPMV: t = time_tile_op<VC_SPMV, V, T>(ctx, *use, err, dinv, nullptr, vec[1], vec[2], nullptr); break;
                case VC_RESTRICT: t = time_tile_op<VC_RESTRICT, V, T>(ctx, *use, err, dinv, vec[0], vec[1], vec[2], nullptr); break;
                default: t = time_tile_op<VC_ADDJAC, V, T>(ctx, *use, err, dinv, vec[0], vec[1], vec[2], vec[3]); break;
            }
            CFA_CHECK_LAUNCH();
            if (nc == 0 || t < best_us) { best_us = t; best = c; }
            us[nc] = t;
            shifts[nc++] = c;
        }
        autotune_store(kind, vb, nvals, M.rows, M.nnz, best, us, shifts, nc);
    }
    if (best != 0) CFA_PROPAGATE(replan(tiles, best));
    return CFA_OK;
}

// The tile heights of a level's matrices whose kernels carry no reduction: every matrix of the
// levels >= 1, and level 0's transfers (level 0's A carries the CG's dots in its last sweep).
template <class V, class T>
static cfa_status tune_level(cfa_ctx* ctx, cfa_amg* amg, AmgLevel& L, int vb) {
    const bool lv0 = &L == &amg->levels[0];
    const int n = L.A.rows, nc = L.R.rows;
    DevBuf<T> buf;
    const size_t len = (size_t)std::max(n, nc) + 1;
    CFA_CUDA(buf.ensure(4 * len));
    CFA_CUDA(cudaMemsetAsync(buf.p, 0, 4 * len * sizeof(T), ctx->stream));
    T* vec[4] = {buf.p, buf.p + len, buf.p + 2 * len, buf.p + 3 * len};   // b, x, y, coarse x
    const T* dinv = std::is_same<T, float>::value ? (const T*)(const void*)L.dinv32.p : (const T*)(const void*)L.dinv.p;
    auto vals = [&](const DCsr& M) { return (const double*)M.v.p; };
    if (!lv0) CFA_PROPAGATE((tune_one<V, T>(ctx, amg, "A", VC_JAC, L.A, vals(L.A), nullptr, vb, L.tA, dinv, vec)));
    SetupScratch& S = amg->scratch;
    if (L.fusedQ) CFA_PROPAGATE((tune_one<V, T>(ctx, amg, "Q", VC_RESTRICT, S.fQ, S.fQ.v.p, nullptr, vb, L.tQ, dinv, vec)));
    else CFA_PROPAGATE((tune_one<V, T>(ctx, amg, "R", VC_SPMV, L.R, vals(L.R), nullptr, vb, L.tR, dinv, vec)));
    if (L.fusedW) CFA_PROPAGATE((tune_one<V, T>(ctx, amg, "W", VC_ADDJAC, S.fW, S.fW.v.p, S.fW1.p, vb, L.tW, dinv, vec)));
    else CFA_PROPAGATE((tune_one<V, T>(ctx, amg, "P", VC_ADD, L.P, vals(L.P), nullptr, vb, L.tP, dinv, vec)));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));   // buf is released on return
    return CFA_OK;
}

// Kernel shapes of one level, its FP32 copies (mixed precision) and its tile-streamed A, P, R in
// the hierarchy precision.
// Relative residual at which a mixed-precision solve's V-cycles switch from FP64 to FP32
// (CFA_FP64_PHASE; 0 keeps them FP32 throughout).
static double fp64_phase_env() {
    const char* e = std::getenv("CFA_FP64_PHASE");
    if (!e || !*e) return 1e-1;
    const double v = std::atof(e);
    return v > 0.0 && v < 1.0 ? v : 0.0;
}

static cfa_status prepare_level(cfa_ctx* ctx, cfa_amg* amg, AmgLevel& L) {
    const cfa_amg_opts& o = amg->opts;
    L.A.tpr = threads_per_row(L.A.rows, L.A.nnz);
    L.P.tpr = threads_per_row(L.P.rows, L.P.nnz);
    L.R.tpr = threads_per_row(L.R.rows, L.R.nnz);
    if (o.precision == CFA_MIXED) {
        CFA_PROPAGATE(to_float(ctx, L.A));
        CFA_PROPAGATE(to_float(ctx, L.P));
        CFA_PROPAGATE(to_float(ctx, L.R));
        CFA_CUDA(L.dinv32.ensure(L.A.rows));
        CFA_LAUNCH(ctx, k_to_float, std::min(ceil_div(L.A.rows, kThreads), 8 * ctx->num_sms), kThreads, 0,
                   (long long)L.A.rows, L.dinv.p, L.dinv32.p);
    }
    CFA_CHECK_LAUNCH();
    if (!amg->tiled) return CFA_OK;
    const int vb = o.precision == CFA_MIXED ? 4 : 8;
    L.fusedQ = L.fusedW = false;
    // levels the composite operator replaces run no tile kernel
    const int l = (int)(&L - &amg->levels[0]);
    if (amg->comp_level >= 0 && l >= amg->comp_level) {
        if (o.precision == CFA_MIXED) CFA_PROPAGATE(level_vectors(ctx, amg, L, L.A.rows));
        return level_vectors64(ctx, L, L.A.rows);
    }
    if (fuse_level(amg, L)) CFA_PROPAGATE(build_fused(ctx, amg, L, vb, fuse_prolongation(amg, L)));
    for (DCsr* M : {&L.A, &L.P, &L.R}) {
        TiledCsr& T = M == &L.A ? L.tA : M == &L.P ? L.tP : L.tR;
        HostBuf<int>& hr = amg->scratch.h_rp;
        CFA_CUDA(hr.ensure(M->rows + 1));
        CFA_CUDA(cudaMemcpyAsync(hr.p, M->rp.p, (M->rows + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CFA_CUDA(cudaStreamSynchronize(ctx->stream));
        T.stages = level_tile_stages();
        CFA_PROPAGATE(plan_tiled(ctx, hr.p, M->rows, 1, vb, T));
        CFA_PROPAGATE(pack_tiled(ctx, M->rp.p, M->ci.p, M->v.p, nullptr, nullptr, T));
        if (amg->phase_switch > 0.0) {   // the FP64 copy for the solves' FP64 phase
            TiledCsr& T64 = M == &L.A ? L.tA64 : M == &L.P ? L.tP64 : L.tR64;
            T64.stages = level_tile_stages();
            CFA_PROPAGATE(plan_tiled(ctx, hr.p, M->rows, 1, 8, T64));
            CFA_PROPAGATE(pack_tiled(ctx, M->rp.p, M->ci.p, M->v.p, nullptr, nullptr, T64));
        }
    }
    if (o.precision == CFA_MIXED) CFA_PROPAGATE(level_vectors(ctx, amg, L, L.A.rows));   // FP32 V-cycle vectors
    CFA_PROPAGATE(level_vectors64(ctx, L, L.A.rows));
    if (autotune_enabled()) {
        if (o.precision != CFA_MIXED) CFA_PROPAGATE((tune_level<double, double>(ctx, amg, L, vb)));
        else if (vcycle_fp32(amg)) CFA_PROPAGATE((tune_level<float, float>(ctx, amg, L, vb)));
        else CFA_PROPAGATE((tune_level<float, double>(ctx, amg, L, vb)));
    }
    return CFA_OK;
}

// The V-cycle's coarse tail plan, and the kernels' shared-memory limits raised now, outside any
// stream capture (a dry V-cycle).
static cfa_status prepare_vcycle(cfa_ctx* ctx, cfa_amg* amg) {
    if (!amg->tiled) return CFA_OK;
    CFA_PROPAGATE(plan_tail(ctx, amg));
    vcycle_tiled_top(ctx, amg, nullptr, nullptr, nullptr, true);
    if (amg->phase_switch > 0.0) vcycle_tiled_top(ctx, amg, nullptr, nullptr, nullptr, true, nullptr, nullptr, nullptr, true);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

// Largest level (rows) whose V-cycle below is formed as one dense operator (CFA_COMPOSITE_ROWS
// overrides; 0: never). At 2048 rows the FP64 matrix is 32 MB, read in about the time of one
// dependent launch of the chain it replaces.
static int composite_rows(const cfa_amg* amg) {
    if (amg->vc_composite_rows >= 0) return amg->vc_composite_rows;
    const char* e = std::getenv("CFA_COMPOSITE_ROWS");
    return e ? std::atoi(e) : 2048;
}

// Forms the composite of the first level l >= 1 with at most composite_rows() rows (the V-cycle's
// level 0 keeps its kernels: its last sweep carries the CG's dots). Runs the V-cycle's operations
// of levels l.. on the identity block in FP64, in the order of vcycle_tiled.
static cfa_status build_composite(cfa_ctx* ctx, cfa_amg* amg) {
    amg->comp_level = -1;
    amg->comp_n = 0;
    const int limit = composite_rows(amg);
    const int L = (int)amg->levels.size();
    int lc = -1;
    for (int l = 1; l < L; ++l)
        if (amg->levels[l].A.rows <= limit) { lc = l; break; }
    if (lc < 0) return CFA_OK;
    const int nb = amg->levels[lc].A.rows;
    const int s = amg->opts.smooth_steps;
    // per level k >= lc: right-hand sides, iterate, scratch, residual (rows(k) x nb); coarse pair
    std::vector<DevBuf<double>> blk(4 * (L - lc) + 2);
    for (int k = lc; k < L; ++k)
        for (int q = 0; q < 4; ++q) CFA_CUDA(blk[4 * (k - lc) + q].ensure((size_t)amg->levels[k].A.rows * nb));
    const int cn = amg->coarse_n;
    CFA_CUDA(blk[4 * (L - lc)].ensure((size_t)cn * nb));
    CFA_CUDA(blk[4 * (L - lc) + 1].ensure((size_t)cn * nb));
    auto grid = [&](long long entries) { return ceil_div(entries, kThreads); };
    CFA_LAUNCH(ctx, k_bm_eye, grid((long long)nb * nb), kThreads, 0, nb, blk[0].p);
    // the V-cycle of level k on the block in blk[4(k - lc)]; returns the block holding its result
    std::function<double*(int)> level = [&](int k) -> double* {
        AmgLevel& Lk = amg->levels[k];
        const int m = Lk.A.rows;
        const long long me = (long long)m * nb;
        double* B = blk[4 * (k - lc)].p;
        double* X = blk[4 * (k - lc) + 1].p;
        double* T = blk[4 * (k - lc) + 2].p;
        double* Rr = blk[4 * (k - lc) + 3].p;
        const DCsr& A = Lk.A;
        CFA_LAUNCH(ctx, k_bm<BM_PRE>, grid(me), kThreads, 0, m, nb, A.rp.p, A.ci.p, A.v.p, Lk.dinv.p, Lk.omega,
                   s >= 2 ? 1 : 0, (const double*)B, (const double*)nullptr, X);
        for (int q = 2; q < s; ++q) {
            CFA_LAUNCH(ctx, k_bm<BM_JAC>, grid(me), kThreads, 0, m, nb, A.rp.p, A.ci.p, A.v.p, Lk.dinv.p, Lk.omega, 0,
                       (const double*)B, (const double*)X, T);
            std::swap(X, T);
        }
        CFA_LAUNCH(ctx, k_bm<BM_RES>, grid(me), kThreads, 0, m, nb, A.rp.p, A.ci.p, A.v.p, Lk.dinv.p, Lk.omega, 0,
                   (const double*)B, (const double*)X, Rr);
        const bool last = k + 1 == L;
        const int mc = Lk.R.rows;
        double* Bc = last ? blk[4 * (L - lc)].p : blk[4 * (k + 1 - lc)].p;
        CFA_LAUNCH(ctx, k_bm<BM_SPMV>, grid((long long)mc * nb), kThreads, 0, mc, nb, Lk.R.rp.p, Lk.R.ci.p,
                   Lk.R.v.p, (const double*)nullptr, 0.0, 0, (const double*)nullptr, (const double*)Rr, Bc);
        const double* Xc;
        if (last) {
            double* Xd = blk[4 * (L - lc) + 1].p;
            CFA_LAUNCH(ctx, k_bm_dense, grid((long long)cn * nb), kThreads, 0, cn, nb,
                       (const double*)amg->coarse_inv.p, (const double*)Bc, Xd);
            Xc = Xd;
        } else {
            Xc = level(k + 1);
        }
        CFA_LAUNCH(ctx, k_bm<BM_ADD>, grid(me), kThreads, 0, m, nb, Lk.P.rp.p, Lk.P.ci.p, Lk.P.v.p,
                   (const double*)nullptr, 0.0, 0, (const double*)nullptr, Xc, X);
        for (int q = 0; q < s; ++q) {
            CFA_LAUNCH(ctx, k_bm<BM_JAC>, grid(me), kThreads, 0, m, nb, A.rp.p, A.ci.p, A.v.p, Lk.dinv.p, Lk.omega, 0,
                       (const double*)B, (const double*)X, T);
            std::swap(X, T);
        }
        return X;
    };
    const double* M = level(lc);
    CFA_CUDA(amg->comp.ensure((size_t)nb * nb));
    CFA_CUDA(cudaMemcpyAsync(amg->comp.p, M, (size_t)nb * nb * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CFA_CHECK_LAUNCH();
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));   // the blocks are released on return
    amg->comp_level = lc;
    amg->comp_n = nb;
    return CFA_OK;
}

static cfa_status amg_setup(cfa_ctx* ctx, cfa_amg* amg, int n, int nnz, const int* d_rp, const int* d_ci,
                            const double* d_v) {
    const auto t0 = std::chrono::steady_clock::now();
    auto tp = t0;
    auto phase = [&](int ph) {
        cudaStreamSynchronize(ctx->stream);
        const auto now = std::chrono::steady_clock::now();
        amg->phase_ms[ph] += std::chrono::duration<double, std::milli>(now - tp).count();
        tp = now;
    };
    const cfa_amg_opts& o = amg->opts;
    // the previous hierarchy's levels are recycled: their buffers only grow (the reference keeps
    // them as `spare`, src/cfa/linalg.cuh:964, :1266-1272)
    std::vector<AmgLevel> pool = std::move(amg->levels);
    amg->levels.clear();
    auto take = [&](size_t l) {
        AmgLevel L;
        if (l < pool.size()) L = std::move(pool[l]);
        else if (l == pool.size() && amg->coarse_holder.A.rp.p) L.A = std::move(amg->coarse_holder.A);
        return L;
    };
    amg->version = next_uid();
    AmgLevel cur = take(0);
    CFA_PROPAGATE(copy_csr(ctx, n, nnz, d_rp, d_ci, d_v, cur.A));
    phase(0);
    for (;;) {
        DCsr& A = cur.A;
        if (!(A.rows > o.coarse_target && (int)amg->levels.size() < o.max_levels - 1)) break;
        const int m = A.rows;
        AmgLevel& L = cur;
        CFA_CUDA(L.dinv.ensure(m));
        CFA_LAUNCH(ctx, k_amg_dinv, ceil_div(m, kThreads), kThreads, 0, m, A.rp.p, A.ci.p, A.v.p, L.dinv.p);
        double rho = 1.0;
        CFA_PROPAGATE(spectral_radius(ctx, amg, A, L.dinv.p, &rho));
        const double omega = 4.0 / (3.0 * rho);
        phase(1);
        // strength on the device; aggregation by the sequential host loop or the device rounds
        SetupScratch& S = amg->scratch;
        CFA_CUDA(S.strong.ensure(std::max(A.nnz, 1)));
        CFA_LAUNCH(ctx, k_strength, ceil_div(m, kThreads), kThreads, 0, m, A.rp.p, A.ci.p, A.v.p, L.dinv.p, o.theta,
                   S.strong.p);
        CFA_CUDA(L.agg.ensure(m));
        int na = 0;
        if (!agg_on_host(amg)) {
            CFA_PROPAGATE(aggregate_device(ctx, S, A, L.agg.p, &na));
            if (na >= (int)(0.85 * m) || na == 0) break;   // coarsening stalled (:1019)
        } else {
            CFA_CUDA(S.h_rp.ensure(m + 1));
            CFA_CUDA(S.h_ci.ensure(std::max(A.nnz, 1)));
            CFA_CUDA(S.h_strong.ensure(std::max(A.nnz, 1)));
            CFA_CUDA(cudaMemcpyAsync(S.h_rp.p, A.rp.p, (m + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            CFA_CUDA(cudaMemcpyAsync(S.h_ci.p, A.ci.p, (size_t)A.nnz * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            CFA_CUDA(cudaMemcpyAsync(S.h_strong.p, S.strong.p, (size_t)A.nnz, cudaMemcpyDeviceToHost, ctx->stream));
            CFA_CUDA(cudaStreamSynchronize(ctx->stream));
            CFA_CUDA(S.h_agg.ensure(m));
            na = aggregate_host(m, S.h_rp.p, S.h_ci.p, S.h_strong.p, S.h_agg.p);
            if (na >= (int)(0.85 * m) || na == 0) break;   // coarsening stalled (:1019)
            const int* agg = S.h_agg.p;
            std::vector<int> size(na, 0);
            for (int i = 0; i < m; ++i) size[agg[i]]++;
            CFA_CUDA(S.h_p0v.ensure(m));
            CFA_CUDA(S.h_p0rp.ensure(m + 1));
            for (int i = 0; i < m; ++i) { S.h_p0v.p[i] = 1.0 / std::sqrt((double)size[agg[i]]); S.h_p0rp.p[i] = i; }
            S.h_p0rp.p[m] = m;
            CFA_CUDA(S.p0v.ensure(m));
            CFA_CUDA(S.p0rp.ensure(m + 1));
            CFA_CUDA(cudaMemcpyAsync(L.agg.p, agg, m * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
            CFA_CUDA(cudaMemcpyAsync(S.p0v.p, S.h_p0v.p, m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            CFA_CUDA(cudaMemcpyAsync(S.p0rp.p, S.h_p0rp.p, (m + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        }
        DevBuf<double>& d_p0v = S.p0v;
        DevBuf<int>& d_p0rp = S.p0rp;
        phase(2);
        // AP0 = A P0, then P = P0 - omega D^-1 A P0
        DCsr& AP0 = S.AP0;
        CFA_PROPAGATE(spgemm(ctx, S, m, na, A.rp.p, A.ci.p, A.v.p, d_p0rp.p, L.agg.p, d_p0v.p, AP0));
        DevBuf<int>& cnt = S.cnt;
        CFA_CUDA(cnt.ensure(m));
        CFA_LAUNCH(ctx, k_p_rows, ceil_div(m, kThreads), kThreads, 0, m, AP0.rp.p, AP0.ci.p, AP0.v.p, L.agg.p, d_p0v.p,
                   L.dinv.p, omega, (const int*)nullptr, (int*)nullptr, (double*)nullptr, cnt.p);
        CFA_CUDA(S.h_cnt.ensure(m));
        CFA_CUDA(S.h_rp.ensure(m + 1));
        CFA_CUDA(cudaMemcpyAsync(S.h_cnt.p, cnt.p, m * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CFA_CUDA(cudaStreamSynchronize(ctx->stream));
        int* h_prp = S.h_rp.p;
        h_prp[0] = 0;
        for (int i = 0; i < m; ++i) h_prp[i + 1] = h_prp[i] + S.h_cnt.p[i];
        L.P.rows = m;
        L.P.cols = na;
        L.P.nnz = h_prp[m];
        CFA_CUDA(L.P.rp.ensure(m + 1));
        CFA_CUDA(L.P.ci.ensure(std::max(L.P.nnz, 1)));
        CFA_CUDA(L.P.v.ensure(std::max(L.P.nnz, 1)));
        CFA_CUDA(cudaMemcpyAsync(L.P.rp.p, h_prp, (m + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        CFA_LAUNCH(ctx, k_p_rows, ceil_div(m, kThreads), kThreads, 0, m, AP0.rp.p, AP0.ci.p, AP0.v.p, L.agg.p, d_p0v.p,
                   L.dinv.p, omega, L.P.rp.p, L.P.ci.p, L.P.v.p, cnt.p);
        CFA_CHECK_LAUNCH();
        phase(3);
        // R = P^T, A_c = R (A P)
        CFA_PROPAGATE(transpose(ctx, S, L.P, L.R));
        phase(4);
        AmgLevel next = take(amg->levels.size() + 1);
        DCsr& AP = S.AP;
        CFA_PROPAGATE(spgemm(ctx, S, m, na, A.rp.p, A.ci.p, A.v.p, L.P.rp.p, L.P.ci.p, L.P.v.p, AP));
        CFA_PROPAGATE(spgemm(ctx, S, na, na, L.R.rp.p, L.R.ci.p, L.R.v.p, AP.rp.p, AP.ci.p, AP.v.p, next.A));
        std::swap(L.AP, S.AP);   // kept for the level's fused transfers
        phase(5);
        L.omega = omega;
        CFA_PROPAGATE(level_vectors(ctx, amg, L, m));
        amg->levels.push_back(std::move(cur));
        cur = std::move(next);
    }
    // coarsest level: dense Cholesky inverse on the device
    amg->coarse_holder = std::move(cur);
    DCsr& A = amg->coarse_holder.A;
    const int cn = A.rows;
    amg->coarse_n = cn;
    DevBuf<double>& M = amg->scratch.M;
    DevBuf<double>& colbuf = amg->scratch.colbuf;
    DevBuf<int>& err = amg->scratch.ierr;
    CFA_CUDA(M.ensure((size_t)cn * cn + 1));
    CFA_CUDA(colbuf.ensure((size_t)cn * cn + 1));
    CFA_CUDA(amg->coarse_inv.ensure((size_t)cn * cn + 1));
    CFA_CUDA(err.ensure(1));
    CFA_LAUNCH(ctx, k_dense_build, ceil_div(cn, 64), 64, 0, cn, A.rp.p, A.ci.p, A.v.p, M.p);
    if (coarse_blocked(cn)) {
        static std::once_flag coarse_once;
        std::call_once(coarse_once, [] {
            cudaFuncSetAttribute(k_coarse_cholesky, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmemMax);
            cudaFuncSetAttribute(k_coarse_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmemMax);
        });
        CFA_LAUNCH(ctx, k_coarse_cholesky, 1, kCholThreads, chol_smem(cn), cn, M.p, colbuf.p, err.p);
        CFA_LAUNCH(ctx, k_coarse_inverse, ceil_div(cn, kInvCols), kInvCols, inv_smem(cn), cn, (const double*)M.p,
                   (const double*)colbuf.p, amg->coarse_inv.p);
    } else {   // coarsest levels beyond the shared-memory panels (cn > ~770): one column per step
        CFA_LAUNCH(ctx, k_cholesky, 1, 256, 0, cn, M.p, err.p);
        CFA_LAUNCH(ctx, k_chol_inverse, ceil_div(cn, 32), 32, 0, cn, M.p, amg->coarse_inv.p, colbuf.p);
    }
    CFA_CHECK_LAUNCH();
    int h_err = 0;
    CFA_CUDA(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_PROPAGATE(build_composite(ctx, amg));
    phase(7);
    CFA_CUDA(amg->cb64.ensure(cn + 1));
    CFA_CUDA(amg->cx64.ensure(cn + 1));
    if (o.precision == CFA_MIXED) {
        CFA_CUDA(amg->cb32.ensure(cn + 1));
        CFA_CUDA(amg->cx32.ensure(cn + 1));
    }
    // precision, kernel shapes and tile-streamed copies of the V-cycle
    const char* te = std::getenv("CFA_TILES");
    amg->tiled = !(te && te[0] == '0') && !amg->levels.empty();
    amg->phase_switch = !(amg->tiled && o.precision == CFA_MIXED) ? 0.0
                        : amg->vc_fp64_phase >= 0.0                  ? amg->vc_fp64_phase
                                                                     : fp64_phase_env();
    if (amg->tiled) {
        CFA_CUDA(amg->err.ensure(1));
        CFA_CUDA(cudaMemsetAsync(amg->err.p, 0, sizeof(int), ctx->stream));
    }
    static const bool setup_log = [] {
        const char* e = std::getenv("CFA_SETUP_LOG");
        return e && e[0] == '1';
    }();
    for (AmgLevel& L : amg->levels) {
        const auto t0l = std::chrono::steady_clock::now();
        CFA_PROPAGATE(prepare_level(ctx, amg, L));
        if (setup_log) {
            cudaStreamSynchronize(ctx->stream);
            fprintf(stderr, "[cfa setup] level %d: rows %d, tiles/fused %.3f ms (fusedQ %d, fusedW %d, R A by %s)\n",
                    (int)(&L - &amg->levels[0]), L.A.rows,
                    std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0l).count(),
                    (int)L.fusedQ, (int)L.fusedW, L.ra_spgemm ? "SpGEMM" : "transpose");
        }
    }
    {
        const auto t0v = std::chrono::steady_clock::now();
        CFA_PROPAGATE(prepare_vcycle(ctx, amg));
        if (setup_log) {
            cudaStreamSynchronize(ctx->stream);
            fprintf(stderr, "[cfa setup] prepare_vcycle %.3f ms\n",
                    std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0v).count());
        }
    }
    phase(6);
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    amg->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (h_err) return set_error(ctx, CFA_COARSE_NOT_SPD, "coarsest AMG operator not SPD", __FILE__, __LINE__);
    return CFA_OK;
}

}  // namespace cfa

using namespace cfa;

// AmgPreconditioner::remap (src/cfa/linalg.cuh:1074-1157). The prolongator of a new node is the
// mean of the rows of its graph neighbours that already have one, built pass by pass outwards on
// the host in node order (the reference's host algorithm; equal columns are summed in the order
// they were gathered, a stable sort), uploaded, transposed on the device in the setup's exact
// order; level 0 takes the new operator and its inverse diagonal. remapped = false when it set
// the hierarchy up anew instead (no levels, or new nodes none of whose neighbours has a row).
static cfa_status amg_remap(cfa_ctx* ctx, cfa_amg* amg, int n, int nnz, const int* d_rp, const int* d_ci,
                            const double* d_v, const int* h_rp, const int* h_ci, const int* n2o, bool& remapped) {
    remapped = false;
    if (amg->levels.empty()) return amg_setup(ctx, amg, n, nnz, d_rp, d_ci, d_v);
    const auto t0 = std::chrono::steady_clock::now();
    AmgLevel& L = amg->levels[0];
    const int old_rows = L.P.rows;
    for (int i = 0; i < n; ++i)
        if (n2o[i] < -1 || n2o[i] >= old_rows)
            return set_error(ctx, CFA_BAD_ARG, "new_to_old entry outside the old level-0 rows", __FILE__, __LINE__);
    // the current level-0 prolongator on the host
    std::vector<int> prp(old_rows + 1), pci(std::max(L.P.nnz, 1));
    std::vector<double> pv(std::max(L.P.nnz, 1));
    CFA_CUDA(cudaMemcpyAsync(prp.data(), L.P.rp.p, (old_rows + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(pci.data(), L.P.ci.p, (size_t)L.P.nnz * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(pv.data(), L.P.v.p, (size_t)L.P.nnz * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    // rows of new nodes, pass by pass from neighbours set in earlier passes
    std::vector<int> extra_of(n, -1), ex_rp(1, 0), pending, still, set_now;
    std::vector<std::pair<int, double>> ex, acc;
    std::vector<char> has_row(n);
    for (int i = 0; i < n; ++i) {
        has_row[i] = n2o[i] >= 0;
        if (n2o[i] < 0) pending.push_back(i);
    }
    while (!pending.empty()) {
        still.clear();
        set_now.clear();
        for (int i : pending) {
            acc.clear();
            int cnt = 0;
            for (int a = h_rp[i]; a < h_rp[i + 1]; ++a) {
                const int k = h_ci[a];
                if (k == i || !has_row[k]) continue;
                ++cnt;
                if (n2o[k] >= 0) {
                    const int j = n2o[k];
                    for (int b = prp[j]; b < prp[j + 1]; ++b) acc.push_back({pci[b], pv[b]});
                } else {
                    for (int b = ex_rp[extra_of[k]]; b < ex_rp[extra_of[k] + 1]; ++b) acc.push_back(ex[b]);
                }
            }
            if (cnt == 0) { still.push_back(i); continue; }
            std::stable_sort(acc.begin(), acc.end(),
                             [](const std::pair<int, double>& x, const std::pair<int, double>& y) { return x.first < y.first; });
            const size_t row0 = ex.size();
            for (const auto& e : acc) {
                if (ex.size() > row0 && ex.back().first == e.first) ex.back().second += e.second;
                else ex.push_back(e);
            }
            for (size_t q = row0; q < ex.size(); ++q) ex[q].second /= cnt;
            extra_of[i] = (int)ex_rp.size() - 1;
            ex_rp.push_back((int)ex.size());
            set_now.push_back(i);
        }
        if (set_now.empty()) return amg_setup(ctx, amg, n, nnz, d_rp, d_ci, d_v);   // isolated new nodes
        for (int i : set_now) has_row[i] = 1;
        pending.swap(still);
    }
    std::vector<int> nrp(n + 1, 0);
    for (int i = 0; i < n; ++i)
        nrp[i + 1] = nrp[i] + (n2o[i] >= 0 ? prp[n2o[i] + 1] - prp[n2o[i]] : ex_rp[extra_of[i] + 1] - ex_rp[extra_of[i]]);
    const int pnnz = nrp[n];
    std::vector<int> nci(std::max(pnnz, 1));
    std::vector<double> nv(std::max(pnnz, 1));
    for (int i = 0; i < n; ++i) {
        int o = nrp[i];
        if (n2o[i] >= 0) {
            for (int b = prp[n2o[i]]; b < prp[n2o[i] + 1]; ++b, ++o) { nci[o] = pci[b]; nv[o] = pv[b]; }
        } else {
            for (int b = ex_rp[extra_of[i]]; b < ex_rp[extra_of[i] + 1]; ++b, ++o) { nci[o] = ex[b].first; nv[o] = ex[b].second; }
        }
    }
    // level 0: new operator, inverse diagonal, P (uploaded), R = P^T
    amg->version = next_uid();
    L.AP.rows = 0;   // A P of the old level 0 no longer holds
    L.P.rows = n;
    L.P.nnz = pnnz;
    CFA_CUDA(L.P.rp.ensure(n + 1));
    CFA_CUDA(L.P.ci.ensure(std::max(pnnz, 1)));
    CFA_CUDA(L.P.v.ensure(std::max(pnnz, 1)));
    CFA_CUDA(cudaMemcpyAsync(L.P.rp.p, nrp.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(L.P.ci.p, nci.data(), (size_t)pnnz * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(L.P.v.p, nv.data(), (size_t)pnnz * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CFA_PROPAGATE(transpose(ctx, amg->scratch, L.P, L.R));
    CFA_PROPAGATE(copy_csr(ctx, n, nnz, d_rp, d_ci, d_v, L.A));
    CFA_CUDA(L.dinv.ensure(n));
    CFA_LAUNCH(ctx, k_amg_dinv, ceil_div(n, kThreads), kThreads, 0, n, L.A.rp.p, L.A.ci.p, L.A.v.p, L.dinv.p);
    CFA_CUDA(L.agg.ensure(n));
    CFA_CUDA(cudaMemsetAsync(L.agg.p, 0xff, (size_t)n * sizeof(int), ctx->stream));   // no aggregates after a remap
    CFA_PROPAGATE(level_vectors(ctx, amg, L, n));
    if (amg->tiled) CFA_CUDA(cudaMemsetAsync(amg->err.p, 0, sizeof(int), ctx->stream));
    CFA_PROPAGATE(prepare_level(ctx, amg, L));
    CFA_PROPAGATE(prepare_vcycle(ctx, amg));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    amg->remaps++;
    amg->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    remapped = true;
    return CFA_OK;
}

extern "C" {

void cfa_amg_default_opts(cfa_amg_opts* o) {
    if (!o) return;
    o->theta = 0.08;
    o->smooth_steps = 2;
    o->coarse_target = 300;
    o->max_levels = 15;
    o->precision = CFA_FP64;
}

cfa_status cfa_amg_create(cfa_ctx* ctx, const cfa_amg_opts* opts, cfa_amg** out) {
    if (!out) return CFA_BAD_ARG;
    CFA_ENTER(ctx);
    auto* a = new cfa_amg();
    if (opts) a->opts = *opts; else cfa_amg_default_opts(&a->opts);
    if (a->opts.smooth_steps < 1 || a->opts.max_levels < 1 ||
        (a->opts.precision != CFA_FP64 && a->opts.precision != CFA_MIXED)) {
        delete a;
        return set_error(ctx, CFA_BAD_ARG, "bad AMG options", __FILE__, __LINE__);
    }
    *out = a;
    return CFA_OK;
}

cfa_status cfa_amg_destroy(cfa_amg* amg) {
    delete amg;
    return CFA_OK;
}

cfa_status cfa_amg_setup(cfa_ctx* ctx, cfa_amg* amg, int n, int nnz, const int* rp, const int* ci, const double* v) {
    CFA_ENTER(ctx);
    CFA_ARG(amg && n > 0 && nnz > 0 && rp && ci && v);
    return amg_setup(ctx, amg, n, nnz, rp, ci, v);
}

cfa_status cfa_amg_remap(cfa_ctx* ctx, cfa_amg* amg, int n, int nnz, const int* rp, const int* ci, const double* v,
                         const int* h_rp, const int* h_ci, const int* h_new_to_old) {
    CFA_ENTER(ctx);
    CFA_ARG(amg && n > 0 && nnz > 0 && rp && ci && v && h_rp && h_ci && h_new_to_old);
    bool remapped = false;
    return amg_remap(ctx, amg, n, nnz, rp, ci, v, h_rp, h_ci, h_new_to_old, remapped);
}

int cfa_amg_remaps(const cfa_amg* amg) { return amg ? amg->remaps : 0; }

cfa_status cfa_amg_apply(cfa_ctx* ctx, cfa_amg* amg, const double* r, double* z) {
    CFA_ENTER(ctx);
    CFA_ARG(amg && r && z && amg->coarse_n > 0);
    return amg_vcycle(ctx, amg, r, z, nullptr);
}

cfa_status cfa_amg_info(const cfa_amg* amg, int* num_levels, int* coarse_n, double* setup_ms) {
    if (!amg) return CFA_BAD_ARG;
    if (num_levels) *num_levels = (int)amg->levels.size() + 1;
    if (coarse_n) *coarse_n = amg->coarse_n;
    if (setup_ms) *setup_ms = amg->setup_ms;
    return CFA_OK;
}

cfa_status cfa_amg_level(const cfa_amg* amg, int l, int* info, const int** agg, const int** Arp, const int** Aci,
                         const double** Av, const int** Prp, const int** Pci, const double** Pv, const int** Rrp,
                         const int** Rci, const double** Rv, double* omega) {
    if (!amg || l < 0 || l >= (int)amg->levels.size()) return CFA_BAD_ARG;
    const AmgLevel& L = amg->levels[l];
    if (info) { info[0] = L.A.rows; info[1] = L.A.nnz; info[2] = L.P.cols; info[3] = L.P.nnz; info[4] = L.R.nnz; }
    if (agg) *agg = L.agg.p;
    if (Arp) *Arp = L.A.rp.p;
    if (Aci) *Aci = L.A.ci.p;
    if (Av) *Av = L.A.v.p;
    if (Prp) *Prp = L.P.rp.p;
    if (Pci) *Pci = L.P.ci.p;
    if (Pv) *Pv = L.P.v.p;
    if (Rrp) *Rrp = L.R.rp.p;
    if (Rci) *Rci = L.R.ci.p;
    if (Rv) *Rv = L.R.v.p;
    if (omega) *omega = L.omega;
    return CFA_OK;
}

cfa_status cfa_amg_phases(const cfa_amg* amg, double* ms8) {
    if (!amg || !ms8) return CFA_BAD_ARG;
    for (int k = 0; k < 8; ++k) ms8[k] = amg->phase_ms[k];
    return CFA_OK;
}

cfa_status cfa_amg_coarse_inverse(const cfa_amg* amg, const double** inv) {
    if (!amg || !inv) return CFA_BAD_ARG;
    *inv = amg->coarse_inv.p;
    return CFA_OK;
}

cfa_status cfa_amg_set_vcycle(cfa_amg* amg, int composite_rows, int fuse_levels, int fold_rows) {
    if (!amg || fuse_levels > 2) return CFA_BAD_ARG;
    amg->vc_composite_rows = composite_rows < 0 ? -1 : composite_rows;
    amg->vc_fuse = fuse_levels < 0 ? -1 : fuse_levels;
    amg->vc_fold_rows = fold_rows < 0 ? -1 : fold_rows;
    return CFA_OK;
}

cfa_status cfa_amg_set_aggregation(cfa_amg* amg, int on_device) {
    if (!amg || on_device > 1) return CFA_BAD_ARG;
    amg->vc_agg_device = on_device < 0 ? -1 : on_device;
    return CFA_OK;
}

cfa_status cfa_amg_set_fp64_phase(cfa_amg* amg, double switch_rel) {
    if (!amg || !(switch_rel < 1.0)) return CFA_BAD_ARG;
    amg->vc_fp64_phase = switch_rel < 0.0 ? -1.0 : switch_rel;
    return CFA_OK;
}

cfa_status cfa_amg_composite(const cfa_amg* amg, int* level, int* rows, const double** m) {
    if (!amg) return CFA_BAD_ARG;
    if (level) *level = amg->comp_level;
    if (rows) *rows = amg->comp_n;
    if (m) *m = amg->comp_level >= 0 ? amg->comp.p : nullptr;
    return CFA_OK;
}

}  // extern "C"
