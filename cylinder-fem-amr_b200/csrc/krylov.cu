// Krylov solvers with every scalar on the device.
//
// The reference drives PCG and BiCGSTAB from the host and copies each dot product back, with a
// blocking D2H copy per dot (3 per CG iteration, 4 per BiCGSTAB2 iteration; src/cfa/linalg.cuh:
// 172-177, :674-679). Here each dot product is fused into the kernel that produces its operand:
// every block publishes fixed-order partials, the last block to finish sums them in a fixed
// order and computes the recurrence scalars (alpha, beta, omega, stopping flags) into a state
// struct in device memory that the following kernels read. A solve is one CUDA graph: the
// initialisation kernels followed by a conditional WHILE node whose body is one iteration; the
// body's kernels clear the condition when the solve stops, so the loop runs on the device with
// no host round trip. Results are deterministic run to run.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <cstdlib>
#include <mutex>

#include "amg.cuh"
#include "ilu.cuh"
#include "mesh.cuh"
#include "tiled.cuh"

namespace cfa {

// =============================================================================================
// shared pieces
// =============================================================================================

#define ROWS_BEGIN(TPR, n)                                                                        \
    {                                                                                             \
        const int lane = threadIdx.x % (TPR);                                                     \
        const int gw_ = (blockIdx.x * blockDim.x + threadIdx.x) / 32;                             \
        const int nw_ = gridDim.x * blockDim.x / 32;                                              \
        constexpr int rpw_ = 32 / (TPR);                                                          \
        for (int base_ = gw_ * rpw_; base_ < (n); base_ += nw_ * rpw_) {                          \
            const int row = base_ + (threadIdx.x & 31) / (TPR);                                   \
            const bool valid = row < (n);

#define ROWS_END \
        }        \
    }

template <int TPR>
__device__ __forceinline__ double group_reduce(double s) {
#pragma unroll
    for (int o = TPR / 2; o > 0; o /= 2) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    return s;
}

// plain SpMV (k_spmv_csr / k_spmv_csr_multi semantics), NR right-hand sides of stride n
template <int TPR, int NR>
__global__ void k_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ val,
                       const double* __restrict__ x, double* __restrict__ y) {
    CFA_GRID_DEP();
    ROWS_BEGIN(TPR, n)
    double s[NR];
#pragma unroll
    for (int c = 0; c < NR; ++c) s[c] = 0.0;
    if (valid)
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
            const double a = val[k];
            const int j = ci[k];
#pragma unroll
            for (int c = 0; c < NR; ++c) s[c] += a * x[(size_t)c * n + j];
        }
#pragma unroll
    for (int c = 0; c < NR; ++c) s[c] = group_reduce<TPR>(s[c]);
    if (valid && lane == 0)
#pragma unroll
        for (int c = 0; c < NR; ++c) y[(size_t)c * n + row] = s[c];
    ROWS_END
}

// Operator pass 1 (OSS only): pn = z + beta p (beta NULL: pn = z), g = M_L^-1 B pn (k_oss_apply_B,
// src/cfa/fem_kernels.cuh:855-868), pn written for the own row when p_new != NULL.
template <int TPR>
__global__ void k_op_b(int n, int nnz, const int* __restrict__ rp, const int* __restrict__ ci,
                       const double* __restrict__ oss, const double* __restrict__ inv_m, const double* __restrict__ z,
                       const double* __restrict__ p, const double* __restrict__ beta_ptr, double* __restrict__ p_new,
                       double* __restrict__ gx, double* __restrict__ gy, const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    const double beta = beta_ptr ? *beta_ptr : 0.0;
    const double* Bx = oss;
    const double* By = oss + nnz;
    ROWS_BEGIN(TPR, n)
    double sx = 0.0, sy = 0.0;
    if (valid)
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
            const int j = ci[k];
            const double pj = beta_ptr ? z[j] + beta * p[j] : z[j];
            sx += Bx[k] * pj;
            sy += By[k] * pj;
        }
    sx = group_reduce<TPR>(sx);
    sy = group_reduce<TPR>(sy);
    if (valid && lane == 0) {
        const double im = inv_m[row];
        gx[row] = sx * im;
        gy[row] = sy * im;
        if (p_new) p_new[row] = beta_ptr ? z[row] + beta * p[row] : z[row];
    }
    ROWS_END
}

// CG state (all on the device)

// Operator pass 2: q = K pn - [not Dirichlet] (B^T_x g_x + B^T_y g_y) (k_spmv_csr + k_oss_apply_BT,
// src/cfa/fem_kernels.cuh:871-885). FUSEP: pn = z + beta p computed on the fly (no OSS pass 1),
// written to p_new for the own row. DOT: pq = pn . q in the last block, alpha = rz / pq and
// the breakdown guard |pq| < 1e-30 of solve_pcg (src/cfa/linalg.cuh:232-236).
template <int TPR, bool OSS, bool FUSEP, bool DOT>
__global__ void __launch_bounds__(kThreads)
k_op_k(int n, int nnz, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ K,
       const double* __restrict__ oss, const int* __restrict__ tag, OutletBc bc, const double* __restrict__ z,
       const double* __restrict__ p, const double* __restrict__ beta_ptr, double* __restrict__ pn_buf,
       const double* __restrict__ gx, const double* __restrict__ gy, double* __restrict__ q, CgState* __restrict__ st,
       double* __restrict__ part, unsigned int* __restrict__ counter, CondArg cond, const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    __shared__ double sh[kWarps];
    const double beta = (FUSEP && beta_ptr) ? *beta_ptr : 0.0;
    const double* BTx = oss + 2 * (size_t)nnz;
    const double* BTy = oss + 3 * (size_t)nnz;
    double acc = 0.0;
    ROWS_BEGIN(TPR, n)
    double s = 0.0, so = 0.0;
    if (valid) {
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
            const int j = ci[k];
            const double pj = FUSEP ? (beta_ptr ? z[j] + beta * p[j] : z[j]) : pn_buf[j];
            s += K[k] * pj;
            if (OSS) so += BTx[k] * gx[j] + BTy[k] * gy[j];
        }
    }
    s = group_reduce<TPR>(s);
    if (OSS) so = group_reduce<TPR>(so);
    if (valid && lane == 0) {
        if (OSS && !pressure_dirichlet(row, tag[row], bc)) s -= so;
        q[row] = s;
        const double pi = FUSEP ? (beta_ptr ? z[row] + beta * p[row] : z[row]) : pn_buf[row];
        if (FUSEP && pn_buf) pn_buf[row] = pi;
        if (DOT) acc += pi * s;
    }
    ROWS_END
    if (!DOT) return;
    double v[1] = {acc};
    block_sum<1>(v, sh);
    if (publish_partials<1>(v, part, counter)) {
        reduce_partials<1>(v, part, counter, sh);
        if (threadIdx.x == 0) {
            const double pq = v[0];
            if (fabs(pq) < 1.0e-30) {
                st->done = 1;
                st->converged = 0;
                st->status = CFA_BREAKDOWN;
                set_cond(cond, 0);
            } else {
                st->alpha = st->rz / pq;
            }
        }
    }
}

// ---- the OSS operator assembled into one matrix ----
// A = K - diag(not Dirichlet) B^T M^-1 B (apply_oss_projection, src/cfa/device.cuh:316-323, with
// k_oss_apply_B / k_oss_apply_BT, src/cfa/fem_kernels.cuh:855-885, applied to the operator
// instead of a vector): one row pass of about 19 entries per row instead of two passes over
// K, Bx, By, BTx, BTy (7 entries each). The pattern of row i is the two-ring of node i, the
// union of the K rows of its neighbours.
constexpr int kRing2Max = 96;

// Sorted union of the K rows of the neighbours of row i in buf; -1 when longer than kRing2Max.
__device__ int ring2_row(int i, const int* __restrict__ rp, const int* __restrict__ ci, int* buf) {
    int len = 0;
    for (int e = rp[i]; e < rp[i + 1]; ++e) {
        const int k = ci[e];
        for (int f = rp[k]; f < rp[k + 1]; ++f) {
            const int j = ci[f];
            int q = len;
            while (q > 0 && buf[q - 1] > j) --q;
            if (q > 0 && buf[q - 1] == j) continue;
            if (len == kRing2Max) return -1;
            for (int r = len; r > q; --r) buf[r] = buf[r - 1];
            buf[q] = j;
            ++len;
        }
    }
    return len;
}

__global__ void k_ring2_count(int n, const int* __restrict__ rp, const int* __restrict__ ci, int* __restrict__ cnt,
                              int* __restrict__ err) {
    CFA_GRID_DEP();
    int buf[kRing2Max];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) { cnt[n] = 0; return; }
    const int len = ring2_row(i, rp, ci, buf);
    if (len < 0) { atomicExch(err, 1); cnt[i] = 0; return; }
    cnt[i] = len;
}

__global__ void k_ring2_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci, const int* __restrict__ rp2,
                             int* __restrict__ ci2) {
    CFA_GRID_DEP();
    int buf[kRing2Max];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int len = ring2_row(i, rp, ci, buf);
    for (int q = 0; q < len; ++q) ci2[rp2[i] + q] = buf[q];
}

// Position of column j in the sorted row [f0, f1) of ci, or -1.
__device__ __forceinline__ int find_in_row(const int* __restrict__ ci, int f0, int f1, int j) {
    int lo = f0, hi = f1 - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ci[mid] < j) lo = mid + 1;
        else hi = mid;
    }
    return (lo < f1 && ci[lo] == j) ? lo : -1;
}

// Symbolic plan of the fused values, one thread per two-ring entry s = (i, j): its row, the
// position of j in K's row i (or -1) and, in pass 2, the pairs (a, f) of the products
// BT_ik m_k^-1 B_kj that reach it: a = (i, k) in K's pattern, f = (k, j), k ascending.
__global__ void k_ring2_slots(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                              const int* __restrict__ rp2, const int* __restrict__ ci2, int* __restrict__ slot_row,
                              int* __restrict__ kpos, int* __restrict__ cnt, const int* __restrict__ pair_ptr,
                              int* __restrict__ pa, int* __restrict__ pf) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int s = rp2[i]; s < rp2[i + 1]; ++s) {
        const int j = ci2[s];
        int c = pair_ptr ? pair_ptr[s] : 0;
        if (!pair_ptr) {
            slot_row[s] = i;
            kpos[s] = find_in_row(ci, rp[i], rp[i + 1], j);
        }
        for (int a = rp[i]; a < rp[i + 1]; ++a) {
            const int k = ci[a];
            const int f = find_in_row(ci, rp[k], rp[k + 1], j);
            if (f < 0) continue;
            if (pair_ptr) { pa[c] = a; pf[c] = f; }
            ++c;
        }
        if (!pair_ptr) cnt[s] = c;
    }
}

// Values of the fused operator, one thread per two-ring entry (i, j), written straight into the
// value section of its tile: K_ij minus, over its pairs in order (k ascending),
// BTx_ik m_k^-1 Bx_kj + BTy_ik m_k^-1 By_kj; Dirichlet rows keep K only.
__global__ void __launch_bounds__(kThreads)
k_oss_fuse(long long nnz2, int n, int nnz, const int* __restrict__ ci, const double* __restrict__ K,
           const double* __restrict__ oss, const int* __restrict__ tag, OutletBc bc, const double* __restrict__ inv_m,
           const int* __restrict__ rp2, const int* __restrict__ slot_row, const int* __restrict__ kpos,
           const int* __restrict__ pair_ptr, const int* __restrict__ pa, const int* __restrict__ pf, TileView tv,
           unsigned char* __restrict__ data) {
    CFA_GRID_DEP();
    const double* Bx = oss;
    const double* By = oss + nnz;
    const double* BTx = oss + 2 * (size_t)nnz;
    const double* BTy = oss + 3 * (size_t)nnz;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nnz2;
         s += (long long)gridDim.x * blockDim.x) {
        const int i = slot_row[s];
        const int kp = kpos[s];
        double acc = kp >= 0 ? K[kp] : 0.0;
        if (!pressure_dirichlet(i, tag[i], bc))
            for (int q = pair_ptr[s]; q < pair_ptr[s + 1]; ++q) {
                const int a = pa[q], f = pf[q];
                const double im = inv_m[ci[a]];
                acc -= (BTx[a] * im) * Bx[f] + (BTy[a] * im) * By[f];
            }
        const int t = i / tv.tile_rows;
        const int r0 = t * tv.tile_rows;
        const int nr = min(tv.tile_rows, n - r0);
        const int e0 = rp2[r0], ne = rp2[r0 + nr] - e0;
        reinterpret_cast<double*>(data + tv.off[t] + tile_val_off(nr, ne, 8, 0))[s - e0] = acc;
    }
}

// ---- tile-streamed forms of the two operator passes (tiled.cuh) ----
// pass 1: tiles of {Bx, By}; pn = z + beta p (beta NULL: pn = z)
template <int TPR>
__global__ void __launch_bounds__(kTileThreads)
k_opt_b(TileView tv, const double* __restrict__ inv_m, const double* __restrict__ z, const double* __restrict__ p,
        const double* __restrict__ beta_ptr, double* __restrict__ p_new, double* __restrict__ gx,
        double* __restrict__ gy, const int* __restrict__ done) {
    extern __shared__ __align__(128) unsigned char tsmem[];
    const bool fuse = beta_ptr != nullptr;
    double beta = 0.0;
    // the tiles are packed at the start of the solve, ahead of at least one other kernel
    tile_loop_dep(tv, tsmem, [&] {
        if (done && *done) return false;
        if (fuse) beta = *beta_ptr;
        return true;
    }, [&](int, int r0, int nr, const unsigned char* ch) {
        const int* rr = reinterpret_cast<const int*>(ch);
        const int ne = rr[nr];
        const int* cs = reinterpret_cast<const int*>(ch + tile_ci_off(nr));
        const double* bx = reinterpret_cast<const double*>(ch + tile_val_off(nr, ne, 8, 0));
        const double* by = reinterpret_cast<const double*>(ch + tile_val_off(nr, ne, 8, 1));
        for (int base = 0; base < nr; base += kTileThreads / TPR) {
            const int lr = base + (int)threadIdx.x / TPR, lane = threadIdx.x % TPR;
            const bool valid = lr < nr;
            const int row = r0 + lr;
            double im = 0.0, zi = 0.0, pi = 0.0;
            if (valid && lane == 0) {
                im = inv_m[row];
                zi = z[row];
                if (fuse) pi = p[row];
            }
            double sx = 0.0, sy = 0.0;
            if (valid) {
                constexpr int U = kGatherBatch / 2;
                const int end = rr[lr + 1];
                for (int e0 = rr[lr] + lane; e0 < end; e0 += U * TPR) {
                    double ax[U], ay[U], gz[U], gp[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int e = e0 + u * TPR;
                        if (e < end) {
                            const int j = cs[e];
                            ax[u] = bx[e];
                            ay[u] = by[e];
                            gz[u] = z[j];
                            if (fuse) gp[u] = p[j];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (e0 + u * TPR < end) {
                            const double pj = fuse ? gz[u] + beta * gp[u] : gz[u];
                            sx += ax[u] * pj;
                            sy += ay[u] * pj;
                        }
                }
            }
            sx = group_reduce<TPR>(sx);
            sy = group_reduce<TPR>(sy);
            if (valid && lane == 0) {
                gx[row] = sx * im;
                gy[row] = sy * im;
                if (p_new) p_new[row] = fuse ? zi + beta * pi : zi;
            }
        }
    });
}

// pass 2: tiles of {K, BTx, BTy} (OSS) or {K}; FUSEP as k_op_k; DOT: pn.q -> alpha
template <int TPR, bool OSS, bool FUSEP, bool DOT>
__global__ void __launch_bounds__(kTileThreads)
k_opt_k(TileView tv, const int* __restrict__ tag, OutletBc bc, const double* __restrict__ z,
        const double* __restrict__ p, const double* __restrict__ beta_ptr, double* __restrict__ pn_buf,
        const double* __restrict__ gx, const double* __restrict__ gy, double* __restrict__ q, CgState* __restrict__ st,
        double* __restrict__ part, unsigned int* __restrict__ counter, CondArg cond, const int* __restrict__ done) {
    extern __shared__ __align__(128) unsigned char tsmem[];
    __shared__ double sh[kWarps];
    const bool fuse = FUSEP && beta_ptr != nullptr;
    double beta = 0.0;
    double acc = 0.0;
    // the tiles are packed at the start of the solve, ahead of at least one other kernel
    const bool go = tile_loop_dep(tv, tsmem, [&] {
        if (done && *done) return false;
        if (fuse) beta = *beta_ptr;
        return true;
    }, [&](int, int r0, int nr, const unsigned char* ch) {
        const int* rr = reinterpret_cast<const int*>(ch);
        const int ne = rr[nr];
        const int* cs = reinterpret_cast<const int*>(ch + tile_ci_off(nr));
        const double* kv = reinterpret_cast<const double*>(ch + tile_val_off(nr, ne, 8, 0));
        const double* btx = reinterpret_cast<const double*>(ch + tile_val_off(nr, ne, 8, 1));
        const double* bty = reinterpret_cast<const double*>(ch + tile_val_off(nr, ne, 8, 2));
        for (int base = 0; base < nr; base += kTileThreads / TPR) {
            const int lr = base + (int)threadIdx.x / TPR, lane = threadIdx.x % TPR;
            const bool valid = lr < nr;
            const int row = r0 + lr;
            bool dir = true;
            double pi = 0.0;
            if (valid && lane == 0) {
                if (OSS) dir = pressure_dirichlet(row, tag[row], bc);
                pi = FUSEP ? (fuse ? z[row] + beta * p[row] : z[row]) : pn_buf[row];
            }
            double s = 0.0, so = 0.0;
            if (valid) {
                constexpr int U = kGatherBatch / 2;
                const int end = rr[lr + 1];
                for (int e0 = rr[lr] + lane; e0 < end; e0 += U * TPR) {
                    double ak[U], g0[U], g1[U], ax[U], ay[U], hx[U], hy[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int e = e0 + u * TPR;
                        if (e < end) {
                            const int j = cs[e];
                            ak[u] = kv[e];
                            if (FUSEP) {
                                g0[u] = z[j];
                                if (fuse) g1[u] = p[j];
                            } else {
                                g0[u] = pn_buf[j];
                            }
                            if (OSS) {
                                ax[u] = btx[e];
                                ay[u] = bty[e];
                                hx[u] = gx[j];
                                hy[u] = gy[j];
                            }
                        }
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (e0 + u * TPR < end) {
                            const double pj = (FUSEP && fuse) ? g0[u] + beta * g1[u] : g0[u];
                            s += ak[u] * pj;
                            if (OSS) so += ax[u] * hx[u] + ay[u] * hy[u];
                        }
                }
            }
            s = group_reduce<TPR>(s);
            if (OSS) so = group_reduce<TPR>(so);
            if (valid && lane == 0) {
                if (OSS && !dir) s -= so;
                q[row] = s;
                if (FUSEP && pn_buf) pn_buf[row] = pi;
                if (DOT) acc += pi * s;
            }
        }
    });
    if (!go || !DOT) return;
    double v[1] = {acc};
    block_sum<1>(v, sh);
    if (publish_partials<1>(v, part, counter)) {
        reduce_partials<1>(v, part, counter, sh);
        if (threadIdx.x == 0) {
            const double pq = v[0];
            if (fabs(pq) < 1.0e-30) {
                st->done = 1;
                st->converged = 0;
                st->status = CFA_BREAKDOWN;
                set_cond(cond, 0);
            } else {
                st->alpha = st->rz / pq;
            }
        }
    }
}

// ||b|| (solve_pcg :205-209)
__global__ void __launch_bounds__(kThreads)
k_cg_bnorm(int n, const double* __restrict__ b, CgState* __restrict__ st, double* __restrict__ part,
           unsigned int* __restrict__ counter, CondArg cond) {
    CFA_GRID_DEP();
    __shared__ double sh[kWarps];
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] += b[i] * b[i];
    block_sum<1>(v, sh);
    if (publish_partials<1>(v, part, counter)) {
        reduce_partials<1>(v, part, counter, sh);
        if (threadIdx.x == 0) {
            st->bnorm = sqrt(v[0]);
            st->iter = 0;
            st->done = 0;
            st->converged = 1;
            st->status = 0;
            st->nullb = 0;
            st->rel = 0.0;
            st->beta = 0.0;
            st->zero = 0.0;
            if (st->bnorm < 1.0e-14) {
                st->done = 1;
                st->nullb = 1;
                set_cond(cond, 0);
            }
        }
    }
}

// r = b - q, ||r|| test (:213-218)
__global__ void __launch_bounds__(kThreads)
k_cg_resid0(int n, const double* __restrict__ b, const double* __restrict__ q, double* __restrict__ r,
            CgState* __restrict__ st, double* __restrict__ part, unsigned int* __restrict__ counter, CondArg cond) {
    CFA_GRID_DEP();
    if (st->done) return;
    __shared__ double sh[kWarps];
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ri = b[i] + -1.0 * q[i];
        r[i] = ri;
        v[0] += ri * ri;
    }
    block_sum<1>(v, sh);
    if (publish_partials<1>(v, part, counter)) {
        reduce_partials<1>(v, part, counter, sh);
        if (threadIdx.x == 0) {
            const double rn = sqrt(v[0]);
            st->rel = rn / st->bnorm;
            if (rn < st->tol * st->bnorm) {
                st->done = 1;
                st->converged = 1;
                set_cond(cond, 0);
            }
        }
    }
}

__global__ void k_cg_nullx(int n, double* __restrict__ x, double* __restrict__ p0, const CgState* __restrict__ st) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (st->nullb) x[i] = 0.0;
    p0[i] = 0.0;
}

// 1 / diag (k_extract_inv_diag, src/cfa/linalg.cuh:28-48)
__global__ void k_inv_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ val,
                           double* __restrict__ dinv) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 1.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) if (ci[k] == i) { d = val[k]; break; }
    dinv[i] = (fabs(d) > 1.0e-14) ? (1.0 / d) : 1.0;
}

// x += alpha pn, r -= alpha q, p = pn, ||r|| test (:237-247); JAC: z = D^-1 r and r.z -> beta
// SC (float or double, with JAC false): also c = omega0 D0^-1 r in the AMG's level-0 vector type,
// the pre-smoothing's first iterate, which the V-cycle's level-0 pre-smoothing then gathers in
// place of D0^-1 and r (PreScale); the product is formed as that pass forms it.
template <bool JAC, class SC = double>
__global__ void __launch_bounds__(kThreads)
k_cg_update(int n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ pn, double* __restrict__ p,
            const double* __restrict__ q, const double* __restrict__ dinv, double* __restrict__ z,
            CgState* __restrict__ st, double* __restrict__ part, unsigned int* __restrict__ counter, CondArg cond,
            const SC* __restrict__ dinv0 = nullptr, SC omega0 = SC(0), SC* __restrict__ c0 = nullptr) {
    CFA_GRID_DEP();
    if (st->done) return;
    __shared__ double sh[2 * kWarps];
    const double alpha = st->alpha;
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double pi = pn[i];
        x[i] += alpha * pi;
        const double ri = r[i] + -alpha * q[i];
        r[i] = ri;
        p[i] = pi;
        if (c0) c0[i] = SC(omega0 * dinv0[i]) * (SC)ri;   // the level-0 pre-smoothing's (omega D^-1) b, rounded
        v[0] += ri * ri;
        if (JAC) {
            const double zi = dinv[i] * ri;
            z[i] = zi;
            v[1] += ri * zi;
        }
    }
    block_sum<2>(v, sh);
    if (publish_partials<2>(v, part, counter)) {
        reduce_partials<2>(v, part, counter, sh);
        if (threadIdx.x == 0) {
            const double rn = sqrt(v[0]);
            st->rel = rn / st->bnorm;
            const int it = st->iter + 1;
            st->iter = it;
            if (rn < st->tol * st->bnorm) {
                st->done = 1;
                st->converged = 1;
                set_cond(cond, 0);
            } else if (it >= st->max_iter) {
                st->done = 1;
                st->converged = 0;
                st->status = CFA_NOT_CONVERGED;
                set_cond(cond, 0);
            } else if (JAC) {
                const double rz_new = v[1];
                st->beta = rz_new / (st->rz + 1.0e-30);
                st->rz = rz_new;
            }
        }
    }
}

// r.z after the preconditioner: first = initial rz (p = z); else beta = rz_new / (rz + 1e-30)
// (solve_pcg, :249-252). With `flexible` (an FP32 preconditioner, which is not exactly the same
// linear operator at every application) beta is the Polak-Ribiere form
// z_new.(r_new - r_old) / rz_old = -alpha z_new.q / rz_old, which keeps CG's convergence rate;
// for a fixed preconditioner both forms are equal in exact arithmetic.
__global__ void __launch_bounds__(kThreads)
k_cg_rz(int n, const double* __restrict__ r, const double* __restrict__ z, const double* __restrict__ q, int first,
        int flexible, CgState* __restrict__ st, double* __restrict__ part, unsigned int* __restrict__ counter,
        CondArg cond) {
    CFA_GRID_DEP();
    if (st->done) return;
    __shared__ double sh[2 * kWarps];
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double zi = z[i];
        v[0] += r[i] * zi;
        if (flexible) v[1] += zi * q[i];
    }
    block_sum<2>(v, sh);
    if (publish_partials<2>(v, part, counter)) {
        reduce_partials<2>(v, part, counter, sh);
        if (threadIdx.x == 0) {
            if (first) {
                st->rz = v[0];
                st->beta = 0.0;
                set_cond(cond, 1);
            } else {
                st->beta = flexible ? -st->alpha * v[1] / (st->rz + 1.0e-30) : v[0] / (st->rz + 1.0e-30);
                st->rz = v[0];
            }
        }
    }
}

// pq = pn . q when a host-side operator added its part to q after the operator kernel; alpha and
// the breakdown guard as in k_op_k's DOT epilogue (solve_pcg, src/cfa/linalg.cuh:231-236)
__global__ void __launch_bounds__(kThreads)
k_cg_pq(int n, const double* __restrict__ pn, const double* __restrict__ q, CgState* __restrict__ st,
        double* __restrict__ part, unsigned int* __restrict__ counter, CondArg cond) {
    CFA_GRID_DEP();
    if (st->done) return;
    __shared__ double sh[kWarps];
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] += pn[i] * q[i];
    block_sum<1>(v, sh);
    if (publish_partials<1>(v, part, counter)) {
        reduce_partials<1>(v, part, counter, sh);
        if (threadIdx.x == 0) {
            const double pq = v[0];
            if (fabs(pq) < 1.0e-30) {
                st->done = 1;
                st->converged = 0;
                st->status = CFA_BREAKDOWN;
                set_cond(cond, 0);
            } else {
                st->alpha = st->rz / pq;
            }
        }
    }
}

// =============================================================================================
// two-component BiCGSTAB (GpuBicgstab2::solve, src/cfa/linalg.cuh:656-754)
// =============================================================================================
struct B2State {
    double tol;
    double rn0[2], bd[2], rho[2], rho_old[2], alpha[2], omega[2], rel[2];
    double cb[2], co[2], ca[2], a1[2], a2[2], cw[2];
    int active[2], iters[2], conv[2], s_done[2];
    int iter, max_iter, done, pad;
};

__device__ __forceinline__ void b2_stop(B2State* st, int c, int it, int ok) {
    st->active[c] = 0;
    st->iters[c] = it;
    st->conv[c] = ok;
}

// start of an iteration (:699-707): breakdown on rho, p-update coefficients
__device__ __forceinline__ void b2_begin_iteration(B2State* st, CondArg cond) {
    const int iter = st->iter;
    if (iter >= st->max_iter) { st->done = 1; set_cond(cond, 0); return; }
    for (int c = 0; c < 2; ++c) {
        st->cb[c] = 0.0;
        st->co[c] = 0.0;
        if (st->active[c] && fabs(st->rho[c]) < st->bd[c]) b2_stop(st, c, iter, 0);
        if (st->active[c] && iter > 0) {
            st->cb[c] = (st->rho[c] / st->rho_old[c]) * (st->alpha[c] / (st->omega[c] + 1.0e-30));
            st->co[c] = st->omega[c];
        }
    }
    if (!(st->active[0] || st->active[1])) { st->done = 1; set_cond(cond, 0); }
}

// The solver's vectors hold the two components interleaved per row: r[i] = (u_i, v_i) as one
// double2 (the reference keeps [u | v] with stride n, linalg.cuh:666-669). Each row's pair is one
// 16-byte access, and the SpMV gathers both components of a neighbour with one load.
//
// v = A x (x given as the caller's two arrays), r = b - v, r0 = p = r, v = 0, ||r|| (:681-697)
template <int TPR>
__global__ void __launch_bounds__(kThreads)
k_b2_init(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ val,
          const double* __restrict__ xu, const double* __restrict__ xv, const double* __restrict__ bu,
          const double* __restrict__ bv, double2* __restrict__ r, double2* __restrict__ r0, double2* __restrict__ p,
          double2* __restrict__ vv, B2State* __restrict__ st, double* __restrict__ part, unsigned int* __restrict__ counter,
          CondArg cond) {
    CFA_GRID_DEP();
    __shared__ double sh[2 * kWarps];
    double acc[2] = {0.0, 0.0};
    ROWS_BEGIN(TPR, n)
    double su = 0.0, sv = 0.0;
    if (valid)
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
            const double a = val[k];
            const int j = ci[k];
            su += a * xu[j];
            sv += a * xv[j];
        }
    su = group_reduce<TPR>(su);
    sv = group_reduce<TPR>(sv);
    if (valid && lane == 0) {
        const double ru = bu[row] - 1.0 * su, rv = bv[row] - 1.0 * sv;
        const double2 rr = make_double2(ru, rv);
        r[row] = rr;
        r0[row] = rr;
        p[row] = rr;
        vv[row] = make_double2(0.0, 0.0);
        acc[0] += ru * ru;
        acc[1] += rv * rv;
    }
    ROWS_END
    block_sum<2>(acc, sh);
    if (publish_partials<2>(acc, part, counter)) {
        reduce_partials<2>(acc, part, counter, sh);
        if (threadIdx.x == 0) {
            for (int c = 0; c < 2; ++c) {
                st->rn0[c] = sqrt(acc[c]);
                st->rho[c] = acc[c];
                st->bd[c] = 1.0e-30 * st->rn0[c] * st->rn0[c] + 1.0e-300;
                st->rho_old[c] = 1.0; st->alpha[c] = 1.0; st->omega[c] = 1.0;
                st->iters[c] = 0; st->conv[c] = 1; st->rel[c] = 0.0; st->s_done[c] = 0;
                st->active[c] = st->rn0[c] >= 1.0e-13;
            }
            st->iter = 0;
            st->done = 0;
            set_cond(cond, 1);
            b2_begin_iteration(st, cond);
        }
    }
}

// p = r + cb (p - co v) (k_bicg2_p)
// The ILU apply's first pass done here (ilu_pair_staging): the new pair also goes to its
// colour position in the apply's work vector, in the work precision (w32 or w64; both null: not
// staged).
__device__ __forceinline__ void b2_stage(int i, double2 v, const int* __restrict__ pos, float2* __restrict__ w32,
                                         double2* __restrict__ w64) {
    if (w32) w32[pos[i]] = make_float2((float)v.x, (float)v.y);
    else if (w64) w64[pos[i]] = v;
}

__global__ void k_b2_p(int n, const double2* __restrict__ r, const double2* __restrict__ v, double2* __restrict__ p,
                       const B2State* __restrict__ st, const int* __restrict__ pos, float2* __restrict__ w32,
                       double2* __restrict__ w64) {
    CFA_GRID_DEP();
    if (st->done) return;
    const double cb0 = st->cb[0], cb1 = st->cb[1], co0 = st->co[0], co1 = st->co[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double2 rr = r[i], vv = v[i];
        double2 pp = p[i];
        pp.x = rr.x + cb0 * (pp.x - co0 * vv.x);
        pp.y = rr.y + cb1 * (pp.y - co1 * vv.y);
        p[i] = pp;
        b2_stage(i, pp, pos, w32, w64);
    }
}

// v = A phat, r0 . v -> alpha (:711-719)
template <int TPR>
__global__ void __launch_bounds__(kThreads)
k_b2_v(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ val,
       const double2* __restrict__ phat, const double2* __restrict__ r0, double2* __restrict__ vv, B2State* __restrict__ st,
       double* __restrict__ part, unsigned int* __restrict__ counter, CondArg cond) {
    CFA_GRID_DEP();
    if (st->done) return;
    __shared__ double sh[2 * kWarps];
    double acc[2] = {0.0, 0.0};
    ROWS_BEGIN(TPR, n)
    double su = 0.0, sv = 0.0;
    if (valid)
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
            const double a = val[k];
            const int j = ci[k];
            const double2 g = phat[j];
            su += a * g.x;
            sv += a * g.y;
        }
    su = group_reduce<TPR>(su);
    sv = group_reduce<TPR>(sv);
    if (valid && lane == 0) {
        vv[row] = make_double2(su, sv);
        const double2 q = r0[row];
        acc[0] += q.x * su;
        acc[1] += q.y * sv;
    }
    ROWS_END
    block_sum<2>(acc, sh);
    if (publish_partials<2>(acc, part, counter)) {
        reduce_partials<2>(acc, part, counter, sh);
        if (threadIdx.x == 0) {
            const int iter = st->iter;
            for (int c = 0; c < 2; ++c) {
                st->ca[c] = 0.0;
                if (st->active[c] && fabs(acc[c]) < st->bd[c]) b2_stop(st, c, iter, 0);
                if (st->active[c]) { st->alpha[c] = st->rho[c] / acc[c]; st->ca[c] = st->alpha[c]; }
            }
            if (!(st->active[0] || st->active[1])) { st->done = 1; set_cond(cond, 0); }
        }
    }
}

// s = r - ca v (k_bicg2_s)
__global__ void k_b2_s(int n, const double2* __restrict__ r, const double2* __restrict__ v, double2* __restrict__ s,
                       const B2State* __restrict__ st, const int* __restrict__ pos, float2* __restrict__ w32,
                       double2* __restrict__ w64) {
    CFA_GRID_DEP();
    if (st->done) return;
    const double a0 = st->ca[0], a1 = st->ca[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double2 rr = r[i], vv = v[i];
        const double2 ss = make_double2(rr.x - a0 * vv.x, rr.y - a1 * vv.y);
        s[i] = ss;
        b2_stage(i, ss, pos, w32, w64);
    }
}

// t = A shat; s.s, t.t, t.s -> omega, s-stop (:723-736)
template <int TPR>
__global__ void __launch_bounds__(kThreads)
k_b2_t(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ val,
       const double2* __restrict__ shat, const double2* __restrict__ s, double2* __restrict__ t, B2State* __restrict__ st,
       double* __restrict__ part, unsigned int* __restrict__ counter) {
    CFA_GRID_DEP();
    if (st->done) return;
    __shared__ double sh[6 * kWarps];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    ROWS_BEGIN(TPR, n)
    double su = 0.0, sv = 0.0;
    if (valid)
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
            const double a = val[k];
            const int j = ci[k];
            const double2 g = shat[j];
            su += a * g.x;
            sv += a * g.y;
        }
    su = group_reduce<TPR>(su);
    sv = group_reduce<TPR>(sv);
    if (valid && lane == 0) {
        t[row] = make_double2(su, sv);
        const double2 sr = s[row];
        const double s0 = sr.x, s1 = sr.y;
        acc[0] += s0 * s0; acc[1] += s1 * s1;
        acc[2] += su * su; acc[3] += sv * sv;
        acc[4] += su * s0; acc[5] += sv * s1;
    }
    ROWS_END
    block_sum<6>(acc, sh);
    if (publish_partials<6>(acc, part, counter)) {
        reduce_partials<6>(acc, part, counter, sh);
        if (threadIdx.x == 0) {
            for (int c = 0; c < 2; ++c) {
                st->a1[c] = 0.0; st->a2[c] = 0.0; st->cw[c] = 0.0; st->s_done[c] = 0;
                if (!st->active[c]) continue;
                st->a1[c] = st->alpha[c];
                const double s_norm = sqrt(acc[c]);
                if (s_norm < st->tol * st->rn0[c] || s_norm < 1.0e-11) { st->s_done[c] = 1; continue; }
                const double tt = acc[2 + c];
                st->omega[c] = (tt > st->bd[c]) ? (acc[4 + c] / tt) : 0.0;
                st->a2[c] = st->omega[c];
                st->cw[c] = st->omega[c];
            }
        }
    }
}

// x += a1 phat + a2 shat, r = s - cw t; r.r, r0.r -> stop tests, rho (:737-750); then the
// start of the next iteration
__global__ void __launch_bounds__(kThreads)
k_b2_xr(int n, double* __restrict__ xu, double* __restrict__ xv, const double2* __restrict__ phat,
        const double2* __restrict__ shat, const double2* __restrict__ s, const double2* __restrict__ t,
        double2* __restrict__ r, const double2* __restrict__ r0, B2State* __restrict__ st, double* __restrict__ part,
        unsigned int* __restrict__ counter, CondArg cond) {
    CFA_GRID_DEP();
    if (st->done) return;
    __shared__ double sh[4 * kWarps];
    const double a10 = st->a1[0], a11 = st->a1[1], a20 = st->a2[0], a21 = st->a2[1], w0 = st->cw[0], w1 = st->cw[1];
    double acc[4] = {0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double2 ph = phat[i], sh2 = shat[i], ss = s[i], tt = t[i], q = r0[i];
        xu[i] += a10 * ph.x + a20 * sh2.x;
        xv[i] += a11 * ph.y + a21 * sh2.y;
        const double ru = ss.x - w0 * tt.x, rv = ss.y - w1 * tt.y;
        r[i] = make_double2(ru, rv);
        acc[0] += ru * ru; acc[1] += rv * rv;
        acc[2] += q.x * ru; acc[3] += q.y * rv;
    }
    block_sum<4>(acc, sh);
    if (publish_partials<4>(acc, part, counter)) {
        reduce_partials<4>(acc, part, counter, sh);
        if (threadIdx.x == 0) {
            const int iter = st->iter;
            for (int c = 0; c < 2; ++c) if (st->s_done[c] && st->active[c]) b2_stop(st, c, iter + 1, 1);
            if (!(st->active[0] || st->active[1])) {
                st->done = 1;
                set_cond(cond, 0);
            } else {
                for (int c = 0; c < 2; ++c) {
                    if (!st->active[c]) continue;
                    const double r_norm = sqrt(acc[c]);
                    st->rel[c] = r_norm / st->rn0[c];
                    if (r_norm < st->tol * st->rn0[c] || r_norm < 1.0e-11) { b2_stop(st, c, iter + 1, 1); continue; }
                    st->rho_old[c] = st->rho[c];
                    st->rho[c] = acc[2 + c];
                    if (iter + 1 == st->max_iter) b2_stop(st, c, st->max_iter, 0);
                }
                st->iter = iter + 1;
                if (!(st->active[0] || st->active[1])) { st->done = 1; set_cond(cond, 0); }
                else b2_begin_iteration(st, cond);
            }
        }
    }
}

// ---- tile-streamed forms of the BiCGSTAB2 SpMV + dot kernels (tiles of {A}, FP64) ----
// MODE 0: init  (x -> v = A x, r = b - v, r0 = p = r, v = 0, r.r)
// MODE 1: v = A phat, r0.v -> alpha
// MODE 2: t = A shat, s.s t.t t.s -> omega / s-stop
template <int TPR, int MODE>
__global__ void __launch_bounds__(kTileThreads)
k_b2t(TileView tv, int n, const double* __restrict__ xu, const double* __restrict__ xv, const double* __restrict__ bu,
      const double* __restrict__ bv, const double2* __restrict__ in, const double2* __restrict__ aux,
      double2* __restrict__ out, double2* __restrict__ r, double2* __restrict__ r0, double2* __restrict__ p,
      B2State* __restrict__ st, double* __restrict__ part, unsigned int* __restrict__ counter, CondArg cond) {
    extern __shared__ __align__(128) unsigned char tsmem[];
    constexpr int NV = MODE == 2 ? 6 : 2;
    __shared__ double sh[NV * kWarps];
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = 0.0;
    // the tiles are packed by the kernel just before MODE 0 (its first copies wait); MODES 1 and 2
    // read them later in the solve
    const bool go = tile_loop_dep<MODE != 0>(tv, tsmem, [&] { return MODE == 0 || !st->done; },
                                             [&](int, int r0_, int nr, const unsigned char* ch) {
        const int* rr = reinterpret_cast<const int*>(ch);
        const int ne = rr[nr];
        const int* cs = reinterpret_cast<const int*>(ch + tile_ci_off(nr));
        const double* av = reinterpret_cast<const double*>(ch + tile_val_off(nr, ne, 8, 0));
        for (int base = 0; base < nr; base += kTileThreads / TPR) {
            const int lr = base + (int)threadIdx.x / TPR, lane = threadIdx.x % TPR;
            const bool valid = lr < nr;
            double su = 0.0, sv = 0.0;
            if (valid) {
                const int end = rr[lr + 1];
                for (int e0 = rr[lr] + lane; e0 < end; e0 += kGatherBatch * TPR) {
                    double a[kGatherBatch], g0[kGatherBatch], g1[kGatherBatch];
#pragma unroll
                    for (int u = 0; u < kGatherBatch; ++u) {
                        const int e = e0 + u * TPR;
                        if (e < end) {
                            const int j = cs[e];
                            a[u] = av[e];
                            if (MODE == 0) {
                                g0[u] = xu[j];
                                g1[u] = xv[j];
                            } else {
                                const double2 g = in[j];
                                g0[u] = g.x;
                                g1[u] = g.y;
                            }
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kGatherBatch; ++u)
                        if (e0 + u * TPR < end) {
                            su += a[u] * g0[u];
                            sv += a[u] * g1[u];
                        }
                }
            }
            su = group_reduce<TPR>(su);
            sv = group_reduce<TPR>(sv);
            if (valid && lane == 0) {
                const int row = r0_ + lr;
                if (MODE == 0) {
                    const double ru = bu[row] - 1.0 * su, rv = bv[row] - 1.0 * sv;
                    const double2 rr = make_double2(ru, rv);
                    r[row] = rr;
                    r0[row] = rr;
                    p[row] = rr;
                    out[row] = make_double2(0.0, 0.0);
                    acc[0] += ru * ru;
                    acc[1] += rv * rv;
                } else if (MODE == 1) {
                    out[row] = make_double2(su, sv);
                    const double2 q = aux[row];
                    acc[0] += q.x * su;
                    acc[1] += q.y * sv;
                } else {
                    out[row] = make_double2(su, sv);
                    const double2 sr = aux[row];
                    const double s0 = sr.x, s1 = sr.y;
                    acc[0] += s0 * s0; acc[1] += s1 * s1;
                    acc[2 % NV] += su * su; acc[3 % NV] += sv * sv;
                    acc[4 % NV] += su * s0; acc[5 % NV] += sv * s1;
                }
            }
        }
    });
    if (!go) return;
    block_sum<NV>(acc, sh);
    if (!publish_partials<NV>(acc, part, counter)) return;
    reduce_partials<NV>(acc, part, counter, sh);
    if (threadIdx.x != 0) return;
    if (MODE == 0) {
        for (int c = 0; c < 2; ++c) {
            st->rn0[c] = sqrt(acc[c]);
            st->rho[c] = acc[c];
            st->bd[c] = 1.0e-30 * st->rn0[c] * st->rn0[c] + 1.0e-300;
            st->rho_old[c] = 1.0; st->alpha[c] = 1.0; st->omega[c] = 1.0;
            st->iters[c] = 0; st->conv[c] = 1; st->rel[c] = 0.0; st->s_done[c] = 0;
            st->active[c] = st->rn0[c] >= 1.0e-13;
        }
        st->iter = 0;
        st->done = 0;
        set_cond(cond, 1);
        b2_begin_iteration(st, cond);
    } else if (MODE == 1) {
        const int iter = st->iter;
        for (int c = 0; c < 2; ++c) {
            st->ca[c] = 0.0;
            if (st->active[c] && fabs(acc[c]) < st->bd[c]) b2_stop(st, c, iter, 0);
            if (st->active[c]) { st->alpha[c] = st->rho[c] / acc[c]; st->ca[c] = st->alpha[c]; }
        }
        if (!(st->active[0] || st->active[1])) { st->done = 1; set_cond(cond, 0); }
    } else {
        for (int c = 0; c < 2; ++c) {
            st->a1[c] = 0.0; st->a2[c] = 0.0; st->cw[c] = 0.0; st->s_done[c] = 0;
            if (!st->active[c]) continue;
            st->a1[c] = st->alpha[c];
            const double s_norm = sqrt(acc[c]);
            if (s_norm < st->tol * st->rn0[c] || s_norm < 1.0e-11) { st->s_done[c] = 1; continue; }
            const double tt = acc[2 + c];
            st->omega[c] = (tt > st->bd[c]) ? (acc[4 + c] / tt) : 0.0;
            st->a2[c] = st->omega[c];
            st->cw[c] = st->omega[c];
        }
    }
}

// =============================================================================================
// Jacobi BiCGSTAB (GpuLinearSolver::solve_bicgstab, :261-347), host-driven like the reference
// but with the fused dot kernels (kept simple: it is the non-default solver and a test oracle).
// =============================================================================================
__global__ void __launch_bounds__(kThreads)
k_dot(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
      double* __restrict__ part, unsigned int* __restrict__ counter) {
    CFA_GRID_DEP();
    __shared__ double sh[kWarps];
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] += a[i] * b[i];
    block_sum<1>(v, sh);
    if (publish_partials<1>(v, part, counter)) {
        reduce_partials<1>(v, part, counter, sh);
        if (threadIdx.x == 0) *out = v[0];
    }
}

__global__ void k_axpby(int n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                        double* __restrict__ out) {
    CFA_GRID_DEP();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a * x[i] + b * y[i];
}
__global__ void k_axpy(int n, double a, const double* __restrict__ x, double* __restrict__ y) {
    CFA_GRID_DEP();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += a * x[i];
}
__global__ void k_vmul(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
    CFA_GRID_DEP();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a[i] * b[i];
}
__global__ void k_bicg_p(int n, const double* __restrict__ r, const double* __restrict__ v, double beta, double omega,
                         double* __restrict__ p) {
    CFA_GRID_DEP();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        p[i] = r[i] + beta * (p[i] - omega * v[i]);
}

// =============================================================================================
// solver workspaces and graphs
// =============================================================================================
// Operator row shape: TPR from the mean row length (P1: about 7 per row)
static int op_tpr(int n, long long nnz) {
    const double per_row = n > 0 ? (double)nnz / n : 1.0;
    if (per_row <= 2.5) return 2;
    if (per_row <= 5.0) return 4;
    if (per_row <= 12.0) return 8;
    return 16;
}

#define OP_TPR_SWITCH(tpr, ...)                                                                \
    do {                                                                                       \
        switch (tpr) {                                                                         \
            case 2: { constexpr int TPR = 2; __VA_ARGS__; } break;                              \
            case 4: { constexpr int TPR = 4; __VA_ARGS__; } break;                              \
            case 8: { constexpr int TPR = 8; __VA_ARGS__; } break;                              \
            default: { constexpr int TPR = 16; __VA_ARGS__; } break;                            \
        }                                                                                      \
    } while (0)

struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    std::vector<const void*> key;
    long long init_kernels = 0, body_kernels = 0;
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        key.clear();
    }
    ~GraphCache() { reset(); }
};

// A straight-line captured graph (no conditional node), replayed while its key holds
struct SegGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> key;
    long long kernels = 0;
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
    }
    ~SegGraph() { reset(); }
};

struct PcgWork {
    int cap = 0;
    DevBuf<double> r, z, p, pn, q, gx, gy, dinv;
    DevBuf<double> c0;                 // omega0 D0^-1 r for the V-cycle's level 0 (float or double elements)
    DevBuf<CgState> st;
    // tile-streamed copy of the operator: K - B^T M^-1 B as one matrix on the two-ring pattern
    // (fused), else pass 1: Bx, By; pass 2: K [, BTx, BTy]
    TiledCsr tb, tk;
    bool fused = false;
    DevBuf<int> rp2, ci2, cnt2;       // two-ring pattern of the fused OSS operator
    DevBuf<int> slot_row, kpos, pair_ptr, pa, pf;   // its per-entry plan (k_ring2_slots)
    DevBuf<unsigned char> scan_tmp;
    std::vector<const void*> tile_key;
    std::vector<const void*> prepared;   // operator whose values the tiles hold (standalone apply)
    bool tiled = false;
    DevBuf<int> err;
    DevBuf<double> part;
    DevBuf<unsigned int> counter;
    GraphCache graph;
    GraphCache graph2;   // the second phase of a mixed-precision solve (FP32 V-cycles)
    SegGraph seg[3];   // the pieces of one iteration between host hooks (cfa_pcg_solve_host_ops)
    DevBuf<unsigned long long> fp;
};

struct B2Work {
    int cap = 0;
    DevBuf<double> r, r0, p, v, s, t, phat, shat;
    DevBuf<B2State> st;
    TiledCsr tA;                     // tile-streamed copy of the momentum matrix (packed per solve)
    std::vector<const void*> tile_key;
    bool tiled = false;
    DevBuf<int> err;
    DevBuf<double> part;
    DevBuf<unsigned int> counter;
    GraphCache graph;
};

struct SolverWork {
    PcgWork pcg;
    B2Work b2;
};

static SolverWork* work(cfa_ctx* ctx) {
    if (!ctx->work) ctx->work = new SolverWork();
    return ctx->work;
}

void free_solver_work(cfa_ctx* ctx) {
    delete ctx->work;
    ctx->work = nullptr;
}

static bool graphs_enabled() {
    const char* e = std::getenv("CFA_GRAPHS");
    return !(e && e[0] == '0');
}

// Captures `init` then a WHILE node with `body` into `gc` (the init kernels set the condition).
template <class Init, class Body>
static cfa_status build_graph(cfa_ctx* ctx, GraphCache& gc, Init init, Body body) {
    gc.reset();
    cudaGraph_t g = nullptr;
    CFA_CUDA(cudaGraphCreate(&g, 0));
    gc.graph = g;
    cudaGraphConditionalHandle handle;
    CFA_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
    CondArg cond{handle, 1};
    // init part, captured into g (launch counts of captures are added per replay instead)
    long long l0 = ctx->launches;
    CFA_CUDA(cudaStreamBeginCaptureToGraph(ctx->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    cfa_status s = init(cond);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &captured);
    gc.init_kernels = ctx->launches - l0;
    ctx->launches = l0;
    if (s != CFA_OK) return s;
    CFA_CUDA(e);
    // the WHILE node depends on every leaf of the init part
    size_t nn = 0;
    CFA_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CFA_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
    std::vector<cudaGraphNode_t> leaves;
    for (cudaGraphNode_t nd : nodes) {
        size_t ndep = 0;
        CFA_CUDA(cudaGraphNodeGetDependentNodes(nd, nullptr, &ndep));
        if (ndep == 0) leaves.push_back(nd);
    }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    CFA_CUDA(cudaGraphAddNode(&wnode, g, leaves.data(), leaves.size(), &cp));
    cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
    l0 = ctx->launches;
    CFA_CUDA(cudaStreamBeginCaptureToGraph(ctx->stream, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    s = body(cond);
    e = cudaStreamEndCapture(ctx->stream, &captured);
    gc.body_kernels = ctx->launches - l0;
    ctx->launches = l0;
    if (s != CFA_OK) return s;
    CFA_CUDA(e);
    CFA_CUDA(cudaGraphInstantiate(&gc.exec, g, 0));
    return CFA_OK;
}

// ---------------------------------------------------------------------------------------------
// PCG
// ---------------------------------------------------------------------------------------------
// Order-free fingerprint of a CSR pattern: the sum (mod 2^64) of a 64-bit mix of every
// (position, value) of row_ptr and col_ind; the mix is the splitmix64 finalizer (Steele, Lea and
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014).
__device__ __forceinline__ unsigned long long fp_mix(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void k_pattern_fingerprint(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                      unsigned long long* __restrict__ out) {
    CFA_GRID_DEP();
    const long long total = (long long)n + 1 + rp[n];
    unsigned long long h = 0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        if (k <= n) h += fp_mix(((unsigned long long)k << 32) ^ (unsigned)rp[k]);
        else h += fp_mix((((unsigned long long)(k - n - 1)) << 32) ^ (unsigned)ci[k - n - 1] ^ 0xa5a5a5a5a5a5a5a5ull);
    }
#pragma unroll
    for (int o = 16; o > 0; o /= 2) h += __shfl_down_sync(0xffffffffu, h, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, h);
}

struct PcgArgs {
    int n, nnz;
    const int *rp, *ci;
    const double* val;
    const double *b;
    double* x;
    const cfa_oss_operator* oss;
    cfa_amg* amg;
    int max_iter;
    double tol;
    // host-side hooks (cfa_pcg_solve_host_ops): extra adds its operator into out, prec replaces
    // the AMG / Jacobi preconditioner
    cfa_host_op extra = nullptr;
    void* extra_user = nullptr;
    cfa_host_op prec = nullptr;
    void* prec_user = nullptr;
    unsigned long long fp = 0;   // fingerprint of the pattern (rp, ci): plans follow its content
    int vc64 = 0;                // the V-cycle in FP64 on a mixed hierarchy (the solve's first phase)
    bool host_ops() const { return extra || prec; }
};

#define TILE_TPR_SWITCH(tpr, ...)                                                              \
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

// Launches tiled pass 2 for one template configuration
template <bool OSS, bool FUSEP, bool DOT>
static void launch_opt_k(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a, const double* z, const double* p,
                         const double* beta_ptr, double* pn, double* q, CondArg cond, const int* done) {
    const cfa_mesh* m = a.oss ? a.oss->mesh : nullptr;
    OutletBc bc = m ? m->bc : OutletBc{};
    TileView tv = W.tk.view(W.err.p);
    tv.l2hint = l2_hint_operator();
    TileLaunch L;
    TILE_TPR_SWITCH(W.tk.tpr,
        L = tile_launch(ctx, W.tk, (const void*)k_opt_k<TPR, OSS, FUSEP, DOT>);
        CFA_LAUNCH(ctx, (k_opt_k<TPR, OSS, FUSEP, DOT>), L.grid, kTileThreads, L.smem, tv,
                   m ? m->tag : (const int*)nullptr, bc, z, p, beta_ptr, pn, (const double*)W.gx.p,
                   (const double*)W.gy.p, q, W.st.p, W.part.p, W.counter.p, cond, done));
}

static cfa_status pcg_operator(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a, const double* z, const double* p,
                               const double* beta_ptr, double* pn, double* q, bool dot, CondArg cond,
                               const int* done) {
    if (W.tiled) {
        if (a.oss && !W.fused) {
            const TileView tv = W.tb.view(W.err.p);
            TileLaunch L;
            TILE_TPR_SWITCH(W.tb.tpr,
                L = tile_launch(ctx, W.tb, (const void*)k_opt_b<TPR>);
                CFA_LAUNCH(ctx, (k_opt_b<TPR>), L.grid, kTileThreads, L.smem, tv, a.oss->d_inv_m, z, p, beta_ptr, pn,
                           W.gx.p, W.gy.p, done));
            if (dot) launch_opt_k<true, false, true>(ctx, W, a, z, p, beta_ptr, pn, q, cond, done);
            else launch_opt_k<true, false, false>(ctx, W, a, z, p, beta_ptr, pn, q, cond, done);
        } else {
            if (dot) launch_opt_k<false, true, true>(ctx, W, a, z, p, beta_ptr, pn, q, cond, done);
            else launch_opt_k<false, true, false>(ctx, W, a, z, p, beta_ptr, pn, q, cond, done);
        }
        return CFA_OK;
    }
    const int tpr = op_tpr(a.n, a.nnz);
    const int grid = row_grid(ctx, a.n, tpr);
    CgState* st = W.st.p;
    if (a.oss) {
        const cfa_mesh* m = a.oss->mesh;
        OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_op_b<TPR>), grid, kThreads, 0, a.n, a.nnz, a.rp, a.ci, a.oss->d_oss_val,
                                      a.oss->d_inv_m, z, p, beta_ptr, pn, W.gx.p, W.gy.p, done));
        if (dot)
            OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_op_k<TPR, true, false, true>), grid, kThreads, 0, a.n, a.nnz, a.rp,
                                          a.ci, a.val, a.oss->d_oss_val, m->tag, m->bc, z, p, beta_ptr, pn, W.gx.p,
                                          W.gy.p, q, st, W.part.p, W.counter.p, cond, done));
        else
            OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_op_k<TPR, true, false, false>), grid, kThreads, 0, a.n, a.nnz, a.rp,
                                          a.ci, a.val, a.oss->d_oss_val, m->tag, m->bc, z, p, beta_ptr, pn, W.gx.p,
                                          W.gy.p, q, st, W.part.p, W.counter.p, cond, done));
    } else {
        OutletBc nobc;
        if (dot)
            OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_op_k<TPR, false, true, true>), grid, kThreads, 0, a.n, a.nnz, a.rp,
                                          a.ci, a.val, (const double*)nullptr, (const int*)nullptr, nobc, z, p, beta_ptr,
                                          pn, (const double*)nullptr, (const double*)nullptr, q, st, W.part.p,
                                          W.counter.p, cond, done));
        else
            OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_op_k<TPR, false, true, false>), grid, kThreads, 0, a.n, a.nnz, a.rp,
                                          a.ci, a.val, (const double*)nullptr, (const int*)nullptr, nobc, z, p, beta_ptr,
                                          pn, (const double*)nullptr, (const double*)nullptr, q, st, W.part.p,
                                          W.counter.p, cond, done));
    }
    return CFA_OK;
}

// This operator's values into the tile-streamed layout (fused: the K - B^T M^-1 B values).
static cfa_status pack_operator(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a) {
    if (a.oss && W.fused) {
        const cfa_mesh* m = a.oss->mesh;
        const long long nnz2 = W.tk.nnz;
        CFA_LAUNCH(ctx, k_oss_fuse, (int)std::min<long long>((nnz2 + kThreads - 1) / kThreads, 16LL * ctx->num_sms),
                   kThreads, 0, nnz2, a.n, a.nnz, a.ci, a.val, a.oss->d_oss_val, m->tag, m->bc, a.oss->d_inv_m,
                   (const int*)W.rp2.p, (const int*)W.slot_row.p, (const int*)W.kpos.p, (const int*)W.pair_ptr.p,
                   (const int*)W.pa.p, (const int*)W.pf.p, W.tk.view(W.err.p), W.tk.data.p);
        tile_fence(ctx);
    } else if (a.oss) {
        const double* o = a.oss->d_oss_val;
        const size_t nz = (size_t)a.nnz;
        CFA_PROPAGATE(pack_tiled(ctx, a.rp, a.ci, o, o + nz, nullptr, W.tb));
        CFA_PROPAGATE(pack_tiled(ctx, a.rp, a.ci, a.val, o + 2 * nz, o + 3 * nz, W.tk));
    } else {
        CFA_PROPAGATE(pack_tiled(ctx, a.rp, a.ci, a.val, nullptr, nullptr, W.tk));
    }
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

static cfa_status pcg_init(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a, CondArg cond) {
    const int n = a.n;
    const int gv = row_grid(ctx, n, 1);
    CgState* st = W.st.p;
    const int* done = &st->done;
    if (W.tiled) CFA_PROPAGATE(pack_operator(ctx, W, a));   // this solve's operator values
    CFA_LAUNCH(ctx, k_cg_bnorm, gv, kThreads, 0, n, a.b, st, W.part.p, W.counter.p, cond);
    if (!a.amg && !a.prec) CFA_LAUNCH(ctx, k_inv_diag, ceil_div(n, kThreads), kThreads, 0, n, a.rp, a.ci, a.val, W.dinv.p);
    // q = A x (pn scratch receives x)
    CFA_PROPAGATE(pcg_operator(ctx, W, a, a.x, a.x, nullptr, W.pn.p, W.q.p, false, cond, done));
    if (a.extra) {
        CFA_CHECK_LAUNCH();
        a.extra(a.x, W.q.p, a.extra_user);
    }
    CFA_LAUNCH(ctx, k_cg_resid0, gv, kThreads, 0, n, a.b, W.q.p, W.r.p, st, W.part.p, W.counter.p, cond);
    if (a.prec) {
        CFA_CHECK_LAUNCH();
        a.prec(W.r.p, W.z.p, a.prec_user);
    } else if (a.amg) {
        CFA_PROPAGATE(amg_vcycle(ctx, a.amg, W.r.p, W.z.p, done, a.vc64 != 0));
    } else {
        CFA_LAUNCH(ctx, k_vmul, gv, kThreads, 0, n, W.dinv.p, W.r.p, W.z.p);
    }
    CFA_LAUNCH(ctx, k_cg_nullx, ceil_div(n, kThreads), kThreads, 0, n, a.x, W.p.p, st);
    CFA_LAUNCH(ctx, k_cg_rz, gv, kThreads, 0, n, W.r.p, W.z.p, (const double*)W.q.p, 1, 0, st, W.part.p,
               W.counter.p, cond);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

// One iteration in the pieces that the host hooks separate: piece 0 is the operator (with the
// dot unless an extra operator follows), then extra(pn, q); piece 1 is pq, the update and the
// preconditioner unless it is a host hook, then prec(r, z); piece 2 is r.z after a host
// preconditioner (empty otherwise).
static bool pcg_piece_empty(const PcgArgs& a, int piece) { return piece == 2 && !a.prec; }

// The beta of the PCG with the FP32 V-cycle: Polak-Ribiere (flexible) unless CFA_PCG_FLEXIBLE=0.
static int pcg_flexible(const cfa_amg* amg) {
    if (amg->opts.precision != CFA_MIXED) return 0;
    const char* e = std::getenv("CFA_PCG_FLEXIBLE");
    return (e && e[0] == '0') ? 0 : 1;
}

static cfa_status pcg_piece(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a, int piece, CondArg cond) {
    const int n = a.n;
    const int gv = row_grid(ctx, n, 1);
    CgState* st = W.st.p;
    const int* done = &st->done;
    if (piece == 0) {
        // q = A pn with pn = z + beta p
        CFA_PROPAGATE(pcg_operator(ctx, W, a, W.z.p, W.p.p, &st->beta, W.pn.p, W.q.p, !a.extra, cond, done));
    } else if (piece == 1) {
        if (a.extra)
            CFA_LAUNCH(ctx, k_cg_pq, gv, kThreads, 0, n, (const double*)W.pn.p, (const double*)W.q.p, st, W.part.p,
                       W.counter.p, cond);
        if (a.amg || a.prec) {
            // the update (x, r, p, |r|, the stopping test) folded into the V-cycle's level 0 where
            // the hierarchy allows it (opt-in), else its own kernel, which also forms the level-0
            // pre-smoothing's scaled residual where the V-cycle takes it
            const bool fuse_update = !a.prec && amg_can_fuse_update(a.amg);
            PreScale ps{};
            const bool prescale = !a.prec && !fuse_update && amg_prescale(a.amg, &ps, a.vc64 != 0);
            if (!fuse_update) {
                if (prescale && ps.fp32)
                    CFA_LAUNCH(ctx, (k_cg_update<false, float>), gv, kThreads, 0, n, a.x, W.r.p, W.pn.p, W.p.p, W.q.p,
                               (const double*)nullptr, (double*)nullptr, st, W.part.p, W.counter.p, cond,
                               (const float*)ps.dinv, (float)ps.omega, reinterpret_cast<float*>(W.c0.p));
                else if (prescale)
                    CFA_LAUNCH(ctx, (k_cg_update<false, double>), gv, kThreads, 0, n, a.x, W.r.p, W.pn.p, W.p.p,
                               W.q.p, (const double*)nullptr, (double*)nullptr, st, W.part.p, W.counter.p, cond,
                               (const double*)ps.dinv, ps.omega, W.c0.p);
                else
                    CFA_LAUNCH(ctx, (k_cg_update<false, double>), gv, kThreads, 0, n, a.x, W.r.p, W.pn.p, W.p.p,
                               W.q.p, (const double*)nullptr, (double*)nullptr, st, W.part.p, W.counter.p, cond,
                               (const double*)nullptr, 0.0, (double*)nullptr);
            }
            if (!a.prec) {
                // z = M^-1 r with r.z (and z.q) folded into the V-cycle's last sweep where it can be
                const int flexible = pcg_flexible(a.amg);
                const RzFuse f{W.q.p, flexible, &st->rz, &st->beta, &st->alpha, W.part.p, W.counter.p};
                const CgFuse g{W.r.p, W.q.p, W.pn.p, a.x, W.p.p, st, W.part.p, W.counter.p, cond};
                bool fused = false;
                CFA_PROPAGATE(amg_vcycle_rz(ctx, a.amg, W.r.p, W.z.p, done, f, &fused, fuse_update ? &g : nullptr,
                                            prescale ? (const void*)W.c0.p : nullptr, a.vc64 != 0));
                if (!fused)
                    CFA_LAUNCH(ctx, k_cg_rz, gv, kThreads, 0, n, W.r.p, W.z.p, (const double*)W.q.p, 0, flexible, st,
                               W.part.p, W.counter.p, cond);
            }
        } else {
            CFA_LAUNCH(ctx, (k_cg_update<true, double>), gv, kThreads, 0, n, a.x, W.r.p, W.pn.p, W.p.p, W.q.p, W.dinv.p, W.z.p,
                       st, W.part.p, W.counter.p, cond, (const double*)nullptr, 0.0, (double*)nullptr);
        }
    } else if (a.prec) {
        CFA_LAUNCH(ctx, k_cg_rz, gv, kThreads, 0, n, W.r.p, W.z.p, (const double*)W.q.p, 0, 0, st, W.part.p,
                   W.counter.p, cond);
    }
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

// Between the two phases of a mixed-precision solve: where the FP64 phase stopped at its switch
// threshold (converged there, iterations left), the solve continues to the final tolerance: the
// stop is undone and the WHILE condition of the second phase set. Otherwise (the final
// tolerance already met, a breakdown, the iteration limit) the second phase does nothing. A
// warm start below the threshold stops the first phase at its initial residual (no iteration;
// p is still zero there, so the resumed V-cycle's beta multiplies nothing).
__global__ void k_cg_phase(CgState* st, double tol, CondArg cond) {
    CFA_GRID_DEP();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (st->converged && st->status == CFA_OK && st->iter < st->max_iter && !(st->rel < tol)) {
        st->tol = tol;
        st->done = 0;
        st->converged = 0;
        set_cond(cond, 1);
    } else if (st->converged) {
        st->tol = tol;
    }
}

// The second phase's start: z = M^-1 r for the residual the first phase stopped at (its V-cycle
// was skipped there), with the dots and the flexible beta as the iteration's own V-cycle forms them.
static cfa_status pcg_resume(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a, double tol, CondArg cond) {
    const int n = a.n;
    CgState* st = W.st.p;
    const int* done = &st->done;
    CFA_LAUNCH(ctx, k_cg_phase, 1, 32, 0, st, tol, cond);
    const int flexible = pcg_flexible(a.amg);
    const RzFuse f{W.q.p, flexible, &st->rz, &st->beta, &st->alpha, W.part.p, W.counter.p};
    bool fused = false;
    CFA_PROPAGATE(amg_vcycle_rz(ctx, a.amg, W.r.p, W.z.p, done, f, &fused, nullptr, nullptr, a.vc64 != 0));
    if (!fused)
        CFA_LAUNCH(ctx, k_cg_rz, row_grid(ctx, n, 1), kThreads, 0, n, W.r.p, W.z.p, (const double*)W.q.p, 0, flexible,
                   st, W.part.p, W.counter.p, cond);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

static void pcg_hook(const PcgArgs& a, PcgWork& W, int after_piece) {
    if (after_piece == 0 && a.extra) a.extra(W.pn.p, W.q.p, a.extra_user);
    if (after_piece == 1 && a.prec) a.prec(W.r.p, W.z.p, a.prec_user);
}

static cfa_status pcg_body(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a, CondArg cond) {
    for (int piece = 0; piece < 3; ++piece) {
        if (pcg_piece_empty(a, piece)) continue;
        CFA_PROPAGATE(pcg_piece(ctx, W, a, piece, cond));
        pcg_hook(a, W, piece);
    }
    return CFA_OK;
}

// Replays `sg` (capturing it first when its key changed)
template <class F>
static cfa_status run_segment(cfa_ctx* ctx, SegGraph& sg, const std::vector<const void*>& key, F fn) {
    if (!sg.exec || sg.key != key) {
        sg.reset();
        const long long l0 = ctx->launches;
        CFA_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const cfa_status s = fn();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        sg.kernels = ctx->launches - l0;
        ctx->launches = l0;
        if (s != CFA_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (s != CFA_OK) return s;
            CFA_CUDA(e);
        }
        const cudaError_t ei = cudaGraphInstantiate(&sg.exec, g, 0);
        cudaGraphDestroy(g);
        CFA_CUDA(ei);
        sg.key = key;
    }
    CFA_CUDA(cudaGraphLaunch(sg.exec, ctx->stream));
    ctx->launches += sg.kernels;
    return CFA_OK;
}

// The iteration with host hooks: each piece a captured graph, the hooks called between them
static cfa_status pcg_body_segments(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a, const std::vector<const void*>& key) {
    CondArg none{0, 0};
    for (int piece = 0; piece < 3; ++piece) {
        if (pcg_piece_empty(a, piece)) continue;
        CFA_PROPAGATE(run_segment(ctx, W.seg[piece], key, [&] { return pcg_piece(ctx, W, a, piece, none); }));
        pcg_hook(a, W, piece);
    }
    return CFA_OK;
}

static std::vector<const void*> operator_key(int n, int nnz, const int* rp, const int* ci, const double* val,
                                             const cfa_oss_operator* oss) {
    return {rp, ci, val, oss ? oss->d_oss_val : nullptr, oss ? oss->d_inv_m : nullptr,
            (const void*)(intptr_t)(oss ? oss->mesh->uid : 0), (const void*)(intptr_t)n, (const void*)(intptr_t)nnz};
}

static cfa_status ensure_pcg_vectors(cfa_ctx* ctx, PcgWork& W, int n) {
    if (n > W.cap) {
        W.graph.reset();
        W.graph2.reset();
        for (SegGraph& g : W.seg) g.reset();
        for (DevBuf<double>* b : {&W.r, &W.z, &W.p, &W.pn, &W.q, &W.gx, &W.gy, &W.dinv, &W.c0}) CFA_CUDA(b->ensure(n));
        CFA_CUDA(W.st.ensure(1));
        CFA_CUDA(W.counter.ensure(1));
        CFA_CUDA(cudaMemsetAsync(W.counter.p, 0, sizeof(unsigned int), ctx->stream));
        W.cap = n;
    }
    if (!W.err.p) {
        CFA_CUDA(W.err.ensure(1));
        CFA_CUDA(cudaMemsetAsync(W.err.p, 0, sizeof(int), ctx->stream));
    }
    CFA_CUDA(W.part.ensure(8 * 8 * (size_t)ctx->num_sms + 64));
    return CFA_OK;
}

static bool tiles_enabled() {
    const char* e = std::getenv("CFA_TILES");
    return !(e && e[0] == '0');
}

template <int TPR>
static void allow_operator_tpr() {
    allow_tile_kernel((const void*)k_opt_b<TPR>);
    allow_tile_kernel((const void*)k_opt_k<TPR, true, false, true>);
    allow_tile_kernel((const void*)k_opt_k<TPR, true, false, false>);
    allow_tile_kernel((const void*)k_opt_k<TPR, false, true, true>);
    allow_tile_kernel((const void*)k_opt_k<TPR, false, true, false>);
}

static void allow_operator_kernels() {
    static std::once_flag once;
    std::call_once(once, [] {
        allow_operator_tpr<1>(); allow_operator_tpr<2>(); allow_operator_tpr<4>();
        allow_operator_tpr<8>(); allow_operator_tpr<16>(); allow_operator_tpr<32>();
    });
}

static bool oss_fused_enabled() {
    const char* e = std::getenv("CFA_OSS_FUSED");
    return !(e && e[0] == '0');
}

// Two-ring pattern (rp2, ci2) of the fused OSS operator; ok = false when a row is longer than
// kRing2Max (the operator then stays in two passes).
static cfa_status plan_ring2(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a, bool& ok) {
    const int n = a.n;
    ok = false;
    CFA_CUDA(W.cnt2.ensure(n + 1));
    CFA_CUDA(W.rp2.ensure(n + 1));
    CFA_CUDA(W.err.ensure(1));
    CFA_CUDA(cudaMemsetAsync(W.err.p, 0, sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_ring2_count, ceil_div(n + 1, kThreads), kThreads, 0, n, a.rp, a.ci, W.cnt2.p, W.err.p);
    size_t tmp = 0;
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, W.cnt2.p, W.rp2.p, n + 1, ctx->stream));
    CFA_CUDA(W.scan_tmp.ensure(tmp + 16));
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(W.scan_tmp.p, tmp, W.cnt2.p, W.rp2.p, n + 1, ctx->stream));
    int h[2] = {0, 0};
    CFA_CUDA(cudaMemcpyAsync(&h[0], W.err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(&h[1], W.rp2.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    CFA_CUDA(cudaMemsetAsync(W.err.p, 0, sizeof(int), ctx->stream));
    if (h[0]) return CFA_OK;
    const int nnz2 = h[1];
    CFA_CUDA(W.ci2.ensure(std::max(nnz2, 1)));
    CFA_LAUNCH(ctx, k_ring2_fill, ceil_div(n, kThreads), kThreads, 0, n, a.rp, a.ci, (const int*)W.rp2.p, W.ci2.p);
    // per-entry plan: row, K position, pair counts, then the pairs
    CFA_CUDA(W.slot_row.ensure(std::max(nnz2, 1)));
    CFA_CUDA(W.kpos.ensure(std::max(nnz2, 1)));
    CFA_CUDA(W.cnt2.ensure(nnz2 + 1));
    CFA_CUDA(W.pair_ptr.ensure(nnz2 + 1));
    CFA_CUDA(cudaMemsetAsync(W.cnt2.p + nnz2, 0, sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_ring2_slots, ceil_div(n, kThreads), kThreads, 0, n, a.rp, a.ci, (const int*)W.rp2.p,
               (const int*)W.ci2.p, W.slot_row.p, W.kpos.p, W.cnt2.p, (const int*)nullptr, (int*)nullptr,
               (int*)nullptr);
    tmp = 0;
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, W.cnt2.p, W.pair_ptr.p, nnz2 + 1, ctx->stream));
    CFA_CUDA(W.scan_tmp.ensure(tmp + 16));
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(W.scan_tmp.p, tmp, W.cnt2.p, W.pair_ptr.p, nnz2 + 1, ctx->stream));
    int npairs = 0;
    CFA_CUDA(cudaMemcpyAsync(&npairs, W.pair_ptr.p + nnz2, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    CFA_CUDA(W.pa.ensure(std::max(npairs, 1)));
    CFA_CUDA(W.pf.ensure(std::max(npairs, 1)));
    CFA_LAUNCH(ctx, k_ring2_slots, ceil_div(n, kThreads), kThreads, 0, n, a.rp, a.ci, (const int*)W.rp2.p,
               (const int*)W.ci2.p, (int*)nullptr, (int*)nullptr, (int*)nullptr, (const int*)W.pair_ptr.p, W.pa.p,
               W.pf.p);
    CFA_CHECK_LAUNCH();
    ok = true;
    return CFA_OK;
}

// Plans the tile-streamed operator for this pattern (host row pointer needed: one sync).
static cfa_status plan_operator_tiles(cfa_ctx* ctx, PcgWork& W, const PcgArgs& a) {
    W.tiled = tiles_enabled();
    if (!W.tiled) return CFA_OK;
    allow_operator_kernels();
    std::vector<const void*> key = {a.rp, a.ci, (const void*)(intptr_t)a.n, (const void*)(intptr_t)a.nnz,
                                    (const void*)(intptr_t)(a.oss ? 1 : 0), (const void*)(uintptr_t)a.fp};
    if (key == W.tile_key) return CFA_OK;
    std::vector<int> h_rp(a.n + 1);
    CFA_CUDA(cudaMemcpyAsync(h_rp.data(), a.rp, (a.n + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    W.fused = false;
    if (a.oss && oss_fused_enabled()) {
        bool ok = false;
        CFA_PROPAGATE(plan_ring2(ctx, W, a, ok));
        if (ok) {
            std::vector<int> h_rp2(a.n + 1);
            CFA_CUDA(cudaMemcpyAsync(h_rp2.data(), W.rp2.p, (a.n + 1) * sizeof(int), cudaMemcpyDeviceToHost,
                                     ctx->stream));
            CFA_CUDA(cudaStreamSynchronize(ctx->stream));
            CFA_PROPAGATE(plan_tiled(ctx, h_rp2.data(), a.n, 1, 8, W.tk));
            CFA_PROPAGATE(pack_tiled(ctx, W.rp2.p, W.ci2.p, nullptr, nullptr, nullptr, W.tk));   // pattern only
            W.fused = true;
        }
    }
    if (a.oss && !W.fused) {
        CFA_PROPAGATE(plan_tiled(ctx, h_rp.data(), a.n, 2, 8, W.tb));
        CFA_PROPAGATE(plan_tiled(ctx, h_rp.data(), a.n, 3, 8, W.tk));
    } else if (!a.oss) {
        CFA_PROPAGATE(plan_tiled(ctx, h_rp.data(), a.n, 1, 8, W.tk));
    }
    W.tile_key = key;
    W.graph.reset();
    W.graph2.reset();
    for (SegGraph& g : W.seg) g.reset();
    return CFA_OK;
}

// nnz = rp[n] and the pattern's fingerprint, one synchronisation
static cfa_status pattern_info(cfa_ctx* ctx, int n, const int* rp, const int* ci, int& nnz, unsigned long long& fp) {
    PcgWork& W = work(ctx)->pcg;
    CFA_CUDA(W.fp.ensure(1));
    CFA_CUDA(cudaMemsetAsync(W.fp.p, 0, sizeof(unsigned long long), ctx->stream));
    CFA_LAUNCH(ctx, k_pattern_fingerprint, std::min(ceil_div(8 * n + 1, kThreads), 4 * ctx->num_sms), kThreads, 0, n, rp,
               ci, W.fp.p);
    CFA_CUDA(cudaMemcpyAsync(&ctx->h_pinned[0], W.fp.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(&ctx->h_pinned[1], rp + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(&fp, &ctx->h_pinned[0], sizeof(fp));
    std::memcpy(&nnz, &ctx->h_pinned[1], sizeof(nnz));
    return CFA_OK;
}

static cfa_status pcg_solve(cfa_ctx* ctx, const PcgArgs& a, cfa_solve_report* rep) {
    PcgWork& W = work(ctx)->pcg;
    const int n = a.n;
    CFA_PROPAGATE(ensure_pcg_vectors(ctx, W, n));
    CFA_PROPAGATE(plan_operator_tiles(ctx, W, a));
    W.prepared.clear();
    // a mixed hierarchy's FP64 first phase, down to the switch threshold, then the FP32 V-cycles
    const double sw = (a.amg && !a.host_ops()) ? amg_fp64_phase(a.amg) : 0.0;
    const bool two = sw > a.tol;
    PcgArgs a1 = a;
    a1.vc64 = two ? 1 : 0;
    // parameters
    CgState init{};
    init.tol = two ? sw : a.tol;
    init.max_iter = a.max_iter;
    CFA_CUDA(cudaMemcpyAsync(W.st.p, &init, sizeof(CgState), cudaMemcpyHostToDevice, ctx->stream));
    CFA_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    long long extra_body = 0;
    const cfa_mesh* om = a.oss ? a.oss->mesh : nullptr;
    const std::vector<const void*> key = {a.rp, a.ci, a.val, a.b, a.x, a.oss ? a.oss->d_oss_val : nullptr,
                                          a.oss ? a.oss->d_inv_m : nullptr, (const void*)(intptr_t)(om ? om->uid : 0),
                                          (const void*)(intptr_t)(om ? om->bc.outlet_dirichlet : 0),
                                          (const void*)(intptr_t)(om ? om->bc.pin : 0),
                                          (const void*)(intptr_t)(a.amg ? a.amg->version : 0),
                                          (const void*)(intptr_t)n, (const void*)(intptr_t)a.nnz,
                                          (const void*)(intptr_t)((a.extra ? 1 : 0) | (a.prec ? 2 : 0)),
                                          (const void*)(uintptr_t)a.fp};
    if (graphs_enabled() && !a.host_ops()) {
        std::vector<const void*> key1 = key;
        key1.push_back((const void*)(intptr_t)(two ? 1 : 0));
        if (!W.graph.exec || W.graph.key != key1) {
            CFA_PROPAGATE(build_graph(ctx, W.graph, [&](CondArg c) { return pcg_init(ctx, W, a1, c); },
                                      [&](CondArg c) { return pcg_body(ctx, W, a1, c); }));
            W.graph.key = key1;
        }
        CFA_CUDA(cudaGraphLaunch(W.graph.exec, ctx->stream));
        extra_body = W.graph.body_kernels;
        ctx->launches += W.graph.init_kernels;
        if (two) {
            if (!W.graph2.exec || W.graph2.key != key) {
                CFA_PROPAGATE(build_graph(ctx, W.graph2, [&](CondArg c) { return pcg_resume(ctx, W, a, a.tol, c); },
                                          [&](CondArg c) { return pcg_body(ctx, W, a, c); }));
                W.graph2.key = key;
            }
            CFA_CUDA(cudaGraphLaunch(W.graph2.exec, ctx->stream));
            ctx->launches += W.graph2.init_kernels;
        }
    } else {
        CondArg none{0, 0};
        CFA_PROPAGATE(pcg_init(ctx, W, a1, none));
        const bool segments = graphs_enabled();   // host hooks: one graph per piece of the iteration
        for (int phase = 0; phase < (two ? 2 : 1); ++phase) {
            const PcgArgs& ap = phase == 0 ? a1 : a;
            if (phase == 1) CFA_PROPAGATE(pcg_resume(ctx, W, a, a.tol, none));
            int polled = 0;
            for (int it = 0; it < a.max_iter; ++it) {
                if (segments) CFA_PROPAGATE(pcg_body_segments(ctx, W, ap, key));
                else CFA_PROPAGATE(pcg_body(ctx, W, ap, none));
                if (++polled == 8 || it + 1 == a.max_iter) {
                    polled = 0;
                    int d = 0;
                    CFA_CUDA(cudaMemcpyAsync(&d, &W.st.p->done, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
                    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
                    if (d) break;
                }
            }
        }
    }
    CFA_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    CgState h;
    int h_err = 0;
    CFA_CUDA(cudaMemcpyAsync(&h, W.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(&h_err, W.err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    int h_amg_err = 0;
    if (a.amg && a.amg->err.p)
        CFA_CUDA(cudaMemcpyAsync(&h_amg_err, a.amg->err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h_amg_err) cudaMemsetAsync(a.amg->err.p, 0, sizeof(int), ctx->stream);
    if (h_err || h_amg_err) {
        cudaMemsetAsync(W.err.p, 0, sizeof(int), ctx->stream);
        return set_error(ctx, CFA_TIMEOUT, "a bounded wait of a tile pipeline timed out", __FILE__, __LINE__);
    }
    float ms = 0.f;
    CFA_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->launches += extra_body * (long long)(h.iter + (h.status == CFA_BREAKDOWN ? 1 : 0));
    if (rep) {
        rep->iterations[0] = h.iter;
        rep->iterations[1] = 0;
        rep->converged[0] = h.converged;
        rep->converged[1] = 1;
        rep->rel_residual[0] = h.rel;
        rep->rel_residual[1] = 0.0;
        rep->solve_ms = ms;
    }
    if (h.status == CFA_BREAKDOWN) return CFA_BREAKDOWN;
    return h.converged ? CFA_OK : CFA_NOT_CONVERGED;
}

// ---------------------------------------------------------------------------------------------
// BiCGSTAB2
// ---------------------------------------------------------------------------------------------
struct B2Args {
    int n, nnz;
    const int *rp, *ci;
    const double* val;
    const double *bu, *bv;
    double *xu, *xv;
    const cfa_ilu* ilu;
    int max_iter;
    double tol;
};

// the interleaved pair view of a work vector (2 n doubles, 16-byte aligned)
static inline double2* pair(double* p) { return reinterpret_cast<double2*>(p); }
static inline const double2* pair(const double* p) { return reinterpret_cast<const double2*>(p); }

template <int MODE>
static void launch_b2t(cfa_ctx* ctx, B2Work& W, const B2Args& a, const double* in, const double* aux, double* out,
                       CondArg cond) {
    const TileView tv = W.tA.view(W.err.p);
    TileLaunch L;
    TILE_TPR_SWITCH(W.tA.tpr,
        L = tile_launch(ctx, W.tA, (const void*)k_b2t<TPR, MODE>);
        CFA_LAUNCH(ctx, (k_b2t<TPR, MODE>), L.grid, kTileThreads, L.smem, tv, a.n, (const double*)a.xu,
                   (const double*)a.xv, a.bu, a.bv, pair(in), pair(aux), pair(out), pair(W.r.p), pair(W.r0.p),
                   pair(W.p.p), W.st.p, W.part.p, W.counter.p, cond));
}

template <int TPR>
static void allow_b2_tpr() {
    allow_tile_kernel((const void*)k_b2t<TPR, 0>);
    allow_tile_kernel((const void*)k_b2t<TPR, 1>);
    allow_tile_kernel((const void*)k_b2t<TPR, 2>);
}

static cfa_status plan_b2_tiles(cfa_ctx* ctx, B2Work& W, const B2Args& a) {
    const char* e = std::getenv("CFA_TILES");
    W.tiled = !(e && e[0] == '0');
    if (!W.tiled) return CFA_OK;
    static std::once_flag once;
    std::call_once(once, [] {
        allow_b2_tpr<1>(); allow_b2_tpr<2>(); allow_b2_tpr<4>(); allow_b2_tpr<8>(); allow_b2_tpr<16>(); allow_b2_tpr<32>();
    });
    if (!W.err.p) {
        CFA_CUDA(W.err.ensure(1));
        CFA_CUDA(cudaMemsetAsync(W.err.p, 0, sizeof(int), ctx->stream));
    }
    // the ILU handle's uid changes with every set_pattern, and its pattern is the matrix's, so a
    // new mesh at the same addresses gets a new plan
    std::vector<const void*> key = {a.rp, a.ci, (const void*)(intptr_t)a.n, (const void*)(intptr_t)a.nnz,
                                    (const void*)(intptr_t)a.ilu->uid};
    if (key == W.tile_key) return CFA_OK;
    std::vector<int> h_rp(a.n + 1);
    CFA_CUDA(cudaMemcpyAsync(h_rp.data(), a.rp, (a.n + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    CFA_PROPAGATE(plan_tiled(ctx, h_rp.data(), a.n, 1, 8, W.tA));
    W.tile_key = key;
    W.graph.reset();
    return CFA_OK;
}

static cfa_status b2_init(cfa_ctx* ctx, B2Work& W, const B2Args& a, CondArg cond) {
    if (W.tiled) {
        CFA_PROPAGATE(pack_tiled(ctx, a.rp, a.ci, a.val, nullptr, nullptr, W.tA));
        launch_b2t<0>(ctx, W, a, nullptr, nullptr, W.v.p, cond);
        CFA_CHECK_LAUNCH();
        return CFA_OK;
    }
    const int tpr = op_tpr(a.n, a.nnz);
    const int grid = row_grid(ctx, a.n, tpr);
    OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_b2_init<TPR>), grid, kThreads, 0, a.n, a.rp, a.ci, a.val, (const double*)a.xu,
                                  (const double*)a.xv, a.bu, a.bv, pair(W.r.p), pair(W.r0.p), pair(W.p.p),
                                  pair(W.v.p), W.st.p, W.part.p, W.counter.p, cond));
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

static cfa_status b2_body(cfa_ctx* ctx, B2Work& W, const B2Args& a, CondArg cond) {
    const int n = a.n;
    const int tpr = op_tpr(a.n, a.nnz);
    const int grid = row_grid(ctx, n, tpr);
    const int gv = row_grid(ctx, n, 1);
    const int* done = &W.st.p->done;
    // p and s written into the ILU apply's work vector as they are formed (its first pass)
    IluStaging stg{};
    const bool staged = ilu_pair_staging(a.ilu, &stg);
    const int* spos = staged ? stg.pos : nullptr;
    float2* w32 = staged && stg.fp32 ? static_cast<float2*>(stg.w) : nullptr;
    double2* w64 = staged && !stg.fp32 ? static_cast<double2*>(stg.w) : nullptr;
    CFA_LAUNCH(ctx, k_b2_p, gv, kThreads, 0, n, pair(W.r.p), pair(W.v.p), pair(W.p.p), W.st.p, spos, w32, w64);
    CFA_PROPAGATE(ilu_apply_pair(ctx, a.ilu, W.p.p, W.phat.p, done, staged));
    if (W.tiled) launch_b2t<1>(ctx, W, a, W.phat.p, W.r0.p, W.v.p, cond);
    else
        OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_b2_v<TPR>), grid, kThreads, 0, n, a.rp, a.ci, a.val, pair(W.phat.p),
                                      pair(W.r0.p), pair(W.v.p), W.st.p, W.part.p, W.counter.p, cond));
    CFA_LAUNCH(ctx, k_b2_s, gv, kThreads, 0, n, pair(W.r.p), pair(W.v.p), pair(W.s.p), W.st.p, spos, w32, w64);
    CFA_PROPAGATE(ilu_apply_pair(ctx, a.ilu, W.s.p, W.shat.p, done, staged));
    if (W.tiled) launch_b2t<2>(ctx, W, a, W.shat.p, W.s.p, W.t.p, cond);
    else
        OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_b2_t<TPR>), grid, kThreads, 0, n, a.rp, a.ci, a.val, pair(W.shat.p),
                                      pair(W.s.p), pair(W.t.p), W.st.p, W.part.p, W.counter.p));
    CFA_LAUNCH(ctx, k_b2_xr, gv, kThreads, 0, n, a.xu, a.xv, pair(W.phat.p), pair(W.shat.p),
               pair(W.s.p), pair(W.t.p), pair(W.r.p), pair(W.r0.p), W.st.p, W.part.p, W.counter.p, cond);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

static cfa_status b2_solve(cfa_ctx* ctx, const B2Args& a, cfa_solve_report* rep) {
    B2Work& W = work(ctx)->b2;
    const int n = a.n;
    if (n > W.cap) {
        W.graph.reset();
        for (DevBuf<double>* b : {&W.r, &W.r0, &W.p, &W.v, &W.s, &W.t, &W.phat, &W.shat}) CFA_CUDA(b->ensure(2 * (size_t)n));
        CFA_CUDA(W.st.ensure(1));
        CFA_CUDA(W.counter.ensure(1));
        CFA_CUDA(cudaMemsetAsync(W.counter.p, 0, sizeof(unsigned int), ctx->stream));
        W.cap = n;
    }
    CFA_CUDA(W.part.ensure(8 * 8 * (size_t)ctx->num_sms + 64));   // NV <= 8 partials x max grid
    CFA_PROPAGATE(plan_b2_tiles(ctx, W, a));
    B2State init{};
    init.tol = a.tol;
    init.max_iter = a.max_iter;
    CFA_CUDA(cudaMemcpyAsync(W.st.p, &init, sizeof(B2State), cudaMemcpyHostToDevice, ctx->stream));
    CFA_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    long long extra_body = 0;
    if (graphs_enabled()) {
        std::vector<const void*> key = {a.rp, a.ci, a.val, a.bu, a.bv, a.xu, a.xv, (const void*)(intptr_t)a.ilu->uid,
                                        (const void*)(intptr_t)n, (const void*)(intptr_t)a.nnz};
        if (!W.graph.exec || W.graph.key != key) {
            CFA_PROPAGATE(build_graph(ctx, W.graph, [&](CondArg c) { return b2_init(ctx, W, a, c); },
                                      [&](CondArg c) { return b2_body(ctx, W, a, c); }));
            W.graph.key = key;
        }
        CFA_CUDA(cudaGraphLaunch(W.graph.exec, ctx->stream));
        extra_body = W.graph.body_kernels;
        ctx->launches += W.graph.init_kernels;
    } else {
        CondArg none{0, 0};
        CFA_PROPAGATE(b2_init(ctx, W, a, none));
        int polled = 0;
        for (int it = 0; it < a.max_iter; ++it) {
            CFA_PROPAGATE(b2_body(ctx, W, a, none));
            if (++polled == 4 || it + 1 == a.max_iter) {
                polled = 0;
                int d = 0;
                CFA_CUDA(cudaMemcpyAsync(&d, &W.st.p->done, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
                CFA_CUDA(cudaStreamSynchronize(ctx->stream));
                if (d) break;
            }
        }
    }
    CFA_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    B2State h;
    int h_err = 0;
    CFA_CUDA(cudaMemcpyAsync(&h, W.st.p, sizeof(B2State), cudaMemcpyDeviceToHost, ctx->stream));
    if (W.err.p) CFA_CUDA(cudaMemcpyAsync(&h_err, W.err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h_err) {
        cudaMemsetAsync(W.err.p, 0, sizeof(int), ctx->stream);
        return set_error(ctx, CFA_TIMEOUT, "a bounded wait of a tile pipeline timed out", __FILE__, __LINE__);
    }
    float ms = 0.f;
    CFA_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->launches += extra_body * (long long)(h.iter + 1);
    if (rep) {
        for (int c = 0; c < 2; ++c) {
            rep->iterations[c] = h.iters[c];
            rep->converged[c] = h.conv[c];
            rep->rel_residual[c] = h.rel[c];
        }
        rep->solve_ms = ms;
    }
    return (h.conv[0] && h.conv[1]) ? CFA_OK : CFA_NOT_CONVERGED;
}

}  // namespace cfa

using namespace cfa;

extern "C" {

cfa_status cfa_spmv(cfa_ctx* ctx, int n, const int* rp, const int* ci, const double* val, const double* x, double* y) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && rp && ci && val && x && y);
    const int tpr = 4;
    CFA_LAUNCH(ctx, (k_spmv<4, 1>), row_grid(ctx, n, tpr), kThreads, 0, n, rp, ci, val, x, y);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_spmv_multi(cfa_ctx* ctx, int n, int nrhs, const int* rp, const int* ci, const double* val,
                          const double* x, double* y) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && (nrhs == 1 || nrhs == 2) && rp && ci && val && x && y);
    if (nrhs == 1) CFA_LAUNCH(ctx, (k_spmv<4, 1>), row_grid(ctx, n, 4), kThreads, 0, n, rp, ci, val, x, y);
    else CFA_LAUNCH(ctx, (k_spmv<4, 2>), row_grid(ctx, n, 4), kThreads, 0, n, rp, ci, val, x, y);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_pressure_operator_prepare(cfa_ctx* ctx, int n, int nnz, const int* rp, const int* ci, const double* val,
                                         const cfa_oss_operator* oss) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && nnz > 0 && rp && ci && val);
    CFA_ARG(!oss || (oss->mesh && oss->d_oss_val && oss->d_inv_m && oss->mesh->n == n));
    PcgWork& W = work(ctx)->pcg;
    CFA_PROPAGATE(ensure_pcg_vectors(ctx, W, n));
    int nnz_dev = 0;
    unsigned long long fp = 0;
    CFA_PROPAGATE(pattern_info(ctx, n, rp, ci, nnz_dev, fp));
    CFA_ARG(nnz_dev == nnz);
    PcgArgs a{n, nnz, rp, ci, val, nullptr, nullptr, oss, nullptr, 0, 0.0};
    a.fp = fp;
    CFA_PROPAGATE(plan_operator_tiles(ctx, W, a));
    W.prepared.clear();
    if (!W.tiled) return CFA_OK;
    CFA_PROPAGATE(pack_operator(ctx, W, a));
    W.prepared = operator_key(n, nnz, rp, ci, val, oss);
    return CFA_OK;
}

cfa_status cfa_pressure_operator_layout(const cfa_ctx* ctx, int* passes, long long* stored_nnz) {
    CFA_ENTER(ctx);
    if (!ctx->work) return CFA_BAD_ARG;
    const PcgWork& W = ctx->work->pcg;
    if (W.prepared.empty()) return CFA_BAD_ARG;
    const bool two = W.tiled && W.tb.nnz > 0 && !W.fused;
    if (passes) *passes = two ? 2 : 1;
    if (stored_nnz) *stored_nnz = W.tk.nnz;
    return CFA_OK;
}

cfa_status cfa_pressure_operator(cfa_ctx* ctx, int n, int nnz, const int* rp, const int* ci, const double* val,
                                 const cfa_oss_operator* oss, const double* x, double* y) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && nnz > 0 && rp && ci && val && x && y);
    CFA_ARG(!oss || (oss->mesh && oss->d_oss_val && oss->d_inv_m && oss->mesh->n == n));
    PcgWork& W = work(ctx)->pcg;
    CFA_PROPAGATE(ensure_pcg_vectors(ctx, W, n));
    W.tiled = tiles_enabled() && !W.prepared.empty() && W.prepared == operator_key(n, nnz, rp, ci, val, oss);
    PcgArgs a{n, nnz, rp, ci, val, nullptr, nullptr, oss, nullptr, 0, 0.0};
    CondArg none{0, 0};
    CFA_PROPAGATE(pcg_operator(ctx, W, a, x, x, nullptr, W.pn.p, y, false, none, nullptr));
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_oss_apply(cfa_ctx* ctx, const cfa_mesh* m, const double* oss_val, const double* inv_m, const double* in,
                         double* out) {
    CFA_ENTER(ctx);
    CFA_ARG(m && oss_val && inv_m && in && out);
    // out -= B^T M^-1 B in: pass 1 into the PCG scratch g, pass 2 with K = 0 contributions
    PcgWork& W = work(ctx)->pcg;
    const int n = m->n;
    CFA_PROPAGATE(ensure_pcg_vectors(ctx, W, n));
    W.tiled = false;
    DevBuf<double> zeroK;
    CFA_CUDA(zeroK.ensure(std::max(m->nnz, 1)));
    CFA_CUDA(cudaMemsetAsync(zeroK.p, 0, (size_t)m->nnz * sizeof(double), ctx->stream));
    cfa_oss_operator op{m, oss_val, inv_m};
    PcgArgs a{n, m->nnz, m->rp, m->ci, zeroK.p, nullptr, nullptr, &op, nullptr, 0, 0.0};
    CondArg none{0, 0};
    CFA_PROPAGATE(pcg_operator(ctx, W, a, in, in, nullptr, W.pn.p, W.q.p, false, none, nullptr));
    // out += q (q = -B^T g on non-Dirichlet rows, 0 elsewhere)
    CFA_LAUNCH(ctx, k_axpy, row_grid(ctx, n, 1), kThreads, 0, n, 1.0, (const double*)W.q.p, out);
    CFA_CHECK_LAUNCH();
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFA_OK;
}

cfa_status cfa_pcg_solve(cfa_ctx* ctx, int n, const int* rp, const int* ci, const double* val, const double* b,
                         double* x, const cfa_oss_operator* oss, cfa_amg* amg, const cfa_solve_opts* opts,
                         cfa_solve_report* rep) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && rp && ci && val && b && x && opts && opts->max_iter >= 0);
    CFA_ARG(!oss || (oss->mesh && oss->d_oss_val && oss->d_inv_m && oss->mesh->n == n));
    CFA_ARG(!amg || (amg->coarse_n > 0 && (amg->levels.empty() ? amg->coarse_n == n : amg->levels[0].A.rows == n)));
    int nnz = 0;
    unsigned long long fp = 0;
    CFA_PROPAGATE(pattern_info(ctx, n, rp, ci, nnz, fp));
    PcgArgs a{n, nnz, rp, ci, val, b, x, oss, amg, opts->max_iter, opts->tol};
    a.fp = fp;
    if (opts->max_iter == 0) {
        if (rep) { *rep = cfa_solve_report{}; rep->converged[0] = 0; rep->converged[1] = 1; }
        return CFA_NOT_CONVERGED;
    }
    return pcg_solve(ctx, a, rep);
}

cfa_status cfa_pcg_solve_host_ops(cfa_ctx* ctx, int n, const int* rp, const int* ci, const double* val,
                                  const double* b, double* x, cfa_host_op extra_op, void* extra_user, cfa_amg* amg,
                                  cfa_host_op precond, void* precond_user, const cfa_solve_opts* opts,
                                  cfa_solve_report* rep) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && rp && ci && val && b && x && opts && opts->max_iter >= 0 && !(amg && precond));
    CFA_ARG(!amg || (amg->coarse_n > 0 && (amg->levels.empty() ? amg->coarse_n == n : amg->levels[0].A.rows == n)));
    int nnz = 0;
    unsigned long long fp = 0;
    CFA_PROPAGATE(pattern_info(ctx, n, rp, ci, nnz, fp));
    PcgArgs a{n, nnz, rp, ci, val, b, x, nullptr, amg, opts->max_iter, opts->tol};
    a.fp = fp;
    a.extra = extra_op;
    a.extra_user = extra_user;
    a.prec = precond;
    a.prec_user = precond_user;
    if (opts->max_iter == 0) {
        if (rep) { *rep = cfa_solve_report{}; rep->converged[0] = 0; rep->converged[1] = 1; }
        return CFA_NOT_CONVERGED;
    }
    return pcg_solve(ctx, a, rep);
}

cfa_status cfa_bicgstab2_solve(cfa_ctx* ctx, int n, const int* rp, const int* ci, const double* val, const double* bu,
                               const double* bv, double* xu, double* xv, const cfa_ilu* ilu, const cfa_solve_opts* opts,
                               cfa_solve_report* rep) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && rp && ci && val && bu && bv && xu && xv && ilu && opts && ilu->n == n && opts->max_iter > 0);
    B2Args a{n, ilu->nnz, rp, ci, val, bu, bv, xu, xv, ilu, opts->max_iter, opts->tol};
    return b2_solve(ctx, a, rep);
}

cfa_status cfa_bicgstab_solve(cfa_ctx* ctx, int n, const int* rp, const int* ci, const double* val, const double* b,
                              double* x, const cfa_solve_opts* opts, cfa_solve_report* rep) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && rp && ci && val && b && x && opts);
    DevBuf<double> r, r0, p, v, s, t, phat, shat, dinv, dots;
    for (DevBuf<double>* buf : {&r, &r0, &p, &v, &s, &t, &phat, &shat, &dinv}) CFA_CUDA(buf->ensure(n));
    CFA_CUDA(dots.ensure(8));
    DevBuf<unsigned int> counter;
    CFA_CUDA(counter.ensure(1));
    CFA_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned int), ctx->stream));
    const int gv = row_grid(ctx, n, 1);
    DevBuf<double> part;
    CFA_CUDA(part.ensure(gv + 16));
    auto spmv = [&](const double* in, double* out) {
        CFA_LAUNCH(ctx, (k_spmv<4, 1>), row_grid(ctx, n, 4), kThreads, 0, n, rp, ci, val, in, out);
    };
    auto dot = [&](const double* aa, const double* bb) -> double {
        CFA_LAUNCH(ctx, k_dot, gv, kThreads, 0, n, aa, bb, dots.p, part.p, counter.p);
        double h = 0.0;
        cudaMemcpyAsync(&h, dots.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        return h;
    };
    CFA_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    CFA_LAUNCH(ctx, k_inv_diag, ceil_div(n, kThreads), kThreads, 0, n, rp, ci, val, dinv.p);
    spmv(x, v.p);
    CFA_LAUNCH(ctx, k_axpby, gv, kThreads, 0, n, 1.0, b, -1.0, (const double*)v.p, r.p);
    CFA_CUDA(cudaMemcpyAsync(r0.p, r.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(p.p, r.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CFA_CUDA(cudaMemsetAsync(v.p, 0, n * sizeof(double), ctx->stream));
    const double r_norm0 = std::sqrt(dot(r.p, r.p));
    int iter = 0;
    bool fin = false;
    double rel = 0.0;
    if (r_norm0 < 1.0e-13) {
        fin = true;
    } else {
        double rho_old = 1.0, alpha = 1.0, omega = 1.0;
        const double breakdown = 1.0e-30 * r_norm0 * r_norm0 + 1.0e-300;
        for (; iter < opts->max_iter; ++iter) {
            const double rho_new = dot(r0.p, r.p);
            if (std::fabs(rho_new) < breakdown) break;
            if (iter > 0) {
                const double beta = (rho_new / rho_old) * (alpha / (omega + 1.0e-30));
                CFA_LAUNCH(ctx, k_bicg_p, gv, kThreads, 0, n, (const double*)r.p, (const double*)v.p, beta, omega, p.p);
            }
            CFA_LAUNCH(ctx, k_vmul, gv, kThreads, 0, n, (const double*)dinv.p, (const double*)p.p, phat.p);
            spmv(phat.p, v.p);
            const double r0v = dot(r0.p, v.p);
            if (std::fabs(r0v) < breakdown) break;
            alpha = rho_new / r0v;
            CFA_LAUNCH(ctx, k_axpby, gv, kThreads, 0, n, 1.0, (const double*)r.p, -alpha, (const double*)v.p, s.p);
            const double s_norm = std::sqrt(dot(s.p, s.p));
            if (s_norm < opts->tol * r_norm0 || s_norm < 1.0e-11) {
                CFA_LAUNCH(ctx, k_axpy, gv, kThreads, 0, n, alpha, (const double*)phat.p, x);
                ++iter;
                fin = true;
                break;
            }
            CFA_LAUNCH(ctx, k_vmul, gv, kThreads, 0, n, (const double*)dinv.p, (const double*)s.p, shat.p);
            spmv(shat.p, t.p);
            const double tt = dot(t.p, t.p);
            omega = (tt > breakdown) ? (dot(t.p, s.p) / tt) : 0.0;
            CFA_LAUNCH(ctx, k_axpy, gv, kThreads, 0, n, alpha, (const double*)phat.p, x);
            CFA_LAUNCH(ctx, k_axpy, gv, kThreads, 0, n, omega, (const double*)shat.p, x);
            CFA_LAUNCH(ctx, k_axpby, gv, kThreads, 0, n, 1.0, (const double*)s.p, -omega, (const double*)t.p, r.p);
            const double r_norm = std::sqrt(dot(r.p, r.p));
            rel = r_norm / r_norm0;
            if (r_norm < opts->tol * r_norm0 || r_norm < 1.0e-11) { ++iter; fin = true; break; }
            rho_old = rho_new;
        }
    }
    CFA_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    CFA_CHECK_LAUNCH();
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    if (rep) {
        rep->iterations[0] = iter; rep->iterations[1] = 0;
        rep->converged[0] = fin; rep->converged[1] = 1;
        rep->rel_residual[0] = rel; rep->rel_residual[1] = 0.0;
        rep->solve_ms = ms;
    }
    return fin ? CFA_OK : CFA_NOT_CONVERGED;
}

}  // extern "C"

// =============================================================================================
// cfa_oss_apply_noalloc: the OSS apply with its intermediate vector in static device memory
// =============================================================================================
namespace cfa {

// Largest mesh (nodes) cfa_oss_apply_noalloc accepts; its scratch is 2 * kOssStaticRows doubles
// (8 MiB), reserved when the library's device code is loaded on a device.
constexpr int kOssStaticRows = 1 << 19;

// g = M_L^-1 B x of the OSS apply: [0, n) the x component, [kOssStaticRows, + n) the y component.
// Nothing in it needs to start at zero: each call writes every entry it later reads.
static __device__ __align__(256) double g_oss_static[2 * kOssStaticRows];

// Pass 2 of the OSS apply on its own: out -= B^T_x g_x + B^T_y g_y on rows that are not pressure
// Dirichlet rows (k_oss_apply_BT, src/cfa/fem_kernels.cuh:871-885); the same per-row summation
// order as the operator kernel of cfa_oss_apply.
template <int TPR>
__global__ void k_oss_bt_sub(int n, int nnz, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ oss, const int* __restrict__ tag, OutletBc bc,
                             const double* __restrict__ gx, const double* __restrict__ gy, double* __restrict__ out) {
    CFA_GRID_DEP();
    const double* BTx = oss + 2 * (size_t)nnz;
    const double* BTy = oss + 3 * (size_t)nnz;
    ROWS_BEGIN(TPR, n)
    double so = 0.0;
    if (valid)
        for (int k = rp[row] + lane; k < rp[row + 1]; k += TPR) {
            const int j = ci[k];
            so += BTx[k] * gx[j] + BTy[k] * gy[j];
        }
    so = group_reduce<TPR>(so);
    if (valid && lane == 0 && !pressure_dirichlet(row, tag[row], bc)) out[row] -= so;
    ROWS_END
}

// Makes a device current for the lifetime of the object and restores the caller's device after.
struct CurrentDevice {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit CurrentDevice(int device) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
        else prev = -1;
    }
    ~CurrentDevice() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Device address of g_oss_static on the current device (the context's), looked up on the first
// call there and kept for the life of the process.
static cfa_status oss_static_scratch(cfa_ctx* ctx, double** out) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static double* addr[kMaxDevices] = {};
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return set_error(ctx, CFA_BAD_ARG, "device ordinal out of range", __FILE__, __LINE__);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[ctx->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_oss_static);
        if (e != cudaSuccess) return set_error(ctx, CFA_CUDA_ERROR, cudaGetErrorString(e), __FILE__, __LINE__);
        addr[ctx->device] = static_cast<double*>(p);
    }
    *out = addr[ctx->device];
    return CFA_OK;
}

}  // namespace cfa

extern "C" {

cfa_status cfa_oss_apply_noalloc(cfa_ctx* ctx, const cfa_mesh* m, const double* oss_val, const double* inv_m,
                                 const double* in, double* out) {
    CFA_ENTER(ctx);
    CFA_ARG(m && oss_val && inv_m && in && out);
    const int n = m->n;
    if (n > kOssStaticRows)
        return set_error(ctx, CFA_BAD_ARG,
                         "cfa_oss_apply_noalloc: the mesh has more nodes than its static scratch holds (524288)",
                         __FILE__, __LINE__);
    // the scratch address and the launches belong to the context's device, whichever device the
    // caller has current
    CurrentDevice on_device(ctx->device);
    if (on_device.err != cudaSuccess)
        return set_error(ctx, CFA_CUDA_ERROR, cudaGetErrorString(on_device.err), __FILE__, __LINE__);
    double* g = nullptr;
    CFA_PROPAGATE(oss_static_scratch(ctx, &g));
    double* gx = g;
    double* gy = g + kOssStaticRows;
    const int tpr = op_tpr(n, m->nnz);
    const int grid = row_grid(ctx, n, tpr);
    OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_op_b<TPR>), grid, kThreads, 0, n, m->nnz, m->rp, m->ci, oss_val, inv_m, in,
                                  (const double*)nullptr, (const double*)nullptr, (double*)nullptr, gx, gy,
                                  (const int*)nullptr));
    OP_TPR_SWITCH(tpr, CFA_LAUNCH(ctx, (k_oss_bt_sub<TPR>), grid, kThreads, 0, n, m->nnz, m->rp, m->ci, oss_val,
                                  m->tag, m->bc, (const double*)gx, (const double*)gy, out));
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

}  // extern "C"
