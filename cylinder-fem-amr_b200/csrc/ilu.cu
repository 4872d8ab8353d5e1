// Multicolour ILU(0): the greedy colouring on the host exactly as MulticolourIlu0::set_pattern
// (src/cfa/linalg.cuh:456-528), the split pattern and elimination program from it on the
// device (k_ilu_program); factor colour by colour in FP64
// (k_ilu0_factor_colour, :366-392); sweeps colour by colour with one thread per row handling
// both right-hand sides, so the factors are read once per apply (the reference's
// k_ilu0_lower/upper_colour, :406-433, use a thread per row and component and read them twice).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>

#include "ilu.cuh"

namespace cfa {

constexpr int kIluMaxRow = 32;   // ILU_MAX_ROW (src/cfa/linalg.cuh:361)

// Row i of colour c (k_ilu0_factor_colour, src/cfa/linalg.cuh:363-392): for its L entries k in
// elimination order, l_ik = a_ik / u_kk and a_ij -= l_ik u_kj within the pattern. The matching of
// row k's columns against row i's pattern is done once per pattern (the elimination program
// built in cfa_ilu_create), so the arithmetic -- the same operations in the same order as the
// reference kernel -- is a plain gather loop.
__global__ void k_ilu_factor_colour(int m, const int* __restrict__ rows, const int* __restrict__ rp,
                                    const int* __restrict__ ep, const int4* __restrict__ elim,
                                    const int2* __restrict__ upd, int t0, double* __restrict__ lu) {
    CFA_GRID_DEP();
    const int tl = blockIdx.x * blockDim.x + threadIdx.x;
    if (tl >= m) return;
    const int t = t0 + tl;
    const int i = rows[t];
    const int s = rp[i], len = rp[i + 1] - s;
    double a[kIluMaxRow];
    for (int q = 0; q < len; ++q) a[q] = lu[s + q];
    const int e1 = ep[t + 1];
    for (int e = ep[t]; e < e1; ++e) {
        const int4 el = elim[e];
        const double lik = a[el.x] / lu[el.y];
        a[el.x] = lik;
        for (int u = el.z; u < el.w; ++u) {
            const int2 up = upd[u];
            a[up.x] -= lik * lu[up.y];
        }
    }
    for (int q = 0; q < len; ++q) lu[s + q] = a[q];
}

// k_ilu0_gather (src/cfa/linalg.cuh:395-402), in the factor precision
template <class T>
__global__ void k_ilu_gather(int nl, int nu, int n, const int* __restrict__ l_src, const int* __restrict__ u_src,
                             const int* __restrict__ d_src, const double* __restrict__ lu, T* __restrict__ lv,
                             T* __restrict__ uv, T* __restrict__ dinv) {
    CFA_GRID_DEP();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nl) lv[e] = (T)lu[l_src[e]];
    if (e < nu) uv[e] = (T)lu[u_src[e]];
    if (e < n) dinv[e] = (T)(1.0 / lu[d_src[e]]);
}

// entries of a row whose loads the sweeps issue together
constexpr int kIluBatch = 4;

// Forward sweep of one colour for NR right-hand sides: y_i = r_i - sum_L l_ie y_e (unit L); the
// last colour also divides by u_ii. T: factor/work precision; FP64 output written when a row is
// final (last colour here, else in the backward sweep).
template <class V, class T, int NR>
__global__ void k_ilu_lower(int m, int n, const int* __restrict__ rows, const int* __restrict__ lp,
                            const int* __restrict__ lc, const V* __restrict__ lv, const V* __restrict__ dinv,
                            int last, const double* __restrict__ r, T* __restrict__ w, double* __restrict__ z,
                            const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int i = rows[t];
    T acc[NR];
#pragma unroll
    for (int c = 0; c < NR; ++c) acc[c] = (T)r[(size_t)c * n + i];
    const int end = lp[t + 1];
    for (int e0 = lp[t]; e0 < end; e0 += kIluBatch) {
        // the loads of a batch of entries first, then the updates in entry order
        V l[kIluBatch];
        T g[kIluBatch][NR];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < end) {
                const int j = lc[e0 + u];
                l[u] = lv[e0 + u];
#pragma unroll
                for (int c = 0; c < NR; ++c) g[u][c] = w[(size_t)c * n + j];
            }
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < end)
#pragma unroll
                for (int c = 0; c < NR; ++c) acc[c] -= (T)l[u] * g[u][c];
    }
    if (last) {
        const T d = (T)dinv[t];
#pragma unroll
        for (int c = 0; c < NR; ++c) {
            acc[c] = acc[c] * d;
            z[(size_t)c * n + i] = (double)acc[c];
        }
    }
#pragma unroll
    for (int c = 0; c < NR; ++c) w[(size_t)c * n + i] = acc[c];
}

// Backward sweep of one colour: z_i = (y_i - sum_U u_ie z_e) / u_ii
template <class V, class T, int NR>
__global__ void k_ilu_upper(int m, int n, const int* __restrict__ rows, const int* __restrict__ up,
                            const int* __restrict__ uc, const V* __restrict__ uv, const V* __restrict__ dinv,
                            T* __restrict__ w, double* __restrict__ z, const int* __restrict__ done) {
    CFA_GRID_DEP();
    if (done && *done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int i = rows[t];
    T acc[NR];
#pragma unroll
    for (int c = 0; c < NR; ++c) acc[c] = w[(size_t)c * n + i];
    const int end = up[t + 1];
    for (int e0 = up[t]; e0 < end; e0 += kIluBatch) {
        V uu[kIluBatch];
        T g[kIluBatch][NR];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < end) {
                const int j = uc[e0 + u];
                uu[u] = uv[e0 + u];
#pragma unroll
                for (int c = 0; c < NR; ++c) g[u][c] = w[(size_t)c * n + j];
            }
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < end)
#pragma unroll
                for (int c = 0; c < NR; ++c) acc[c] -= (T)uu[u] * g[u][c];
    }
    const T d = (T)dinv[t];
#pragma unroll
    for (int c = 0; c < NR; ++c) {
        acc[c] = acc[c] * d;
        w[(size_t)c * n + i] = acc[c];
        z[(size_t)c * n + i] = (double)acc[c];
    }
}

template <class V, class T, int NR>
static void sweeps(cfa_ctx* ctx, const cfa_ilu* h, const V* lv, const V* uv, const V* dinv, T* w,
                   const double* r, double* z, const int* done) {
    const int n = h->n;
    for (int c = 0; c < h->nc; ++c) {
        const int cs = h->colour_start[c], m = h->colour_start[c + 1] - cs;
        if (m == 0) continue;
        CFA_LAUNCH(ctx, (k_ilu_lower<V, T, NR>), ceil_div(m, kThreads), kThreads, 0, m, n, h->rows.p + cs, h->lp.p + cs,
                   h->lc.p, lv, dinv + cs, c == h->nc - 1 ? 1 : 0, r, w, z, done);
    }
    for (int c = h->nc - 2; c >= 0; --c) {
        const int cs = h->colour_start[c], m = h->colour_start[c + 1] - cs;
        if (m == 0) continue;
        CFA_LAUNCH(ctx, (k_ilu_upper<V, T, NR>), ceil_div(m, kThreads), kThreads, 0, m, n, h->rows.p + cs, h->up.p + cs,
                   h->uc.p, uv, dinv + cs, w, z, done);
    }
}

// ---- sweeps for the momentum solve's pair of right-hand sides stored interleaved per row ----
// r[i] = (u_i, v_i) as one double2, so a row's own and gathered accesses of both components are
// one 16-byte (FP64) or 8-byte (FP32 work vector) load in one sector. Each colour kernel first
// loads the data that do not change during a solve (its rows, their split-pattern offsets, the
// first kIluBatch column indices and factor values, the diagonal), then waits for the previous
// kernel (griddepcontrol.wait), so that with programmatic dependent launch these loads overlap
// the previous colour's tail. With `early` set, each block also signals its dependents at once
// (griddepcontrol.launch_dependents), so the next colour's blocks are scheduled, and do their
// own loads, while this colour still runs. Those loads read only the factors and the pattern,
// written before the solve began. Streamed data go through the evict-first path (__ldcs) when
// `stream_hint` is set, so that the work vector stays in L2 across the colour kernels.
template <class T> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };

template <class X>
__device__ __forceinline__ X ld_stream(const X* p, bool hint) { return hint ? __ldcs(p) : __ldg(p); }

__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Forward sweep of one colour: y_i = r_i - sum_L l_ie y_e for both components (unit L); the last
// colour also divides by u_ii and writes z. T: sweep arithmetic and work-vector precision (SEP:
// w is a separate T work vector; otherwise w is z, FP64 in place).
template <class V, class T, bool SEP>
__global__ void __launch_bounds__(kThreads)
k_ilu_lower_pair(int m, const int* __restrict__ rows, const int* __restrict__ lp, const int* __restrict__ lc,
                 const V* __restrict__ lv, const V* __restrict__ dinv, int last, const double2* __restrict__ r,
                 typename Pair<T>::type* __restrict__ w, double2* __restrict__ z, const int* __restrict__ done,
                 int early, int hint) {
    using T2 = typename Pair<T>::type;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = t < m;
    int i = 0, b = 0, e = 0;
    int j[kIluBatch];
    V l[kIluBatch];
    V d = V(0);
    if (valid) {
        i = ld_stream(rows + t, hint);
        b = ld_stream(lp + t, hint);
        e = ld_stream(lp + t + 1, hint);
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) {
                j[u] = ld_stream(lc + b + u, hint);
                l[u] = ld_stream(lv + b + u, hint);
            }
        if (last) d = ld_stream(dinv + t, hint);
    }
    if (early) pdl_launch_dependents();
    CFA_GRID_DEP();
    if (done && *done) return;
    if (!valid) return;
    const double2 rr = r[i];
    T a0 = (T)rr.x, a1 = (T)rr.y;
    {
        T2 g[kIluBatch];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) g[u] = w[j[u]];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) {
                a0 -= (T)l[u] * g[u].x;
                a1 -= (T)l[u] * g[u].y;
            }
    }
    for (int e0 = b + kIluBatch; e0 < e; e0 += kIluBatch) {
        V lq[kIluBatch];
        T2 g[kIluBatch];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < e) {
                lq[u] = ld_stream(lv + e0 + u, hint);
                g[u] = w[ld_stream(lc + e0 + u, hint)];
            }
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < e) {
                a0 -= (T)lq[u] * g[u].x;
                a1 -= (T)lq[u] * g[u].y;
            }
    }
    if (last) {
        a0 = a0 * (T)d;
        a1 = a1 * (T)d;
        if (SEP) z[i] = make_double2((double)a0, (double)a1);
    }
    T2 o;
    o.x = a0;
    o.y = a1;
    w[i] = o;
}

// Backward sweep of one colour: z_i = (y_i - sum_U u_ie z_e) / u_ii, both components.
template <class V, class T, bool SEP>
__global__ void __launch_bounds__(kThreads)
k_ilu_upper_pair(int m, const int* __restrict__ rows, const int* __restrict__ up, const int* __restrict__ uc,
                 const V* __restrict__ uv, const V* __restrict__ dinv, typename Pair<T>::type* __restrict__ w,
                 double2* __restrict__ z, const int* __restrict__ done, int early, int hint) {
    using T2 = typename Pair<T>::type;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = t < m;
    int i = 0, b = 0, e = 0;
    int j[kIluBatch];
    V q[kIluBatch];
    V d = V(0);
    if (valid) {
        i = ld_stream(rows + t, hint);
        b = ld_stream(up + t, hint);
        e = ld_stream(up + t + 1, hint);
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) {
                j[u] = ld_stream(uc + b + u, hint);
                q[u] = ld_stream(uv + b + u, hint);
            }
        d = ld_stream(dinv + t, hint);
    }
    if (early) pdl_launch_dependents();
    CFA_GRID_DEP();
    if (done && *done) return;
    if (!valid) return;
    const T2 own = w[i];
    T a0 = own.x, a1 = own.y;
    {
        T2 g[kIluBatch];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) g[u] = w[j[u]];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) {
                a0 -= (T)q[u] * g[u].x;
                a1 -= (T)q[u] * g[u].y;
            }
    }
    for (int e0 = b + kIluBatch; e0 < e; e0 += kIluBatch) {
        V qq[kIluBatch];
        T2 g[kIluBatch];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < e) {
                qq[u] = ld_stream(uv + e0 + u, hint);
                g[u] = w[ld_stream(uc + e0 + u, hint)];
            }
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < e) {
                a0 -= (T)qq[u] * g[u].x;
                a1 -= (T)qq[u] * g[u].y;
            }
    }
    a0 = a0 * (T)d;
    a1 = a1 * (T)d;
    T2 o;
    o.x = a0;
    o.y = a1;
    w[i] = o;
    if (SEP) z[i] = make_double2((double)a0, (double)a1);
}

// Runtime switches of the pair sweeps, read once: CFA_ILU_EARLY=0 drops the early dependent
// launch, CFA_ILU_HINT=1 turns on the evict-first loads of the streamed factors (measured slower
// on the 402k- and 4.2M-vertex meshes), CFA_ILU_PERM=0 selects the natural-order sweeps below instead of the
// colour-order ones.
static int env_flag(const char* name, int def) {
    const char* e = std::getenv(name);
    return e ? (e[0] != '0') : def;
}

template <class V, class T, bool SEP>
static void sweeps_pair(cfa_ctx* ctx, const cfa_ilu* h, const V* lv, const V* uv, const V* dinv,
                        typename Pair<T>::type* w, const double2* r, double2* z, const int* done) {
    static const int early = env_flag("CFA_ILU_EARLY", 1);
    static const int hint = env_flag("CFA_ILU_HINT", 0);
    for (int c = 0; c < h->nc; ++c) {
        const int cs = h->colour_start[c], m = h->colour_start[c + 1] - cs;
        if (m == 0) continue;
        CFA_LAUNCH(ctx, (k_ilu_lower_pair<V, T, SEP>), ceil_div(m, kThreads), kThreads, 0, m, h->rows.p + cs,
                   h->lp.p + cs, h->lc.p, lv, dinv + cs, c == h->nc - 1 ? 1 : 0, r, w, z, done, early, hint);
    }
    for (int c = h->nc - 2; c >= 0; --c) {
        const int cs = h->colour_start[c], m = h->colour_start[c + 1] - cs;
        if (m == 0) continue;
        CFA_LAUNCH(ctx, (k_ilu_upper_pair<V, T, SEP>), ceil_div(m, kThreads), kThreads, 0, m, h->rows.p + cs,
                   h->up.p + cs, h->uc.p, uv, dinv + cs, w, z, done, early, hint);
    }
}

// ---- the same sweeps with the work vector in colour order ----
// In the reference's natural row order the rows of one colour are scattered over the whole
// vector, so every colour kernel touches most 32-byte sectors of r, w and z for a sixth of their
// rows. Here the work vector w is held in colour order (position t = the row's place in `rows`):
// the first kernel runs over the rows in natural order, reads r coalesced and puts each row's
// pair at its colour position (colour 0 has no L entries: its forward sweep is this copy); the
// colour kernels read and write their own rows of w contiguously and gather their neighbours
// through column indices mapped to colour positions (lcp, ucp); the last kernel runs in natural
// order again, does colour 0's backward step and writes z coalesced. The arithmetic is that of
// k_ilu_lower_pair / k_ilu_upper_pair, entry for entry.
template <class T>
__global__ void __launch_bounds__(kThreads)
k_ilu_first_perm(int n, const int* __restrict__ pos, const double2* __restrict__ r, typename Pair<T>::type* __restrict__ w,
                 const int* __restrict__ done, int early) {
    using T2 = typename Pair<T>::type;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = i < n ? __ldg(pos + i) : 0;
    if (early) pdl_launch_dependents();
    CFA_GRID_DEP();
    if (done && *done) return;
    if (i >= n) return;
    const double2 v = r[i];
    T2 o;
    o.x = (T)v.x;
    o.y = (T)v.y;
    w[t] = o;
}

// Forward sweep of colour c (positions cs .. cs + m): y_t = y_t - sum_L l_te y_e; the last
// colour also divides by u_tt.
template <class V, class T>
__global__ void __launch_bounds__(kThreads)
k_ilu_lower_perm(int m, int cs, const int* __restrict__ lp, const int* __restrict__ lcp, const V* __restrict__ lv,
                 const V* __restrict__ dinv, int last, typename Pair<T>::type* __restrict__ w,
                 const int* __restrict__ done, int early) {
    using T2 = typename Pair<T>::type;
    const int tl = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = tl < m;
    const int t = cs + tl;
    int b = 0, e = 0;
    int j[kIluBatch];
    V l[kIluBatch];
    V d = V(0);
    if (valid) {
        b = __ldg(lp + t);
        e = __ldg(lp + t + 1);
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) {
                j[u] = __ldg(lcp + b + u);
                l[u] = __ldg(lv + b + u);
            }
        if (last) d = __ldg(dinv + t);
    }
    if (early) pdl_launch_dependents();
    CFA_GRID_DEP();
    if (done && *done) return;
    if (!valid) return;
    const T2 own = w[t];
    T a0 = own.x, a1 = own.y;
    {
        T2 g[kIluBatch];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) g[u] = w[j[u]];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) {
                a0 -= (T)l[u] * g[u].x;
                a1 -= (T)l[u] * g[u].y;
            }
    }
    for (int e0 = b + kIluBatch; e0 < e; e0 += kIluBatch) {
        V lq[kIluBatch];
        T2 g[kIluBatch];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < e) {
                lq[u] = __ldg(lv + e0 + u);
                g[u] = w[__ldg(lcp + e0 + u)];
            }
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < e) {
                a0 -= (T)lq[u] * g[u].x;
                a1 -= (T)lq[u] * g[u].y;
            }
    }
    if (last) {
        a0 = a0 * (T)d;
        a1 = a1 * (T)d;
    }
    T2 o;
    o.x = a0;
    o.y = a1;
    w[t] = o;
}

// Backward step of row t: (y_t - sum_U u_te z_e) / u_tt, both components.
template <class V, class T>
__device__ __forceinline__ typename Pair<T>::type ilu_upper_row(typename Pair<T>::type own, int b, int e,
                                                               const int (&j)[kIluBatch], const V (&q)[kIluBatch], V d,
                                                               const int* __restrict__ ucp, const V* __restrict__ uv,
                                                               const typename Pair<T>::type* __restrict__ w) {
    using T2 = typename Pair<T>::type;
    T a0 = own.x, a1 = own.y;
    {
        T2 g[kIluBatch];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) g[u] = w[j[u]];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (b + u < e) {
                a0 -= (T)q[u] * g[u].x;
                a1 -= (T)q[u] * g[u].y;
            }
    }
    for (int e0 = b + kIluBatch; e0 < e; e0 += kIluBatch) {
        V qq[kIluBatch];
        T2 g[kIluBatch];
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < e) {
                qq[u] = __ldg(uv + e0 + u);
                g[u] = w[__ldg(ucp + e0 + u)];
            }
#pragma unroll
        for (int u = 0; u < kIluBatch; ++u)
            if (e0 + u < e) {
                a0 -= (T)qq[u] * g[u].x;
                a1 -= (T)qq[u] * g[u].y;
            }
    }
    T2 o;
    o.x = a0 * (T)d;
    o.y = a1 * (T)d;
    return o;
}

template <class V>
__device__ __forceinline__ void ilu_upper_prefetch(int t, const int* __restrict__ up, const int* __restrict__ ucp,
                                                   const V* __restrict__ uv, const V* __restrict__ dinv, int& b, int& e,
                                                   int (&j)[kIluBatch], V (&q)[kIluBatch], V& d) {
    b = __ldg(up + t);
    e = __ldg(up + t + 1);
#pragma unroll
    for (int u = 0; u < kIluBatch; ++u)
        if (b + u < e) {
            j[u] = __ldg(ucp + b + u);
            q[u] = __ldg(uv + b + u);
        }
    d = __ldg(dinv + t);
}

// Backward sweep of colour c >= 1 (positions cs .. cs + m), in place in w.
template <class V, class T>
__global__ void __launch_bounds__(kThreads)
k_ilu_upper_perm(int m, int cs, const int* __restrict__ up, const int* __restrict__ ucp, const V* __restrict__ uv,
                 const V* __restrict__ dinv, typename Pair<T>::type* __restrict__ w, const int* __restrict__ done,
                 int early) {
    const int tl = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = tl < m;
    const int t = cs + tl;
    int b = 0, e = 0;
    int j[kIluBatch];
    V q[kIluBatch];
    V d = V(0);
    if (valid) ilu_upper_prefetch(t, up, ucp, uv, dinv, b, e, j, q, d);
    if (early) pdl_launch_dependents();
    CFA_GRID_DEP();
    if (done && *done) return;
    if (!valid) return;
    w[t] = ilu_upper_row<V, T>(w[t], b, e, j, q, d, ucp, uv, w);
}

// The last kernel, rows in natural order: colour 0's backward step (positions below c1) from w,
// every other row's final value copied; z written coalesced in FP64.
template <class V, class T>
__global__ void __launch_bounds__(kThreads)
k_ilu_last_perm(int n, int c1, const int* __restrict__ pos, const int* __restrict__ up, const int* __restrict__ ucp,
                const V* __restrict__ uv, const V* __restrict__ dinv, const typename Pair<T>::type* __restrict__ w,
                double2* __restrict__ z, const int* __restrict__ done) {
    using T2 = typename Pair<T>::type;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const int t = valid ? __ldg(pos + i) : 0;
    const bool c0 = valid && t < c1;
    int b = 0, e = 0;
    int j[kIluBatch];
    V q[kIluBatch];
    V d = V(0);
    if (c0) ilu_upper_prefetch(t, up, ucp, uv, dinv, b, e, j, q, d);
    CFA_GRID_DEP();
    if (done && *done) return;
    if (!valid) return;
    const T2 o = c0 ? ilu_upper_row<V, T>(w[t], b, e, j, q, d, ucp, uv, w) : w[t];
    z[i] = make_double2((double)o.x, (double)o.y);
}

template <class V, class T>
static void sweeps_perm(cfa_ctx* ctx, const cfa_ilu* h, const V* lv, const V* uv, const V* dinv,
                        typename Pair<T>::type* w, const double2* r, double2* z, const int* done, bool staged) {
    static const int early = env_flag("CFA_ILU_EARLY", 1);
    const int n = h->n;
    if (!staged)
        CFA_LAUNCH(ctx, (k_ilu_first_perm<T>), ceil_div(n, kThreads), kThreads, 0, n, (const int*)h->pos.p, r, w,
                   done, early);
    for (int c = 1; c < h->nc; ++c) {
        const int cs = h->colour_start[c], m = h->colour_start[c + 1] - cs;
        if (m == 0) continue;
        CFA_LAUNCH(ctx, (k_ilu_lower_perm<V, T>), ceil_div(m, kThreads), kThreads, 0, m, cs, (const int*)h->lp.p,
                   (const int*)h->lcp.p, lv, dinv, c == h->nc - 1 ? 1 : 0, w, done, early);
    }
    for (int c = h->nc - 2; c >= 1; --c) {
        const int cs = h->colour_start[c], m = h->colour_start[c + 1] - cs;
        if (m == 0) continue;
        CFA_LAUNCH(ctx, (k_ilu_upper_perm<V, T>), ceil_div(m, kThreads), kThreads, 0, m, cs, (const int*)h->up.p,
                   (const int*)h->ucp.p, uv, dinv, w, done, early);
    }
    CFA_LAUNCH(ctx, (k_ilu_last_perm<V, T>), ceil_div(n, kThreads), kThreads, 0, n, h->colour_start[1],
               (const int*)h->pos.p, (const int*)h->up.p, (const int*)h->ucp.p, uv, dinv,
               (const typename Pair<T>::type*)w, z, done);
}

// pos[rows[t]] = t, and the split pattern's column indices as colour positions
__global__ void k_ilu_positions(int n, const int* __restrict__ rows, int* __restrict__ pos) {
    CFA_GRID_DEP();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) pos[rows[t]] = t;
}

__global__ void k_ilu_map_cols(int count, const int* __restrict__ cols, const int* __restrict__ pos,
                               int* __restrict__ out) {
    CFA_GRID_DEP();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < count) out[e] = pos[cols[e]];
}


// Position of the mirrored entry (j, i) of every CSR entry (i, j) (binary search in row j);
// err set when the pattern is not structurally symmetric.
__global__ void k_mirror_positions(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                   int* __restrict__ tpos, int* __restrict__ err) {
    CFA_GRID_DEP();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int a = rp[i]; a < rp[i + 1]; ++a) {
        const int j = ci[a];
        if (j < 0 || j >= n) {   // not a pattern of n rows
            tpos[a] = a;
            atomicExch(err, 1);
            continue;
        }
        int lo = rp[j], hi = rp[j + 1] - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ci[mid] < i) lo = mid + 1;
            else hi = mid;
        }
        if (lo < rp[j + 1] && ci[lo] == i) tpos[a] = lo;
        else { tpos[a] = a; atomicExch(err, 1); }
    }
}

// The split factor of (LU)^T = (U^T D^-1)(D L^T) in the same colour order (rows in colour c only
// depend on colours < c in both triangles): unit lower L'_ij = U_ji / U_jj, upper
// U'_ij = U_ii L_ji, the same diagonal (src/cfa/linalg.cuh:531-541 factor, transposed).
template <class T>
__global__ void k_ilu_gather_transposed(int n, const int* __restrict__ rows, const int* __restrict__ lp,
                                        const int* __restrict__ up, const int* __restrict__ lc,
                                        const int* __restrict__ l_src, const int* __restrict__ u_src,
                                        const int* __restrict__ d_src, const int* __restrict__ diag,
                                        const int* __restrict__ tpos, const double* __restrict__ lu,
                                        T* __restrict__ lv, T* __restrict__ uv, T* __restrict__ dinv) {
    CFA_GRID_DEP();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double d = lu[d_src[t]];
    for (int e = lp[t]; e < lp[t + 1]; ++e) lv[e] = (T)(lu[tpos[l_src[e]]] / lu[diag[lc[e]]]);
    for (int e = up[t]; e < up[t + 1]; ++e) uv[e] = (T)(d * lu[tpos[u_src[e]]]);
    dinv[t] = (T)(1.0 / d);
}

__global__ void k_transpose_values(int nnz, const int* __restrict__ tpos, const double* __restrict__ val,
                                   double* __restrict__ out) {
    CFA_GRID_DEP();
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < nnz) out[a] = val[tpos[a]];
}

cfa_status ilu_apply(cfa_ctx* ctx, const cfa_ilu* h, const double* r, double* z, int nrhs, const int* done) {
    if (h->precision == CFA_MIXED) {
        // FP32 factors, FP64 vectors and arithmetic, in place in z
        if (nrhs == 1) sweeps<float, double, 1>(ctx, h, h->lv32.p, h->uv32.p, h->dinv32.p, z, r, z, done);
        else sweeps<float, double, 2>(ctx, h, h->lv32.p, h->uv32.p, h->dinv32.p, z, r, z, done);
    } else {
        // FP64: the sweeps work in place in z (as the reference)
        if (nrhs == 1) sweeps<double, double, 1>(ctx, h, h->lv64.p, h->uv64.p, h->dinv64.p, z, r, z, done);
        else sweeps<double, double, 2>(ctx, h, h->lv64.p, h->uv64.p, h->dinv64.p, z, r, z, done);
    }
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

bool ilu_pair_staging(const cfa_ilu* h, IluStaging* out) {
    if (!h || h->nc < 2 || !env_flag("CFA_ILU_PERM", 1) || !env_flag("CFA_ILU_STAGED", 1)) return false;
    const bool f32 = h->precision == CFA_MIXED;
    void* w = f32 ? (void*)h->work32.p : (void*)h->work64.p;
    if (!w || !h->pos.p) return false;
    out->pos = h->pos.p;
    out->w = w;
    out->fp32 = f32 ? 1 : 0;
    return true;
}

cfa_status ilu_apply_pair(cfa_ctx* ctx, const cfa_ilu* h, const double* r, double* z, const int* done, bool staged) {
    const double2* r2 = reinterpret_cast<const double2*>(r);
    double2* z2 = reinterpret_cast<double2*>(z);
    // colour order (default) or, with CFA_ILU_PERM=0, the reference's natural row order
    const bool colour_order = env_flag("CFA_ILU_PERM", 1) && h->nc >= 2;
    if (staged && !colour_order)
        return set_error(ctx, CFA_BAD_ARG, "staged ILU apply without the colour-order work vector", __FILE__, __LINE__);
    if (h->precision == CFA_MIXED) {
        // FP32 factors, FP32 sweeps on the handle's FP32 work vector; FP64 in and out
        if (!h->work32.p || h->work32.cap < 2 * (size_t)h->n)
            return set_error(ctx, CFA_BAD_ARG, "ILU handle without its FP32 work vector", __FILE__, __LINE__);
        float2* w = reinterpret_cast<float2*>(h->work32.p);
        if (colour_order) sweeps_perm<float, float>(ctx, h, h->lv32.p, h->uv32.p, h->dinv32.p, w, r2, z2, done, staged);
        else sweeps_pair<float, float, true>(ctx, h, h->lv32.p, h->uv32.p, h->dinv32.p, w, r2, z2, done);
    } else if (colour_order) {
        if (!h->work64.p || h->work64.cap < 2 * (size_t)h->n)
            return set_error(ctx, CFA_BAD_ARG, "ILU handle without its FP64 work vector", __FILE__, __LINE__);
        sweeps_perm<double, double>(ctx, h, h->lv64.p, h->uv64.p, h->dinv64.p,
                                    reinterpret_cast<double2*>(h->work64.p), r2, z2, done, staged);
    } else {
        sweeps_pair<double, double, false>(ctx, h, h->lv64.p, h->uv64.p, h->dinv64.p, z2, r2, z2, done);
    }
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

// Split pattern and elimination program of row t (rows in colour order), counted (FILL false)
// or written (FILL true) at the offsets lp[t], up[t] (= ep[t]: one elimination entry per L
// entry) and uo[t]. The L entries are taken colour by colour and, within a colour, in column
// order, and row k's matches in its own order: the operation sequence of the reference's
// k_ilu0_factor_colour (src/cfa/linalg.cuh:366-392). Thread per row.
template <bool FILL>
__global__ void k_ilu_program(int n, const int* __restrict__ rows, const int* __restrict__ rp,
                              const int* __restrict__ ci, const int* __restrict__ colour, const int* __restrict__ diag,
                              int* __restrict__ lcnt, int* __restrict__ ucnt, int* __restrict__ ocnt,
                              const int* __restrict__ lp, const int* __restrict__ up, const int* __restrict__ uo,
                              int* __restrict__ lc, int* __restrict__ uc, int* __restrict__ l_src,
                              int* __restrict__ u_src, int* __restrict__ d_src, int4* __restrict__ elim,
                              int2* __restrict__ upd) {
    CFA_GRID_DEP();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = rows[t];
    const int s0 = rp[i], len = rp[i + 1] - s0, cii = colour[i];
    int l = FILL ? lp[t] : 0, u = FILL ? up[t] : 0;
    for (int a = s0; a < s0 + len; ++a) {
        const int j = ci[a];
        if (j == i) {
            if (FILL) d_src[t] = a;
        } else if (colour[j] < cii) {
            if (FILL) { lc[l] = j; l_src[l] = a; }
            ++l;
        } else {
            if (FILL) { uc[u] = j; u_src[u] = a; }
            ++u;
        }
    }
    int e = FILL ? lp[t] : 0, o = FILL ? uo[t] : 0;
    for (int c = 0; c < cii; ++c) {
        for (int q = 0; q < len; ++q) {
            const int k = ci[s0 + q];
            if (colour[k] != c) continue;
            const int o0 = o;
            // rows k and i are sorted: one merge finds the common columns
            for (int mm = rp[k], b = 0; mm < rp[k + 1] && b < len;) {
                const int j = ci[mm], cb = ci[s0 + b];
                if (cb < j) { ++b; continue; }
                if (cb == j && colour[j] > c) {
                    if (FILL) upd[o] = make_int2(b, mm);
                    ++o;
                }
                ++mm;
            }
            if (FILL) elim[e] = make_int4(q, diag[k], o0, o);
            ++e;
        }
    }
    if (!FILL) {
        lcnt[t] = l;
        ucnt[t] = u;
        ocnt[t] = o;
    }
}

// set_pattern (src/cfa/linalg.cuh:456-528) into handle h, reusing its device buffers (they grow
// geometrically, as the reference's cap_n / cap_nnz). The greedy colouring (sequential by
// definition) runs on the host in node order; the split pattern and the elimination program
// are built on the device from it.
static cfa_status ilu_pattern(cfa_ctx* ctx, cfa_ilu* h, int n, const int* rp, const int* ci, const int* d_rp,
                              const int* d_ci) {
    (void)d_rp;
    (void)d_ci;
    const int nnz = rp[n];
    std::vector<int> colour(n, -1), diag(n, -1), mark;
    int nc = 0;
    for (int i = 0; i < n; ++i) {
        if (rp[i + 1] - rp[i] > kIluMaxRow)
            return set_error(ctx, CFA_ROW_TOO_LONG, "ILU row longer than 32 entries", __FILE__, __LINE__);
        for (int a = rp[i]; a < rp[i + 1]; ++a) {
            const int c = colour[ci[a]];
            if (c >= 0) mark[c] = i;
            if (ci[a] == i) diag[i] = a;
        }
        int c = 0;
        while (c < nc && mark[c] == i) ++c;
        if (c == nc) { ++nc; mark.push_back(-1); }
        colour[i] = c;
    }
    for (int r = 0; r < n; ++r)
        if (diag[r] < 0) return set_error(ctx, CFA_BAD_ARG, "ILU pattern row without a diagonal", __FILE__, __LINE__);
    h->uid = next_uid();
    h->n = n;
    h->nnz = nnz;
    h->nc = nc;
    h->mirror = false;
    h->transposed = false;
    h->colour_start.assign(nc + 1, 0);
    for (int i = 0; i < n; ++i) h->colour_start[colour[i] + 1]++;
    for (int c = 0; c < nc; ++c) h->colour_start[c + 1] += h->colour_start[c];
    std::vector<int> rows(n), fill(h->colour_start.begin(), h->colour_start.end() - 1);
    for (int i = 0; i < n; ++i) rows[fill[colour[i]]++] = i;

    // the handle's own copy of the pattern (the reference keeps the caller's device arrays; a
    // copy leaves nothing for the caller to keep alive), the colouring and the row order
    auto up_int = [&](DevBuf<int>& d, const int* v, size_t count) -> cudaError_t {
        cudaError_t e = d.ensure(std::max<size_t>(count, 1));
        if (e == cudaSuccess && count)
            e = cudaMemcpyAsync(d.p, v, count * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
        return e;
    };
    CFA_CUDA(up_int(h->own_rp, rp, (size_t)n + 1));
    CFA_CUDA(up_int(h->own_ci, ci, (size_t)nnz));
    h->rp = h->own_rp.p;
    h->ci = h->own_ci.p;
    CFA_CUDA(up_int(h->rows, rows.data(), n));
    CFA_CUDA(up_int(h->colour, colour.data(), n));
    CFA_CUDA(up_int(h->diag, diag.data(), n));

    // counts, offsets (exclusive sums into lp, up, ep and the update offsets), totals
    DevBuf<int> cnt;   // lcnt | ucnt | ocnt, n + 1 each
    CFA_CUDA(cnt.ensure(3 * ((size_t)n + 1)));
    int* lcnt = cnt.p;
    int* ucnt = cnt.p + (n + 1);
    int* ocnt = cnt.p + 2 * (size_t)(n + 1);
    CFA_CUDA(cudaMemsetAsync(cnt.p, 0, 3 * ((size_t)n + 1) * sizeof(int), ctx->stream));
    CFA_CUDA(h->lp.ensure(n + 1));
    CFA_CUDA(h->up.ensure(n + 1));
    CFA_CUDA(h->ep.ensure(n + 1));
    DevBuf<int> uo;
    CFA_CUDA(uo.ensure(n + 1));
    CFA_LAUNCH(ctx, k_ilu_program<false>, ceil_div(n, kThreads), kThreads, 0, n, (const int*)h->rows.p, h->rp, h->ci,
               (const int*)h->colour.p, (const int*)h->diag.p, lcnt, ucnt, ocnt, (const int*)nullptr,
               (const int*)nullptr, (const int*)nullptr, (int*)nullptr, (int*)nullptr, (int*)nullptr, (int*)nullptr,
               (int*)nullptr, (int4*)nullptr, (int2*)nullptr);
    size_t tmp_bytes = 0;
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, lcnt, h->lp.p, n + 1, ctx->stream));
    DevBuf<unsigned char> tmp;
    CFA_CUDA(tmp.ensure(std::max<size_t>(tmp_bytes, 1)));
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, lcnt, h->lp.p, n + 1, ctx->stream));
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, ucnt, h->up.p, n + 1, ctx->stream));
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, ocnt, uo.p, n + 1, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(h->ep.p, h->lp.p, ((size_t)n + 1) * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
    int tot[3] = {0, 0, 0};
    CFA_CUDA(cudaMemcpyAsync(&tot[0], h->lp.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(&tot[1], h->up.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(&tot[2], uo.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    h->nl = tot[0];
    h->nu = tot[1];
    h->n_elim = tot[0];
    h->n_upd = tot[2];

    for (DevBuf<int>* b : {&h->lc, &h->l_src}) CFA_CUDA(b->ensure(std::max(h->nl, 1)));
    for (DevBuf<int>* b : {&h->uc, &h->u_src}) CFA_CUDA(b->ensure(std::max(h->nu, 1)));
    CFA_CUDA(h->d_src.ensure(n));
    CFA_CUDA(h->elim.ensure(std::max(h->n_elim, 1)));
    CFA_CUDA(h->upd.ensure(std::max(h->n_upd, 1)));
    CFA_LAUNCH(ctx, k_ilu_program<true>, ceil_div(n, kThreads), kThreads, 0, n, (const int*)h->rows.p, h->rp, h->ci,
               (const int*)h->colour.p, (const int*)h->diag.p, (int*)nullptr, (int*)nullptr, (int*)nullptr,
               (const int*)h->lp.p, (const int*)h->up.p, (const int*)uo.p, h->lc.p, h->uc.p, h->l_src.p, h->u_src.p,
               h->d_src.p, h->elim.p, h->upd.p);
    // colour positions of the rows and of the split pattern's columns (the colour-order sweeps)
    CFA_CUDA(h->pos.ensure(n));
    CFA_CUDA(h->lcp.ensure(std::max(h->nl, 1)));
    CFA_CUDA(h->ucp.ensure(std::max(h->nu, 1)));
    CFA_LAUNCH(ctx, k_ilu_positions, ceil_div(n, kThreads), kThreads, 0, n, (const int*)h->rows.p, h->pos.p);
    if (h->nl > 0)
        CFA_LAUNCH(ctx, k_ilu_map_cols, ceil_div(h->nl, kThreads), kThreads, 0, h->nl, (const int*)h->lc.p,
                   (const int*)h->pos.p, h->lcp.p);
    if (h->nu > 0)
        CFA_LAUNCH(ctx, k_ilu_map_cols, ceil_div(h->nu, kThreads), kThreads, 0, h->nu, (const int*)h->uc.p,
                   (const int*)h->pos.p, h->ucp.p);
    CFA_CUDA(h->lu.ensure(nnz));
    if (h->precision == CFA_MIXED) {
        CFA_CUDA(h->lv32.ensure(std::max(h->nl, 1)));
        CFA_CUDA(h->uv32.ensure(std::max(h->nu, 1)));
        CFA_CUDA(h->dinv32.ensure(n));
        CFA_CUDA(h->work32.ensure(2 * (size_t)n));
    } else {
        CFA_CUDA(h->lv64.ensure(std::max(h->nl, 1)));
        CFA_CUDA(h->uv64.ensure(std::max(h->nu, 1)));
        CFA_CUDA(h->dinv64.ensure(n));
        CFA_CUDA(h->work64.ensure(2 * (size_t)n));
    }
    CFA_CHECK_LAUNCH();
    // the scratch buffers (cnt, uo, tmp) are released on return: wait for the kernels using them
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFA_OK;
}

}  // namespace cfa

using namespace cfa;

extern "C" {

cfa_status cfa_ilu_create(cfa_ctx* ctx, int n, const int* rp, const int* ci, const int* d_rp, const int* d_ci,
                          cfa_precision precision, cfa_ilu** out) {
    if (!out) return CFA_BAD_ARG;
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && rp && ci && d_rp && d_ci);
    CFA_ARG(precision == CFA_FP64 || precision == CFA_MIXED);
    *out = nullptr;
    auto* h = new cfa_ilu();
    h->precision = precision;
    const cfa_status st = ilu_pattern(ctx, h, n, rp, ci, d_rp, d_ci);
    if (st != CFA_OK) {
        delete h;
        return st;
    }
    *out = h;
    return CFA_OK;
}

cfa_status cfa_ilu_set_pattern(cfa_ctx* ctx, cfa_ilu* h, int n, const int* rp, const int* ci, const int* d_rp,
                               const int* d_ci) {
    CFA_ENTER(ctx);
    CFA_ARG(h && n > 0 && rp && ci && d_rp && d_ci);
    return ilu_pattern(ctx, h, n, rp, ci, d_rp, d_ci);
}

cfa_status cfa_ilu_destroy(cfa_ilu* ilu) {
    delete ilu;
    return CFA_OK;
}

cfa_status cfa_ilu_factor(cfa_ctx* ctx, cfa_ilu* h, const double* val) {
    CFA_ENTER(ctx);
    CFA_ARG(h && val);
    CFA_CUDA(cudaMemcpyAsync(h->lu.p, val, (size_t)h->nnz * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    for (int c = 1; c < h->nc; ++c) {
        const int cs = h->colour_start[c], m = h->colour_start[c + 1] - cs;
        if (m == 0) continue;
        CFA_LAUNCH(ctx, k_ilu_factor_colour, ceil_div(m, 128), 128, 0, m, (const int*)h->rows.p, h->rp,
                   (const int*)h->ep.p, (const int4*)h->elim.p, (const int2*)h->upd.p, cs, h->lu.p);
    }
    const int len = std::max(h->n, std::max(h->nl, h->nu));
    if (h->precision == CFA_MIXED)
        CFA_LAUNCH(ctx, k_ilu_gather<float>, ceil_div(len, kThreads), kThreads, 0, h->nl, h->nu, h->n, h->l_src.p,
                   h->u_src.p, h->d_src.p, h->lu.p, h->lv32.p, h->uv32.p, h->dinv32.p);
    else
        CFA_LAUNCH(ctx, k_ilu_gather<double>, ceil_div(len, kThreads), kThreads, 0, h->nl, h->nu, h->n, h->l_src.p,
                   h->u_src.p, h->d_src.p, h->lu.p, h->lv64.p, h->uv64.p, h->dinv64.p);
    CFA_CHECK_LAUNCH();
    h->transposed = false;
    return CFA_OK;
}

}  // extern "C"

namespace cfa {
// Mirror positions of the handle's pattern, computed once (synchronises the first time).
static cfa_status ensure_mirror(cfa_ctx* ctx, cfa_ilu* h) {
    if (h->mirror) return CFA_OK;
    CFA_CUDA(h->tpos.ensure(std::max(h->nnz, 1)));
    DevBuf<int> err;
    CFA_CUDA(err.ensure(1));
    CFA_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_mirror_positions, ceil_div(h->n, kThreads), kThreads, 0, h->n, h->rp, h->ci, h->tpos.p, err.p);
    int herr = 0;
    CFA_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    if (herr) return set_error(ctx, CFA_BAD_ARG, "pattern not structurally symmetric", __FILE__, __LINE__);
    h->mirror = true;
    return CFA_OK;
}
}  // namespace cfa

extern "C" {

cfa_status cfa_ilu_factor_transposed(cfa_ctx* ctx, cfa_ilu* h, const double* val) {
    CFA_ENTER(ctx);
    CFA_ARG(h && val);
    CFA_PROPAGATE(ensure_mirror(ctx, h));
    CFA_PROPAGATE(cfa_ilu_factor(ctx, h, val));
    if (h->precision == CFA_MIXED)
        CFA_LAUNCH(ctx, k_ilu_gather_transposed<float>, ceil_div(h->n, kThreads), kThreads, 0, h->n, h->rows.p,
                   h->lp.p, h->up.p, h->lc.p, h->l_src.p, h->u_src.p, h->d_src.p, h->diag.p, h->tpos.p, h->lu.p,
                   h->lv32.p, h->uv32.p, h->dinv32.p);
    else
        CFA_LAUNCH(ctx, k_ilu_gather_transposed<double>, ceil_div(h->n, kThreads), kThreads, 0, h->n, h->rows.p,
                   h->lp.p, h->up.p, h->lc.p, h->l_src.p, h->u_src.p, h->d_src.p, h->diag.p, h->tpos.p, h->lu.p,
                   h->lv64.p, h->uv64.p, h->dinv64.p);
    CFA_CHECK_LAUNCH();
    h->transposed = true;
    return CFA_OK;
}

cfa_status cfa_csr_transpose_values(cfa_ctx* ctx, cfa_ilu* h, const double* val, double* val_t) {
    CFA_ENTER(ctx);
    CFA_ARG(h && val && val_t && val != val_t);
    CFA_PROPAGATE(ensure_mirror(ctx, h));
    CFA_LAUNCH(ctx, k_transpose_values, ceil_div(h->nnz, kThreads), kThreads, 0, h->nnz, (const int*)h->tpos.p, val,
               val_t);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

cfa_status cfa_ilu_apply(cfa_ctx* ctx, const cfa_ilu* h, const double* r, double* z, int nrhs) {
    CFA_ENTER(ctx);
    CFA_ARG(h && r && z && (nrhs == 1 || nrhs == 2));
    CFA_ARG(r != z);
    return ilu_apply(ctx, h, r, z, nrhs, nullptr);
}

cfa_status cfa_ilu_apply_interleaved(cfa_ctx* ctx, const cfa_ilu* h, const double* r, double* z) {
    CFA_ENTER(ctx);
    CFA_ARG(h && r && z && r != z);
    CFA_ARG(((uintptr_t)r % 16) == 0 && ((uintptr_t)z % 16) == 0);
    return ilu_apply_pair(ctx, h, r, z, nullptr);
}

cfa_status cfa_ilu_colours(const cfa_ilu* h, int* n_colours, int* colour_start) {
    if (!h) return CFA_BAD_ARG;
    if (n_colours) *n_colours = h->nc;
    if (colour_start) std::copy(h->colour_start.begin(), h->colour_start.end(), colour_start);
    return CFA_OK;
}

cfa_status cfa_ilu_device_arrays(const cfa_ilu* h, const int** colour, const int** rows, const double** lu) {
    if (!h) return CFA_BAD_ARG;
    if (colour) *colour = h->colour.p;
    if (rows) *rows = h->rows.p;
    if (lu) *lu = h->lu.p;
    return CFA_OK;
}

}  // extern "C"
