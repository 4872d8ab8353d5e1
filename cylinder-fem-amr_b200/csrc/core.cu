// Context, CSR pattern build (a1), mesh assembly plan (a2), SpMV kernels (a10, a18).
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>

#include "internal.cuh"
#include "mesh.cuh"

namespace cfa {

cfa_status set_error(cfa_ctx* ctx, cfa_status s, const char* what, const char* file, int line) {
    if (ctx) {
        char buf[512];
        snprintf(buf, sizeof(buf), "%s (%s:%d)", what, file, line);
        ctx->err = buf;
    }
    return s;
}

bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("CFA_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

long long next_uid() {
    static std::atomic<long long> uid{0};
    return ++uid;
}

cfa_status ensure_partials(cfa_ctx* ctx, size_t count) {
    if (count <= ctx->part_cap) return CFA_OK;
    if (ctx->d_part) cudaFree(ctx->d_part);
    ctx->d_part = nullptr;
    ctx->part_cap = 0;
    size_t c = std::max<size_t>(count, 64 * 1024);
    CFA_CUDA(cudaMalloc(&ctx->d_part, c * sizeof(double)));
    ctx->part_cap = c;
    return CFA_OK;
}

// ---------------------------------------------------------------------------------------------
// CSR pattern (src/cfa/mesh.cuh:198-249): node -> element incidence sorted by element (a stable
// radix sort of (node, element) pairs), then one thread per node collects, sorts and dedups
// its neighbours in registers/local memory.
// ---------------------------------------------------------------------------------------------
__global__ void k_incidence_keys(int ne, const int* __restrict__ ev, int* __restrict__ keys, int* __restrict__ vals) {
    CFA_GRID_DEP();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * ne) return;
    keys[t] = ev[t];
    vals[t] = ((t / 3) << 2) | (t % 3);   // element << 2 | local vertex
}

__global__ void k_incidence_ptr(int n, int m, const int* __restrict__ sorted_keys, int* __restrict__ ptr) {
    CFA_GRID_DEP();
    // ptr[i] = first position with key >= i (sorted keys), ptr[n] = m
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > m) return;
    int cur = t < m ? sorted_keys[t] : n;
    int prev = t > 0 ? sorted_keys[t - 1] : -1;
    for (int i = prev + 1; i <= cur && i <= n; ++i) ptr[i] = t;
}

constexpr int kMaxRowBuild = 128;

__device__ __forceinline__ int collect_row(int i, const int* __restrict__ ev, const int* __restrict__ inc_ptr,
                                           const int* __restrict__ inc, int* row, bool* overflow) {
    int m = 0;
    row[m++] = i;
    for (int s = inc_ptr[i]; s < inc_ptr[i + 1]; ++s) {
        const int e = inc[s] >> 2;
        for (int k = 0; k < 3; ++k) {
            const int v = ev[3 * e + k];
            // insertion keeping row[0, m) sorted and unique
            int q = m;
            while (q > 0 && row[q - 1] > v) --q;
            if (q > 0 && row[q - 1] == v) continue;
            if (m >= kMaxRowBuild) { *overflow = true; return m; }
            for (int r = m; r > q; --r) row[r] = row[r - 1];
            row[q] = v;
            ++m;
        }
    }
    return m;
}

__global__ void k_csr_row_len(int n, const int* __restrict__ ev, const int* __restrict__ inc_ptr,
                              const int* __restrict__ inc, int* __restrict__ len, int* __restrict__ err) {
    CFA_GRID_DEP();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int row[kMaxRowBuild];
    bool overflow = false;
    int m = collect_row(i, ev, inc_ptr, inc, row, &overflow);
    if (overflow) atomicExch(err, 1);
    len[i] = m;
}

__global__ void k_csr_row_fill(int n, const int* __restrict__ ev, const int* __restrict__ inc_ptr,
                               const int* __restrict__ inc, const int* __restrict__ rp, int* __restrict__ ci) {
    CFA_GRID_DEP();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int row[kMaxRowBuild];
    bool overflow = false;
    int m = collect_row(i, ev, inc_ptr, inc, row, &overflow);
    const int base = rp[i];
    if (overflow || m != rp[i + 1] - base) return;
    for (int q = 0; q < m; ++q) ci[base + q] = row[q];
}

__global__ void k_scatter_positions(int n, const int* __restrict__ ev, const int* __restrict__ inc_ptr,
                                    const int* __restrict__ inc, const int* __restrict__ rp,
                                    const int* __restrict__ ci, int* __restrict__ pos, int* __restrict__ err) {
    CFA_GRID_DEP();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b0 = rp[i], b1 = rp[i + 1];
    for (int s = inc_ptr[i]; s < inc_ptr[i + 1]; ++s) {
        const int e = inc[s] >> 2;
        for (int k = 0; k < 3; ++k) {
            const int col = ev[3 * e + k];
            int lo = b0, hi = b1 - 1, found = -1;
            while (lo <= hi) {
                int mid = (lo + hi) >> 1, c = ci[mid];
                if (c == col) { found = mid; break; }
                if (c < col) lo = mid + 1; else hi = mid - 1;
            }
            if (found < 0) atomicExch(err, 1);
            pos[3 * s + k] = found;
        }
    }
}

// Builds the sorted incidence (inc_ptr[n+1], inc[3 ne]) into the given buffers.
static cfa_status build_incidence(cfa_ctx* ctx, int n, int ne, const int* d_ev, DevBuf<int>& inc_ptr,
                                  DevBuf<int>& inc) {
    const int m = 3 * ne;
    DevBuf<int> keys, vals, keys_out;
    CFA_CUDA(keys.ensure(m));
    CFA_CUDA(vals.ensure(m));
    CFA_CUDA(keys_out.ensure(m));
    CFA_CUDA(inc.ensure(m));
    CFA_CUDA(inc_ptr.ensure(n + 1));
    if (m > 0) CFA_LAUNCH(ctx, k_incidence_keys, ceil_div(m, kThreads), kThreads, 0, ne, d_ev, keys.p, vals.p);
    int bits = 1;
    while ((1LL << bits) <= n) ++bits;
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.p, keys_out.p, vals.p, inc.p, m, 0, bits, ctx->stream);
    DevBuf<char> tmp;
    CFA_CUDA(tmp.ensure(tmp_bytes + 16));
    CFA_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, keys.p, keys_out.p, vals.p, inc.p, m, 0, bits,
                                             ctx->stream));
    ctx->launches += 4;
    CFA_LAUNCH(ctx, k_incidence_ptr, ceil_div(m + 1, kThreads), kThreads, 0, n, m, keys_out.p, inc_ptr.p);
    CFA_CHECK_LAUNCH();
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFA_OK;
}

}  // namespace cfa

using namespace cfa;

// =============================================================================================
// C ABI: context
// =============================================================================================
extern "C" {

cfa_status cfa_ctx_create(void* stream, cfa_ctx** out) {
    if (!out) return CFA_BAD_ARG;
    *out = nullptr;
    auto* ctx = new cfa_ctx();
    ctx->stream = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaGetDevice(&ctx->device);
    // Graphs cannot be captured on the legacy default stream: for a NULL stream the context owns
    // a blocking stream, which keeps the legacy stream's ordering with the caller's other work.
    if (e == cudaSuccess && ctx->stream == nullptr) {
        e = cudaStreamCreate(&ctx->stream);
        ctx->own_stream = e == cudaSuccess;
    }
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_counters, 64 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(ctx->d_counters, 0, 64 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_pinned, 64 * sizeof(double));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cfa_ctx_destroy(ctx);
        return CFA_CUDA_ERROR;
    }
    pool_stream_live(ctx->stream, ctx->device);
    ctx->pooled = true;
    *out = ctx;
    return CFA_OK;
}

cfa_status cfa_ctx_destroy(cfa_ctx* ctx) {
    if (!ctx) return CFA_OK;
    free_solver_work(ctx);
    if (ctx->pooled) {
        // the stream's cached blocks become idle once its work has finished
        cudaStreamSynchronize(ctx->stream);
        pool_stream_retire(ctx->stream);
    }
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->d_part) cudaFree(ctx->d_part);
    if (ctx->d_counters) cudaFree(ctx->d_counters);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return CFA_OK;
}

const char* cfa_ctx_last_error(const cfa_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

const char* cfa_status_string(cfa_status s) {
    switch (s) {
        case CFA_OK: return "ok";
        case CFA_NOT_CONVERGED: return "not converged";
        case CFA_BREAKDOWN: return "Krylov breakdown";
        case CFA_ROW_TOO_LONG: return "row longer than 32 entries";
        case CFA_COARSE_NOT_SPD: return "coarsest AMG operator not SPD";
        case CFA_CUDA_ERROR: return "CUDA error";
        case CFA_TIMEOUT: return "device wait timed out";
        case CFA_BAD_ARG: return "bad argument";
        case CFA_NO_MEMORY: return "out of memory";
    }
    return "unknown status";
}

long long cfa_ctx_kernel_launches(const cfa_ctx* ctx) { return ctx ? ctx->launches : 0; }

cfa_status cfa_mem_trim(cfa_ctx* ctx) {
    if (ctx) CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    pool_trim(ctx ? ctx->stream : nullptr);
    return CFA_OK;
}

cfa_status cfa_mem_cached(size_t* device_bytes, size_t* pinned_bytes) {
    if (!device_bytes || !pinned_bytes) return CFA_BAD_ARG;
    pool_stats(device_bytes, pinned_bytes);
    return CFA_OK;
}

cfa_status cfa_ctx_sync(cfa_ctx* ctx) {
    CFA_ENTER(ctx);
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFA_OK;
}

// =============================================================================================
// C ABI: CSR pattern
// =============================================================================================
cfa_status cfa_csr_count(cfa_ctx* ctx, int n, int ne, const int* d_ev, int* d_rp, int* nnz_out) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && ne >= 0 && d_ev && d_rp && nnz_out);
    DevBuf<int> inc_ptr, inc, len, err;
    CFA_PROPAGATE(build_incidence(ctx, n, ne, d_ev, inc_ptr, inc));
    CFA_CUDA(len.ensure(n + 1));
    CFA_CUDA(err.ensure(1));
    CFA_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
    CFA_LAUNCH(ctx, k_csr_row_len, ceil_div(n, kThreads), kThreads, 0, n, d_ev, inc_ptr.p, inc.p, len.p, err.p);
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, len.p, d_rp, n + 1, ctx->stream);
    DevBuf<char> tmp;
    CFA_CUDA(tmp.ensure(tmp_bytes + 16));
    CFA_CUDA(cudaMemsetAsync(len.p + n, 0, sizeof(int), ctx->stream));
    CFA_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, len.p, d_rp, n + 1, ctx->stream));
    ctx->launches += 2;
    int h[2];
    CFA_CUDA(cudaMemcpyAsync(&h[0], d_rp + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(&h[1], err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h[1]) return set_error(ctx, CFA_BAD_ARG, "node degree too high for the CSR build", __FILE__, __LINE__);
    *nnz_out = h[0];
    return CFA_OK;
}

cfa_status cfa_csr_fill(cfa_ctx* ctx, int n, int ne, const int* d_ev, const int* d_rp, int* d_ci) {
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && ne >= 0 && d_ev && d_rp && d_ci);
    DevBuf<int> inc_ptr, inc;
    CFA_PROPAGATE(build_incidence(ctx, n, ne, d_ev, inc_ptr, inc));
    CFA_LAUNCH(ctx, k_csr_row_fill, ceil_div(n, kThreads), kThreads, 0, n, d_ev, inc_ptr.p, inc.p, d_rp, d_ci);
    CFA_CHECK_LAUNCH();
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFA_OK;
}

// =============================================================================================
// C ABI: mesh + assembly plan
// =============================================================================================
cfa_status cfa_mesh_create(cfa_ctx* ctx, int n, int ne, const int* d_ev, const double* d_x, const double* d_y,
                           const int* d_tag, const int* d_rp, const int* d_ci, cfa_mesh** out) {
    if (!out) return CFA_BAD_ARG;
    CFA_ENTER(ctx);
    CFA_ARG(n > 0 && ne > 0 && d_ev && d_x && d_y && d_tag && d_rp && d_ci);
    auto* m = new cfa_mesh();
    m->uid = next_uid();
    m->n = n;
    m->ne = ne;
    m->ev = d_ev;
    m->x = d_x;
    m->y = d_y;
    m->tag = d_tag;
    m->rp = d_rp;
    m->ci = d_ci;
    cfa_status s = build_incidence(ctx, n, ne, d_ev, m->inc_ptr, m->inc);
    if (s != CFA_OK) { delete m; return s; }
    DevBuf<int> err;
    cudaError_t e = m->pos.ensure(9 * (size_t)ne);
    if (e == cudaSuccess) e = err.ensure(1);
    if (e == cudaSuccess) e = cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream);
    if (e != cudaSuccess) { delete m; return set_error(ctx, CFA_CUDA_ERROR, cudaGetErrorString(e), __FILE__, __LINE__); }
    ctx->launches++;
    k_scatter_positions<<<ceil_div(n, kThreads), kThreads, 0, ctx->stream>>>(n, d_ev, m->inc_ptr.p, m->inc.p, d_rp,
                                                                               d_ci, m->pos.p, err.p);
    int h_nnz = 0, h_err = 0;
    e = cudaMemcpyAsync(&h_nnz, d_rp + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { delete m; return set_error(ctx, CFA_CUDA_ERROR, cudaGetErrorString(e), __FILE__, __LINE__); }
    if (h_err) { delete m; return set_error(ctx, CFA_BAD_ARG, "element edge missing from the CSR pattern", __FILE__, __LINE__); }
    m->nnz = h_nnz;
    *out = m;
    return CFA_OK;
}

cfa_status cfa_mesh_destroy(cfa_mesh* mesh) {
    delete mesh;
    return CFA_OK;
}

cfa_status cfa_mesh_set_outlet(cfa_mesh* mesh, int outlet_dirichlet, int pin, double outlet_scale) {
    if (!mesh) return CFA_BAD_ARG;
    if (outlet_dirichlet && (pin < 0 || pin >= mesh->n)) return CFA_BAD_ARG;
    mesh->bc.outlet_dirichlet = outlet_dirichlet ? 1 : 0;
    mesh->bc.pin = pin;
    mesh->bc.outlet_scale = outlet_scale;
    return CFA_OK;
}

}  // extern "C"
