// Internal definitions shared by the cfa_b200 translation units: the context, device buffers,
// launch accounting, and warp/block reductions whose summation order is fixed (results do not
// depend on scheduling: every reduction is a fixed tree over a fixed partition).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "cfa_b200.h"

namespace cfa {

constexpr int kThreads = 256;          // block size of the row kernels
constexpr int kWarps = kThreads / 32;

// BoundaryTag (src/cfa/common.cuh:68-74)
enum BoundaryTag : int { BC_INTERIOR = 0, BC_INLET = 1, BC_OUTLET = 2, BC_WALL = 3, BC_CYLINDER = 4 };

struct SolverWork;

}  // namespace cfa

struct cfa_ctx {
    cudaStream_t stream = nullptr;
    bool own_stream = false;              // created here when the caller passed the legacy stream
    bool pooled = false;                  // its stream is registered with the block cache
    int device = 0;
    int num_sms = 148;
    std::string err;
    long long launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // small device scratch: reduction partials and counters shared by the context's calls
    double* d_part = nullptr;
    size_t part_cap = 0;
    unsigned int* d_counters = nullptr;   // zero between kernels (each last block resets its own)
    double* h_pinned = nullptr;           // pinned staging for small reports
    cfa::SolverWork* work = nullptr;      // Krylov workspaces and cached solve graphs
};

namespace cfa {

cfa_status set_error(cfa_ctx* ctx, cfa_status s, const char* what, const char* file, int line);

#define CFA_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return ::cfa::set_error(ctx, CFA_CUDA_ERROR, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define CFA_CHECK_LAUNCH() CFA_CUDA(cudaGetLastError())

#define CFA_ARG(cond)                                                                         \
    do {                                                                                      \
        if (!(cond)) return ::cfa::set_error(ctx, CFA_BAD_ARG, "bad argument: " #cond, __FILE__, __LINE__); \
    } while (0)

#define CFA_PROPAGATE(expr)                                                                   \
    do {                                                                                      \
        cfa_status s_ = (expr);                                                               \
        if (s_ != CFA_OK) return s_;                                                          \
    } while (0)

// Launch on the context's stream and count it (kernel: a __global__ function, parenthesised
// when it is a template-id with commas).
#define CFA_LAUNCH(ctx, kernel, grid, block, smem, ...) ::cfa::launch((ctx), kernel, (grid), (block), (smem), __VA_ARGS__)

// Block cache behind the buffers (pool.cu). A scope names the stream (a context's) that the
// allocations of the current thread are ordered on; CFA_ENTER opens one at every C ABI entry.
struct StreamScope {
    cudaStream_t prev_stream;
    int prev_device;
    StreamScope(cudaStream_t s, int device);
    ~StreamScope();
    StreamScope(const StreamScope&) = delete;
    StreamScope& operator=(const StreamScope&) = delete;
};
cudaStream_t scope_stream();
void pool_stream_live(cudaStream_t s, int device);
void pool_stream_retire(cudaStream_t s);    // after the stream has been synchronised
cudaError_t pool_alloc(void** p, size_t* bytes, cudaStream_t* owner, int* device);
void pool_release(void* p, size_t bytes, cudaStream_t owner, int device);
cudaError_t pinned_alloc(void** p, size_t* bytes);
void pinned_release(void* p, size_t bytes, cudaStream_t owner);
void pool_trim(cudaStream_t s);
void pool_stats(size_t* device_cached, size_t* pinned_cached);

#define CFA_ENTER(ctx_)                  \
    if (!(ctx_)) return CFA_BAD_ARG;     \
    ::cfa::StreamScope cfa_scope_((ctx_)->stream, (ctx_)->device)

// Growable device buffer (geometric growth, as the reference's workspaces, linalg.cuh:132-151);
// its blocks come from the cache, ordered on the stream of the scope that allocated them.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    size_t bytes = 0;
    cudaStream_t owner = nullptr;
    int dev = -1;
    cudaError_t ensure(size_t count) {
        if (count <= cap && p) return cudaSuccess;
        release();
        size_t b = (count + count / 2 + 64) * sizeof(T);
        void* q = nullptr;
        cudaError_t e = pool_alloc(&q, &b, &owner, &dev);
        if (e != cudaSuccess) return e;
        p = static_cast<T*>(q);
        bytes = b;
        cap = b / sizeof(T);
        return cudaSuccess;
    }
    void release() {
        if (p) pool_release(p, bytes, owner, dev);
        p = nullptr;
        cap = bytes = 0;
        owner = nullptr;
        dev = -1;
    }
    ~DevBuf() { release(); }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), cap(o.cap), bytes(o.bytes), owner(o.owner), dev(o.dev) { o.forget(); }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p; cap = o.cap; bytes = o.bytes; owner = o.owner; dev = o.dev;
            o.forget();
        }
        return *this;
    }

  private:
    void forget() { p = nullptr; cap = bytes = 0; owner = nullptr; dev = -1; }
};

// Programmatic dependent launch. Kernels go out with cudaLaunchAttributeProgrammaticStreamSerialization,
// so a kernel's blocks may be scheduled as the previous kernel's blocks exit (in a captured graph
// the edge becomes a programmatic one). Every kernel of this library starts with CFA_GRID_DEP():
// griddepcontrol.wait returns once the preceding grid has completed and its writes are visible,
// before this kernel reads or writes anything. For a kernel launched without the attribute it is
// a no-op. It removes part of the launch gap between the short dependent kernels of a V-cycle
// (402k-vertex step 17.4 -> 16.8 ms). For kernels that wait at entry an explicit early launch_dependents
// was slower (17.7 ms): blocks of the next kernel parked on the SMs while the current one still
// ran. The tile kernels (tiled.cuh: tile_loop_dep) and the ILU sweeps (ilu.cu) load constant data
// (their first tiles, the factors) before they wait, so there the early signal pays.
#define CFA_GRID_DEP() asm volatile("griddepcontrol.wait;" ::: "memory")

bool pdl_enabled();   // CFA_PDL=0 in the environment turns the attribute off

template <class... P, class... A>
inline void launch(cfa_ctx* ctx, void (*kernel)(P...), int grid, int block, size_t smem, A&&... args) {
    ctx->launches++;
    if (!pdl_enabled()) {
        kernel<<<grid, block, smem, ctx->stream>>>(static_cast<P>(args)...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...);
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Grid for a grid-stride row kernel: enough blocks to cover the rows, at most 8 per SM.
inline int row_grid(const cfa_ctx* ctx, long long rows, int tpr) {
    long long need = (rows * tpr + kThreads - 1) / kThreads;
    long long cap = 8LL * ctx->num_sms;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

// Threads per row from the mean row length, the reference's rule (csr_threads_per_row,
// src/cfa/linalg.cuh:918-926).
inline int threads_per_row(int rows, long long nnz) {
    double per_row = rows > 0 ? (double)nnz / rows : 1.0;
    double target = per_row / (rows < 20000 ? 2.0 : 4.0);
    int tpr = 1;
    while (tpr < 32 && 2 * tpr <= target) tpr *= 2;
    return tpr;
}

cfa_status ensure_partials(cfa_ctx* ctx, size_t count);
void free_solver_work(cfa_ctx* ctx);
// Process-unique id for handles and hierarchy versions: cached solve graphs key on it, because a
// new handle can be allocated at the address of a freed one.
long long next_uid();

// ---------------------------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum over a block of kThreads threads in a fixed tree; the result is valid in thread 0.
// `sh` holds kWarps doubles per value.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = warp_sum(v[k]);
        if (lane == 0) sh[k * kWarps + warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < kWarps ? sh[k * kWarps + lane] : 0.0;
            s = warp_sum(s);
            v[k] = s;
        }
    }
    __syncthreads();
}

// Writes this block's NV partials to part[k * gridDim.x + blockIdx.x], then returns true in
// exactly one block, the last to finish, after which every partial is visible to it. The
// counter is reset by the caller's last block (reset_counter).
template <int NV>
__device__ __forceinline__ bool publish_partials(const double (&v)[NV], double* part, unsigned int* counter) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) part[k * gridDim.x + blockIdx.x] = v[k];
        __threadfence();
        unsigned int prev = atomicAdd(counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// In the last block: sums the partials of every block in a fixed order (thread t takes blocks
// t, t + kThreads, ..., then the block tree); result valid in thread 0. Resets the counter.
template <int NV>
__device__ __forceinline__ void reduce_partials(double (&v)[NV], const double* part, unsigned int* counter,
                                                double* sh) {
    const int G = gridDim.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = 0.0;
        for (int b = threadIdx.x; b < G; b += kThreads) s += __ldcg(part + k * G + b);
        v[k] = s;
    }
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) *counter = 0u;
}

}  // namespace cfa
