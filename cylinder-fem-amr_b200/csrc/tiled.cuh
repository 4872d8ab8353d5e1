// Tile-streamed CSR: the B200 data path of the bandwidth-bound row kernels.
//
// A CSR matrix (with one or more value arrays on the same pattern) is repacked into row tiles.
// Each tile is one contiguous, 16-byte aligned chunk:
//     [ row offsets relative to the tile (rows + 1 int32) | column indices (int32) |
//       value array 0 | value array 1 | ... ]                    (every section 16-byte padded)
// so a whole tile moves with ONE bulk asynchronous copy (cp.async.bulk, the TMA's 1-D mode)
// into shared memory. Persistent CTAs walk the tiles (tile = blockIdx.x + k gridDim.x) through a
// kTileStages-deep pipeline: the copies of the next kTileStages - 1 tiles are in flight while
// tile k is computed from shared memory; an mbarrier with transaction counting signals arrival.
// Every wait is bounded: on timeout the kernel records an error code, waits (bounded) for its
// other copies, and returns. Matrix bytes are read once, fully coalesced, at exactly the
// algorithmic volume (plus 16-byte padding per section); only the vector gathers x[col] go
// through L1/L2. The row kernels issue the gathers of up to kGatherBatch entries of a lane before
// they use any of them, so a row costs one L2 round trip instead of one per entry.
#pragma once

#include <cstdint>
#include <vector>

#include "internal.cuh"

namespace cfa {

constexpr int kTileThreads = 256;
constexpr int kTileStages = 3;             // tiles in flight per CTA
constexpr int kTileBudget = 36 * 1024;     // max bytes of one tile (kTileStages per CTA: two CTAs per SM at most)
constexpr int kGatherBatch = 8;            // entries per lane whose gathers are issued together
constexpr unsigned kWaitLimit = 1u << 22;  // bounded mbarrier waits (each try_wait itself blocks a while)

__host__ __device__ inline long long align16(long long b) { return (b + 15) & ~15LL; }

struct TileView {
    const unsigned char* data = nullptr;
    const long long* off = nullptr;   // [ntiles + 1] byte offset of each tile chunk
    const int* row0 = nullptr;        // [ntiles + 1] first row of each tile
    int ntiles = 0, rows = 0, nvals = 0, vbytes = 8;
    int tile_rows = 0;                // rows of every tile but the last (tile t starts at t * tile_rows)
    int max_chunk = 0;                // bytes
    int* err = nullptr;               // device error word (timeout)
    int early = 0;                    // signal dependents as soon as the first copies are issued
    int l2hint = 0;                   // L2 policy of the tile copies: 0 normal, 1 evict first, 2 evict last
    int stages = kTileStages;         // pipeline depth, 2 .. kTileStages (the matrix's own)
};

// L2 policies of the tile streams: the pressure operator's tiles (CFA_L2_OP, default 1) and the
// V-cycle's level tiles (CFA_L2_VC, default 0), each 0 (normal), 1 (evict first) or 2 (evict
// last). The operator's stream is read once per CG iteration and is larger than what the rest of
// the iteration touches; marked evict-first it no longer pushes the V-cycle's levels and the
// Krylov vectors out of L2 (402k-vertex step 13.56 -> 13.36 ms). Evict-last on the level tiles changed
// nothing measurable.
int l2_hint_operator();
int l2_hint_vcycle();

// Tile kernels signal their dependent launch (griddepcontrol.launch_dependents) right after
// issuing their first tile copies, so the next kernel's blocks are scheduled and issue their own
// first copies while this kernel runs (402k-vertex step 15.72 -> 15.11 ms); CFA_TILE_EARLY=0 turns it off.
bool tile_early_enabled();

// Host-side description + device buffers of a tiled matrix.
struct TiledCsr {
    int rows = 0, nnz = 0, ntiles = 0, nvals = 0, vbytes = 8, tile_rows = 0, max_chunk = 0;
    int tpr = 1;                      // lanes per row of the kernels (tile_rows = kTileThreads / tpr)
    int stages = kTileStages;         // pipeline depth of the kernels streaming this matrix (2 .. kTileStages)
    long long bytes = 0;
    DevBuf<unsigned char> data;
    DevBuf<long long> off;
    DevBuf<int> row0;
    DevBuf<int> e0;                   // [ntiles + 1] first CSR entry of each tile
    TileView view(int* err) const {
        TileView v;
        v.data = data.p; v.off = off.p; v.row0 = row0.p; v.ntiles = ntiles; v.rows = rows;
        v.nvals = nvals; v.vbytes = vbytes; v.max_chunk = max_chunk; v.err = err; v.tile_rows = tile_rows;
        v.early = tile_early_enabled() ? 1 : 0;
        v.stages = stages;
        return v;
    }
};

// Chunk geometry of a tile with nr rows and ne entries
__host__ __device__ inline long long tile_ci_off(int nr) { return align16(4LL * (nr + 1)); }
__host__ __device__ inline long long tile_val_off(int nr, int ne, int vbytes, int k) {
    return tile_ci_off(nr) + align16(4LL * ne) + k * align16((long long)vbytes * ne);
}
__host__ __device__ inline long long tile_bytes(int nr, int ne, int nvals, int vbytes) {
    return tile_val_off(nr, ne, vbytes, nvals);
}

// Plans the tiles from the host row pointer: tpr (lanes per row) is the smallest power of two
// with at most about kGatherBatch entries per lane on average, raised until a tile of
// kTileThreads / tpr rows fits kTileBudget (at tpr = 32 the tile rows are halved instead).
// Allocates the device buffers (the pattern and values are packed by pack_tiled).
// row_shift != 0 scales the rows of a tile by 2^row_shift (lanes per row unchanged, so every row's
// sum keeps its order); CFA_BAD_ARG when such a tile would exceed the budget.
cfa_status plan_tiled(cfa_ctx* ctx, const int* h_rp, int rows, int nvals, int vbytes, TiledCsr& T, int row_shift = 0);

// ---------------------------------------------------------------------------------------------
// Autotuner (off unless cfa_autotune_set(1) or CFA_AUTOTUNE=1). For a tiled matrix whose kernels
// carry no fused reduction, it times the tile heights 2^k * (kTileThreads / lanes per row),
// k in {-2, -1, 0, 1}, on the kernel that reads the matrix and keeps the fastest. Lanes per row
// stay those of the row-length rule, so the results do not depend on the choice. Choices are
// cached per pattern class (kind, precision, value arrays, log2 rows, entries per row to a
// quarter) for the life of the process and logged (cfa_autotune_log).
// ---------------------------------------------------------------------------------------------
bool autotune_enabled();
// The cached row shift of a pattern class, if any.
bool autotune_lookup(const char* kind, int vbytes, int nvals, int rows, long long nnz, int* shift);
void autotune_store(const char* kind, int vbytes, int nvals, int rows, long long nnz, int shift,
                    const double* us, const int* shifts, int ncand);

// Packs pattern + values (FP64 sources; converted to float when vbytes == 4) into T.
// A NULL source leaves its value section to be filled by its producer. Asynchronous; ends with
// tile_fence, so the next kernel may read the tiles before its griddepcontrol.wait.
// Kernels that write tile values themselves (a producer) must be followed by tile_fence too.
cfa_status pack_tiled(cfa_ctx* ctx, const int* d_rp, const int* d_ci, const double* v0, const double* v1,
                      const double* v2, TiledCsr& T);

// ---------------------------------------------------------------------------------------------
// device side: mbarrier + bulk copy
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// The same copy with an L2 cache policy made by createpolicy.
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, unsigned bytes, uint64_t* bar,
                                              uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ uint64_t l2_policy(int hint) {
    uint64_t p;
    if (hint == 1)
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    else
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase) {
    for (unsigned it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// Issues the copy of tile t into stage s (one thread).
__device__ __forceinline__ void tile_issue(const TileView& tv, int t, unsigned char* dst, uint64_t* bar) {
    const long long o0 = tv.off[t], o1 = tv.off[t + 1];
    const unsigned bytes = (unsigned)(o1 - o0);
    mbar_expect_tx(bar, bytes);
    if (tv.l2hint)
        bulk_g2s_hint(dst, tv.data + o0, bytes, bar, l2_policy(tv.l2hint));
    else
        bulk_g2s(dst, tv.data + o0, bytes, bar);
}

// Runs body(tile, row0, nrows, chunk) for every tile of this CTA (all threads call it; the
// body must not return early for some threads and must synchronise nothing itself).
// Dynamic shared memory: kTileStages * align16(max_chunk) bytes. Returns false on a timeout.
template <class Body>
__device__ __forceinline__ bool tile_loop(const TileView& tv, unsigned char* smem, Body&& body) {
    const int S = tv.stages;   // 2 .. kTileStages
    __shared__ uint64_t bar[kTileStages];
    __shared__ int abort_flag;
    const long long stride = align16(tv.max_chunk);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < S; ++k) mbar_init(&bar[k], 1);
        mbar_fence_init();
        abort_flag = 0;
    }
    __syncthreads();
    const int t0 = blockIdx.x;
    if (t0 >= tv.ntiles) return true;
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < S - 1; ++k) {
            const int t = t0 + k * (int)gridDim.x;
            if (t < tv.ntiles) tile_issue(tv, t, smem + k * stride, &bar[k]);
        }
    unsigned phase = 0u;   // bit k: parity of the next completion of stage k
    int s = 0;             // stage of tile t
    for (int t = t0; t < tv.ntiles; t += gridDim.x) {
        // refill the stage consumed in the previous iteration with the tile S - 1 ahead
        const int sn = s == 0 ? S - 1 : s - 1;
        const int tn = t + (S - 1) * (int)gridDim.x;
        if (threadIdx.x == 0 && tn < tv.ntiles) {
            fence_proxy_async();
            tile_issue(tv, tn, smem + sn * stride, &bar[sn]);
        }
        // every thread waits on the stage's mbarrier itself (the wait's acquire makes the copied
        // bytes visible to it); a warp computes only if all its lanes saw the tile arrive, so the
        // lane groups of the body stay whole, and the one barrier per tile (the stage's reuse)
        // also carries a timeout to the whole CTA
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar[s], (phase >> s) & 1u));
        if (!ok) {
            if ((threadIdx.x & 31) == 0) atomicExch(tv.err, (int)CFA_TIMEOUT);
            abort_flag = 1;
        } else {
            const int r0 = t * tv.tile_rows;
            body(t, r0, min(tv.tile_rows, tv.rows - r0), smem + s * stride);
        }
        __syncthreads();
        if (abort_flag) {
            // let the copies still in flight land before the CTA exits, bounded
            for (int k = 0; k < S; ++k) {
                const int sk = (s + k) % S;
                if (t + k * (int)gridDim.x < tv.ntiles) mbar_wait(&bar[sk], (phase >> sk) & 1u);
            }
            return false;
        }
        phase ^= 1u << s;
        s = s + 1 == S ? 0 : s + 1;
    }
    return true;
}

// tile_loop for a kernel launched as a programmatic dependent of the previous kernel, which
// replaces the kernel's own griddepcontrol.wait at entry. With PRE, the tiles must hold a matrix
// that no kernel still running or just finished has written (written before the previous
// kernel started: every kernel of this library waits for its predecessor before it ends), so the
// first kTileStages - 1 copies are issued BEFORE griddepcontrol.wait and their latency overlaps
// the end of the previous kernel; without PRE they are issued after it (tiles packed by the
// kernel just before). After the wait every thread evaluates gate() (it may read what earlier
// kernels wrote, e.g. a stop flag or a scalar, and must give the same answer in every thread);
// if it is false the copies already issued are waited for (bounded) and false is returned
// without running the body. The kernel must not touch memory that earlier kernels write before
// this call.
template <bool PRE = true, class Gate, class Body>
__device__ __forceinline__ bool tile_loop_dep(const TileView& tv, unsigned char* smem, Gate&& gate, Body&& body) {
    const int S = tv.stages;   // 2 .. kTileStages
    __shared__ uint64_t bar[kTileStages];
    __shared__ int abort_flag;
    const long long stride = align16(tv.max_chunk);
    const int t0 = blockIdx.x;
    auto issue_first = [&] {
#pragma unroll
        for (int k = 0; k < S - 1; ++k) {
            const int t = t0 + k * (int)gridDim.x;
            if (t < tv.ntiles) tile_issue(tv, t, smem + k * stride, &bar[k]);
        }
    };
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < S; ++k) mbar_init(&bar[k], 1);
        mbar_fence_init();
        abort_flag = 0;
        if (PRE) issue_first();
    }
    if (PRE && tv.early) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    CFA_GRID_DEP();
    __syncthreads();
    const bool go = gate();
    if (!PRE && go && threadIdx.x == 0) issue_first();
    if (!go) {
        if (threadIdx.x == 0)
            for (int k = 0; k < S - 1; ++k)
                if (t0 + k * (int)gridDim.x < tv.ntiles) mbar_wait(&bar[k], 0u);
        return false;
    }
    if (t0 >= tv.ntiles) return true;
    unsigned phase = 0u;   // bit k: parity of the next completion of stage k
    int s = 0;             // stage of tile t
    for (int t = t0; t < tv.ntiles; t += gridDim.x) {
        const int sn = s == 0 ? S - 1 : s - 1;
        const int tn = t + (S - 1) * (int)gridDim.x;
        if (threadIdx.x == 0 && tn < tv.ntiles) {
            fence_proxy_async();
            tile_issue(tv, tn, smem + sn * stride, &bar[sn]);
        }
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar[s], (phase >> s) & 1u));
        if (!ok) {
            if ((threadIdx.x & 31) == 0) atomicExch(tv.err, (int)CFA_TIMEOUT);
            abort_flag = 1;
        } else {
            const int r0 = t * tv.tile_rows;
            body(t, r0, min(tv.tile_rows, tv.rows - r0), smem + s * stride);
        }
        __syncthreads();
        if (abort_flag) {
            for (int k = 0; k < S; ++k) {
                const int sk = (s + k) % S;
                if (t + k * (int)gridDim.x < tv.ntiles) mbar_wait(&bar[sk], (phase >> sk) & 1u);
            }
            return true;
        }
        phase ^= 1u << s;
        s = s + 1 == S ? 0 : s + 1;
    }
    return true;
}

// One-block kernel that only waits for the previous kernel (see tile_loop_dep).
void tile_fence(cfa_ctx* ctx);

// Launch shape of a tile kernel: persistent grid limited by shared memory (kTileStages tiles).
struct TileLaunch {
    int grid = 1, smem = 0, tpr = 1;
};
TileLaunch tile_launch(const cfa_ctx* ctx, const TiledCsr& T, const void* kernel);
// Raises the kernel's dynamic shared memory limit to kTileStages tiles of the budget (once per kernel;
// call outside stream capture).
void allow_tile_kernel(const void* kernel);

}  // namespace cfa
