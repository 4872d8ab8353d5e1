// Tile planning and packing for the tile-streamed CSR kernels (tiled.cuh).
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>

#include <cstdlib>
#include <cstring>

#include "tiled.cuh"

namespace cfa {

static int l2_hint_env(const char* name, int dflt) {
    const char* e = std::getenv(name);
    if (!e || !*e) return dflt;
    const int v = std::atoi(e);
    return v >= 0 && v <= 2 ? v : dflt;
}

int l2_hint_operator() { return l2_hint_env("CFA_L2_OP", 1); }
int l2_hint_vcycle() { return l2_hint_env("CFA_L2_VC", 0); }

bool tile_early_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("CFA_TILE_EARLY");
        return !(e && e[0] == '0');
    }();
    return on;
}


__global__ void k_pack_tiles(int ntiles, const long long* __restrict__ off, const int* __restrict__ row0,
                             const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v0,
                             const double* __restrict__ v1, const double* __restrict__ v2, int nvals, int vbytes,
                             unsigned char* __restrict__ data) {
    CFA_GRID_DEP();
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int r0 = row0[t], nr = row0[t + 1] - r0;
        const int e0 = rp[r0], ne = rp[r0 + nr] - e0;
        unsigned char* ch = data + off[t];
        int* rr = reinterpret_cast<int*>(ch);
        for (int r = threadIdx.x; r <= nr; r += blockDim.x) rr[r] = rp[r0 + r] - e0;
        int* cs = reinterpret_cast<int*>(ch + tile_ci_off(nr));
        for (int e = threadIdx.x; e < ne; e += blockDim.x) cs[e] = ci[e0 + e];
        const double* src[3] = {v0, v1, v2};
        for (int k = 0; k < nvals; ++k) {
            if (!src[k]) continue;   // value section left to its producer
            unsigned char* vs = ch + tile_val_off(nr, ne, vbytes, k);
            const double* sv = src[k] + e0;
            if (vbytes == 8) {
                double* d = reinterpret_cast<double*>(vs);
                for (int e = threadIdx.x; e < ne; e += blockDim.x) d[e] = sv[e];
            } else {
                float* d = reinterpret_cast<float*>(vs);
                for (int e = threadIdx.x; e < ne; e += blockDim.x) d[e] = (float)sv[e];
            }
        }
    }
}

cfa_status plan_tiled(cfa_ctx* ctx, const int* h_rp, int rows, int nvals, int vbytes, TiledCsr& T, int row_shift) {
    const double per_row = rows > 0 ? (double)h_rp[rows] / rows : 1.0;
    int tpr = 1;
    while (tpr < 32 && per_row > (double)kGatherBatch * tpr) tpr *= 2;
    int tr = kTileThreads / tpr;
    for (;;) {
        long long mx = 0;
        for (int r0 = 0; r0 < rows; r0 += tr) {
            const int r1 = std::min(rows, r0 + tr);
            mx = std::max(mx, tile_bytes(r1 - r0, h_rp[r1] - h_rp[r0], nvals, vbytes));
        }
        if (mx <= kTileBudget || tr <= 1) {
            T.max_chunk = (int)mx;
            break;
        }
        if (tpr < 32) {
            tpr *= 2;
            tr = kTileThreads / tpr;
        } else {
            tr /= 2;
        }
    }
    T.tpr = tpr;
    if (T.max_chunk > kTileBudget) return set_error(ctx, CFA_BAD_ARG, "matrix row too long for the tile budget", __FILE__, __LINE__);
    if (row_shift != 0) {
        tr = row_shift > 0 ? tr << row_shift : std::max(1, tr >> -row_shift);
        long long mx = 0;
        for (int r0 = 0; r0 < rows; r0 += tr) {
            const int r1 = std::min(rows, r0 + tr);
            mx = std::max(mx, tile_bytes(r1 - r0, h_rp[r1] - h_rp[r0], nvals, vbytes));
        }
        if (mx > kTileBudget) return CFA_BAD_ARG;   // not a usable candidate (no error recorded)
        T.max_chunk = (int)mx;
    }
    T.rows = rows;
    T.nnz = h_rp[rows];
    T.nvals = nvals;
    T.vbytes = vbytes;
    T.tile_rows = tr;
    T.ntiles = (rows + tr - 1) / tr;
    std::vector<long long> off(T.ntiles + 1, 0);
    std::vector<int> row0(T.ntiles + 1), e0(T.ntiles + 1);
    for (int t = 0; t < T.ntiles; ++t) {
        const int r0 = t * tr, r1 = std::min(rows, r0 + tr);
        row0[t] = r0;
        e0[t] = h_rp[r0];
        off[t + 1] = off[t] + tile_bytes(r1 - r0, h_rp[r1] - h_rp[r0], nvals, vbytes);
    }
    row0[T.ntiles] = rows;
    e0[T.ntiles] = h_rp[rows];
    T.bytes = off[T.ntiles];
    CFA_CUDA(T.data.ensure(T.bytes + 16));
    CFA_CUDA(T.off.ensure(T.ntiles + 1));
    CFA_CUDA(T.row0.ensure(T.ntiles + 1));
    CFA_CUDA(T.e0.ensure(T.ntiles + 1));
    CFA_CUDA(cudaMemcpyAsync(T.off.p, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(T.row0.p, row0.data(), row0.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CFA_CUDA(cudaMemcpyAsync(T.e0.p, e0.data(), e0.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CFA_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFA_OK;
}

cfa_status pack_tiled(cfa_ctx* ctx, const int* d_rp, const int* d_ci, const double* v0, const double* v1,
                      const double* v2, TiledCsr& T) {
    if (T.ntiles == 0) return CFA_OK;
    const int grid = std::min(T.ntiles, 16 * ctx->num_sms);
    CFA_LAUNCH(ctx, k_pack_tiles, grid, kTileThreads, 0, T.ntiles, (const long long*)T.off.p, (const int*)T.row0.p,
               d_rp, d_ci, v0, v1, v2, T.nvals, T.vbytes, T.data.p);
    tile_fence(ctx);
    CFA_CHECK_LAUNCH();
    return CFA_OK;
}

// ---- autotuner cache and log ----
namespace {
struct TuneState {
    std::mutex mu;
    int enabled = -1;   // -1: not set, read CFA_AUTOTUNE
    std::unordered_map<std::string, int> best;
    std::string log;
};
TuneState& tune_state() {
    static TuneState st;
    return st;
}
std::string tune_key(const char* kind, int vbytes, int nvals, int rows, long long nnz) {
    int lg = 0;
    while ((1LL << (lg + 1)) <= rows) ++lg;
    const long long q = rows > 0 ? (4 * nnz + rows / 2) / rows : 0;   // entries per row to a quarter
    return std::string(kind) + "/v" + std::to_string(vbytes) + "/n" + std::to_string(nvals) + "/r2^" +
           std::to_string(lg) + "/e" + std::to_string(q);
}
}  // namespace

bool autotune_enabled() {
    TuneState& st = tune_state();
    std::lock_guard<std::mutex> lock(st.mu);
    if (st.enabled < 0) {
        const char* e = std::getenv("CFA_AUTOTUNE");
        st.enabled = (e && e[0] == '1') ? 1 : 0;
    }
    return st.enabled == 1;
}

bool autotune_lookup(const char* kind, int vbytes, int nvals, int rows, long long nnz, int* shift) {
    TuneState& st = tune_state();
    std::lock_guard<std::mutex> lock(st.mu);
    auto it = st.best.find(tune_key(kind, vbytes, nvals, rows, nnz));
    if (it == st.best.end()) return false;
    *shift = it->second;
    return true;
}

void autotune_store(const char* kind, int vbytes, int nvals, int rows, long long nnz, int shift, const double* us,
                    const int* shifts, int ncand) {
    TuneState& st = tune_state();
    std::lock_guard<std::mutex> lock(st.mu);
    const std::string key = tune_key(kind, vbytes, nvals, rows, nnz);
    st.best[key] = shift;
    std::string line = "{\"class\": \"" + key + "\", \"rows\": " + std::to_string(rows) + ", \"nnz\": " +
                       std::to_string(nnz) + ", \"row_shift\": " + std::to_string(shift) + ", \"us\": {";
    for (int k = 0; k < ncand; ++k) {
        char buf[64];
        snprintf(buf, sizeof buf, "%s\"%d\": %.2f", k ? ", " : "", shifts[k], us[k]);
        line += buf;
    }
    st.log += line + "}}\n";
}

// Waits for the previous kernel and ends: a kernel launched after it can start (and read tiles
// before its own griddepcontrol.wait) only once every block of this one has passed its wait, so
// whatever the kernels before this one wrote is complete and visible to it.
__global__ void k_tile_fence() { CFA_GRID_DEP(); }

void tile_fence(cfa_ctx* ctx) { launch(ctx, k_tile_fence, 1, 32, 0); }

void allow_tile_kernel(const void* kernel) {
    static std::mutex mu;
    static std::unordered_map<const void*, bool> done;
    std::lock_guard<std::mutex> lock(mu);
    if (done[kernel]) return;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileStages * kTileBudget + 64);
    done[kernel] = true;
}

// Resident blocks per SM of a tile kernel with this much dynamic shared memory, as the runtime
// computes it from the kernel's registers too (cached; 0 when the query fails).
static int tile_occupancy(const void* kernel, int smem) {
    static std::mutex mu;
    static std::unordered_map<std::string, int> cache;
    char key[64];
    std::snprintf(key, sizeof(key), "%p/%d", kernel, smem);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kTileThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    cache.emplace(key, n);
    return n;
}

TileLaunch tile_launch(const cfa_ctx* ctx, const TiledCsr& T, const void* kernel) {
    TileLaunch L;
    L.smem = (int)(T.stages * align16(T.max_chunk) + 16);
    int per_sm = std::max(1, std::min(2048 / kTileThreads, (227 * 1024 - 1024) / std::max(L.smem + 64, 1)));
    // a grid beyond what is resident would leave its last blocks, each with its share of the
    // tiles, to run after the first ones finish: the kernel's registers may allow fewer blocks
    // than the shared memory does
    if (kernel) {
        const int occ = tile_occupancy(kernel, L.smem);
        if (occ > 0) per_sm = std::min(per_sm, occ);
    }
    L.grid = std::max(1, std::min(T.ntiles, per_sm * ctx->num_sms));
    L.tpr = T.tpr;
    return L;
}

}  // namespace cfa

extern "C" {

cfa_status cfa_autotune_set(int enabled) {
    cfa::TuneState& st = cfa::tune_state();
    std::lock_guard<std::mutex> lock(st.mu);
    st.enabled = enabled ? 1 : 0;
    return CFA_OK;
}

cfa_status cfa_autotune_log(char* buf, size_t cap, size_t* len) {
    cfa::TuneState& st = cfa::tune_state();
    std::lock_guard<std::mutex> lock(st.mu);
    if (len) *len = st.log.size();
    if (buf && cap) {
        const size_t k = std::min(cap - 1, st.log.size());
        memcpy(buf, st.log.data(), k);
        buf[k] = '\0';
    }
    return CFA_OK;
}

}  // extern "C"
