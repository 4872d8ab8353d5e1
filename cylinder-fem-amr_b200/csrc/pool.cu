// Block cache behind DevBuf and HostBuf.
//
// The reference sizes its workspaces with cudaMalloc/cudaFree at every resize
// (src/cfa/linalg.cuh:132-151). cudaFree waits for the whole device, so with several contexts
// solving different systems concurrently (one stream each) every resize in one of them stalls
// all the others, and each system built from scratch pays a few hundred of these calls. Here a
// block a buffer lets go returns to a free list of the stream it was allocated for and is handed
// out again, in that stream's order, to a later allocation on the same stream; no device-wide
// synchronisation happens. When a context is destroyed, its stream is synchronised and its blocks
// become idle, free for any stream of the device. cudaMalloc is paid once per block.
//
// Ownership: a block belongs to the stream of the context whose call allocated it (the scope
// opened by CFA_ENTER). A handle used from a second context must have that context ordered
// after the first (cfa_ctx_sync), the same rule as for any buffer shared between streams.
// Allocations outside a context's call (no scope) use cudaMalloc/cudaFree directly.
#include <map>
#include <mutex>
#include <unordered_map>

#include "internal.cuh"

namespace cfa {

namespace {

thread_local cudaStream_t tl_stream = nullptr;
thread_local int tl_device = -1;

constexpr size_t kRound = 512;                 // block sizes are multiples of this
constexpr size_t kSlack = 64 << 10;            // a cached block may exceed the request by 4x + this

struct Pool {
    std::mutex m;
    struct Live { int device, refs; };
    std::unordered_map<cudaStream_t, Live> live;                         // contexts' streams
    std::unordered_map<cudaStream_t, std::multimap<size_t, void*>> lists; // per live stream
    std::unordered_map<int, std::multimap<size_t, void*>> idle;           // per device
    std::multimap<size_t, void*> pinned;
    size_t cached = 0;          // device bytes held in lists and idle
    size_t cap = 0;             // at most this many (a quarter of the device's memory)
    size_t pinned_cached = 0;
};

Pool& pool() {
    static Pool* P = new Pool();   // never destroyed: buffers of static objects may outlive exit order
    return *P;
}

size_t round_up(size_t b) { return (b + kRound - 1) / kRound * kRound; }

// Best fit from `l`: the smallest block of at least `b` bytes, if it is at most 4b + kSlack.
void* take(std::multimap<size_t, void*>& l, size_t b, size_t* got) {
    auto it = l.lower_bound(b);
    if (it == l.end() || it->first > 4 * b + kSlack) return nullptr;
    void* p = it->second;
    *got = it->first;
    l.erase(it);
    return p;
}

size_t free_all(std::multimap<size_t, void*>& l) {
    size_t b = 0;
    for (auto& kv : l) {
        cudaFree(kv.second);
        b += kv.first;
    }
    l.clear();
    return b;
}

}  // namespace

StreamScope::StreamScope(cudaStream_t s, int device) : prev_stream(tl_stream), prev_device(tl_device) {
    tl_stream = s;
    tl_device = device;
}

StreamScope::~StreamScope() {
    tl_stream = prev_stream;
    tl_device = prev_device;
}

cudaStream_t scope_stream() { return tl_stream; }

void pool_stream_live(cudaStream_t s, int device) {
    Pool& P = pool();
    std::lock_guard<std::mutex> g(P.m);
    auto it = P.live.find(s);
    if (it == P.live.end()) P.live.emplace(s, Pool::Live{device, 1});
    else it->second.refs++;
    if (!P.cap) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) P.cap = tot / 4;
        if (!P.cap) P.cap = size_t(8) << 30;
    }
}

void pool_stream_retire(cudaStream_t s) {
    Pool& P = pool();
    std::lock_guard<std::mutex> g(P.m);
    auto it = P.live.find(s);
    if (it == P.live.end() || --it->second.refs > 0) return;
    auto& idle = P.idle[it->second.device];
    auto lt = P.lists.find(s);
    if (lt != P.lists.end()) {
        idle.insert(lt->second.begin(), lt->second.end());
        P.lists.erase(lt);
    }
    P.live.erase(it);
}

cudaError_t pool_alloc(void** p, size_t* bytes, cudaStream_t* owner, int* device) {
    Pool& P = pool();
    const size_t b = round_up(*bytes);
    cudaStream_t s = tl_stream;
    *owner = nullptr;
    *device = -1;
    if (s) {
        std::lock_guard<std::mutex> g(P.m);
        auto it = P.live.find(s);
        if (it != P.live.end()) {
            *owner = s;
            *device = it->second.device;
            size_t got = 0;
            void* q = take(P.lists[s], b, &got);
            if (!q) q = take(P.idle[*device], b, &got);
            if (q) {
                P.cached -= got;
                *p = q;
                *bytes = got;
                return cudaSuccess;
            }
        }
    }
    cudaError_t e = cudaMalloc(p, b);
    if (e == cudaErrorMemoryAllocation && *owner) {
        // give back what this device's idle list and this stream's list hold, then retry
        cudaGetLastError();
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        const bool sync = cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone &&
                          cudaStreamSynchronize(s) == cudaSuccess;
        std::lock_guard<std::mutex> g(P.m);
        P.cached -= free_all(P.idle[*device]);
        if (sync) P.cached -= free_all(P.lists[s]);
        e = cudaMalloc(p, b);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        *owner = nullptr;
        return e;
    }
    *bytes = b;
    return cudaSuccess;
}

void pool_release(void* p, size_t bytes, cudaStream_t owner, int device) {
    if (!p) return;
    if (!owner) {
        cudaFree(p);
        return;
    }
    Pool& P = pool();
    {
        std::lock_guard<std::mutex> g(P.m);
        if (P.cached + bytes <= P.cap) {
            auto it = P.live.find(owner);
            if (it != P.live.end() && it->second.device == device) P.lists[owner].emplace(bytes, p);
            else P.idle[device].emplace(bytes, p);   // its stream was synchronised when it retired
            P.cached += bytes;
            return;
        }
    }
    cudaFree(p);
}

cudaError_t pinned_alloc(void** p, size_t* bytes) {
    Pool& P = pool();
    const size_t b = round_up(*bytes);
    {
        std::lock_guard<std::mutex> g(P.m);
        size_t got = 0;
        void* q = take(P.pinned, b, &got);
        if (q) {
            P.pinned_cached -= got;
            *p = q;
            *bytes = got;
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMallocHost(p, b);
    if (e == cudaSuccess) *bytes = b;
    return e;
}

void pinned_release(void* p, size_t bytes, cudaStream_t owner) {
    if (!p) return;
    // the block may still be the target of a copy on its stream: wait for that stream (never for
    // one that is being captured, whose copies have not been issued), else let cudaFreeHost wait
    bool idle = false;
    if (owner) {
        Pool& P = pool();
        bool live;
        {
            std::lock_guard<std::mutex> g(P.m);
            live = P.live.count(owner) != 0;
        }
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (live && cudaStreamIsCapturing(owner, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone)
            idle = cudaStreamSynchronize(owner) == cudaSuccess;
        cudaGetLastError();
    }
    if (idle) {
        Pool& P = pool();
        std::lock_guard<std::mutex> g(P.m);
        if (P.pinned_cached + bytes <= (size_t(4) << 30)) {
            P.pinned.emplace(bytes, p);
            P.pinned_cached += bytes;
            return;
        }
    }
    cudaFreeHost(p);
}

void pool_trim(cudaStream_t s) {
    Pool& P = pool();
    std::lock_guard<std::mutex> g(P.m);
    for (auto& kv : P.idle) P.cached -= free_all(kv.second);
    if (s) {
        auto lt = P.lists.find(s);
        if (lt != P.lists.end()) P.cached -= free_all(lt->second);
    }
    for (auto& kv : P.pinned) cudaFreeHost(kv.second);
    P.pinned.clear();
    P.pinned_cached = 0;
}

void pool_stats(size_t* device_cached, size_t* pinned_cached) {
    Pool& P = pool();
    std::lock_guard<std::mutex> g(P.m);
    *device_cached = P.cached;
    *pinned_cached = P.pinned_cached;
}

}  // namespace cfa
