// Caching allocator for the device and pinned host memory of the solver
// objects (multigrid levels, control blocks, partial sums).
//
// cudaMalloc, cudaMallocHost and cudaFree are slow (tens of microseconds to
// milliseconds each), and cudaFree may synchronise the whole device.  A
// process that builds and drops many solvers — a serving loop meeting grid
// shapes it has not seen, a batch of hundreds of uneven grids — spends its
// time there and stalls every stream in flight.  With the pool on
// (gb_pool_set), freed blocks are kept, binned by a size class (sizes are
// rounded up to four classes per power of two, at most 25% over), and handed
// out again; only gb_pool_release, or a cache above its limit, returns
// memory to the driver.  Blocks of a class up to SMALL_MAX are carved from
// slabs of SLAB bytes (pinned host: HSMALL_MAX from HSLAB), so that a cold
// build, whose classes are not cached yet, calls the driver once per slab
// instead of once per buffer; carved blocks go back to the cache, and their
// slabs stay with the process.
//
// The contract that makes this safe: an object is freed only when no work
// that uses it is in flight (cudaFree gave that for free by synchronising).
// With the pool off (the default) every call goes straight to the driver.
#include <map>
#include <mutex>
#include <unordered_map>

#include "gb_objects.cuh"

namespace gb {
namespace {

constexpr size_t SLAB = (size_t)256 << 20, SMALL_MAX = (size_t)64 << 20;
constexpr size_t HSLAB = (size_t)1 << 20, HSMALL_MAX = (size_t)16 << 10;

struct Block {
    size_t bytes;   // class size
    int device;     // -1: pinned host
    bool carved;    // from a slab (never given back to the driver alone)
};

struct Slab {
    char* base = nullptr;
    size_t used = 0, size = 0;
};

struct Pool {
    std::mutex mu;
    bool on = false;
    size_t limit = (size_t)16 << 30;      // cached bytes kept at most
    size_t live_bytes = 0, cached_bytes = 0;
    std::unordered_map<void*, Block> live;                 // handed out
    std::multimap<std::pair<int, size_t>, std::pair<void*, bool>> cached;
    std::map<int, Slab> slab;                              // per device / host
};

Pool& pool() {
    static Pool* p = new Pool();   // never destroyed: frees may come at exit
    return *p;
}

size_t size_class(size_t bytes) {
    if (bytes <= 4096) return (bytes + 255) & ~(size_t)255;
    int k = 63 - __builtin_clzll((unsigned long long)bytes);
    const size_t step = (size_t)1 << (k - 2);
    return (bytes + step - 1) / step * step;
}

void driver_free(void* p, int device) {
    if (device < 0)
        cudaFreeHost(p);
    else
        cudaFree(p);
}

// drop cached blocks that came from the driver one by one, largest first,
// until at most `keep` cached bytes remain (or only carved ones)
void trim_locked(Pool& P, size_t keep) {
    while (P.cached_bytes > keep) {
        auto it = P.cached.end();
        for (auto j = P.cached.begin(); j != P.cached.end(); ++j)
            if (!j->second.second && (it == P.cached.end() || j->first.second > it->first.second))
                it = j;
        if (it == P.cached.end()) return;
        driver_free(it->second.first, it->first.first);
        P.cached_bytes -= it->first.second;
        P.cached.erase(it);
    }
}

cudaError_t driver_alloc(void** out, size_t bytes, bool host) {
    return host ? cudaMallocHost(out, bytes) : cudaMalloc(out, bytes);
}

// a class-`cls` block carved from the device's (or the host's) slab
cudaError_t carve(Pool& P, void** out, size_t cls, int device, bool host) {
    Slab& sl = P.slab[device];
    if (!sl.base || sl.used + cls > sl.size) {
        void* b = nullptr;
        const size_t sz = host ? HSLAB : SLAB;
        cudaError_t e = driver_alloc(&b, sz, host);
        if (e != cudaSuccess) return e;
        sl.base = (char*)b;       // the old slab's rest stays unused
        sl.used = 0;
        sl.size = sz;
    }
    *out = sl.base + sl.used;
    sl.used += cls;
    return cudaSuccess;
}

int take(void** out, size_t bytes, bool host) {
    *out = nullptr;
    if (bytes == 0) bytes = 1;
    Pool& P = pool();
    int device = -1;
    if (!host) GB_CUDA_TRY(cudaGetDevice(&device));
    std::lock_guard<std::mutex> g(P.mu);
    if (!P.on) {
        cudaError_t e = host ? cudaMallocHost(out, bytes) : cudaMalloc(out, bytes);
        if (e != cudaSuccess)
            return fail(GB_ECUDA, "allocation of %zu bytes: %s", bytes, cudaGetErrorString(e));
        return 0;
    }
    const size_t cls = size_class(bytes);
    bool carved = cls <= (host ? HSMALL_MAX : SMALL_MAX);
    auto it = P.cached.find({device, cls});
    if (it != P.cached.end()) {
        *out = it->second.first;
        carved = it->second.second;
        P.cached.erase(it);
        P.cached_bytes -= cls;
    } else {
        cudaError_t e = carved ? carve(P, out, cls, device, host) : driver_alloc(out, cls, host);
        if (e != cudaSuccess && P.cached_bytes > 0) {
            cudaGetLastError();
            trim_locked(P, 0);    // give the cache back and try once more
            e = carved ? carve(P, out, cls, device, host) : driver_alloc(out, cls, host);
        }
        if (e != cudaSuccess)
            return fail(GB_ECUDA, "allocation of %zu bytes: %s", cls, cudaGetErrorString(e));
    }
    P.live[*out] = Block{cls, device, carved};
    P.live_bytes += cls;
    return 0;
}

void give(void* p, bool host) {
    if (!p) return;
    Pool& P = pool();
    std::lock_guard<std::mutex> g(P.mu);
    auto it = P.live.find(p);
    if (it == P.live.end()) {       // allocated with the pool off
        driver_free(p, host ? -1 : 0);
        return;
    }
    const Block b = it->second;
    P.live.erase(it);
    P.live_bytes -= b.bytes;
    if (!P.on) {
        if (!b.carved) {
            driver_free(p, b.device);
            return;
        }
        // a carved block stays cached; wait as cudaFree would have, since
        // the caller made no promise about work in flight
        cudaDeviceSynchronize();
    }
    P.cached.insert({{b.device, b.bytes}, {p, b.carved}});
    P.cached_bytes += b.bytes;
    if (P.cached_bytes > P.limit) trim_locked(P, P.limit);
}

}  // namespace

int dmalloc(void** p, size_t bytes) { return take(p, bytes, false); }
void dfree(void* p) { give(p, false); }
int hmalloc(void** p, size_t bytes) { return take(p, bytes, true); }
void hfree(void* p) { give(p, true); }

}  // namespace gb

extern "C" int gb_pool_set(int on, size_t cache_limit) {
    gb::Pool& P = gb::pool();
    std::lock_guard<std::mutex> g(P.mu);
    P.on = on != 0;
    P.limit = cache_limit;
    gb::trim_locked(P, P.on ? P.limit : 0);
    return 0;
}

extern "C" int gb_pool_release(void) {
    gb::Pool& P = gb::pool();
    std::lock_guard<std::mutex> g(P.mu);
    gb::trim_locked(P, 0);
    return 0;
}

extern "C" int gb_pool_stats(size_t* live, size_t* cached) {
    gb::Pool& P = gb::pool();
    std::lock_guard<std::mutex> g(P.mu);
    if (live) *live = P.live_bytes;
    if (cached) *cached = P.cached_bytes;
    return 0;
}
