// Library-wide utilities: error string, SM count, device exclusive scan.
#include "common.cuh"

#include <algorithm>
#include <cstring>
#include <thread>
#include <atomic>
#include <chrono>
#include <map>
#include <memory>
#include <string>
#include <vector>
#include <cstdlib>
#include <mutex>

namespace mlp {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

void set_last_error(const std::string& s) { g_last_error = s; }
const char* last_error() { return g_last_error.c_str(); }

static thread_local int t_pdl_off = 0;
PdlOff::PdlOff() { t_pdl_off++; }
PdlOff::~PdlOff() { t_pdl_off--; }

bool pdl_enabled() { return t_pdl_off == 0; }

static bool trace_on() {
    static int on = -1;
    if (on < 0) {
        const char* e = getenv("MLP_TRACE");
        on = (e && e[0] == '1') ? 1 : 0;
    }
    return on == 1;
}
static thread_local std::vector<std::pair<std::string, double>> g_trace;

void trace(const char* label) {
    if (!trace_on()) return;
    double t = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
    g_trace.emplace_back(label, t);
}

void trace_flush() {
    if (!trace_on() || g_trace.empty()) return;
    double t0 = g_trace.front().second, prev = t0;
    for (auto& e : g_trace) {
        fprintf(stderr, "[mlp trace] %-28s +%8.3f ms (total %8.3f)\n", e.first.c_str(), e.second - prev, e.second - t0);
        prev = e.second;
    }
    g_trace.clear();
}

// ---- scratch arena ----------------------------------------------------------
namespace {
struct DevArena {
    std::mutex mu;
    struct Chunk { char* base; size_t cap, off; };
    std::vector<Chunk> chunks;
};
DevArena& dev_arena(int dev) {
    static std::mutex m;
    static std::map<int, std::unique_ptr<DevArena>> all;
    std::lock_guard<std::mutex> lk(m);
    auto& a = all[dev];
    if (!a) a.reset(new DevArena());
    return *a;
}
thread_local DevArena* t_arena = nullptr;
thread_local int t_arena_depth = 0;
}  // namespace

ArenaScope::ArenaScope() {
    CK(cudaGetDevice(&dev));
    if (t_arena_depth++ == 0) {
        DevArena& a = dev_arena(dev);
        a.mu.lock();
        for (auto& c : a.chunks) c.off = 0;
        t_arena = &a;
    }
}

ArenaScope::~ArenaScope() {
    if (--t_arena_depth == 0) {
        // the scope's work must be finished before the memory is reused
        cudaDeviceSynchronize();
        pool_recycle(dev);
        DevArena* a = t_arena;
        t_arena = nullptr;
        a->mu.unlock();
    }
}

void* arena_take(size_t bytes) {
    DevArena* a = t_arena;
    if (!a) return nullptr;
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto& c : a->chunks)
        if (c.off + bytes <= c.cap) {
            void* p = c.base + c.off;
            c.off += bytes;
            return p;
        }
    size_t cap = std::max<size_t>(bytes, (size_t)64 << 20);
    char* base = nullptr;
    CK(cudaMalloc(&base, cap));
    a->chunks.push_back({base, cap, bytes});
    return base;
}

// ---- device buffer pool -------------------------------------------------------
namespace {
struct Pool {
    std::mutex mu;
    struct Block { int dev; size_t bytes; bool pending; };
    std::map<void*, Block> live;                           // handed out or pending
    std::map<int, std::multimap<size_t, void*>> free_;     // per device: reusable blocks by size
    std::map<int, std::vector<void*>> pending;             // released, maybe still in use
};
Pool& pool() {
    static Pool* p = new Pool();  // never destroyed: buffers may be released during exit
    return *p;
}
// Size classes: four per octave above 4 KB (at most 25% slack).
size_t size_class(size_t b) {
    if (b <= 4096) return 4096;
    int lg = 63 - __builtin_clzll((unsigned long long)(b - 1));
    size_t step = (size_t)1 << (lg - 2);
    return (b + step - 1) & ~(step - 1);
}
}  // namespace

// ---- large host-to-device copies ----------------------------------------------
// A copy from pageable host memory is staged by the driver through its own
// pinned buffers one piece at a time. Large inputs (the matrix arrays, 93 MB
// at 60x220x85) go through two pinned staging buffers of this library
// instead: host threads copy a chunk into one buffer while the DMA engine
// moves the other, so the transfer runs near the link rate. The staging
// buffers are pinned host memory (not device memory), made once per process.
static constexpr size_t STAGE_BYTES = (size_t)16 << 20;
static std::mutex g_stage_mu;
static void* g_stage[2] = {nullptr, nullptr};
static cudaEvent_t g_stage_ev[2] = {nullptr, nullptr};

static void parallel_memcpy(void* dst, const void* src, size_t bytes) {
    unsigned T = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    if (bytes < ((size_t)1 << 20)) T = 1;
    if (T == 1) { std::memcpy(dst, src, bytes); return; }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++) {
        size_t a = bytes * t / T, b = bytes * (t + 1) / T;
        th.emplace_back([=] { std::memcpy((char*)dst + a, (const char*)src + a, b - a); });
    }
    for (auto& x : th) x.join();
}

// The staging buffers' events mark the last copy that used each buffer
// (either direction); callers hold g_stage_mu.
static void stage_init(cudaStream_t s) {
    if (g_stage[0]) return;
    for (int k = 0; k < 2; k++) {
        CK(cudaMallocHost(&g_stage[k], STAGE_BYTES));
        CK(cudaEventCreateWithFlags(&g_stage_ev[k], cudaEventDisableTiming));
        CK(cudaEventRecord(g_stage_ev[k], s));
    }
}

void h2d_large(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes < ((size_t)8 << 20)) {
        if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return;
    }
    std::lock_guard<std::mutex> lk(g_stage_mu);
    stage_init(s);
    size_t off = 0;
    for (int k = 0; off < bytes; k ^= 1) {
        size_t len = std::min(STAGE_BYTES, bytes - off);
        CK(cudaEventSynchronize(g_stage_ev[k]));  // the buffer's previous copy has left it
        parallel_memcpy(g_stage[k], (const char*)src + off, len);
        CK(cudaMemcpyAsync((char*)dst + off, g_stage[k], len, cudaMemcpyHostToDevice, s));
        CK(cudaEventRecord(g_stage_ev[k], s));
        off += len;
    }
}

void d2h_large(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes < ((size_t)8 << 20)) {
        if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return;
    }
    std::lock_guard<std::mutex> lk(g_stage_mu);
    stage_init(s);
    const size_t nch = (bytes + STAGE_BYTES - 1) / STAGE_BYTES;
    auto issue = [&](size_t c) {
        const int k = (int)(c & 1);
        const size_t off = c * STAGE_BYTES, len = std::min(STAGE_BYTES, bytes - off);
        CK(cudaEventSynchronize(g_stage_ev[k]));  // the buffer's previous copy is done
        CK(cudaMemcpyAsync(g_stage[k], (const char*)src + off, len, cudaMemcpyDeviceToHost, s));
        CK(cudaEventRecord(g_stage_ev[k], s));
    };
    issue(0);
    if (nch > 1) issue(1);
    for (size_t c = 0; c < nch; c++) {
        const int k = (int)(c & 1);
        const size_t off = c * STAGE_BYTES, len = std::min(STAGE_BYTES, bytes - off);
        CK(cudaEventSynchronize(g_stage_ev[k]));  // the chunk has arrived
        parallel_memcpy((char*)dst + off, g_stage[k], len);
        if (c + 2 < nch) issue(c + 2);
    }
}

void* pool_alloc(size_t bytes) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    size_t cls = size_class(bytes);
    Pool& P = pool();
    {
        std::lock_guard<std::mutex> lk(P.mu);
        auto& fl = P.free_[dev];
        auto it = fl.find(cls);
        if (it != fl.end()) {
            void* p = it->second;
            fl.erase(it);
            P.live[p] = {dev, cls, false};
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, cls);
    if (e != cudaSuccess) {
        // out of memory: give the cached blocks back and try once more
        cudaGetLastError();
        CK(cudaDeviceSynchronize());
        {
            std::lock_guard<std::mutex> lk(P.mu);
            for (void* q : P.pending[dev]) { P.free_[dev].emplace(P.live[q].bytes, q); P.live.erase(q); }
            P.pending[dev].clear();
            for (auto& kv : P.free_[dev]) cudaFree(kv.second);
            P.free_[dev].clear();
        }
        CK(cudaMalloc(&p, cls));
    }
    std::lock_guard<std::mutex> lk(P.mu);
    P.live[p] = {dev, cls, false};
    return p;
}

void pool_release(void* p) {
    if (!p) return;
    Pool& P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    auto it = P.live.find(p);
    if (it == P.live.end() || it->second.pending) return;
    it->second.pending = true;
    P.pending[it->second.dev].push_back(p);
}

// Cached free bytes kept per device; above this the largest cached blocks are
// given back with cudaFree (the caller has just synchronised the device).
static constexpr size_t POOL_KEEP_BYTES = (size_t)16 << 30;

void pool_recycle(int dev) {
    Pool& P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    auto& pend = P.pending[dev];
    for (void* q : pend) {
        auto it = P.live.find(q);
        if (it == P.live.end()) continue;
        P.free_[dev].emplace(it->second.bytes, q);
        P.live.erase(it);
    }
    pend.clear();
    auto& fl = P.free_[dev];
    size_t cached = 0;
    for (auto& kv : fl) cached += kv.first;
    while (cached > POOL_KEEP_BYTES && !fl.empty()) {
        auto last = std::prev(fl.end());
        cached -= last->first;
        cudaFree(last->second);
        fl.erase(last);
    }
}

void pool_sync_recycle() {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceSynchronize());
    pool_recycle(dev);
}

int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    return sms;
}

// ---- exclusive scan -------------------------------------------------------
// Three passes: per-tile sums, a single-block scan of the tile sums, then the
// per-tile scan with its offset. A tile is 1024 threads x 4 items.
static constexpr int SCAN_T = 1024;
static constexpr int SCAN_I = 4;
static constexpr int SCAN_TILE = SCAN_T * SCAN_I;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_tot[32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < (blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        warp_tot[lane] = t;  // inclusive
    }
    __syncthreads();
    uint32_t base = wid ? warp_tot[wid - 1] : 0;
    if (total) *total = warp_tot[(blockDim.x >> 5) - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void k_tile_sums(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ sums) {
    size_t base = (size_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_I;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; k++)
        if (base + k < n) s += in[base + k];
    uint32_t tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(uint32_t* sums, uint32_t nt, uint32_t* total_out) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nt; base += blockDim.x) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < nt ? sums[i] : 0;
        uint32_t tot;
        uint32_t ex = block_excl_scan(v, &tot);
        if (i < nt) sums[i] = ex + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void k_tile_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n,
                            const uint32_t* __restrict__ sums) {
    size_t base = (size_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_I;
    uint32_t v[SCAN_I];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    uint32_t ex = block_excl_scan(s, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_I; k++) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
}

void exclusive_scan_u32_async(const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t s) {
    uint32_t nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nt == 0) nt = 1;
    Tmp<uint32_t> sums(nt);
    k_tile_sums<<<nt, SCAN_T, 0, s>>>(in, n, sums.p);
    CK_LAUNCH();
    k_scan_sums<<<1, SCAN_T, 0, s>>>(sums.p, nt, out + n);
    CK_LAUNCH();
    k_tile_scan<<<nt, SCAN_T, 0, s>>>(in, out, n, sums.p);
    CK_LAUNCH();
    // no synchronisation for `sums`: scratch released here is reused only
    // after the device has been synchronised (arena scopes end with a device
    // synchronisation; released pool blocks wait in a pending list until one)
}

std::vector<uint32_t> read_words(const std::vector<const uint32_t*>& words, cudaStream_t s) {
    std::vector<uint32_t> h(words.size(), 0);
    if (words.empty()) return h;
    Tmp<uint32_t> d(words.size());
    for (size_t i = 0; i < words.size(); i++)
        CK(cudaMemcpyAsync(d.p + i, words[i], 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(h.data(), d.p, 4 * words.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return h;
}

std::vector<uint32_t> exclusive_scans_u32(const std::vector<ScanJob>& jobs, cudaStream_t s) {
    std::vector<const uint32_t*> ends;
    for (const ScanJob& j : jobs) {
        exclusive_scan_u32_async(j.in, j.out, j.n, s);
        ends.push_back(j.out + j.n);
    }
    return read_words(ends, s);
}

uint32_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t s) {
    exclusive_scan_u32_async(in, out, n, s);
    uint32_t tot = 0;
    CK(cudaMemcpyAsync(&tot, out + n, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return tot;
}

}  // namespace mlp
