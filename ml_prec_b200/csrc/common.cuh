// Shared infrastructure of the ml_prec_b200 CUDA library: error state, device
// buffers, CSR containers and small launch helpers. Every entry point of the
// C ABI returns an int status and records a message retrievable through
// mlp_last_error() (include/mlp_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <utility>
#include <stdexcept>
#include <string>
#include <vector>

namespace mlp {

// Status codes of the C ABI (mirrored in include/mlp_b200.h).
enum Status : int {
    OK = 0,
    ERR_ARG = 1,          // invalid argument / size
    ERR_CONFIG = 2,       // bad preconditioner configuration
    ERR_LEVELS = 3,       // "Too many levels"
    ERR_CURVATURE = 4,    // <Ap, p> <= 0 in PCG
    ERR_NOT_FINITE = 5,   // NaN / Inf in a scalar
    ERR_MAXIT = 6,        // iteration cap reached
    ERR_CUDA = 7,         // CUDA runtime error
    ERR_NO_ITER = 8,      // "No need to iterate"
    ERR_LIMIT = 9,        // a documented size limit was exceeded
    ERR_INTERNAL = 10,    // a device-side consistency check failed
};

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define MLP_THROW(code, msg)                                                     \
    do {                                                                         \
        throw ::mlp::Error((code), std::string(msg) + " (" + __FILE__ + ":" +    \
                                       std::to_string(__LINE__) + ")");          \
    } while (0)

#define CK(call)                                                                 \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess)                                                   \
            MLP_THROW(::mlp::ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void count_launches(uint64_t n);
uint64_t launch_count();
#define CK_LAUNCH()                 \
    do {                            \
        ::mlp::count_launches(1);   \
        CK(cudaGetLastError());     \
    } while (0)

void set_last_error(const std::string& s);
const char* last_error();

// Device buffer pool. Released buffers are kept for reuse instead of being
// given back with cudaFree (which synchronises the device and, with cudaMalloc,
// dominated repeated setups). A released buffer may still be in use by queued
// work, so it becomes reusable only at pool_recycle(dev), which callers invoke
// right after a cudaDeviceSynchronize (the end of a build scope, the destroy
// entry points); pool_sync_recycle() does both.
// Host-to-device copy of a large pageable array through pinned staging buffers
// (parallel host copies overlapped with the DMA); small copies go directly.
void h2d_large(void* dst, const void* src, size_t bytes, cudaStream_t s);
// The reverse: device to pageable host memory through the same staging
// buffers (the DMA fills one while host threads drain the other); returns
// when the data are in dst.
void d2h_large(void* dst, const void* src, size_t bytes, cudaStream_t s);

void* pool_alloc(size_t bytes);
void pool_release(void* p);
void pool_recycle(int dev);
void pool_sync_recycle();

// Device buffer (RAII) on the pool.
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    explicit DBuf(size_t count) { alloc(count); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DBuf() { release(); }
    // 16 bytes of slack past the end: kernels that stage a row range with
    // 16-byte vector loads may read (never use) up to 15 bytes beyond it.
    void alloc(size_t count) {
        release();
        n = count;
        if (count) p = static_cast<T*>(pool_alloc(count * sizeof(T) + 16));
    }
    void release() {
        if (p) pool_release(p);
        p = nullptr;
        n = 0;
    }
    void zero(cudaStream_t s) { if (n) CK(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void upload(const T* h, size_t count, cudaStream_t s) {
        if (count > n) alloc(count);
        if (count) CK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    std::vector<T> download(cudaStream_t s, size_t count = (size_t)-1) const {
        if (count == (size_t)-1) count = n;
        std::vector<T> h(count);
        if (count) CK(cudaMemcpyAsync(h.data(), p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return h;
    }
};

// Scratch arena for the temporaries of a hierarchy build or an assembly. Each
// device keeps a list of chunks that are reused from one build to the next
// (temporaries then cost neither cudaMalloc nor cudaFree, whose implicit
// synchronisation and page mapping dominated short setups). An ArenaScope
// takes the device's lock for its lifetime, so builds in one process are
// serialised; Tmp<T> buffers created inside a scope come from the arena, outside
// one they fall back to the buffer pool.
void* arena_take(size_t bytes);  // null when no scope is active
struct ArenaScope {
    ArenaScope();
    ~ArenaScope();
    ArenaScope(const ArenaScope&) = delete;
    ArenaScope& operator=(const ArenaScope&) = delete;
    int dev;
};

template <class T>
struct Tmp {
    T* p = nullptr;
    size_t n = 0;
    bool owned = false;
    Tmp() = default;
    explicit Tmp(size_t count) { alloc(count); }
    Tmp(const Tmp&) = delete;
    Tmp& operator=(const Tmp&) = delete;
    ~Tmp() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        if (!count) return;
        size_t bytes = count * sizeof(T) + 16;
        p = static_cast<T*>(arena_take(bytes));
        if (!p) {
            p = static_cast<T*>(pool_alloc(bytes));
            owned = true;
        }
    }
    void release() {
        if (p && owned) pool_release(p);
        p = nullptr;
        n = 0;
        owned = false;
    }
    void zero(cudaStream_t s) { if (n) CK(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void upload(const T* h, size_t count, cudaStream_t s) {
        if (count > n) alloc(count);
        if (count) CK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    std::vector<T> download(cudaStream_t s, size_t count = (size_t)-1) const {
        if (count == (size_t)-1) count = n;
        std::vector<T> h(count);
        if (count) CK(cudaMemcpyAsync(h.data(), p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return h;
    }
};

// CSR matrix on the device: 32-bit indices, FP64 values (plus an optional FP32
// copy of the values for the reduced-precision preconditioner).
struct DCSR {
    uint32_t nrow = 0, ncol = 0, nnz = 0;
    uint32_t tile_max = 0;  // largest nnz of a 256-row tile (0 = not computed)
    DBuf<uint32_t> ia, ja;
    DBuf<double> a;
    DBuf<float> a32;
    void alloc(uint32_t r, uint32_t c, uint32_t z) {
        nrow = r; ncol = c; nnz = z;
        ia.alloc((size_t)r + 1);
        ja.alloc(z ? z : 1);
        a.alloc(z ? z : 1);
    }
};

// Programmatic dependent launch. Kernels of the apply plan start with
// pdl_wait() (returns once the preceding kernel in the stream has finished and
// its writes are visible; a no-op when launched without the attribute) and
// then pdl_trigger() (lets the next kernel be scheduled while this one runs),
// so the launch latency of each kernel overlaps its predecessor.
// MLP_TIMELINE_HOOK: the in-graph timeline of the apply (mlp_prec_timeline)
// stamps the time each kernel of solve.cu passes this wait; elsewhere empty.
#ifndef MLP_TIMELINE_HOOK
#define MLP_TIMELINE_HOOK()
#endif
__device__ __forceinline__ void pdl_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    MLP_TIMELINE_HOOK();
}
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

bool pdl_enabled();
// While one is alive on a thread, launches recorded there carry no
// programmatic dependent launch: in a graph of many concurrent branches (the
// ensemble) an early-scheduled dependent CTA holds an SM slot that another
// branch's kernel could use (one launch of 64 members: 75 ms without against
// 88 ms with).
struct PdlOff {
    PdlOff();
    ~PdlOff();
};

// Host-side phase timer of the setup, printed to stderr when MLP_TRACE=1.
void trace(const char* label);
void trace_flush();

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                     Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

inline unsigned grid_for(size_t n, unsigned block) {
    size_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 0x7fffffff) g = 0x7fffffff;
    return (unsigned)g;
}

int num_sms();

// Exclusive scan of 32-bit counts on the device; returns the total (synchronises).
uint32_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t s);
// Same, total left on the device at out[n] (no host synchronisation).
void exclusive_scan_u32_async(const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t s);
// Several scans with one host synchronisation; returns their totals.
struct ScanJob {
    const uint32_t* in;
    uint32_t* out;
    uint32_t n;
};
std::vector<uint32_t> exclusive_scans_u32(const std::vector<ScanJob>& jobs, cudaStream_t s);
// Copies `words` 32-bit device words (any addresses) to the host with one
// synchronisation.
std::vector<uint32_t> read_words(const std::vector<const uint32_t*>& words, cudaStream_t s);

}  // namespace mlp
