// k_persist: runs a recorded chain of preconditioner steps in one cooperative
// launch, with a grid-wide barrier between consecutive steps (persist.cuh).
//
// Work of a step is spread over every warp of the grid the way the separate
// kernel spreads it over its threads: a row kernel with LPR lanes per row
// gives each warp 32 / LPR consecutive rows, lane l of a row adds the row's
// entries l, l + LPR, ... in order with a fused multiply-add and the lanes
// combine with the xor butterfly, exactly as k_phase1 / k_phase2 / k_update /
// k_spmv do; the dense product takes a warp per row as k_dense_gemv does.
// Only the assignment of rows to warps differs, which does not change any
// row's arithmetic, so results are bit-identical to the separate launches.
//
// Memory ordering: vectors written in one step are read by other CTAs in the
// next, so they are read with plain loads (never the read-only path) after a
// barrier whose arrival is a release and whose wait is an acquire at GPU
// scope; the matrices are constant for the whole launch and go through the
// read-only path.
#include <algorithm>
#include <cstdlib>

#include "persist.cuh"

namespace mlp {

namespace {

__device__ __forceinline__ double fmadd_p(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmadd_p(float a, float b, float c) { return __fmaf_rn(a, b, c); }

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Polls of one barrier wait before it gives up (about a second: each poll is
// an L2 round trip, every 64th adds a short sleep).
constexpr uint32_t PK_SPIN_LIMIT = 1u << 22;

// Grid barrier. Thread 0 of each CTA publishes the CTA's writes (a release
// add, ordered after the other threads' writes by the CTA barrier before it),
// then waits with acquire loads until all CTAs of this barrier have arrived;
// the CTA barrier after it orders the other threads' next loads after that
// acquire. No separate fences: on B200 they made each barrier 0.5 us slower
// (1.9 against 1.4 us at 148 CTAs).
// Returns false when a wait ran out of its limit here or in another CTA; the
// caller then stops running steps.
__device__ __forceinline__ bool pk_barrier(PBar* bar, unsigned& target) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        target += gridDim.x;
        red_release_add_u32(&bar->count, 1u);
        int ok = 1;
        for (uint32_t it = 0;; it++) {
            unsigned v = ld_acquire_u32(&bar->count);
            if ((int)(v - target) >= 0) break;
            if ((it & 63u) == 63u) {
                if (*(volatile int*)&bar->err) { ok = 0; break; }
                if (it >= PK_SPIN_LIMIT) { atomicExch(&bar->err, 1); ok = 0; break; }
                __nanosleep(64);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct WarpIdx {
    uint32_t lane, g, W;  // lane, global warp index, warps in the grid
    __device__ __forceinline__ WarpIdx()
        : lane(threadIdx.x & 31u),
          g(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)),
          W(gridDim.x * (blockDim.x >> 5)) {}
};

// Rows [0, rows) in groups of 32 / LPR per warp; body(row, active, sub) runs
// for every lane (inactive lanes take part in the shuffles with zeros).
template <int LPR, class Body>
__device__ __forceinline__ void for_rows(uint32_t rows, Body body) {
    constexpr uint32_t RPW = 32 / LPR;
    WarpIdx w;
    for (uint32_t base = w.g * RPW; base < rows; base += w.W * RPW) {
        uint32_t row = base + w.lane / LPR;
        body(row, row < rows, (int)(w.lane % LPR));
    }
}

// Lane-split row sum of k_phase1 / k_phase2 / k_update / k_spmv (RowPre::sum
// followed by the butterfly).
template <class T, int LPR, class V>
__device__ __forceinline__ T row_sum(uint32_t row, bool active, int sub, const uint32_t* __restrict__ ia,
                                     const uint32_t* __restrict__ ja, const T* __restrict__ a, V val) {
    T s = 0;
    if (active) {
        uint32_t e = __ldg(ia + row + 1);
        for (uint32_t j = __ldg(ia + row) + sub; j < e; j += LPR) s = fmadd_p(__ldg(a + j), val(__ldg(ja + j)), s);
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

template <class Body>
__device__ __forceinline__ void for_each(uint32_t lo, uint32_t hi, Body body) {
    uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += stride) body(i);
}

template <class T, int LPR>
__device__ __forceinline__ void step_rows(const PStep<T>& st) {
    const uint32_t* ia = st.ia;
    const uint32_t* ja = st.ja;
    const T* a = st.a;
    switch (st.op) {
        case PS_PHASE1: {
            const uint32_t R = st.n0;
            const T* src = static_cast<const T*>(st.v[0]);
            T* w = static_cast<T*>(st.v[1]);
            for_rows<LPR>(R, [&](uint32_t row, bool act, int sub) {
                T s = row_sum<T, LPR>(row, act, sub, ia, ja, a, [&](uint32_t c) { return src[c]; });
                if (act && sub == 0) w[row] = s;
            });
            break;
        }
        case PS_PHASE2: {
            const uint32_t M = st.n0;
            const T* w = static_cast<const T*>(st.v[0]);
            T* out = static_cast<T*>(st.v[1]);
            for_rows<LPR>(M, [&](uint32_t row, bool act, int sub) {
                T s = row_sum<T, LPR>(row, act, sub, ia, ja, a, [&](uint32_t c) { return c < M ? w[c] : out[c]; });
                if (act && sub == 0) out[row] = s;
            });
            break;
        }
        case PS_UPDATE: {
            const uint32_t N = st.n0;
            const T* u0 = static_cast<const T*>(st.v[0]);
            T* x = static_cast<T*>(st.v[1]);
            T* r = static_cast<T*>(st.v[2]);
            for_rows<LPR>(N, [&](uint32_t row, bool act, int sub) {
                T s = row_sum<T, LPR>(row, act, sub, ia, ja, a, [&](uint32_t c) { return u0[c]; });
                if (act && sub == 0) {
                    x[row] += u0[row];
                    r[row] -= s;
                }
            });
            break;
        }
        case PS_RESID: {
            const uint32_t N = st.n0;
            const T* x = static_cast<const T*>(st.v[0]);
            T* y = static_cast<T*>(st.v[1]);
            const T* f = static_cast<const T*>(st.v[2]);
            for_rows<LPR>(N, [&](uint32_t row, bool act, int sub) {
                T s = row_sum<T, LPR>(row, act, sub, ia, ja, a, [&](uint32_t c) { return x[c]; });
                if (act && sub == 0) y[row] = f[row] - s;
            });
            break;
        }
        default:
            break;
    }
}

// k_dense_gemv: a warp per row, lane l adds columns l, l + 32, ... in order
// (in the operator's type CT), then the butterfly.
template <class T, class CT>
__device__ __forceinline__ void dense_rows(uint32_t n, const CT* __restrict__ C, const T* f, T* x) {
    WarpIdx w;
    for (uint32_t row = w.g; row < n; row += w.W) {
        const CT* c = C + (size_t)row * n;
        CT s = 0;
        for (uint32_t j = w.lane; j < n; j += 32) s = fmadd_p(__ldg(c + j), (CT)f[j], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (w.lane == 0) x[row] = (T)s;
    }
}

template <class T>
__device__ void run_step(const PStep<T>& st) {
    switch (st.op) {
        case PS_PHASE1:
        case PS_PHASE2:
        case PS_UPDATE:
        case PS_RESID:
            if (st.op == PS_UPDATE && st.mode == 0) {
                // the last correction of a level call: x += u0
                const T* u0 = static_cast<const T*>(st.v[0]);
                T* x = static_cast<T*>(st.v[1]);
                for_each(0, st.n0, [&](uint32_t i) { x[i] += u0[i]; });
                break;
            }
            switch (st.lpr) {
                case 1: step_rows<T, 1>(st); break;
                case 2: step_rows<T, 2>(st); break;
                case 4: step_rows<T, 4>(st); break;
                case 8: step_rows<T, 8>(st); break;
                case 16: step_rows<T, 16>(st); break;
                default: step_rows<T, 32>(st); break;
            }
            if (st.op == PS_PHASE1 && st.n1 > st.n0) {
                // diagonal rows [R, N): out = dval * src
                const uint32_t R = st.n0;
                const T* src = static_cast<const T*>(st.v[0]);
                T* out = static_cast<T*>(st.v[2]);
                const T* dv = st.dval;
                for_each(R, st.n1, [&](uint32_t q) { out[q] = __ldg(dv + (q - R)) * src[q]; });
            }
            break;
        case PS_DENSE: {
            const uint32_t n = st.n0;
            const T* f = static_cast<const T*>(st.v[0]);
            T* x = static_cast<T*>(st.v[1]);
            if (st.mode == 1) dense_rows<T, double>(n, static_cast<const double*>(st.v[2]), f, x);
            else dense_rows<T, T>(n, st.a, f, x);
            break;
        }
        case PS_SCALE: {
            T* v = static_cast<T*>(st.v[0]);
            const T al = (T)st.s0;
            for_each(0, st.n0, [&](uint32_t i) { v[i] *= al; });
            break;
        }
        case PS_CHEB2: {
            T* x2 = static_cast<T*>(st.v[0]);
            const T* u1 = static_cast<const T*>(st.v[1]);
            const T ma = (T)st.s0, c = (T)st.s1;
            for_each(0, st.n0, [&](uint32_t i) { x2[i] = fmadd_p(x2[i], ma, c * u1[i]); });
            break;
        }
        case PS_CHEBK: {
            T* x2 = static_cast<T*>(st.v[0]);
            const T* u1 = static_cast<const T*>(st.v[1]);
            const T* u0 = static_cast<const T*>(st.v[2]);
            const T al = (T)st.s0, be = (T)st.s1;
            for_each(0, st.n0, [&](uint32_t i) {
                T a1 = u1[i];
                x2[i] = fmadd_p(be, a1 - u0[i], fmadd_p(-al, x2[i], a1));
            });
            break;
        }
        case PS_COPY: {
            const T* src = static_cast<const T*>(st.v[0]);
            T* dst = static_cast<T*>(st.v[1]);
            for_each(0, st.n0, [&](uint32_t i) { dst[i] = src[i]; });
            break;
        }
        case PS_TOF32: {
            const double* src = static_cast<const double*>(st.v[0]);
            float* dst = static_cast<float*>(st.v[1]);
            for_each(0, st.n0, [&](uint32_t i) { dst[i] = (float)src[i]; });
            break;
        }
        case PS_TOF64: {
            const float* src = static_cast<const float*>(st.v[0]);
            double* dst = static_cast<double*>(st.v[1]);
            for_each(0, st.n0, [&](uint32_t i) { dst[i] = (double)src[i]; });
            break;
        }
        default:
            break;
    }
}

// Sum of v over the CTA (valid in thread 0), fixed order: warp butterflies,
// then warp 0 adds the warp sums.
template <int NT>
__device__ __forceinline__ double cta_sum(double v) {
    __shared__ double sh[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < (NT / 32) ? sh[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;
}

template <class T, int NT>
__global__ void __launch_bounds__(NT, 2) k_persist(const PStep<T>* __restrict__ steps, uint32_t nsteps,
                                                            PBar* bar) {
    constexpr uint32_t NW = sizeof(PStep<T>) / 4;
    __shared__ __align__(16) uint32_t sbuf[2][NW];
    __shared__ uint32_t spc[2];
    __shared__ double s_init[PK_MAXLOOP];
    __shared__ uint32_t s_cnt[PK_MAXLOOP];
    __shared__ uint32_t s_next, s_total;
    const uint32_t* gsrc = reinterpret_cast<const uint32_t*>(steps);
    auto fetch = [&](uint32_t pc, int b) {
        if (threadIdx.x < NW) sbuf[b][threadIdx.x] = __ldg(gsrc + (size_t)pc * NW + threadIdx.x);
        if (threadIdx.x == 0) spc[b] = pc;
    };
    fetch(0, 0);
    if (threadIdx.x == 0) {
        spc[1] = 0xffffffffu;
        s_total = 0;
    }
    __syncthreads();
    unsigned target = 0;
    uint32_t pc = 0;
    int cur = 0;
    bool ok = true;
    while (pc < nsteps) {
        if (spc[cur] != pc) {  // after a jump: the step was not prefetched
            __syncthreads();
            fetch(pc, cur);
            __syncthreads();
        }
        const PStep<T>& st = *reinterpret_cast<const PStep<T>*>(sbuf[cur]);
        // the next descriptor in program order is fetched while this step runs
        if (pc + 1 < nsteps) fetch(pc + 1, cur ^ 1);
        uint32_t next = pc + 1;
        bool sync_grid = true;
        if (st.op == PS_NORM2) {
            const T* v = static_cast<const T*>(st.v[0]);
            double part = 0;
            for_each(0, st.n0, [&](uint32_t i) {
                double t = (double)v[i];
                part += t * t;
            });
            part = cta_sum<NT>(part);
            if (threadIdx.x == 0) bar->red[blockIdx.x] = part;
        } else if (st.op == PS_LOOPTEST || st.op == PS_JUMP) {
            // a decision every CTA takes alike: thread 0 computes it from data
            // all CTAs see the same, and the CTA reads it back from shared memory
            if (threadIdx.x < 32) {
                uint32_t slot = st.mode & 255u;
                uint32_t nx = pc + 1;
                if (st.op == PS_LOOPTEST) {
                    double t = 0;
                    for (uint32_t b = threadIdx.x; b < gridDim.x; b += 32) t += ((volatile double*)bar->red)[b];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                    double nrm = sqrt(t);
                    if (threadIdx.x == 0) {
                        if (st.mode & 256u) {
                            s_init[slot] = nrm;
                            s_cnt[slot] = 0;
                        } else if (nrm / s_init[slot] < st.s0) {
                            nx = st.target;
                        }
                    }
                } else if (threadIdx.x == 0) {
                    if (++s_cnt[slot] >= PK_LOOP_CAP || ++s_total >= PK_TOTAL_CAP) {
                        atomicCAS(&bar->err, 0, 2);
                        nx = nsteps;  // stop
                    } else {
                        nx = st.target;
                    }
                }
                if (threadIdx.x == 0) s_next = nx;
            }
            __syncthreads();
            next = s_next;
            sync_grid = false;  // nothing was written to global memory
        } else {
            run_step<T>(st);
        }
        if (next < nsteps) {
            if (sync_grid) {
                if (!pk_barrier(bar, target)) {
                    ok = false;
                    break;
                }
            } else {
                __syncthreads();
            }
        }
        pc = next;
        cur ^= 1;
    }
    (void)ok;
    // Every CTA has left its last barrier wait once exitc reaches the grid
    // size, so the last one to leave resets the counters for the next launch.
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned e = atomicAdd(&bar->exitc, 1u);
        if (e == gridDim.x - 1) {
            atomicExch(&bar->count, 0u);
            atomicExch(&bar->exitc, 0u);
        }
    }
}

}  // namespace

template <class T>
unsigned persist_grid() {
    static unsigned g = 0;
    if (!g) {
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist<T, PK_THREADS>, PK_THREADS, 0));
        if (per_sm < 1) MLP_THROW(ERR_INTERNAL, "persistent apply kernel does not fit on an SM");
        // two CTAs per SM where they fit
        g = (unsigned)num_sms() * (unsigned)std::min(per_sm, 2);
        if (g > sizeof(PBar::red) / sizeof(double))
            MLP_THROW(ERR_INTERNAL, "persistent apply grid exceeds its reduction buffer");
    }
    return g;
}

template <class T>
void launch_persist(const PStep<T>* steps, uint32_t nsteps, PBar* bar, cudaStream_t s) {
    if (!nsteps) return;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(persist_grid<T>());
    cfg.blockDim = dim3(PK_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k_persist<T, PK_THREADS>, steps, nsteps, bar));
}

template unsigned persist_grid<double>();
template unsigned persist_grid<float>();
template void launch_persist<double>(const PStep<double>*, uint32_t, PBar*, cudaStream_t);
template void launch_persist<float>(const PStep<float>*, uint32_t, PBar*, cudaStream_t);


}  // namespace mlp
