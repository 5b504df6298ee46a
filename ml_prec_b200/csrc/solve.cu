// Solve phase: CSR SpMV, the level-scheduled triangular solves, the recursive
// multi-split / Chebyshev apply recorded as a launch plan (replayed as one CUDA
// graph), and the device-resident PCG loop.
//
// Every vector of level l lives in the level's frame order (setup.cuh): the
// next level's vectors are slices [M, M+n) of this level's, so the recursion
// moves no data between levels.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

// In-graph timeline (mlp_prec_timeline): while c_tl_buf is set, thread 0 of
// block 0 of every kernel of this file writes %globaltimer into it when it
// passes the dependent-launch wait, so consecutive stamps bound each launch's
// time inside the graph (with programmatic dependent launch the next kernel's
// wait returns when this one has finished). Off (null) the cost is one
// constant-cache load in one thread per kernel.
namespace mlp {
__constant__ unsigned long long* c_tl_buf;
__constant__ unsigned c_tl_cap;
__device__ unsigned g_tl_n;
__device__ __forceinline__ void tl_stamp() {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long* b = c_tl_buf;
        if (b) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            unsigned i = atomicAdd(&g_tl_n, 1u);
            if (i < c_tl_cap) b[i] = t;
        }
    }
}
}  // namespace mlp
#define MLP_TIMELINE_HOOK() ::mlp::tl_stamp()

#include "persist.cuh"
#include "small.cuh"
#include "solve.cuh"

namespace mlp {

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// a * b + c rounded once. Row sums that must agree bit for bit between
// kernels (the separate and merged sweep steps) use it explicitly rather than
// relying on the compiler's contraction of s += a * b.
__device__ __forceinline__ double fmadd(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmadd(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// y = A x  (or y = f - A x when f != null). LPR lanes cooperate on one row and
// reduce with shuffles; rows of a 7-point stencil use 8 lanes.
template <class T, int LPR>
__global__ void __launch_bounds__(256) k_spmv(uint32_t n, const uint32_t* __restrict__ ia,
                                              const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                              const T* __restrict__ x, T* __restrict__ y,
                                              const T* __restrict__ f) {
    pdl_wait();
    pdl_trigger();
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t row = gid / LPR;
    int lane = gid % LPR;
    bool active = row < n;
    T s = 0;
    if (active) {
        uint32_t e = ia[row + 1];
        for (uint32_t j = ia[row] + lane; j < e; j += LPR) s = fmadd(a[j], x[ja[j]], s);
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (active && lane == 0) y[row] = f ? f[row] - s : s;
}

// Staged CSR SpMV: a CTA takes tiles of ST_ROWS consecutive rows; the tile's
// column indices and values are copied into shared memory with 16-byte vector
// loads (coalesced, independent of the row structure), then each thread
// reduces one row from shared memory, gathering x through L2.
static constexpr uint32_t ST_ROWS = 256;
static constexpr uint32_t ST_MAX_NNZ = 3072;

// Row sum of a staged tile: sum_j s_a[j - ba] * x[s_ja[j - bj]] over [j, je),
// accumulated in column order; the column indices and x values of four
// entries are loaded before their products are added, so the x gathers of a
// row are in flight together instead of one after another.
template <class T, class XF>
__device__ __forceinline__ T staged_row(uint32_t j, uint32_t je, const uint32_t* s_ja, uint32_t bj, const T* s_a,
                                        uint32_t ba, XF xv) {
    T acc = 0;
    for (; j + 4 <= je; j += 4) {
        uint32_t c0 = s_ja[j - bj], c1 = s_ja[j + 1 - bj], c2 = s_ja[j + 2 - bj], c3 = s_ja[j + 3 - bj];
        T x0 = xv(c0), x1 = xv(c1), x2 = xv(c2), x3 = xv(c3);
        acc = fmadd(s_a[j - ba], x0, acc);
        acc = fmadd(s_a[j + 1 - ba], x1, acc);
        acc = fmadd(s_a[j + 2 - ba], x2, acc);
        acc = fmadd(s_a[j + 3 - ba], x3, acc);
    }
    for (; j < je; j++) acc = fmadd(s_a[j - ba], xv(s_ja[j - bj]), acc);
    return acc;
}

// Pipelined staged tiles. The dynamic shared memory holds two tile buffers
// and three row-start buffers; while a tile's rows are summed, the next
// tile's column indices (and, with SA, its values) and the row starts of the
// one after are already on their way (cp.async, 16 bytes per copy, from the
// 16-byte boundaries at or below the tile's first entries). Without SA the
// values are read from global memory in the summing loop (each row's values
// are contiguous; the tile's lines are reused through L1), which halves the
// shared memory of a CTA so twice as many warps fit on an SM. The matrix
// copies of the first tile are issued before griddepcontrol.wait (the matrix
// is constant); x is only read after it. Rows are summed in column order
// (staged_row), so the result equals the unpipelined order.
constexpr uint32_t PIPE_IAS = ST_ROWS + 8;
template <class T>
__host__ __device__ constexpr uint32_t pipe_cap(uint32_t tile_max) { return (tile_max + 8 + 3) & ~3u; }
template <class T, bool SA>
__host__ __device__ constexpr size_t pipe_smem_bytes(uint32_t tile_max) {
    return 2ull * pipe_cap<T>(tile_max) * ((SA ? sizeof(T) : 0) + 4) + 3ull * PIPE_IAS * 4;
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all_groups() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <class T, bool SA, class Val, class Epi>
__device__ __forceinline__ void spmv_pipe_v(uint32_t n, const uint32_t* __restrict__ ia,
                                            const uint32_t* __restrict__ ja, const T* __restrict__ a, Val val,
                                            uint32_t cap, Epi epi) {
    extern __shared__ __align__(16) unsigned char pipe_smem[];
    constexpr uint32_t VA = 16 / sizeof(T);
    T* s_a = reinterpret_cast<T*>(pipe_smem);                                // 2 x cap (SA only)
    uint32_t* s_ja = reinterpret_cast<uint32_t*>(s_a + (SA ? 2 * cap : 0));  // 2 x cap
    uint32_t* s_ia = s_ja + 2 * cap;                                         // 3 x PIPE_IAS
    const uint32_t ntiles = (n + ST_ROWS - 1) / ST_ROWS;
    const uint32_t G = gridDim.x;
    auto issue_ia = [&](uint32_t t, int b) {
        uint32_t r0 = t * ST_ROWS, nr = min(ST_ROWS, n - r0);
        uint32_t nv = (nr + 1 + 3) / 4;  // r0 is a multiple of 4: 16-byte aligned
        for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) cp_async16(s_ia + b * PIPE_IAS + 4 * v, ia + r0 + 4 * v);
    };
    auto issue_tile = [&](uint32_t t, int bi, int b) {
        uint32_t nr = min(ST_ROWS, n - t * ST_ROWS);
        const uint32_t* sia = s_ia + bi * PIPE_IAS;
        uint32_t e0 = sia[0], e1 = sia[nr];
        uint32_t bj = e0 & ~3u, nvj = (e1 - bj + 3) / 4;
        for (uint32_t v = threadIdx.x; v < nvj; v += blockDim.x) cp_async16(s_ja + b * cap + 4 * v, ja + bj + 4 * v);
        if (SA) {
            uint32_t ba = e0 & ~(VA - 1), nva = (e1 - ba + VA - 1) / VA;
            for (uint32_t v = threadIdx.x; v < nva; v += blockDim.x) cp_async16(s_a + b * cap + VA * v, a + ba + VA * v);
        }
    };
    const uint32_t t0 = blockIdx.x;
    if (t0 < ntiles) {
        issue_ia(t0, 0);
        cp_async_commit();
        cp_async_wait_all_groups();
        __syncthreads();
        issue_tile(t0, 0, 0);
        if (t0 + G < ntiles) issue_ia(t0 + G, 1);
        cp_async_commit();
    }
    pdl_wait();
    pdl_trigger();
    uint32_t i = 0;
    for (uint32_t t = t0; t < ntiles; t += G, i++) {
        cp_async_wait_all_groups();
        __syncthreads();
        uint32_t tn = t + G;
        if (tn < ntiles) {
            issue_tile(tn, (i + 1) % 3, (i + 1) & 1);
            if (tn + G < ntiles) issue_ia(tn + G, (i + 2) % 3);
            cp_async_commit();
        }
        uint32_t r0 = t * ST_ROWS, nr = min(ST_ROWS, n - r0);
        const uint32_t* sia = s_ia + (i % 3) * PIPE_IAS;
        uint32_t e0 = sia[0];
        uint32_t bj = e0 & ~3u, ba = e0 & ~(VA - 1);
        if (threadIdx.x < nr) {
            T acc = SA ? staged_row<T>(sia[threadIdx.x], sia[threadIdx.x + 1], s_ja + (i & 1) * cap, bj,
                                       s_a + (i & 1) * cap, ba, val)
                       : staged_row<T>(sia[threadIdx.x], sia[threadIdx.x + 1], s_ja + (i & 1) * cap, bj, a, 0, val);
            epi(r0 + threadIdx.x, acc);
        }
    }
}

template <class T, bool SA, class Epi>
__device__ __forceinline__ void spmv_pipe(uint32_t n, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                                          const T* __restrict__ a, const T* __restrict__ x, uint32_t cap, Epi epi) {
    spmv_pipe_v<T, SA>(n, ia, ja, a, [&](uint32_t c) { return x[c]; }, cap, epi);
}

// The sweep steps of a large level on the same tile pipeline (rows summed
// serially in column order): phase 1 (w = P1 src on rows < R, then the
// diagonal rows out = dval src), phase 2 (out_q = sum G_qj (j < M ? w_j :
// out_j)) and the correction (x += u0; r -= A u0).
template <class T>
__global__ void __launch_bounds__(ST_ROWS) k_phase1_staged(uint32_t R, uint32_t N, const uint32_t* __restrict__ ia,
                                                           const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                           const T* __restrict__ dval, const T* __restrict__ src,
                                                           T* __restrict__ w, T* __restrict__ out, uint32_t cap) {
    spmv_pipe_v<T, false>(R, ia, ja, a, [&](uint32_t c) { return src[c]; }, cap,
                          [&](uint32_t row, T acc) { w[row] = acc; });
    for (uint32_t q = R + blockIdx.x * blockDim.x + threadIdx.x; q < N; q += gridDim.x * blockDim.x)
        out[q] = dval[q - R] * src[q];
}
template <class T>
__global__ void __launch_bounds__(ST_ROWS) k_phase2_staged(uint32_t M, const uint32_t* __restrict__ ia,
                                                           const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                           const T* __restrict__ w, T* out, uint32_t cap) {
    spmv_pipe_v<T, false>(M, ia, ja, a, [&](uint32_t c) { return c < M ? w[c] : out[c]; }, cap,
                          [&](uint32_t row, T acc) { out[row] = acc; });
}
template <class T>
__global__ void __launch_bounds__(ST_ROWS) k_update_staged(uint32_t N, const uint32_t* __restrict__ ia,
                                                           const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                           const T* __restrict__ u0, T* __restrict__ x,
                                                           T* __restrict__ r, uint32_t cap) {
    spmv_pipe_v<T, false>(N, ia, ja, a, [&](uint32_t c) { return u0[c]; }, cap, [&](uint32_t row, T acc) {
        x[row] += u0[row];
        r[row] -= acc;
    });
}

template <class T, int MODE, bool SA>  // MODE 0: y = A x, 1: y = f - A x
__global__ void __launch_bounds__(ST_ROWS) k_spmv_staged(uint32_t n, const uint32_t* __restrict__ ia,
                                                         const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                         const T* __restrict__ x, T* __restrict__ y,
                                                         const T* __restrict__ f, uint32_t cap) {
    spmv_pipe<T, SA>(n, ia, ja, a, x, cap, [&](uint32_t row, T acc) { y[row] = MODE ? f[row] - acc : acc; });
}

__global__ void k_tile_max(uint32_t n, const uint32_t* __restrict__ ia, uint32_t* __restrict__ out) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r0 = t * ST_ROWS;
    if (r0 >= n) return;
    uint32_t r1 = min(n, r0 + ST_ROWS);
    atomicMax(out, ia[r1] - ia[r0]);
}

static void pipe_prepare_all(uint32_t tile_max);

void csr_tile_stats(DCSR& m, cudaStream_t s) {
    if (!m.nrow) { m.tile_max = 0; return; }
    Tmp<uint32_t> d(1);
    d.zero(s);
    uint32_t nt = (m.nrow + ST_ROWS - 1) / ST_ROWS;
    k_tile_max<<<grid_for(nt, 256), 256, 0, s>>>(m.nrow, m.ia.p, d.p);
    CK_LAUNCH();
    CK(cudaMemcpyAsync(&m.tile_max, d.p, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // the staged kernels' launch shapes are worked out here, outside any stream capture
    if (m.tile_max && m.tile_max <= ST_MAX_NNZ) pipe_prepare_all(m.tile_max);
}

void csr_tile_stats_batch(const std::vector<DCSR*>& ms, const std::vector<const uint32_t*>& extra,
                          std::vector<uint32_t>& extra_out, cudaStream_t s) {
    Tmp<uint32_t> d(ms.size() + 1);
    d.zero(s);
    std::vector<const uint32_t*> words;
    for (size_t i = 0; i < ms.size(); i++) {
        const DCSR& m = *ms[i];
        if (m.nrow) {
            uint32_t nt = (m.nrow + ST_ROWS - 1) / ST_ROWS;
            k_tile_max<<<grid_for(nt, 256), 256, 0, s>>>(m.nrow, m.ia.p, d.p + i);
            CK_LAUNCH();
        }
        words.push_back(d.p + i);
    }
    for (const uint32_t* w : extra) words.push_back(w);
    std::vector<uint32_t> h = read_words(words, s);
    for (size_t i = 0; i < ms.size(); i++) {
        DCSR& m = *ms[i];
        m.tile_max = m.nrow ? h[i] : 0;
        if (m.tile_max && m.tile_max <= ST_MAX_NNZ) pipe_prepare_all(m.tile_max);
    }
    extra_out.assign(h.begin() + ms.size(), h.end());
}

// Largest grid of the staged PCG SpMV (and so the size of its callers'
// reduction scratch): one tile per CTA, at most eight CTAs per SM, the
// occupancy the tile pipeline reaches (pipe_grid); at five per SM the
// in-graph SpMV with (Ap, p) ran at 0.53 of the HBM bandwidth against 0.77
// for the SpMV alone at eight.
static unsigned staged_grid(uint32_t n) {
    uint32_t nt = (n + ST_ROWS - 1) / ST_ROWS;
    return (unsigned)std::max<uint32_t>(1, std::min<uint32_t>(nt, (uint32_t)num_sms() * 8));
}

// Grid of a pipelined staged kernel: the CTAs that fit on the device at once
// with this shared memory (at most eight per SM, and at most one per tile).
template <class K>
static unsigned pipe_grid(K kern, uint32_t n, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<const void*, size_t>, int> occ;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto key = std::make_pair((const void*)kern, smem);
        auto it = occ.find(key);
        if (it == occ.end()) {
            cudaFuncAttributes fa;
            CK(cudaFuncGetAttributes(&fa, kern));
            CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(small_smem_limit() - fa.sharedSizeBytes)));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ST_ROWS, smem));
            occ[key] = per_sm;
        } else {
            per_sm = it->second;
        }
    }
    uint32_t nt = (n + ST_ROWS - 1) / ST_ROWS;
    uint32_t g = (uint32_t)num_sms() * (uint32_t)std::max(1, std::min(per_sm, 8));
    return (unsigned)std::max<uint32_t>(1, std::min<uint32_t>(nt, g));
}

template <class T>
static void launch_spmv(uint32_t n, uint32_t nnz, const uint32_t* ia, const uint32_t* ja, const T* a, const T* x,
                        T* y, const T* f, cudaStream_t s, uint32_t tile_max = 0) {
    if (!n) return;
    if (tile_max && tile_max <= ST_MAX_NNZ && n >= 4 * ST_ROWS) {
        uint32_t cap = pipe_cap<T>(tile_max);
        size_t smem = pipe_smem_bytes<T, false>(tile_max);
        if (f) launch_k(k_spmv_staged<T, 1, false>, pipe_grid(k_spmv_staged<T, 1, false>, n, smem), ST_ROWS, smem, s, n,
                        ia, ja, a, x, y, f, cap);
        else launch_k(k_spmv_staged<T, 0, false>, pipe_grid(k_spmv_staged<T, 0, false>, n, smem), ST_ROWS, smem, s, n,
                      ia, ja, a, x, y, f, cap);
        return;
    }
    double avg = (double)nnz / n;
    int lpr = avg <= 1.5 ? 1 : avg <= 3 ? 2 : avg <= 6 ? 4 : avg <= 12 ? 8 : avg <= 24 ? 16 : 32;
    unsigned blocks = grid_for((size_t)n * lpr, 256);
    switch (lpr) {
        case 1: launch_k(k_spmv<T, 1>, blocks, 256, 0, s, n, ia, ja, a, x, y, f); break;
        case 2: launch_k(k_spmv<T, 2>, blocks, 256, 0, s, n, ia, ja, a, x, y, f); break;
        case 4: launch_k(k_spmv<T, 4>, blocks, 256, 0, s, n, ia, ja, a, x, y, f); break;
        case 8: launch_k(k_spmv<T, 8>, blocks, 256, 0, s, n, ia, ja, a, x, y, f); break;
        case 16: launch_k(k_spmv<T, 16>, blocks, 256, 0, s, n, ia, ja, a, x, y, f); break;
        default: launch_k(k_spmv<T, 32>, blocks, 256, 0, s, n, ia, ja, a, x, y, f); break;
    }
}

void spmv(const DCSR& A, const double* x, double* y, cudaStream_t s) {
    launch_spmv<double>(A.nrow, A.nnz, A.ia.p, A.ja.p, A.a.p, x, y, nullptr, s, A.tile_max);
    CK_LAUNCH();
}

// One wavefront of the L solve (solve_L, multi_split_solve.cc:25-36) over
// contiguous frame rows [r0, r1): w_q = src_q - sum_k L_qk w_k.
template <class T>
__global__ void k_lwave(uint32_t r0, uint32_t r1, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                        const T* __restrict__ a, const T* __restrict__ src, T* __restrict__ w) {
    pdl_wait();
    pdl_trigger();
    uint32_t q = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= r1) return;
    T s = src[q];
    for (uint32_t j = ia[q]; j < ia[q + 1]; j++) s -= a[j] * w[ja[j]];
    w[q] = s;
}

// Coarse rows of the L solve (they read eliminated rows only) fused with the
// diagonal block (solve_diagonal, multi_split_solve.cc:12-22): rows [M, R)
// write w, rows [R, N) write out = dval * src.
template <class T>
__global__ void k_lcoarse_diag(uint32_t M, uint32_t R, uint32_t N, const uint32_t* __restrict__ ia,
                               const uint32_t* __restrict__ ja, const T* __restrict__ a, const T* __restrict__ src,
                               T* __restrict__ w, const T* __restrict__ dval, T* __restrict__ out) {
    pdl_wait();
    pdl_trigger();
    uint32_t q = M + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N) return;
    if (q < R) {
        T s = src[q];
        for (uint32_t j = ia[q]; j < ia[q + 1]; j++) s -= a[j] * w[ja[j]];
        w[q] = s;
    } else {
        out[q] = dval[q - R] * src[q];
    }
}

// One wavefront of the U solve (solve_U, multi_split_solve.cc:39-53):
// out_q = (w_q - sum_{j != q} U_qj out_j) / U_qq, rows given by a list.
template <class T>
__global__ void k_uwave(uint32_t cnt, const uint32_t* __restrict__ rows, const uint32_t* __restrict__ ia,
                        const uint32_t* __restrict__ ja, const T* __restrict__ a, const T* __restrict__ w,
                        T* __restrict__ out) {
    pdl_wait();
    pdl_trigger();
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    uint32_t q = rows[t];
    uint32_t rs = ia[q];
    T z = w[q];
    for (uint32_t j = rs + 1; j < ia[q + 1]; j++) z -= a[j] * out[ja[j]];
    out[q] = z / a[rs];
}

// The deep wavefronts of a level hold few rows each: one CTA runs all of them
// with a barrier between wavefronts instead of one launch per wavefront.
static constexpr uint32_t TAIL_ROWS = 1024;
static constexpr uint32_t TAIL_THREADS = 1024;

template <class T>
__global__ void __launch_bounds__(TAIL_THREADS) k_lwave_tail(uint32_t d0, uint32_t d1, const uint32_t* __restrict__ off,
                                                             const uint32_t* __restrict__ ia,
                                                             const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                             const T* __restrict__ src, T* w) {
    pdl_wait();
    pdl_trigger();
    for (uint32_t d = d0; d < d1; d++) {
        uint32_t r0 = off[d], r1 = off[d + 1];
        for (uint32_t q = r0 + threadIdx.x; q < r1; q += blockDim.x) {
            T s = src[q];
            for (uint32_t j = ia[q]; j < ia[q + 1]; j++) s -= a[j] * w[ja[j]];
            w[q] = s;
        }
        __syncthreads();
    }
}

template <class T>
__global__ void __launch_bounds__(TAIL_THREADS) k_uwave_tail(uint32_t d0, uint32_t d1, const uint32_t* __restrict__ off,
                                                             const uint32_t* __restrict__ rows,
                                                             const uint32_t* __restrict__ ia,
                                                             const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                             const T* __restrict__ w, T* out) {
    pdl_wait();
    pdl_trigger();
    for (uint32_t d = d0; d < d1; d++) {
        uint32_t o0 = off[d], o1 = off[d + 1];
        for (uint32_t t = o0 + threadIdx.x; t < o1; t += blockDim.x) {
            uint32_t q = rows[t];
            uint32_t rs = ia[q];
            T z = w[q];
            for (uint32_t j = rs + 1; j < ia[q + 1]; j++) z -= a[j] * out[ja[j]];
            out[q] = z / a[rs];
        }
        __syncthreads();
    }
}

// First wavefront from which every remaining wavefront is small.
static size_t tail_start(const std::vector<uint32_t>& off) {
    size_t nw = off.empty() ? 0 : off.size() - 1;
    size_t d = nw;
    while (d > 0 && off[d] - off[d - 1] <= TAIL_ROWS) d--;
    return (nw - d >= 2) ? d : nw;
}

template <class T>
__global__ void k_axpy1(uint32_t n, T* __restrict__ x, const T* __restrict__ u) {
    pdl_wait();
    pdl_trigger();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += u[i];
}

template <class T>
__global__ void k_scale(uint32_t n, T* __restrict__ x, T alpha) {
    pdl_wait();
    pdl_trigger();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] *= alpha;
}

template <class T>
__global__ void k_copy(uint32_t n, const T* __restrict__ src, T* __restrict__ dst) {
    pdl_wait();
    pdl_trigger();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

// Chebyshev step 2 (cheb_solve.cc:70-72): x2 = -alpha*x2 + c*u1
template <class T>
__global__ void k_cheb2(uint32_t n, T* __restrict__ x2, const T* __restrict__ u1, T malpha, T c) {
    pdl_wait();
    pdl_trigger();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x2[i] = fmadd(x2[i], malpha, c * u1[i]);
}
// Chebyshev step k >= 3 (cheb_solve.cc:98-99): x2 = u1 - alpha*x2 + beta*(u1-u0)
template <class T>
__global__ void k_chebk(uint32_t n, T* __restrict__ x2, const T* __restrict__ u1, const T* __restrict__ u0,
                        T alpha, T beta) {
    pdl_wait();
    pdl_trigger();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        T a1 = u1[i];
        x2[i] = fmadd(beta, a1 - u0[i], fmadd(-alpha, x2[i], a1));
    }
}

// Dense coarsest level: x = C^{-1} f, one warp per row. The operator's type
// CT may be wider than the vectors' T: the FP32 hierarchy keeps its coarsest
// solve (the dense inverse, or the tabulated small-level operator standing in
// for it) in FP64 and accumulates in FP64. EPI > 0 applies the Chebyshev
// update that follows a tabulated level call to the row's result, with the
// arithmetic of the separate kernel: 1 k_scale (x = v ea), 2 k_cheb2
// (x = v ea + eb u1), 3 k_chebk (x = u1 - ea v + eb (u1 - u0), ea = alpha).
enum { EPI_NONE = 0, EPI_SCALE = 1, EPI_CHEB2 = 2, EPI_CHEBK = 3 };
template <class T, class CT, int EPI>
__device__ __forceinline__ void dense_gemv_body(uint32_t n, const CT* __restrict__ C, const T* __restrict__ f,
                                                T* __restrict__ x, const T* __restrict__ u1,
                                                const T* __restrict__ u0, T ea, T eb) {
    // the operator is constant: its row is loaded before the wait (see RowPre)
    constexpr int CV = 16;
    uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    const CT* c = C + (size_t)(row < n ? row : 0) * n;
    CT cv[CV];
#pragma unroll
    for (int k = 0; k < CV; k++) {
        uint32_t j = lane + 32 * k;
        cv[k] = (row < n && j < n) ? c[j] : CT(0);
    }
    pdl_wait();
    pdl_trigger();
    if (row >= n) return;
    CT s = 0;
#pragma unroll
    for (int k = 0; k < CV; k++) {
        uint32_t j = lane + 32 * k;
        if (j < n) s = fmadd(cv[k], (CT)f[j], s);
    }
    for (uint32_t j = lane + 32 * CV; j < n; j += 32) s = fmadd(c[j], (CT)f[j], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        T v = (T)s;
        if (EPI == EPI_SCALE) {
            v *= ea;
        } else if (EPI == EPI_CHEB2) {
            v = fmadd(v, ea, eb * u1[row]);
        } else if (EPI == EPI_CHEBK) {
            T a1 = u1[row];
            v = fmadd(eb, a1 - u0[row], fmadd(-ea, v, a1));
        }
        x[row] = v;
    }
}
template <class T, class CT = T>
__global__ void k_dense_gemv(uint32_t n, const CT* __restrict__ C, const T* __restrict__ f, T* __restrict__ x) {
    dense_gemv_body<T, CT, EPI_NONE>(n, C, f, x, nullptr, nullptr, T(0), T(0));
}
template <class T, class CT, int EPI>
__global__ void k_dense_gemv_epi(uint32_t n, const CT* __restrict__ C, const T* __restrict__ f, T* __restrict__ x,
                                 const T* __restrict__ u1, const T* __restrict__ u0, T ea, T eb) {
    dense_gemv_body<T, CT, EPI>(n, C, f, x, u1, u0, ea, eb);
}

__global__ void k_to_f32(uint32_t n, const double* __restrict__ a, float* __restrict__ b) {
    pdl_wait();
    pdl_trigger();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
__global__ void k_to_f64(uint32_t n, const float* __restrict__ a, double* __restrict__ b) {
    pdl_wait();
    pdl_trigger();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}
__global__ void k_gather(uint32_t n, const uint32_t* __restrict__ idx, const double* __restrict__ src,
                         double* __restrict__ dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}
__global__ void k_scatter(uint32_t n, const uint32_t* __restrict__ idx, const double* __restrict__ src,
                          double* __restrict__ dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[idx[i]] = src[i];
}

// Replays the recorded launches.
void Plan::run(cudaStream_t s) const {
    for (const auto& op : ops) op(s);
}

void gather(uint32_t n, const uint32_t* idx, const double* src, double* dst, cudaStream_t s) {
    if (!n) return;
    k_gather<<<grid_for(n, 256), 256, 0, s>>>(n, idx, src, dst);
    CK_LAUNCH();
}
void scatter(uint32_t n, const uint32_t* idx, const double* src, double* dst, cudaStream_t s) {
    if (!n) return;
    k_scatter<<<grid_for(n, 256), 256, 0, s>>>(n, idx, src, dst);
    CK_LAUNCH();
}


// ---- explicit-form sweep kernels -------------------------------------------
// The matrices of the apply are constant, so a row kernel loads its row's
// first PRE_K entries (values and column indices) BEFORE griddepcontrol.wait:
// under programmatic dependent launch those loads overlap the tail of the
// previous kernel, and after the wait only the gathers of the vector the
// previous kernel wrote remain on the critical path. The products are added in
// the same order as a plain lane-strided loop.
constexpr int PRE_K = 4;

template <class T, int LPR>
struct RowPre {
    uint32_t jb = 0, je = 0;
    T av[PRE_K];
    uint32_t cv[PRE_K];
    __device__ __forceinline__ void load(bool active, uint32_t row, int lane, const uint32_t* __restrict__ ia,
                                         const uint32_t* __restrict__ ja, const T* __restrict__ a) {
        if (active) {
            jb = ia[row] + lane;
            je = ia[row + 1];
        }
#pragma unroll
        for (int k = 0; k < PRE_K; k++) {
            uint32_t j = jb + k * LPR;
            av[k] = 0;
            cv[k] = 0;
            if (j < je) {
                av[k] = a[j];
                cv[k] = ja[j];
            }
        }
    }
    template <class V>
    __device__ __forceinline__ T sum(V val, const uint32_t* __restrict__ ja, const T* __restrict__ a) const {
        T s = 0;
#pragma unroll
        for (int k = 0; k < PRE_K; k++)
            if (jb + k * LPR < je) s = fmadd(av[k], val(cv[k]), s);
        for (uint32_t j = jb + PRE_K * LPR; j < je; j += LPR) s = fmadd(a[j], val(ja[j]), s);
        return s;
    }
};

// Phase 1 of a level solve: w = P1 src on rows [0, R) (the L solve of the
// eliminated and coarse rows) and out = dval * src on the diagonal rows
// [R, N). The first nb1 blocks take the P1 rows with LPR lanes per row, the
// rest one diagonal row per thread.
template <class T, int LPR>
__global__ void __launch_bounds__(512) k_phase1(uint32_t R, uint32_t N, uint32_t nb1, const uint32_t* __restrict__ ia,
                                                const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                const T* __restrict__ dval, const T* __restrict__ src,
                                                T* __restrict__ w, T* __restrict__ out) {
    if (blockIdx.x < nb1) {
        uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
        uint32_t row = gid / LPR;
        int lane = gid % LPR;
        bool active = row < R;
        RowPre<T, LPR> rp;
        rp.load(active, row, lane, ia, ja, a);
        pdl_wait();
        pdl_trigger();
        T s = rp.sum([&](uint32_t c) { return src[c]; }, ja, a);
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lane == 0) w[row] = s;
    } else {
        uint32_t q = R + (blockIdx.x - nb1) * blockDim.x + threadIdx.x;
        T d = q < N ? dval[q - R] : T(0);
        pdl_wait();
        pdl_trigger();
        if (q < N) out[q] = d * src[q];
    }
}

// Phase 2: out_q = sum_j G_qj y_j on the eliminated rows q < M, where
// y_j = w_j for eliminated columns (j < M) and out_j (the coarse solution the
// recursion wrote) for coarse columns.
template <class T, int LPR>
__global__ void __launch_bounds__(512) k_phase2(uint32_t M, const uint32_t* __restrict__ ia,
                                                const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                const T* __restrict__ w, T* out) {
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t row = gid / LPR;
    int lane = gid % LPR;
    bool active = row < M;
    RowPre<T, LPR> rp;
    rp.load(active, row, lane, ia, ja, a);
    pdl_wait();
    pdl_trigger();
    T s = rp.sum([&](uint32_t c) { return c < M ? w[c] : out[c]; }, ja, a);
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (active && lane == 0) out[row] = s;
}

// Phase 2 with the coarse solve folded in (launch plan; the level below is
// one dense FP64 operator C, n x n). One launch computes
//  * the coarse solution out_{M+k} = C_k . w_C, a warp per row with the
//    arithmetic of k_dense_gemv (blocks [0, nb_c));
//  * the nf rows of G with coarse columns (rows[0, nf)), a warp per row:
//    out_q = sum_{j<M} G_qj w_j (in lanes, as k_phase2 with 32 lanes) + D_q . w_C,
//    D = G_C C built at set-up in FP64 (blocks [nb_c, nb_c + nb_f));
//  * the other rows (rows[nf, M), all columns < M) exactly as k_phase2.
// So the apply needs no separate launch for the coarse solve; the folded rows
// add G_C (C w_C) in the order (G_C C) w_C. In FP32 a folded row's bounds and
// each lane's first G entry are loaded before the dependent-launch wait and its
// first gather is issued with those of w_C (FP32 solve at 60x220x85 on B200
// 11.60 -> 10.69 ms); in FP64 that measured slower (16.23 -> 16.45 ms), so
// there the row is read after the wait.
template <class T, int LPR>
__global__ void __launch_bounds__(256) k_phase2_fold(uint32_t M, uint32_t n, const uint32_t* __restrict__ ia,
                                                     const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                     const double* __restrict__ C, const double* __restrict__ D,
                                                     const uint32_t* __restrict__ rows, uint32_t nf, uint32_t nb_c,
                                                     uint32_t nb_f, const T* __restrict__ w, T* __restrict__ out) {
    if (blockIdx.x < nb_c + nb_f) {
        constexpr int CV = 16;
        const bool coarse = blockIdx.x < nb_c;
        const uint32_t r = (coarse ? blockIdx.x : blockIdx.x - nb_c) * (blockDim.x >> 5) + (threadIdx.x >> 5);
        const int lane = threadIdx.x & 31;
        const uint32_t nr = coarse ? n : nf;
        const double* c = (coarse ? C : D) + (size_t)(r < nr ? r : 0) * n;
        double cv[CV];
#pragma unroll
        for (int k = 0; k < CV; k++) {
            uint32_t j = lane + 32 * k;
            cv[k] = (r < nr && j < n) ? c[j] : 0.0;
        }
        // FP32: a folded row's G row, its bounds and each lane's first entry
        constexpr bool PRE = sizeof(T) == 4;
        uint32_t q = 0, gj = 0, ge = 0, gc = 0;
        T ga = 0;
        if (PRE && !coarse && r < nr) {
            q = rows[r];
            gj = ia[q] + lane;
            ge = ia[q + 1];
            if (gj < ge) {
                gc = ja[gj];
                ga = a[gj];
            }
        }
        pdl_wait();
        pdl_trigger();
        if (r >= nr) return;
        const T* wc = w + M;
        const bool g0 = PRE && !coarse && gj < ge && gc < M;
        const T wg = g0 ? w[gc] : T(0);
        double d = 0;
#pragma unroll
        for (int k = 0; k < CV; k++) {
            uint32_t j = lane + 32 * k;
            if (j < n) d = fmadd(cv[k], (double)wc[j], d);
        }
        for (uint32_t j = lane + 32 * CV; j < n; j += 32) d = fmadd(c[j], (double)wc[j], d);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (coarse) {
            if (lane == 0) out[M + r] = (T)d;
            return;
        }
        T sp = 0;
        if constexpr (PRE) {
            if (g0) sp = fmadd(ga, wg, sp);
            for (uint32_t j = gj + 32; j < ge; j += 32) {
                uint32_t col = ja[j];
                if (col < M) sp = fmadd(a[j], w[col], sp);
            }
        } else {
            q = rows[r];
            for (uint32_t j = ia[q] + lane, e = ia[q + 1]; j < e; j += 32) {
                uint32_t col = ja[j];
                if (col < M) sp = fmadd(a[j], w[col], sp);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sp += __shfl_xor_sync(0xffffffffu, sp, o);
        if (lane == 0) out[q] = (T)((double)sp + d);
        return;
    }
    const uint32_t gid = (blockIdx.x - nb_c - nb_f) * blockDim.x + threadIdx.x;
    const uint32_t k = gid / LPR;
    const int lane = gid % LPR;
    const bool active = k < M - nf;
    const uint32_t row = active ? rows[nf + k] : 0;
    RowPre<T, LPR> rp;
    rp.load(active, row, lane, ia, ja, a);
    pdl_wait();
    pdl_trigger();
    T s = rp.sum([&](uint32_t c) { return w[c]; }, ja, a);
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (active && lane == 0) out[row] = s;
}

// D = G_C C for the folded rows: block i takes row rows[i] of G, thread t the
// columns t, t + blockDim.x, ... of D; the coarse entries of the row are
// added in their stored order.
template <class T>
__global__ void k_fold_build(uint32_t nf, const uint32_t* __restrict__ rows, uint32_t M, uint32_t n,
                             const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                             const T* __restrict__ a, const double* __restrict__ C, double* __restrict__ D) {
    const uint32_t i = blockIdx.x;
    if (i >= nf) return;
    const uint32_t q = rows[i];
    for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        double s = 0;
        for (uint32_t j = ia[q]; j < ia[q + 1]; j++) {
            uint32_t col = ja[j];
            if (col >= M) s = fmadd((double)a[j], C[(size_t)(col - M) * n + t], s);
        }
        D[(size_t)i * n + t] = s;
    }
}

// Correction step of a level sweep: x += u0 and, when more sweeps follow,
// r -= A u0 (the residual f - A x updated in place of recomputing it).
template <class T, int LPR>
__global__ void __launch_bounds__(512) k_update(uint32_t n, const uint32_t* __restrict__ ia,
                                                const uint32_t* __restrict__ ja, const T* __restrict__ a,
                                                const T* __restrict__ u0, T* __restrict__ x, T* __restrict__ r,
                                                int do_r) {
    uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t row = gid / LPR;
    int lane = gid % LPR;
    bool active = row < n;
    RowPre<T, LPR> rp;
    rp.load(active && do_r, row, lane, ia, ja, a);
    pdl_wait();
    pdl_trigger();
    T s = rp.sum([&](uint32_t c) { return u0[c]; }, ja, a);
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (active && lane == 0) {
        x[row] += u0[row];
        if (do_r) r[row] -= s;
    }
}

// ---- merged sweep steps --------------------------------------------------------
// At a small level every kernel boundary costs more than the kernel's work, so
// consecutive steps of the sweep are merged where the data allows, and each
// merged kernel reproduces the separate kernels' arithmetic exactly (same
// products, same lane-split partial sums, same butterfly order), so the merged
// and separate paths give bit-identical results:
//  * step A = correction of sweep it-1 + phase 1 of sweep it:
//      x += u0;  r' = r - Af u0;  w = P1 r';  u0'_D = dval r'_D
//    (or, for the second sweep, r' = f - Af x). A thread of a P1 row
//    recomputes the entries r'_k it needs from Af row k instead of waiting for
//    the whole of r' (r and u0 are double-buffered).
//  * step B = the tabulated coarse product + phase 2:
//      u0_C = C w_C;  u0_E = G [w_E; u0_C]
//    a warp of an E row recomputes the entries of u0_C its G row needs.

// Lane-split sum of a CSR row as LP cooperating lanes compute it (lane l adds
// the entries l, l + LP, ... in order, then the xor butterfly of the lanes),
// evaluated by one thread.
template <class T, int LP, class V>
__device__ __forceinline__ T lane_split_sum(uint32_t jb, uint32_t je, const uint32_t* __restrict__ ja,
                                            const T* __restrict__ a, V val) {
    T p[LP];
#pragma unroll
    for (int l = 0; l < LP; l++) p[l] = 0;
    for (uint32_t j = jb; j < je; j++) {
        // entry j belongs to lane (j - jb) % LP; LP is a power of two
        T av = a[j], xv = val(ja[j]);
        int l = (int)((j - jb) & (LP - 1));
#pragma unroll
        for (int m = 0; m < LP; m++)
            if (m == l) p[m] = fmadd(av, xv, p[m]);
    }
#pragma unroll
    for (int o = LP / 2; o > 0; o >>= 1) {
        T q[LP];
#pragma unroll
        for (int l = 0; l < LP; l++) q[l] = p[l] + p[l ^ o];
#pragma unroll
        for (int l = 0; l < LP; l++) p[l] = q[l];
    }
    return p[0];
}

// lane_split_sum with the row's first K entries (column indices pc, values pa)
// already in registers: their K gathers are issued together, then the sum
// goes on in entry order exactly as lane_split_sum adds it.
template <class T, int LP, int K, class V>
__device__ __forceinline__ T lane_split_sum_pre(uint32_t jb, uint32_t je, const uint32_t (&pc)[K], const T (&pa)[K],
                                                const uint32_t* __restrict__ ja, const T* __restrict__ a, V val) {
    T xv[K];
#pragma unroll
    for (int t = 0; t < K; t++) xv[t] = jb + t < je ? val(pc[t]) : T(0);
    T p[LP];
#pragma unroll
    for (int l = 0; l < LP; l++) p[l] = 0;
#pragma unroll
    for (int t = 0; t < K; t++)
        if (jb + t < je) p[t & (LP - 1)] = fmadd(pa[t], xv[t], p[t & (LP - 1)]);
    for (uint32_t j = jb + K; j < je; j++) {
        T av = a[j], x = val(ja[j]);
        int l = (int)((j - jb) & (LP - 1));
#pragma unroll
        for (int m = 0; m < LP; m++)
            if (m == l) p[m] = fmadd(av, x, p[m]);
    }
#pragma unroll
    for (int o = LP / 2; o > 0; o >>= 1) {
        T q[LP];
#pragma unroll
        for (int l = 0; l < LP; l++) q[l] = p[l] + p[l ^ o];
#pragma unroll
        for (int l = 0; l < LP; l++) p[l] = q[l];
    }
    return p[0];
}

// Step A. Blocks [0, nbu): the rows of Af with LPU lanes per row (the
// correction kernel's layout); blocks [nbu, ...): a warp per P1 row.
// MODE 0: r' = f - Af x (second sweep); MODE 1: x += u0; r' = r - Af u0.
// In FP32 the first Af entries of a P1 row's entries are loaded before the
// dependent-launch wait, with the kernel held to five 256-thread CTAs an SM
// so that a level-2 grid of the 60x220x85 field (706 CTAs) stays one wave:
// FP32 solve 10.69 -> 10.36 ms on B200. In FP64 the same prefetch measured
// slower (16.45 -> 17.04 ms: the extra registers spill or split the grid into
// two waves), so FP64 loads them after the wait.
template <class T>
constexpr int merge_a_min_ctas() { return sizeof(T) == 4 ? 5 : 0; }  // 0: no bound
template <class T, int LPU, int LPP, int MODE>
__global__ void __launch_bounds__(256, merge_a_min_ctas<T>()) k_merge_a(uint32_t N, uint32_t R, uint32_t nbu,
                                                 const uint32_t* __restrict__ af_ia,
                                                 const uint32_t* __restrict__ af_ja, const T* __restrict__ af_a,
                                                 const uint32_t* __restrict__ p1_ia, const uint32_t* __restrict__ p1_ja,
                                                 const T* __restrict__ p1_a, const T* __restrict__ dval,
                                                 const T* __restrict__ f, T* __restrict__ x, const T* __restrict__ r_in,
                                                 T* __restrict__ r_out, const T* __restrict__ u_in, T* __restrict__ u_out,
                                                 T* __restrict__ w) {
    const T* v = MODE == 0 ? x : u_in;  // the vector Af multiplies
    if (blockIdx.x < nbu) {
        uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
        uint32_t row = gid / LPU;
        int lane = gid % LPU;
        bool active = row < N;
        RowPre<T, LPU> rp;
        rp.load(active, row, lane, af_ia, af_ja, af_a);
        T d = (active && row >= R) ? dval[row - R] : T(0);
        pdl_wait();
        pdl_trigger();
        T s = rp.sum([&](uint32_t c) { return v[c]; }, af_ja, af_a);
#pragma unroll
        for (int o = LPU / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lane == 0) {
            T rn;
            if (MODE == 0) {
                rn = f[row] - s;
            } else {
                x[row] += u_in[row];
                rn = r_in[row] - s;
            }
            r_out[row] = rn;
            if (row >= R) u_out[row] = d * rn;
        }
    } else {
        // One warp per P1 row: lane e recomputes the entry r'_k of the row's
        // entries e, e + 32, ... (all lanes at once), then the products are
        // added in entry order with k_phase1's lane split. The row's first 32
        // entries and their Af row bounds (and in FP32 the first AFK entries
        // of those Af rows) are loaded before the wait.
        constexpr bool PRE = sizeof(T) == 4;
        constexpr int AFK = PRE ? 4 : 1;
        const uint32_t q = ((blockIdx.x - nbu) * blockDim.x + threadIdx.x) >> 5;
        const int lane = threadIdx.x & 31;
        const bool act = q < R;
        uint32_t jb = 0, je = 0;
        if (act) {
            jb = p1_ia[q];
            je = p1_ia[q + 1];
        }
        uint32_t k0 = 0, kb0 = 0, ke0 = 0;
        T a0 = 0;
        uint32_t fc[AFK];
        T fa[AFK];
#pragma unroll
        for (int t = 0; t < AFK; t++) {
            fc[t] = 0;
            fa[t] = 0;
        }
        if (jb + lane < je) {
            k0 = p1_ja[jb + lane];
            a0 = p1_a[jb + lane];
            kb0 = af_ia[k0];
            ke0 = af_ia[k0 + 1];
            if constexpr (PRE) {
#pragma unroll
                for (int t = 0; t < AFK; t++)
                    if (kb0 + t < ke0) {
                        fc[t] = af_ja[kb0 + t];
                        fa[t] = af_a[kb0 + t];
                    }
            }
        }
        pdl_wait();
        pdl_trigger();
        if (!act) return;  // the whole warp
        auto vv = [&](uint32_t c) { return v[c]; };
        T p[LPP];
#pragma unroll
        for (int l = 0; l < LPP; l++) p[l] = 0;
        for (uint32_t base = jb; base < je; base += 32) {
            uint32_t j = base + lane;
            T av = 0, rv = 0;
            if (j < je) {
                if (PRE && base == jb) {
                    av = a0;
                    T fk = MODE == 0 ? f[k0] : r_in[k0];
                    rv = fk - lane_split_sum_pre<T, LPU, AFK>(kb0, ke0, fc, fa, af_ja, af_a, vv);
                } else {
                    uint32_t k = k0, kb = kb0, ke = ke0;
                    av = a0;
                    if (base != jb) {
                        k = p1_ja[j];
                        av = p1_a[j];
                        kb = af_ia[k];
                        ke = af_ia[k + 1];
                    }
                    T t = lane_split_sum<T, LPU>(kb, ke, af_ja, af_a, vv);
                    rv = (MODE == 0 ? f[k] : r_in[k]) - t;
                }
            }
            uint32_t cnt = min(32u, je - base);
            for (uint32_t e = 0; e < cnt; e++) {
                T ae = __shfl_sync(0xffffffffu, av, e), re = __shfl_sync(0xffffffffu, rv, e);
                int l = (int)((base - jb + e) & (LPP - 1));
#pragma unroll
                for (int m = 0; m < LPP; m++)
                    if (m == l) p[m] = fmadd(ae, re, p[m]);
            }
        }
#pragma unroll
        for (int o = LPP / 2; o > 0; o >>= 1) {
            T t2[LPP];
#pragma unroll
            for (int l = 0; l < LPP; l++) t2[l] = p[l] + p[l ^ o];
#pragma unroll
            for (int l = 0; l < LPP; l++) p[l] = t2[l];
        }
        if (lane == 0) w[q] = p[0];
    }
}

// Lanes per row of the fixed row-kernel shapes: about two and a half entries
// a lane (the first entries of each lane are loaded before the dependent-launch
// wait). Halving the lanes from about 1.5 entries a lane shortened the grids
// and the solve at 60x220x85: FP64 16.51 -> 16.25 ms, FP32 12.04 -> 11.57 ms.
static int pick_lpr(uint32_t n, uint32_t nnz) {
    double avg = n ? (double)nnz / n : 1;
    return avg <= 2.5 ? 1 : avg <= 5 ? 2 : avg <= 10 ? 4 : avg <= 20 ? 8 : avg <= 40 ? 16 : 32;
}

// Lanes per row of the SpMV launch_spmv picks (the staged tile kernel sums a
// row serially, as one lane does).
static uint32_t spmv_lpr(uint32_t n, uint32_t nnz, uint32_t tile_max) {
    if (tile_max && tile_max <= ST_MAX_NNZ && n >= 4 * ST_ROWS) return 1;
    return (uint32_t)pick_lpr(n, nnz);
}

#define LPR_SWITCH(lpr, KERNEL, ...)                                      \
    switch (lpr) {                                                        \
        case 1: launch_k(KERNEL<T, 1>, __VA_ARGS__); break;               \
        case 2: launch_k(KERNEL<T, 2>, __VA_ARGS__); break;               \
        case 4: launch_k(KERNEL<T, 4>, __VA_ARGS__); break;               \
        case 8: launch_k(KERNEL<T, 8>, __VA_ARGS__); break;               \
        case 16: launch_k(KERNEL<T, 16>, __VA_ARGS__); break;             \
        default: launch_k(KERNEL<T, 32>, __VA_ARGS__); break;             \
    }

// ---------------------------------------------------------------------------
// Launch-shape autotuner. With BuildCfg::autotune the plan builder times, for
// every row kernel of a level (phase 1, phase 2, correction), each candidate
// (lanes per row 1..16 up to twice the average row length, blocks of 128, 256
// or 512 threads, and at levels above MERGE_MAX_N rows the pipelined tile
// kernel, lpr = 0) on the level's own data, three launches per candidate after
// one warm-up, CUDA events on the build stream, and keeps the fastest. The
// choice is cached per (kernel, value type, rows, nonzeros), so an ensemble of
// equal-shaped members, or a rebuild, tunes once. Without it the shape is the
// fixed heuristic (pick_lpr lanes, 256 threads). The lane count changes the
// order in which a row's products are added, so tuned and untuned plans agree
// to rounding.
// ---------------------------------------------------------------------------
struct LaunchShape {
    int lpr = 1;
    unsigned block = 256;
};

namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, uint32_t, uint32_t>, LaunchShape> g_tune;
}  // namespace

template <class Launch>
static LaunchShape tune_shape(int kind, int tsize, uint32_t rows, uint32_t nnz, cudaStream_t s, Launch launch,
                              bool staged_candidate = false) {
    auto key = std::make_tuple(kind, tsize, rows, nnz);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) return it->second;
    }
    double avg = rows ? (double)nnz / rows : 1;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    LaunchShape best;
    float best_ms = 1e30f;
    for (int lpr : {0, 1, 2, 4, 8, 16}) {
        if (lpr == 0 && !staged_candidate) continue;
        if (lpr > 1 && lpr > 2 * std::ceil(avg)) break;
        for (unsigned block : {128u, 256u, 512u}) {
            if (lpr == 0 && block != ST_ROWS) continue;  // the pipelined tile kernel has one shape
            LaunchShape c{lpr, block};
            launch(c, s);
            CK(cudaEventRecord(e0, s));
            for (int r = 0; r < 3; r++) launch(c, s);
            CK(cudaEventRecord(e1, s));
            CK(cudaEventSynchronize(e1));
            CK(cudaGetLastError());
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best_ms) { best_ms = ms; best = c; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
    return best;
}

#define LPR_SWITCH_B(lpr, KERNEL, ...)                                    \
    switch (lpr) {                                                        \
        case 1: launch_k(KERNEL<T, 1>, __VA_ARGS__); break;               \
        case 2: launch_k(KERNEL<T, 2>, __VA_ARGS__); break;               \
        case 4: launch_k(KERNEL<T, 4>, __VA_ARGS__); break;               \
        case 8: launch_k(KERNEL<T, 8>, __VA_ARGS__); break;               \
        case 16: launch_k(KERNEL<T, 16>, __VA_ARGS__); break;             \
        default: launch_k(KERNEL<T, 32>, __VA_ARGS__); break;             \
    }

// ---------------------------------------------------------------------------
// Plan builder: replays the reference's recursion once on the host and records
// the launches.
// ---------------------------------------------------------------------------
static bool is_equal1(double a) { return std::fabs(a - 1.0) <= 2.220446049250313e-16; }

template <class T>
static const T* vals(const DCSR& m);
template <>
const double* vals<double>(const DCSR& m) { return m.a.p; }
template <>
const float* vals<float>(const DCSR& m) { return m.a32.p; }
template <class T>
static const T* dvals(const Level& l);
template <>
const double* dvals<double>(const Level& l) { return l.dval.p; }
template <>
const float* dvals<float>(const Level& l) { return l.dval32.p; }
template <class T>
static const T* cinv(const Level& l);
template <>
const double* cinv<double>(const Level& l) { return l.cinv.p; }
template <>
const float* cinv<float>(const Level& l) { return l.cinv32.p; }

template <class T>
struct Builder {
    Hierarchy& H;
    std::vector<LevelWork<T>>& W;
    Plan& plan;
    const SmallPlan<T>* small = nullptr;
    uint64_t bytes = 0;

    // ---- persistent recording -------------------------------------------
    // While ps is set, the step functions append descriptors for k_persist
    // instead of recording launches; persist_region() wraps a whole level
    // call (and everything below it) into one launch.
    std::vector<PStep<T>>* ps = nullptr;
    std::vector<DBuf<uint8_t>>* pdesc = nullptr;  // owner of the descriptor arrays
    PBar* pbar = nullptr;
    bool persist = false;                         // persistent regions allowed
    uint32_t persist_max_n = 0;                   // largest level that starts a region
    uint32_t persist_regions = 0, persist_steps = 0;

    static PStep<T> pstep(uint32_t op, uint32_t lpr, uint32_t n0, uint32_t n1, const uint32_t* ia,
                          const uint32_t* ja, const T* a, const T* dval, const void* v0, const void* v1,
                          const void* v2 = nullptr, double s0 = 0, double s1 = 0, uint32_t mode = 0) {
        PStep<T> st;
        memset(&st, 0, sizeof st);
        st.op = op;
        st.lpr = lpr < 1 ? 1 : lpr;  // the tile kernels (lpr 0) sum a row serially, as one lane does
        st.mode = mode;
        st.n0 = n0;
        st.n1 = n1;
        st.ia = ia;
        st.ja = ja;
        st.a = a;
        st.dval = dval;
        st.v[0] = const_cast<void*>(v0);
        st.v[1] = const_cast<void*>(v1);
        st.v[2] = const_cast<void*>(v2);
        st.s0 = s0;
        st.s1 = s1;
        return st;
    }

    // Whether the call of level l (and every level below it) can run as one
    // persistent launch: every step there has a descriptor form (the
    // shared-memory small-level kernel has none).
    bool persist_ok(uint32_t l) const {
        if (!persist || ps || autotune || !explicit_solves) return false;
        if (H.lv[l]->N > persist_max_n && !dynamic()) return false;
        if (small && small->valid() && !small->dense.p && small->first >= l) return false;
        return true;
    }

    bool dynamic() const {
        for (uint32_t l = 0; l < H.nlevels; l++)
            if (H.lv[l]->eps != 0) return true;
        return false;
    }

    template <class Body>
    void persist_region(Body body) {
        std::vector<PStep<T>> v;
        uint64_t b0 = bytes;
        ps = &v;
        body();
        ps = nullptr;
        if (v.empty()) return;
        uint64_t region = bytes - b0;
        bytes = b0;  // the region's bytes belong to its one launch
        pdesc->emplace_back();
        DBuf<uint8_t>& d = pdesc->back();
        d.alloc(v.size() * sizeof(PStep<T>));
        CK(cudaMemcpy(d.p, v.data(), v.size() * sizeof(PStep<T>), cudaMemcpyHostToDevice));
        const PStep<T>* dp = reinterpret_cast<const PStep<T>*>(d.p);
        uint32_t n = (uint32_t)v.size();
        PBar* bar = pbar;
        op([=](cudaStream_t s) { launch_persist<T>(dp, n, bar, s); }, "persistent");
        bytes += region;
        persist_regions++;
        persist_steps += n;
    }

    // FP32 hierarchy: the tabulated operator of the small levels in FP64
    const SmallPlan<double>* small64 = nullptr;

    // x = C f with an FP64 operator (vectors of type T, FP64 sums)
    void dense64(uint32_t n, const double* C, const T* f, T* x) {
        if (ps) {
            PStep<T> st = pstep(PS_DENSE, 32, n, 0, nullptr, nullptr, nullptr, nullptr, f, x);
            st.mode = 1;  // the operator is FP64
            st.v[2] = const_cast<double*>(C);
            ps->push_back(st);
        } else {
            op([=](cudaStream_t s) {
                launch_k(k_dense_gemv<T, double>, grid_for((size_t)n * 32, 256), 256, 0, s, n, C, f, x);
            }, "dense");
        }
        bytes += (uint64_t)n * n * 8 + 2ull * n * sizeof(T);
    }

    bool small_call(uint32_t l, const T* f, T* x) {
        if (small64 && small64->valid() && small64->dense.p && l == small64->first) {
            dense64(small64->N0, small64->dense.p, f, x);
            return true;
        }
        if (!small || !small->valid() || l != small->first) return false;
        const SmallPlan<T>* sp = small;
        if (sp->dense.p) {
            uint32_t n = sp->N0;
            const T* C = sp->dense.p;
            if (ps) ps->push_back(pstep(PS_DENSE, 32, n, 0, nullptr, nullptr, C, nullptr, f, x));
            else op([=](cudaStream_t s) {
                launch_k(k_dense_gemv<T>, grid_for((size_t)n * 32, 256), 256, 0, s, n, C, f, x);
            }, "dense");
            bytes += (uint64_t)n * n * sizeof(T) + 2ull * n * sizeof(T);
            return true;
        }
        if (ps) MLP_THROW(ERR_INTERNAL, "small-level kernel inside a persistent region");
        op([=](cudaStream_t s) { launch_small<T>(*sp, f, x, s); }, "small");
        bytes += sp->h.bytes_static + 2ull * sizeof(T) * sp->N0;
        return true;
    }

    // uh_cheb: the call of level l when it is the tabulated small-level
    // operator, with the Chebyshev update that follows it applied in the
    // GEMV's epilogue (one launch in place of two; same arithmetic, so the
    // result is bit-identical). False, and nothing recorded, where level l is
    // not a tabulated operator, inside a persistent region, or with MLP_MERGE=0.
    bool dense_epi(uint32_t l, const T* f, T* x, int mode, const T* u1, const T* u0, T ea, T eb) {
        if (ps || !merge_enabled() || persist_ok(l)) return false;
        const double* C64 = nullptr;
        const T* CT_ = nullptr;
        uint32_t n = 0;
        if (small64 && small64->valid() && small64->dense.p && l == small64->first) {
            C64 = small64->dense.p;
            n = small64->N0;
        } else if (small && small->valid() && l == small->first && small->dense.p) {
            CT_ = small->dense.p;
            n = small->N0;
        } else {
            return false;
        }
        LevelScope scope(cur_level, l);
        check_plan_size();
        unsigned g = grid_for((size_t)n * 32, 256);
        auto rec = [&](auto kern, const auto* Cm) {
            op([=](cudaStream_t s) { launch_k(kern, g, 256, 0, s, n, Cm, f, x, u1, u0, ea, eb); }, "dense_step");
        };
#define DENSE_EPI_CASE(E)                                                      \
    case E:                                                                    \
        if (C64) rec(k_dense_gemv_epi<T, double, E>, C64);                     \
        else rec(k_dense_gemv_epi<T, T, E>, CT_);                              \
        break;
        switch (mode) {
            DENSE_EPI_CASE(EPI_SCALE)
            DENSE_EPI_CASE(EPI_CHEB2)
            DENSE_EPI_CASE(EPI_CHEBK)
            default: MLP_THROW(ERR_INTERNAL, "dense step: unknown update");
        }
#undef DENSE_EPI_CASE
        bytes += (uint64_t)n * n * (C64 ? 8 : sizeof(T)) + (2ull + (uint64_t)mode) * n * sizeof(T);
        return true;
    }

    // Level whose call is being recorded (names the ops for profiling).
    uint32_t cur_level = 0;
    struct LevelScope {
        uint32_t& r;
        uint32_t saved;
        LevelScope(uint32_t& r_, uint32_t l) : r(r_), saved(r_) { r = l; }
        ~LevelScope() { r = saved; }
    };

    void op(std::function<void(cudaStream_t)> f, const char* name = "op") {
        plan.ops.push_back(std::move(f));
        plan.names.push_back(std::string(name) + " L" + std::to_string(cur_level));
        plan.bytes_start.push_back(bytes);
        plan.launches++;
    }

    void lsolve(const Level& L, const T* src, T* w) {
        const uint32_t* ia = L.Lf.ia.p;
        const uint32_t* ja = L.Lf.ja.p;
        const T* a = vals<T>(L.Lf);
        size_t nw = L.lw_off.empty() ? 0 : L.lw_off.size() - 1;
        size_t dt = tail_start(L.lw_off);
        for (size_t d = 0; d < dt; d++) {
            uint32_t r0 = L.lw_off[d], r1 = L.lw_off[d + 1];
            if (r1 <= r0) continue;
            op([=](cudaStream_t s) { launch_k(k_lwave<T>, grid_for(r1 - r0, 128), 128, 0, s, r0, r1, ia, ja, a, src, w); }, "lwave");
        }
        if (dt < nw) {
            const uint32_t* off = L.lw_off_d.p;
            uint32_t d0 = (uint32_t)dt, d1 = (uint32_t)nw;
            op([=](cudaStream_t s) {
                launch_k(k_lwave_tail<T>, 1, TAIL_THREADS, 0, s, d0, d1, off, ia, ja, a, src, w);
            }, "lwave_tail");
        }
    }
    void coarse_diag(const Level& L, const T* src, T* w, T* out) {
        uint32_t M = L.M, R = L.N - L.Md, N = L.N;
        if (N <= M) return;
        const uint32_t* ia = L.Lf.ia.p;
        const uint32_t* ja = L.Lf.ja.p;
        const T* a = vals<T>(L.Lf);
        const T* dv = dvals<T>(L);
        op([=](cudaStream_t s) {
            launch_k(k_lcoarse_diag<T>, grid_for(N - M, 128), 128, 0, s, M, R, N, ia, ja, a, src, w, dv, out);
        }, "lcoarse_diag");
    }
    void usolve(const Level& L, const T* w, T* out) {
        const uint32_t* ia = L.Uf.ia.p;
        const uint32_t* ja = L.Uf.ja.p;
        const T* a = vals<T>(L.Uf);
        const uint32_t* rows = L.uw_rows.p;
        size_t nw = L.uw_off.empty() ? 0 : L.uw_off.size() - 1;
        size_t dt = tail_start(L.uw_off);
        for (size_t d = 0; d < dt; d++) {
            uint32_t o0 = L.uw_off[d], o1 = L.uw_off[d + 1];
            if (o1 <= o0) continue;
            op([=](cudaStream_t s) {
                launch_k(k_uwave<T>, grid_for(o1 - o0, 128), 128, 0, s, o1 - o0, rows + o0, ia, ja, a, w, out);
            }, "uwave");
        }
        if (dt < nw) {
            const uint32_t* off = L.uw_off_d.p;
            uint32_t d0 = (uint32_t)dt, d1 = (uint32_t)nw;
            op([=](cudaStream_t s) {
                launch_k(k_uwave_tail<T>, 1, TAIL_THREADS, 0, s, d0, d1, off, rows, ia, ja, a, w, out);
            }, "uwave_tail");
        }
    }
    void direct(const Level& L, const T* f, T* x) {
        uint32_t n = L.N;
        if (!std::is_same<T, double>::value) {
            dense64(n, L.cinv.p, f, x);  // the coarsest solve stays FP64
            return;
        }
        const T* C = cinv<T>(L);
        if (ps) ps->push_back(pstep(PS_DENSE, 32, n, 0, nullptr, nullptr, C, nullptr, f, x));
        else op([=](cudaStream_t s) { launch_k(k_dense_gemv<T>, grid_for((size_t)n * 32, 256), 256, 0, s, n, C, f, x); }, "dense");
        bytes += (uint64_t)n * n * sizeof(T) + 2ull * n * sizeof(T);
    }
    // One application of the level's split operator on src: phase 1 (L solve
    // and diagonal block), the recursion on the coarse slice, phase 2 (U solve).
    bool autotune = false;
    cudaStream_t stream = nullptr;  // stream of the build (tuning launches)
    cudaStream_t tune_stream() const { return stream; }

    // The pipelined tile kernels are a tuner candidate for the sweep steps of
    // levels above MERGE_MAX_N rows (measured slower than the lane-split row
    // kernels at the 1.12 M-cell levels 0 and 1 with the fixed shapes: solve
    // 20.2 ms against 18.1 ms, the P1 and G rows being 1.6-2.6 entries long).
    static bool staged_ok(const Level& L, const DCSR& m, uint32_t rows) {
        return L.N > MERGE_MAX_N && rows >= 4 * ST_ROWS && m.tile_max && m.tile_max <= ST_MAX_NNZ;
    }

    void phase1(const Level& L, const T* src, T* w, T* out) {
        uint32_t R = L.N - L.Md, N = L.N;
        if (!R && N <= R) return;
        const uint32_t* ia = L.P1.ia.p;
        const uint32_t* ja = L.P1.ja.p;
        const T* a = vals<T>(L.P1);
        const T* dv = dvals<T>(L);
        bool st = staged_ok(L, L.P1, R);
        uint32_t cap = st ? pipe_cap<T>(L.P1.tile_max) : 0;
        size_t smem = st ? pipe_smem_bytes<T, false>(L.P1.tile_max) : 0;
        auto launch = [=](LaunchShape c, cudaStream_t s) {
            if (c.lpr == 0) {
                launch_k(k_phase1_staged<T>, pipe_grid(k_phase1_staged<T>, R, smem), ST_ROWS, smem, s, R, N, ia, ja,
                         a, dv, src, w, out, cap);
                return;
            }
            uint32_t nb1 = R ? grid_for((size_t)R * c.lpr, c.block) : 0;
            uint32_t nb2 = N > R ? grid_for(N - R, c.block) : 0;
            LPR_SWITCH_B(c.lpr, k_phase1, nb1 + nb2, c.block, 0, s, R, N, nb1, ia, ja, a, dv, src, w, out);
        };
        LaunchShape c{pick_lpr(R, L.P1.nnz), 256};
        if (autotune) c = tune_shape(1, sizeof(T), R, L.P1.nnz, tune_stream(), launch, st);
        if (ps) ps->push_back(pstep(PS_PHASE1, (uint32_t)c.lpr, R, N, ia, ja, a, dv, src, w, out));
        else op([=](cudaStream_t s) { launch(c, s); }, "phase1");
        bytes += (uint64_t)L.P1.nnz * (4 + sizeof(T)) + 4ull * (R + 1) + sizeof(T) * (2ull * N + L.Md) ;
    }
    void phase2(const Level& L, const T* w, T* out) {
        uint32_t M = L.M;
        if (!M) return;
        const uint32_t* ia = L.G.ia.p;
        const uint32_t* ja = L.G.ja.p;
        const T* a = vals<T>(L.G);
        bool st = staged_ok(L, L.G, M);
        uint32_t cap = st ? pipe_cap<T>(L.G.tile_max) : 0;
        size_t smem = st ? pipe_smem_bytes<T, false>(L.G.tile_max) : 0;
        auto launch = [=](LaunchShape c, cudaStream_t s) {
            if (c.lpr == 0) {
                launch_k(k_phase2_staged<T>, pipe_grid(k_phase2_staged<T>, M, smem), ST_ROWS, smem, s, M, ia, ja, a, w,
                         out, cap);
                return;
            }
            LPR_SWITCH_B(c.lpr, k_phase2, grid_for((size_t)M * c.lpr, c.block), c.block, 0, s, M, ia, ja, a, w, out);
        };
        LaunchShape c{pick_lpr(M, L.G.nnz), 256};
        if (autotune) c = tune_shape(2, sizeof(T), M, L.G.nnz, tune_stream(), launch, st);
        // n1: the level's rows (the extent of out, whose entries past M the
        // coarse columns read)
        if (ps) ps->push_back(pstep(PS_PHASE2, (uint32_t)c.lpr, M, L.N, ia, ja, a, nullptr, w, out));
        else op([=](cudaStream_t s) { launch(c, s); }, "phase2");
        bytes += (uint64_t)L.G.nnz * (4 + sizeof(T)) + 4ull * (M + 1) + sizeof(T) * (M + L.n + M);
    }
    // ---- folded coarse solve (launch plan) ------------------------------
    bool fold = true;  // MLP_FOLD=0 turns it off
    // Largest D = G_C C kept per level (bytes): the folded phase 2 reads it
    // once per call, so it must stay well below what a launch costs.
    static constexpr size_t FOLD_MAX_BYTES = 8u << 20;

    // Whether the call of level l + 1 is one dense FP64 product (the
    // tabulated small levels or the direct coarsest solve); C and n are its
    // operator and size.
    bool dense_next(uint32_t l, const double*& C, uint32_t& n) const {
        if (l + 1 >= H.nlevels) return false;
        const Level& Ln = *H.lv[l + 1];
        if (small64 && small64->valid() && small64->first <= l + 1) {
            if (small64->first != l + 1 || !small64->dense.p) return false;
            C = small64->dense.p;
            n = small64->N0;
            return true;
        }
        if (small && small->valid() && small->first <= l + 1) {
            if (small->first != l + 1 || !small->dense.p || !std::is_same<T, double>::value) return false;
            C = reinterpret_cast<const double*>(small->dense.p);
            n = small->N0;
            return true;
        }
        if (Ln.direct && Ln.cinv.p) {
            C = Ln.cinv.p;
            n = Ln.N;
            return true;
        }
        return false;
    }

    // Builds (once per level) the row split and D = G_C C for the folded
    // phase 2; false when the level does not qualify.
    bool fold_ready(uint32_t l, const double* C, uint32_t n) {
        LevelWork<T>& w = W[l];
        if (w.fold_state) return w.fold_state > 0;
        w.fold_state = -1;
        const Level& L = *H.lv[l];
        const uint32_t M = L.M;
        if (!M || n != L.n || L.G.nnz == 0) return false;
        std::vector<uint32_t> ia = L.G.ia.download(stream, (size_t)M + 1);
        std::vector<uint32_t> ja = L.G.ja.download(stream, L.G.nnz);
        std::vector<uint32_t> rows, plain;
        for (uint32_t q = 0; q < M; q++) {
            bool has = false;
            for (uint32_t j = ia[q]; j < ia[q + 1]; j++) {
                if (ja[j] >= M + n) return false;  // not a level of this shape
                has |= ja[j] >= M;
            }
            (has ? rows : plain).push_back(q);
        }
        const uint32_t nf = (uint32_t)rows.size();
        if ((size_t)nf * n * sizeof(double) > FOLD_MAX_BYTES) return false;
        rows.insert(rows.end(), plain.begin(), plain.end());
        w.fold_rows.alloc(M);
        w.fold_rows.upload(rows.data(), M, stream);
        w.fold_D.alloc((size_t)(nf ? nf : 1) * n);
        if (nf) {
            k_fold_build<T><<<nf, 256, 0, stream>>>(nf, w.fold_rows.p, M, n, L.G.ia.p, L.G.ja.p, vals<T>(L.G), C,
                                                     w.fold_D.p);
            CK_LAUNCH();
        }
        CK(cudaStreamSynchronize(stream));
        w.fold_nf = nf;
        w.fold_state = 1;
        return true;
    }

    void phase2_fold(uint32_t l, const double* C, uint32_t n, const T* w, T* out) {
        const Level& L = *H.lv[l];
        const LevelWork<T>& lw = W[l];
        const uint32_t M = L.M, nf = lw.fold_nf;
        const uint32_t* ia = L.G.ia.p;
        const uint32_t* ja = L.G.ja.p;
        const T* a = vals<T>(L.G);
        const double* D = lw.fold_D.p;
        const uint32_t* rows = lw.fold_rows.p;
        const uint32_t nb_c = (n + 7) / 8, nb_f = (nf + 7) / 8;
        const int lpr = pick_lpr(M, L.G.nnz);
        const uint32_t nb_p = grid_for((size_t)(M - nf) * (lpr < 1 ? 1 : lpr), 256);
        op([=](cudaStream_t s) {
            LPR_SWITCH_B(lpr < 1 ? 1 : lpr, k_phase2_fold, nb_c + nb_f + (M > nf ? nb_p : 0), 256, 0, s, M, n, ia,
                         ja, a, C, D, rows, nf, nb_c, nb_f, w, out);
        }, "phase2_fold");
        bytes += (uint64_t)L.G.nnz * (4 + sizeof(T)) + 4ull * (M + 1) + 4ull * M + 8ull * n * (n + nf) +
                 sizeof(T) * (M + n + M + n);
    }

    // The coarse call and phase 2 of a sweep of level l: one folded launch
    // where it applies, else the recursion into level l + 1 and phase 2.
    void coarse_phase2(uint32_t l, T* w, T* out) {
        Level& L = *H.lv[l];
        const bool next = l + 1 < H.nlevels && L.n;
        const double* C = nullptr;
        uint32_t n = 0;
        if (next && fold && !ps && explicit_solves && dense_next(l, C, n) && fold_ready(l, C, n)) {
            phase2_fold(l, C, n, w, out);
            return;
        }
        if (next) ms(l + 1, w + L.M, out + L.M);
        phase2(L, w, out);
    }

    void update(const Level& L, const T* u0, T* x, T* r, bool do_r) {
        uint32_t N = L.N;
        const uint32_t* ia = L.Af.ia.p;
        const uint32_t* ja = L.Af.ja.p;
        const T* a = vals<T>(L.Af);
        int dr = do_r ? 1 : 0;
        bool st = do_r && staged_ok(L, L.Af, N);
        uint32_t cap = st ? pipe_cap<T>(L.Af.tile_max) : 0;
        size_t smem = st ? pipe_smem_bytes<T, false>(L.Af.tile_max) : 0;
        auto launch = [=](LaunchShape c, cudaStream_t s) {
            if (c.lpr == 0) {
                launch_k(k_update_staged<T>, pipe_grid(k_update_staged<T>, N, smem), ST_ROWS, smem, s, N, ia, ja, a, u0,
                         x, r, cap);
                return;
            }
            LPR_SWITCH_B(c.lpr, k_update, grid_for((size_t)N * c.lpr, c.block), c.block, 0, s, N, ia, ja, a, u0, x, r,
                         dr);
        };
        LaunchShape c{do_r ? pick_lpr(N, L.Af.nnz) : 1, 256};
        // the tuning runs x += u0 on scratch: every buffer of the plan is
        // rewritten before it is read in an apply
        if (autotune && do_r) c = tune_shape(3, sizeof(T), N, L.Af.nnz, tune_stream(), launch, st);
        if (ps) ps->push_back(pstep(PS_UPDATE, (uint32_t)c.lpr, N, 0, ia, ja, a, nullptr, u0, x, r, 0, 0, dr));
        else op([=](cudaStream_t s) { launch(c, s); }, "update");
        bytes += sizeof(T) * 3ull * N + (do_r ? spmv_bytes(L.Af) : 0);
    }

    uint64_t sweep_bytes(const Level& L) const {
        // L (E and coarse rows), U, dval, src/w/out vectors
        uint64_t b = (uint64_t)L.Lf.nnz * (4 + sizeof(T)) + 4ull * (L.N - L.Md + 1);
        b += (uint64_t)L.Uf.nnz * (4 + sizeof(T)) + 4ull * (L.M + 1) + 4ull * L.M;
        b += (uint64_t)L.Md * sizeof(T);
        b += sizeof(T) * (uint64_t)(L.N + 2ull * (L.N - L.Md) + L.N);
        return b;
    }
    uint64_t spmv_bytes(const DCSR& A) const {
        return (uint64_t)A.nnz * (4 + sizeof(T)) + 4ull * (A.nrow + 1) + 3ull * sizeof(T) * A.nrow;
    }

    // MultiSplitPrec::solve(level, f, x) (multi_split_solve.cc:59-157) with the
    // triangular solves in explicit form: each sweep is phase 1, the recursion
    // and phase 2; the correction sweeps update the residual in place.
    // The recursion applies level l + 1 niter (or ncheb) times per call of
    // level l, so a deep hierarchy with little coarsening multiplies the plan
    // geometrically; past this many steps the build stops with an error.
    static constexpr size_t PLAN_MAX_STEPS = 1000000;
    void check_plan_size() const {
        if (plan.ops.size() + (ps ? ps->size() : 0) > PLAN_MAX_STEPS)
            MLP_THROW(ERR_LIMIT, "the preconditioner's application needs more than " + std::to_string(PLAN_MAX_STEPS) +
                                     " steps (the hierarchy coarsens too little for its inner iterations)");
    }

    void ms(uint32_t l, const T* f, T* x) {
        LevelScope scope(cur_level, l);
        check_plan_size();
        if (persist_ok(l)) {
            persist_region([&] { ms(l, f, x); });
            return;
        }
        if (small_call(l, f, x)) return;
        Level& L = *H.lv[l];
        if (L.direct) { direct(L, f, x); return; }
        if (!explicit_solves) {
            if (L.eps != 0)
                MLP_THROW(ERR_CONFIG, "inner_iter = dynamic needs the persistent apply, which needs the explicit "
                                      "triangular solves (MLP_EXPLICIT=0 is set)");
            ms_waves(l, f, x);
            return;
        }
        if (!ps && ms_merged(l, f, x)) return;
        if (L.eps != 0) { ms_dynamic(l, f, x); return; }
        LevelWork<T>& w = W[l];
        uint32_t N = L.N;
        phase1(L, f, w.w.p, x);
        coarse_phase2(l, w.w.p, x);
        if (L.niter < 2) return;
        {
            const uint32_t* ia = L.Af.ia.p;
            const uint32_t* ja = L.Af.ja.p;
            const T* a = vals<T>(L.Af);
            uint32_t nnz = L.Af.nnz, tm = L.Af.tile_max;
            T* r = w.r.p;
            if (ps) ps->push_back(pstep(PS_RESID, spmv_lpr(N, nnz, tm), N, 0, ia, ja, a, nullptr, x, r, f));
            else op([=](cudaStream_t s) { launch_spmv<T>(N, nnz, ia, ja, a, x, r, f, s, tm); }, "residual");
            bytes += spmv_bytes(L.Af);
        }
        for (uint32_t it = 2; it <= L.niter; it++) {
            phase1(L, w.r.p, w.w.p, w.u0.p);
            coarse_phase2(l, w.w.p, w.u0.p);
            update(L, w.u0.p, x, w.r.p, it < L.niter);
        }
    }

    bool explicit_solves = true;

    // MultiSplitPrec::solve(l, f, x) with dynamic inner iterations
    // (multi_split_solve.cc:95-157 with li.eps != 0): after the first sweep,
    // r = f - A x; stop when ||r|| / ||f|| < eps, else sweep on r and add the
    // correction. The loop runs inside the persistent launch (a test step that
    // every CTA evaluates alike, and a jump back), so the number of sweeps is
    // decided on the device.
    void ms_dynamic(uint32_t l, const T* f, T* x) {
        if (!ps) MLP_THROW(ERR_CONFIG, "inner_iter = dynamic needs the persistent apply (MLP_PERSIST=0 is set)");
        if (l >= PK_MAXLOOP) MLP_THROW(ERR_LIMIT, "dynamic inner iterations on more than 16 levels");
        Level& L = *H.lv[l];
        LevelWork<T>& w = W[l];
        uint32_t N = L.N, M = L.M;
        bool next = l + 1 < H.nlevels && L.n;
        const uint32_t* ia = L.Af.ia.p;
        const uint32_t* ja = L.Af.ja.p;
        const T* a = vals<T>(L.Af);
        T *r = w.r.p, *u0 = w.u0.p;
        auto push = [&](uint32_t op, uint32_t mode, const void* v0, double s0 = 0) {
            PStep<T> st = pstep(op, 1, N, 0, nullptr, nullptr, nullptr, nullptr, v0, nullptr);
            st.mode = mode;
            st.s0 = s0;
            ps->push_back(st);
            return ps->size() - 1;
        };
        push(PS_NORM2, l, f);
        push(PS_LOOPTEST, l | 256u, nullptr);  // init_norm = ||f||
        phase1(L, f, w.w.p, x);
        if (next) ms(l + 1, w.w.p + M, x + M);
        phase2(L, w.w.p, x);
        uint32_t top = (uint32_t)ps->size();
        ps->push_back(pstep(PS_RESID, spmv_lpr(N, L.Af.nnz, L.Af.tile_max), N, 0, ia, ja, a, nullptr, x, r, f));
        push(PS_NORM2, l, r);
        size_t test = push(PS_LOOPTEST, l, nullptr, L.eps);
        phase1(L, r, w.w.p, u0);
        if (next) ms(l + 1, w.w.p + M, u0 + M);
        phase2(L, w.w.p, u0);
        ps->push_back(pstep(PS_UPDATE, 1, N, 0, nullptr, nullptr, nullptr, nullptr, u0, x, nullptr, 0, 0, 0));
        size_t jmp = push(PS_JUMP, l, nullptr);
        (*ps)[jmp].target = top;
        (*ps)[test].target = (uint32_t)ps->size();
        // one extra sweep in the byte count (the number of sweeps is data dependent)
        bytes += spmv_bytes(L.Af) + 3ull * sizeof(T) * N;
    }

    // Merged sweep steps (k_merge_a) at levels of at most MERGE_MAX_N rows
    // without the autotuner (their arithmetic reproduces the fixed launch
    // shapes). On by default (MLP_MERGE=0 turns it off): with a warp per P1 row
    // recomputing its entries of r' in parallel it takes the 1.12 M-cell solve
    // from 18.56 to 18.13 ms on B200 (one thread per row doing it serially had
    // made it 29.7 ms).
    static constexpr uint32_t MERGE_MAX_N = 1u << 17;
    static bool merge_enabled() {
        const char* e = getenv("MLP_MERGE");
        return !(e && e[0] == '0');
    }
    // rows of the residual's matrix (Af, or As for uh_cheb's Chebyshev
    // residual) with the correction kernel's lane count, P1 rows a warp each
    void step_a(const Level& L, int mode, const T* f, T* x, const T* r_in, T* r_out, const T* u_in, T* u_out,
                T* w, const DCSR* Am = nullptr) {
        const DCSR& A_ = Am ? *Am : L.Af;
        uint32_t N = L.N, R = L.N - L.Md;
        bool staged = A_.tile_max && A_.tile_max <= ST_MAX_NNZ && N >= 4 * ST_ROWS;
        int lpu = mode == 0 ? (staged ? 1 : pick_lpr(N, A_.nnz)) : pick_lpr(N, A_.nnz);
        int lpp = pick_lpr(R, L.P1.nnz);
        uint32_t nbu = grid_for((size_t)N * lpu, 256), nbp = R ? grid_for((size_t)R * 32, 256) : 0;
        const uint32_t *aia = A_.ia.p, *aja = A_.ja.p, *pia = L.P1.ia.p, *pja = L.P1.ja.p;
        const T *aa = vals<T>(A_), *pa = vals<T>(L.P1), *dv = dvals<T>(L);
        auto go = [=](auto kern, cudaStream_t s) {
            launch_k(kern, nbu + nbp, 256, 0, s, N, R, nbu, aia, aja, aa, pia, pja, pa, dv, f, x, r_in, r_out, u_in,
                     u_out, w);
        };
#define MERGE_A_CASE(U, P)                                                                          \
    if (lpu == U && lpp == P) {                                                                     \
        if (mode == 0) op([=](cudaStream_t s) { go(k_merge_a<T, U, P, 0>, s); }, "merge_a");                   \
        else op([=](cudaStream_t s) { go(k_merge_a<T, U, P, 1>, s); }, "merge_a");                             \
        return;                                                                                     \
    }
        MERGE_A_CASE(1, 1) MERGE_A_CASE(1, 2) MERGE_A_CASE(1, 4) MERGE_A_CASE(1, 8)
        MERGE_A_CASE(2, 1) MERGE_A_CASE(2, 2) MERGE_A_CASE(2, 4) MERGE_A_CASE(2, 8)
        MERGE_A_CASE(4, 1) MERGE_A_CASE(4, 2) MERGE_A_CASE(4, 4) MERGE_A_CASE(4, 8)
        MERGE_A_CASE(8, 1) MERGE_A_CASE(8, 2) MERGE_A_CASE(8, 4) MERGE_A_CASE(8, 8)
#undef MERGE_A_CASE
        MLP_THROW(ERR_INTERNAL, "merged step: unsupported lane counts");
    }
    bool merge_a_ok(const Level& L) const {
        uint32_t N = L.N, R = L.N - L.Md;
        bool staged = L.Af.tile_max && L.Af.tile_max <= ST_MAX_NNZ && N >= 4 * ST_ROWS;
        int l0 = staged ? 1 : pick_lpr(N, L.Af.nnz), l1 = pick_lpr(N, L.Af.nnz), lp = pick_lpr(R, L.P1.nnz);
        return l0 <= 8 && l1 <= 8 && lp <= 8;
    }
    // uh_cheb: the residual F - As u of a Chebyshev step and phase 1 of the
    // level-l call that follows it as one step-A launch (MODE 0, As in place of
    // Af), where that call takes the plan's regular path (not persistent, not
    // a small or tabulated level) and the residual uses the tile kernel, whose
    // serial row sums step A repeats with one lane per row: the merged and the
    // separate launches give bit-identical results.
    bool ch_merge_ok(uint32_t l) const {
        if (!merge_enabled() || autotune || ps || !explicit_solves || l >= H.nlevels || persist_ok(l)) return false;
        if (small64 && small64->valid() && small64->dense.p && l == small64->first) return false;
        if (small && small->valid() && l == small->first) return false;
        const Level& L = *H.lv[l];
        if (L.direct || L.N > MERGE_MAX_N) return false;
        const DCSR& As = L.As;
        bool staged = As.tile_max && As.tile_max <= ST_MAX_NNZ && L.N >= 4 * ST_ROWS;
        return staged && pick_lpr(L.N - L.Md, L.P1.nnz) <= 8;
    }
    // set by a merged step A: the next ch() call's phase 1 is already done
    bool ch_phase1_done = false;
    // MultiSplitPrec::solve(l, f, x) with merged steps: sweep 1 = phase 1,
    // step B (or the recursion and phase 2); sweep 2 = step A (residual),
    // step B; sweeps 3.. = step A (correction of the previous sweep), step B;
    // then the last correction x += u0.
    bool ms_merged(uint32_t l, const T* f, T* x) {
        Level& L = *H.lv[l];
        if (!merge_enabled() || autotune || L.N > MERGE_MAX_N || L.niter < 2 || !merge_a_ok(L)) return false;
        LevelWork<T>& W_ = W[l];
        if (!W_.r2.p) W_.r2.alloc(L.N);
        if (!W_.u02.p) W_.u02.alloc(L.N);
        T* w = W_.w.p;
        auto stepB = [&](T* out) { coarse_phase2(l, w, out); };
        phase1(L, f, w, x);
        stepB(x);
        T *ra = W_.r.p, *rb = W_.r2.p, *ua = W_.u0.p, *ub = W_.u02.p;
        step_a(L, 0, f, x, nullptr, ra, nullptr, ua, w);
        bytes += spmv_bytes(L.Af) + (uint64_t)L.P1.nnz * (4 + sizeof(T)) + sizeof(T) * (uint64_t)L.N;
        stepB(ua);
        for (uint32_t it = 3; it <= L.niter; it++) {
            step_a(L, 1, f, x, ra, rb, ua, ub, w);
            bytes += spmv_bytes(L.Af) + (uint64_t)L.P1.nnz * (4 + sizeof(T)) + sizeof(T) * 4ull * L.N;
            stepB(ub);
            std::swap(ra, rb);
            std::swap(ua, ub);
        }
        update(L, ua, x, nullptr, false);
        return true;
    }

    // Wavefront form of ms (the L and U solves one wavefront at a time).
    void ms_waves(uint32_t l, const T* f, T* x) {
        LevelScope scope(cur_level, l);
        check_plan_size();
        Level& L = *H.lv[l];
        LevelWork<T>& w = W[l];
        uint32_t N = L.N, M = L.M;
        bool has_next = l + 1 < H.nlevels;
        // step 1, x0 = 0: r = f
        lsolve(L, f, w.w.p);
        coarse_diag(L, f, w.w.p, x);
        if (has_next && L.n) ms(l + 1, w.w.p + M, x + M);
        usolve(L, w.w.p, x);
        bytes += sweep_bytes(L);
        // steps 2..niter: x += B_l (f - A_l x)
        for (uint32_t it = 2; it <= L.niter; it++) {
            const uint32_t* ia = L.Af.ia.p;
            const uint32_t* ja = L.Af.ja.p;
            const T* a = vals<T>(L.Af);
            uint32_t nnz = L.Af.nnz;
            T* r = w.r.p;
            op([=](cudaStream_t s) { launch_spmv<T>(N, nnz, ia, ja, a, x, r, f, s); }, "residual");
            lsolve(L, r, w.w.p);
            coarse_diag(L, r, w.w.p, w.u0.p);
            if (has_next && L.n) ms(l + 1, w.w.p + M, w.u0.p + M);
            usolve(L, w.w.p, w.u0.p);
            T* u0 = w.u0.p;
            op([=](cudaStream_t s) { launch_k(k_axpy1<T>, grid_for(N, 256), 256, 0, s, N, x, (const T*)u0); }, "axpy");
            bytes += sweep_bytes(L) + spmv_bytes(L.Af) + 3ull * sizeof(T) * N;
        }
    }

    // Prec::solve(level, f, x) (cheb_solve.cc:13-123)
    void ch(uint32_t l, const T* f, T* x) {
        LevelScope scope(cur_level, l);
        check_plan_size();
        if (persist_ok(l)) {
            persist_region([&] { ch(l, f, x); });
            return;
        }
        if (small_call(l, f, x)) return;
        Level& L = *H.lv[l];
        LevelWork<T>& w = W[l];
        uint32_t M = L.M;
        if (explicit_solves) {
            if (ch_phase1_done) ch_phase1_done = false;
            else phase1(L, f, w.w.p, x);
        } else {
            lsolve(L, f, w.w.p);
            coarse_diag(L, f, w.w.p, x);
            bytes += sweep_bytes(L);
        }
        if (l + 1 < H.nlevels) {
            Level& Ln = *H.lv[l + 1];
            uint32_t n = Ln.N, nch = L.ncheb;
            const T* F = w.w.p + M;
            double lmin = Ln.lmin, lmax = Ln.lmax;
            double eta = (lmax + lmin) / (lmax - lmin);
            T *u0 = w.cu0.p, *u1 = w.cu1.p, *x2 = w.cx2.p, *tmp = w.ctmp.p;
            const uint32_t* sia = Ln.As.ia.p;
            const uint32_t* sja = Ln.As.ja.p;
            const T* sa = vals<T>(Ln.As);
            uint32_t snnz = Ln.As.nnz, stm = Ln.As.tile_max;
            double alpha = 2 / (lmax + lmin), beta;
            auto scale = [&](T* v, double al) {
                if (is_equal1(al)) return;
                T a = (T)al;
                if (ps) ps->push_back(pstep(PS_SCALE, 1, n, 0, nullptr, nullptr, nullptr, nullptr, v, nullptr, nullptr, (double)a));
                else op([=](cudaStream_t s) { launch_k(k_scale<T>, grid_for(n, 256), 256, 0, s, n, v, a); }, "scale");
            };
            auto resid = [&](const T* u, T* y) {
                if (ps) ps->push_back(pstep(PS_RESID, spmv_lpr(n, snnz, stm), n, 0, sia, sja, sa, nullptr, u, y, F));
                else op([=](cudaStream_t s) { launch_spmv<T>(n, snnz, sia, sja, sa, u, y, F, s, stm); }, "residual");
            };
            // y = F - As u, then out = solve(l + 1, y), followed by the step's
            // update (mode, u1, u0, ea, eb as k_dense_gemv_epi takes them).
            // True when the update went into the level call's epilogue.
            auto resid_solve = [&](T* u, T* y, T* out, int mode, const T* e1, const T* e0, T ea, T eb) {
                if (ch_merge_ok(l + 1)) {
                    LevelScope sc(cur_level, l + 1);  // named by the level whose data it reads
                    step_a(Ln, 0, F, u, nullptr, y, nullptr, out, W[l + 1].w.p, &Ln.As);
                    bytes += (uint64_t)Ln.P1.nnz * (4 + sizeof(T)) + sizeof(T) * (uint64_t)Ln.N;
                    ch_phase1_done = true;
                } else {
                    resid(u, y);
                    if (dense_epi(l + 1, y, out, mode, e1, e0, ea, eb)) return true;
                }
                ch(l + 1, y, out);
                return false;
            };
            // out = alpha solve(l + 1, F)
            auto first = [&](T* out) {
                if (!is_equal1(alpha) && dense_epi(l + 1, F, out, EPI_SCALE, nullptr, nullptr, (T)alpha, T(0)))
                    return;
                ch(l + 1, F, out);
                scale(out, alpha);
            };
            // The last step of the recurrence writes the coarse part of x
            // itself (no copy of the final iterate).
            T* xo = x + M;
            first(nch > 1 ? u1 : xo);
            if (nch == 2) x2 = xo;
            if (nch > 1) {
                alpha = 4 / (lmax - lmin) * cheb_poly(eta, 1) / cheb_poly(eta, 2);
                beta = cheb_poly(eta, 0) / cheb_poly(eta, 2);
                // x2 := -alpha * solve(A u1 - F) + (1+beta) u1 = alpha * solve(F - A u1) + (1+beta) u1
                double c = is_equal1(1 + beta) ? 1.0 : 1 + beta;
                T ma = (T)alpha, cc = (T)c;
                // tmp = F - A u1; the reference forms A u1 - F: negate via the scalars
                if (!resid_solve(u1, tmp, x2, EPI_CHEB2, u1, nullptr, ma, cc)) {
                    if (ps) ps->push_back(pstep(PS_CHEB2, 1, n, 0, nullptr, nullptr, nullptr, nullptr, x2, u1, nullptr, (double)ma, (double)cc));
                    else op([=](cudaStream_t s) { launch_k(k_cheb2<T>, grid_for(n, 256), 256, 0, s, n, x2, (const T*)u1, ma, cc); }, "cheb2");
                }
                bytes += spmv_bytes(Ln.As) + 3ull * sizeof(T) * n;
            }
            for (uint32_t i = 3; i <= nch; i++) {
                T* t = u0; u0 = u1; u1 = x2; x2 = t;  // cheb_solve.cc:87-89
                if (i == nch) x2 = xo;
                alpha = 4 / (lmax - lmin) * cheb_poly(eta, i - 1) / cheb_poly(eta, i);
                beta = cheb_poly(eta, i - 2) / cheb_poly(eta, i);
                // x2 = u1 - alpha*solve(A u1 - F) + beta*(u1-u0) = u1 + alpha*solve(F - A u1) + ...
                T ma = (T)(-alpha), bb = (T)beta;
                T* u0c = u0; T* u1c = u1; T* x2c = x2;
                if (!resid_solve(u1, tmp, x2, EPI_CHEBK, u1c, u0c, ma, bb)) {
                    if (ps) ps->push_back(pstep(PS_CHEBK, 1, n, 0, nullptr, nullptr, nullptr, nullptr, x2c, u1c, u0c, (double)ma, (double)bb));
                    else op([=](cudaStream_t s) { launch_k(k_chebk<T>, grid_for(n, 256), 256, 0, s, n, x2c, (const T*)u1c, (const T*)u0c, ma, bb); }, "chebk");
                }
                bytes += spmv_bytes(Ln.As) + 4ull * sizeof(T) * n;
            }
        }
        if (explicit_solves) phase2(L, w.w.p, x);
        else usolve(L, w.w.p, x);
    }
};

// Chebyshev sign convention: the reference solves with (A u1 - F); the plan
// solves with (F - A u1) (one fused residual kernel) and flips the sign of the
// coefficient that multiplies that solve. The preconditioner is linear, so the
// two forms are the same operator.

template <class T>
static void alloc_work(Hierarchy& H, std::vector<LevelWork<T>>& W) {
    W.clear();
    W.resize(H.nlevels);
    for (uint32_t l = 0; l < H.nlevels; l++) {
        Level& L = *H.lv[l];
        if (L.direct) continue;
        W[l].w.alloc(L.N - L.Md + 1);
        if (H.kind == PREC_MSPLIT) {
            if (L.niter >= 2 || L.eps != 0) { W[l].r.alloc(L.N); W[l].u0.alloc(L.N); }
        } else if (l + 1 < H.nlevels) {
            uint32_t n = H.lv[l + 1]->N;
            W[l].cu0.alloc(n); W[l].cu1.alloc(n); W[l].cx2.alloc(n); W[l].ctmp.alloc(n);
        }
    }
}

__global__ void k_d2f(size_t n, const double* __restrict__ a, float* __restrict__ b) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
static void make_f32(const DBuf<double>& src, DBuf<float>& dst, size_t n, cudaStream_t s) {
    dst.alloc(n ? n : 1);
    if (n) { k_d2f<<<grid_for(n, 256), 256, 0, s>>>(n, src.p, dst.p); CK_LAUNCH(); }
}
static void make_f32(DCSR& m, cudaStream_t s) { make_f32(m.a, m.a32, m.nnz, s); }

// ---- instantiated graphs of released handles ------------------------------
// Instantiating a graph of a few hundred nodes costs about a millisecond. A
// handle built for the same problem shape records the same launches with
// other pointers, so when a handle is released its instantiated graphs are
// kept (by a key naming the device, the size and every launch of the plan),
// and the next handle of that shape updates one in place
// (cudaGraphExecUpdate) instead of instantiating its own; an update the
// runtime refuses falls back to instantiation.
namespace {
struct ExecCache {
    std::mutex mu;
    std::multimap<std::string, cudaGraphExec_t> spare;
    uint64_t updates = 0, instantiations = 0;
};
ExecCache& exec_cache() {
    static ExecCache* c = new ExecCache();  // never destroyed: handles may be released during exit
    return *c;
}
constexpr size_t EXEC_SPARE_MAX = 16;
}  // namespace

std::string plan_key(const Prec& P, const std::string& what) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::string k = what + "|" + std::to_string(dev) + "|" + std::to_string(P.plan.launches);
    for (const std::string& nm : P.plan.names) k += "|" + nm;
    return k;
}

void exec_release(const std::string& key, cudaGraphExec_t ex) {
    if (!ex) return;
    ExecCache& c = exec_cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        if (!key.empty() && c.spare.size() < EXEC_SPARE_MAX && c.spare.count(key) < 2) {
            c.spare.emplace(key, ex);
            return;
        }
    }
    cudaGraphExecDestroy(ex);
}

// An executable graph for g (which is destroyed): a released one of the same
// key updated to g, else a new instantiation.
cudaGraphExec_t exec_for(const std::string& key, cudaGraph_t g) {
    ExecCache& c = exec_cache();
    cudaGraphExec_t ex = nullptr;
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.spare.find(key);
        if (it != c.spare.end()) {
            ex = it->second;
            c.spare.erase(it);
        }
    }
    if (ex) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(ex, g, &info) == cudaSuccess) {
            cudaGraphDestroy(g);
            std::lock_guard<std::mutex> lk(c.mu);
            c.updates++;
            return ex;
        }
        cudaGetLastError();
        cudaGraphExecDestroy(ex);
    }
    cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) MLP_THROW(ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    std::lock_guard<std::mutex> lk(c.mu);
    c.instantiations++;
    return ex;
}

void exec_cache_counts(uint64_t& updates, uint64_t& instantiations) {
    ExecCache& c = exec_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    updates = c.updates;
    instantiations = c.instantiations;
}

Prec::~Prec() {
    exec_release(graph_key, graph);
}
Prec::Prec() = default;

// Shared-memory budget of the small-level kernel; MLP_SMALL_BUDGET (bytes, 0 =
// off) overrides it, which the tests use to exercise both apply paths.
static uint32_t small_budget() {
    const char* e = getenv("MLP_SMALL_BUDGET");
    if (e && *e) return (uint32_t)strtoul(e, nullptr, 10);
    return 200 * 1024;
}

// Persistent regions (k_persist): MLP_PERSIST=1 turns them on, =0 off; unset,
// they are used where they are needed, for dynamic inner iterations (on B200
// the launch-per-step plan with programmatic dependent launch measured faster
// for fixed iterations at 60x220x85: solve 18.0 ms against 29.8 ms). A region
// starts at the first level of at most MLP_PERSIST_MAX_N rows (default
// 524,288, so that a 1.12 M-cell level 0 keeps its bandwidth-bound separate
// kernels).
static bool persist_enabled(const Hierarchy& H) {
    const char* e = getenv("MLP_PERSIST");
    if (e && e[0] == '1') return true;
    if (e && e[0] == '0') return false;
    for (uint32_t l = 0; l < H.nlevels; l++)
        if (H.lv[l]->eps != 0) return true;
    return false;
}
static uint32_t persist_max_n() {
    const char* e = getenv("MLP_PERSIST_MAX_N");
    if (e && *e) return (uint32_t)strtoul(e, nullptr, 10);
    return 1u << 19;
}
// The folded coarse solve (k_phase2_fold) is on unless MLP_FOLD=0.
static bool fold_enabled() {
    const char* e = getenv("MLP_FOLD");
    return !(e && e[0] == '0');
}

template <class T>
static void builder_persist(Builder<T>& B, Prec& P) {
    B.fold = fold_enabled();
    B.persist = persist_enabled(B.H);
    B.persist_max_n = persist_max_n();
    B.pdesc = &P.pdesc;
    B.pbar = P.pbar.p;
}

void check_persist(Prec& P, cudaStream_t s) {
    if (!P.persist_regions) return;
    unsigned h[4];  // count, exitc, err, pad
    CK(cudaMemcpyAsync(h, P.pbar.p, sizeof h, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    int err = (int)h[2];
    if (err) {
        CK(cudaMemsetAsync(P.pbar.p, 0, sizeof h, s));
        CK(cudaStreamSynchronize(s));
        if (err == 2)
            MLP_THROW(ERR_MAXIT, "a dynamic level iteration reached its cap (" + std::to_string(PK_LOOP_CAP) +
                                     " sweeps per level call, " + std::to_string(PK_TOTAL_CAP) + " per apply)");
        MLP_THROW(ERR_INTERNAL, "a grid barrier of the persistent apply gave up waiting");
    }
}

std::unique_ptr<Prec> make_prec(const DCSR& A, const BuildCfg& cfg, bool fp32, cudaStream_t s) {
    ArenaScope arena;
    auto P = std::unique_ptr<Prec>(new Prec());
    P->stream = s;
    P->fp32 = fp32;
    P->H = build_hierarchy(A, cfg, s);
    trace("hierarchy");
    Hierarchy& H = *P->H;
    uint32_t N0 = H.lv[0]->N;
    P->fin_buf.alloc(N0);
    P->fout_buf.alloc(N0);
    P->fin = P->fin_buf.p;
    P->fout = P->fout_buf.p;
    P->pbar.alloc(1);
    P->pbar.zero(s);
    const char* ex = getenv("MLP_EXPLICIT");
    bool explicit_solves = !(ex && ex[0] == '0');
    // With dynamic inner iterations a level call is no fixed linear operator,
    // so the sub-hierarchy is neither tabulated nor packed for the one-CTA
    // kernel; the whole apply runs persistent.
    bool dyn = false;
    for (uint32_t l = 0; l < H.nlevels; l++) dyn = dyn || H.lv[l]->eps != 0;
    if (!fp32) {
        alloc_work<double>(H, P->w64);
        P->sp64.reset(new SmallPlan<double>());
        if (small_budget() && !dyn) build_small<double>(H, *P->sp64, small_budget(), s);
        Builder<double> B{H, P->w64, P->plan, P->sp64.get()};
        B.explicit_solves = explicit_solves;
        B.stream = s;
        B.autotune = cfg.autotune != 0;
        builder_persist(B, *P);
        if (H.kind == PREC_MSPLIT) B.ms(0, P->fin, P->fout);
        else B.ch(0, P->fin, P->fout);
        P->bytes_per_apply = B.bytes;
        P->plan.bytes_total = B.bytes;
        P->persist_regions = B.persist_regions;
        P->persist_steps = B.persist_steps;
    } else {
        for (uint32_t l = 0; l < H.nlevels; l++) {
            Level& L = *H.lv[l];
            make_f32(L.Lf, s); make_f32(L.Uf, s); make_f32(L.Af, s);
            if (!L.direct) { make_f32(L.P1, s); make_f32(L.G, s); }
            if (H.kind == PREC_CHEB && l > 0) make_f32(L.As, s);
            make_f32(L.dval, L.dval32, L.Md, s);
            // the FP32 copy of a dense inverse serves only the one-CTA small-level
            // kernel (sub-hierarchies too large to tabulate); the plan applies the
            // FP64 inverse
            if (L.direct) make_f32(L.cinv, L.cinv32, (size_t)L.N * L.N, s);
        }
        alloc_work<float>(H, P->w32);
        // The small levels: their tabulated operator stands in for the
        // coarsest solve and is kept in FP64 (tabulated from the FP64 levels);
        // when they are not tabulated, the one-CTA kernel runs them in FP32.
        P->sp64.reset(new SmallPlan<double>());
        P->sp32.reset(new SmallPlan<float>());
        if (small_budget() && !dyn) {
            build_small<double>(H, *P->sp64, small_budget(), s);
            if (!P->sp64->dense.p) {
                P->sp64.reset(new SmallPlan<double>());
                build_small<float>(H, *P->sp32, small_budget(), s);
            }
        }
        P->f32.alloc(N0);
        P->z32.alloc(N0);
        Builder<float> B{H, P->w32, P->plan, P->sp32.get()};
        B.small64 = P->sp64.get();
        B.explicit_solves = explicit_solves;
        B.stream = s;
        B.autotune = cfg.autotune != 0;
        builder_persist(B, *P);
        const double* fin = P->fin;
        float* f32 = P->f32.p;
        float* z32 = P->z32.p;
        double* fout = P->fout;
        auto top = [&] {
            if (B.ps) B.ps->push_back(Builder<float>::pstep(PS_TOF32, 1, N0, 0, nullptr, nullptr, nullptr, nullptr, fin, f32));
            else B.op([=](cudaStream_t st) { launch_k(k_to_f32, grid_for(N0, 256), 256, 0, st, N0, fin, f32); }, "to_f32");
            if (H.kind == PREC_MSPLIT) B.ms(0, f32, z32);
            else B.ch(0, f32, z32);
            if (B.ps) B.ps->push_back(Builder<float>::pstep(PS_TOF64, 1, N0, 0, nullptr, nullptr, nullptr, nullptr, z32, fout));
            else B.op([=](cudaStream_t st) { launch_k(k_to_f64, grid_for(N0, 256), 256, 0, st, N0, (const float*)z32, fout); }, "to_f64");
        };
        if (B.persist_ok(0)) B.persist_region(top);
        else top();
        P->bytes_per_apply = B.bytes + 12ull * N0 * 2;
        P->plan.bytes_total = B.bytes;
        P->persist_regions = B.persist_regions;
        P->persist_steps = B.persist_steps;
    }
    CK(cudaStreamSynchronize(s));
    trace("plan + small levels");
    // capture the apply once as a graph
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    P->plan.run(s);
    cudaError_t le = cudaGetLastError();
    CK(cudaStreamEndCapture(s, &g));
    if (le != cudaSuccess) { cudaGraphDestroy(g); MLP_THROW(ERR_CUDA, cudaGetErrorString(le)); }
    P->graph_key = plan_key(*P, "apply");
    P->graph = exec_for(P->graph_key, g);
    trace("graph");
    trace_flush();
    return P;
}

std::vector<OpProfile> profile_apply(Prec& P, uint32_t reps, cudaStream_t s) {
    const Plan& pl = P.plan;
    size_t n = pl.ops.size();
    std::vector<OpProfile> out(n);
    if (!n) return out;
    std::vector<cudaEvent_t> ev(n + 1);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    if (reps < 1) reps = 1;
    for (uint32_t r = 0; r < reps; r++) {
        for (size_t k = 0; k < n; k++) {
            CK(cudaEventRecord(ev[k], s));
            pl.ops[k](s);
        }
        CK(cudaEventRecord(ev[n], s));
        CK(cudaEventSynchronize(ev[n]));
        CK(cudaGetLastError());
        for (size_t k = 0; k < n; k++) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            out[k].ms += ms / reps;
        }
    }
    count_launches((uint64_t)reps * pl.launches);
    for (auto& e : ev) cudaEventDestroy(e);
    for (size_t k = 0; k < n; k++) {
        out[k].name = pl.names[k];
        uint64_t end = k + 1 < n ? pl.bytes_start[k + 1] : pl.bytes_total;
        out[k].bytes = end - pl.bytes_start[k];
    }
    check_persist(P, s);
    return out;
}

// Turns the stamping on with room for `cap` stamps (the stream is idle).
static void tl_begin(DBuf<unsigned long long>& buf, size_t cap, cudaStream_t s) {
    buf.alloc(cap);
    unsigned long long* bp = buf.p;
    unsigned c = (unsigned)cap, zero = 0;
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpyToSymbol(c_tl_cap, &c, sizeof c));
    CK(cudaMemcpyToSymbol(g_tl_n, &zero, sizeof zero));
    CK(cudaMemcpyToSymbol(c_tl_buf, &bp, sizeof bp));
}
// Waits for the stream, turns the stamping off and returns the stamps (at most
// the capacity) and, in `got`, how many kernels stamped.
static std::vector<unsigned long long> tl_end(const DBuf<unsigned long long>& buf, unsigned& got, cudaStream_t s) {
    cudaError_t se = cudaStreamSynchronize(s);
    unsigned long long* nul = nullptr;
    CK(cudaMemcpyToSymbol(c_tl_buf, &nul, sizeof nul));
    CK(cudaMemcpyFromSymbol(&got, g_tl_n, sizeof got));
    CK(se);
    std::vector<unsigned long long> t(std::min<size_t>(got, buf.n));
    if (!t.empty()) CK(cudaMemcpy(t.data(), buf.p, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    return t;
}

std::vector<double> timeline_apply(Prec& P, uint32_t reps, cudaStream_t s) {
    const Plan& pl = P.plan;
    size_t n = pl.ops.size();
    std::vector<double> us(n, 0.0);
    if (!n) return us;
    if (!P.graph) MLP_THROW(ERR_ARG, "the apply has no graph");
    if (reps < 2) reps = 2;
    size_t total = (size_t)reps * n;
    DBuf<unsigned long long> buf;
    tl_begin(buf, total + 64, s);
    cudaError_t le = cudaSuccess;
    for (uint32_t r = 0; r < reps && le == cudaSuccess; r++) le = cudaGraphLaunch(P.graph, s);
    unsigned got = 0;
    std::vector<unsigned long long> t = tl_end(buf, got, s);
    CK(le);
    count_launches((uint64_t)reps * pl.launches);
    if (got != total)
        MLP_THROW(ERR_INTERNAL, "timeline: " + std::to_string(got) + " stamps for " + std::to_string(total) +
                                    " launches (a launch of the plan does not come from the solve kernels)");
    // op k of replay r lasts until the next stamp; the last op of the last
    // replay has none and takes the mean of the earlier replays
    for (size_t k = 0; k < n; k++) {
        double sum = 0;
        uint32_t cnt = 0;
        for (uint32_t r = 0; r < reps; r++) {
            size_t i = (size_t)r * n + k;
            if (i + 1 < total) {
                sum += (double)(t[i + 1] - t[i]) / 1e3;
                cnt++;
            }
        }
        us[k] = cnt ? sum / cnt : 0.0;
    }
    check_persist(P, s);
    return us;
}

void prec_apply_frame(Prec& P, cudaStream_t s) {
    if (P.graph) CK(cudaGraphLaunch(P.graph, s));
    else P.plan.run(s);
    count_launches(P.plan.launches);
}

// ---------------------------------------------------------------------------
// PCG
// ---------------------------------------------------------------------------
static constexpr int RB = 256;  // reduction block
// Iteration cap when the caller passes maxit = 0: the iterations must always
// end, also when eps is below what rounding lets the residual reach.
static constexpr uint32_t PCG_DEFAULT_MAXIT = 10000;

struct PcgDev {
    double rz0, rz1, app, alpha, beta, rr, rz_prev;
    unsigned ticket[4];
    int status;  // 1: <Ap,p> <= 0, 2: not finite
    uint32_t it, maxit;
    double init, eps;
};
static int take_x0_mode();

// All four pointers 16-byte aligned (pairs of doubles move in one access).
__device__ __forceinline__ bool aligned16(const void* a, const void* b, const void* c, const void* e) {
    return (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c | (uintptr_t)e) & 15u) == 0;
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0;
    if (w == 0) {
        t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;  // valid in thread 0
}

// Deterministic grid reduction: block partials in fixed slots, the last block
// to arrive sums them in slot order.
__device__ __forceinline__ bool finish_reduce(double part, double* partials, unsigned* ticket, double* total) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = part;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double v = 0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) v += ((volatile double*)partials)[b];
    v = block_sum(v);
    if (threadIdx.x == 0) { *total = v; *ticket = 0; }
    return true;
}

// Ap = A p, app = (Ap, p), alpha = rz0 / app.
template <int LPR>
__global__ void __launch_bounds__(RB) k_pcg_spmv_dot(uint32_t n, const uint32_t* __restrict__ ia,
                                                     const uint32_t* __restrict__ ja, const double* __restrict__ a,
                                                     const double* __restrict__ p, double* __restrict__ Ap,
                                                     double* partials, PcgDev* d) {
    pdl_wait();
    pdl_trigger();
    double part = 0;
    const uint32_t groups = gridDim.x * (RB / LPR);
    int lane = threadIdx.x % LPR;
    for (uint32_t row = blockIdx.x * (RB / LPR) + threadIdx.x / LPR;; row += groups) {
        bool active = row < n;
        if (__all_sync(0xffffffffu, !active)) break;
        double s = 0;
        if (active) {
            uint32_t e = ia[row + 1];
            for (uint32_t j = ia[row] + lane; j < e; j += LPR) s += a[j] * p[ja[j]];
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lane == 0) {
            Ap[row] = s;
            part += s * p[row];
        }
    }
    part = block_sum(part);
    double tot;
    if (finish_reduce(part, partials, &d->ticket[0], &tot) && threadIdx.x == 0) {
        d->app = tot;
        if (!(tot > 0)) d->status |= (tot != tot) ? 2 : 1;
        d->alpha = d->rz0 / tot;
    }
}

// Staged form of k_pcg_spmv_dot (same tiles as k_spmv_staged).
template <bool SA>
__global__ void __launch_bounds__(ST_ROWS) k_pcg_spmv_dot_staged(uint32_t n, const uint32_t* __restrict__ ia,
                                                                 const uint32_t* __restrict__ ja,
                                                                 const double* __restrict__ a,
                                                                 const double* __restrict__ p,
                                                                 double* __restrict__ Ap, double* partials,
                                                                 PcgDev* d, uint32_t cap) {
    double part = 0;
    spmv_pipe<double, SA>(n, ia, ja, a, p, cap, [&](uint32_t row, double acc) {
        Ap[row] = acc;
        part += acc * p[row];
    });
    part = block_sum(part);
    double tot;
    if (finish_reduce(part, partials, &d->ticket[0], &tot) && threadIdx.x == 0) {
        d->app = tot;
        if (!(tot > 0)) d->status |= (tot != tot) ? 2 : 1;
        d->alpha = d->rz0 / tot;
    }
}

static void pipe_prepare_all(uint32_t tile_max) {
    size_t u64 = pipe_smem_bytes<double, false>(tile_max), u32 = pipe_smem_bytes<float, false>(tile_max);
    pipe_grid(k_spmv_staged<double, 0, false>, 0, u64);
    pipe_grid(k_spmv_staged<double, 1, false>, 0, u64);
    pipe_grid(k_spmv_staged<float, 0, false>, 0, u32);
    pipe_grid(k_spmv_staged<float, 1, false>, 0, u32);
    pipe_grid(k_pcg_spmv_dot_staged<false>, 0, u64);
    pipe_grid(k_phase1_staged<double>, 0, u64);
    pipe_grid(k_phase2_staged<double>, 0, u64);
    pipe_grid(k_update_staged<double>, 0, u64);
    pipe_grid(k_phase1_staged<float>, 0, u32);
    pipe_grid(k_phase2_staged<float>, 0, u32);
    pipe_grid(k_update_staged<float>, 0, u32);
}

// Launch of k_pcg_spmv_dot_staged; its grid never exceeds staged_grid(n), the
// size the reduction scratch of every caller is made for.
static void launch_pcg_spmv_dot_staged(uint32_t n, const DCSR& Af, const double* p, double* Ap, double* partials,
                                       PcgDev* d, cudaStream_t s, bool pdl = false) {
    uint32_t cap = pipe_cap<double>(Af.tile_max);
    size_t smem = pipe_smem_bytes<double, false>(Af.tile_max);
    unsigned g = std::min(pipe_grid(k_pcg_spmv_dot_staged<false>, n, smem), staged_grid(n));
    if (pdl)
        launch_k(k_pcg_spmv_dot_staged<false>, g, ST_ROWS, smem, s, n, (const uint32_t*)Af.ia.p,
                 (const uint32_t*)Af.ja.p, (const double*)Af.a.p, p, Ap, partials, d, cap);
    else
        k_pcg_spmv_dot_staged<false><<<g, ST_ROWS, smem, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p, Ap, partials, d, cap);
}

// x += alpha p; r -= alpha Ap; rr = (r, r). In the device loop (cond != 0)
// the block that completes the reduction also ends the iteration: it counts
// it and keeps the loop going while ||r||/||r0|| > eps (pcg.cc:42), no error
// was flagged and the cap is not hit.
__global__ void __launch_bounds__(RB) k_pcg_update(uint32_t n, double* __restrict__ x, double* __restrict__ r,
                                                   const double* __restrict__ p, const double* __restrict__ Ap,
                                                   double* partials, PcgDev* d, cudaGraphConditionalHandle h,
                                                   int cond) {
    pdl_wait();
    pdl_trigger();
    double alpha = d->alpha;
    double part = 0;
    const uint32_t t0 = blockIdx.x * RB + threadIdx.x, stride = gridDim.x * RB;
    if (aligned16(x, r, p, Ap)) {
        // pairs of elements in 16-byte accesses, two pairs in flight per thread
        double2* x2 = reinterpret_cast<double2*>(x);
        double2* r2 = reinterpret_cast<double2*>(r);
        const double2* p2 = reinterpret_cast<const double2*>(p);
        const double2* a2 = reinterpret_cast<const double2*>(Ap);
        const uint32_t n2 = n >> 1;
        for (uint32_t i = t0; i < n2; i += 2 * stride) {
            const uint32_t j = i + stride;
            const bool two = j < n2;
            double2 xv = x2[i], pv = p2[i], rv = r2[i], av = a2[i];
            double2 xw = two ? x2[j] : xv, pw = two ? p2[j] : pv, rw = two ? r2[j] : rv, aw = two ? a2[j] : av;
            xv.x += alpha * pv.x; xv.y += alpha * pv.y;
            rv.x = rv.x - alpha * av.x; rv.y = rv.y - alpha * av.y;
            x2[i] = xv; r2[i] = rv;
            part += rv.x * rv.x; part += rv.y * rv.y;
            if (two) {
                xw.x += alpha * pw.x; xw.y += alpha * pw.y;
                rw.x = rw.x - alpha * aw.x; rw.y = rw.y - alpha * aw.y;
                x2[j] = xw; r2[j] = rw;
                part += rw.x * rw.x; part += rw.y * rw.y;
            }
        }
        if ((n & 1) && t0 == 0) {
            const uint32_t i = n - 1;
            x[i] += alpha * p[i];
            double ri = r[i] - alpha * Ap[i];
            r[i] = ri;
            part += ri * ri;
        }
    } else {
        for (uint32_t i = t0; i < n; i += stride) {
            x[i] += alpha * p[i];
            double ri = r[i] - alpha * Ap[i];
            r[i] = ri;
            part += ri * ri;
        }
    }
    part = block_sum(part);
    double tot;
    if (finish_reduce(part, partials, &d->ticket[1], &tot) && threadIdx.x == 0) {
        d->rr = tot;
        if (tot != tot || tot > 1e308) d->status |= 2;
        if (cond) {
            d->it++;
            bool go = sqrt(tot) / d->init > d->eps && d->status == 0 && (d->maxit == 0 || d->it < d->maxit);
            cudaGraphSetConditional(h, go ? 1u : 0u);
        }
    }
}

// rz1 = (r, z); beta = rz1/rz0 (or Polak-Ribiere (r - r_prev, z)/rz0); rz0 =
// rz1. The block that completes the last reduction computes beta: with the
// flexible form that is the last block of the second reduction, which every
// block enters after the first, whose total is then already in d->rz1.
__global__ void __launch_bounds__(RB) k_pcg_dot_rz(uint32_t n, const double* __restrict__ r,
                                                   const double* __restrict__ z, const double* __restrict__ rprev,
                                                   double* partials, PcgDev* d, int flexible) {
    pdl_wait();
    pdl_trigger();
    double part = 0, part2 = 0;
    const uint32_t t0 = blockIdx.x * RB + threadIdx.x, stride = gridDim.x * RB;
    if (aligned16(r, z, rprev, r)) {
        const double2* r2 = reinterpret_cast<const double2*>(r);
        const double2* z2 = reinterpret_cast<const double2*>(z);
        const double2* q2 = reinterpret_cast<const double2*>(rprev);
        const uint32_t n2 = n >> 1;
        for (uint32_t i = t0; i < n2; i += stride) {
            double2 rv = r2[i], zv = z2[i];
            part += rv.x * zv.x; part += rv.y * zv.y;
            if (flexible) {
                double2 qv = q2[i];
                part2 += qv.x * zv.x; part2 += qv.y * zv.y;
            }
        }
        if ((n & 1) && t0 == 0) {
            part += r[n - 1] * z[n - 1];
            if (flexible) part2 += rprev[n - 1] * z[n - 1];
        }
    } else {
        for (uint32_t i = t0; i < n; i += stride) {
            part += r[i] * z[i];
            if (flexible) part2 += rprev[i] * z[i];
        }
    }
    part = block_sum(part);
    double tot;
    bool last = finish_reduce(part, partials, &d->ticket[2], &tot);
    if (last && threadIdx.x == 0) {
        d->rz1 = tot;
        if (!flexible) {
            double beta = tot / d->rz0;
            d->beta = beta;
            d->rz0 = tot;
            if (beta != beta) d->status |= 2;
        }
    }
    if (flexible) {
        __syncthreads();
        part2 = block_sum(part2);
        double tot2;
        bool last2 = finish_reduce(part2, partials + gridDim.x, &d->ticket[3], &tot2);
        if (last2 && threadIdx.x == 0) {
            double rz1 = *(volatile double*)&d->rz1;
            double beta = (rz1 - tot2) / d->rz0;
            d->rz_prev = tot2;
            d->beta = beta;
            d->rz0 = rz1;
            if (beta != beta) d->status |= 2;
        }
    }
}

// p = beta p + z (dscal then daxpy, pcg.cc:71-72), PCG_P_PAIRS pairs of
// elements a thread (pair t and t + T, T the grid's threads, so that the grid
// fits one wave). p and z were written before the preceding launch (the (r, z)
// reduction), so they are loaded before the wait; only beta comes from it.
constexpr uint32_t PCG_P_PAIRS = 2;
__global__ void k_pcg_p(uint32_t n, double* __restrict__ p, const double* __restrict__ z, const PcgDev* d) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
    const bool vec = aligned16(p, z, p, z);
    double pv[PCG_P_PAIRS][2], zv[PCG_P_PAIRS][2];
#pragma unroll
    for (uint32_t k = 0; k < PCG_P_PAIRS; k++) {
        const uint32_t i = t + k * T, e = 2 * i;
        pv[k][0] = pv[k][1] = zv[k][0] = zv[k][1] = 0;
        if (vec && e + 1 < n) {
            double2 a = reinterpret_cast<const double2*>(p)[i], b = reinterpret_cast<const double2*>(z)[i];
            pv[k][0] = a.x; pv[k][1] = a.y; zv[k][0] = b.x; zv[k][1] = b.y;
        } else {
            if (e < n) { pv[k][0] = p[e]; zv[k][0] = z[e]; }
            if (e + 1 < n) { pv[k][1] = p[e + 1]; zv[k][1] = z[e + 1]; }
        }
    }
    pdl_wait();
    pdl_trigger();
    const double beta = d->beta;
#pragma unroll
    for (uint32_t k = 0; k < PCG_P_PAIRS; k++) {
        const uint32_t i = t + k * T, e = 2 * i;
        if (vec && e + 1 < n) {
            reinterpret_cast<double2*>(p)[i] = make_double2(beta * pv[k][0] + zv[k][0], beta * pv[k][1] + zv[k][1]);
        } else {
            if (e < n) p[e] = beta * pv[k][0] + zv[k][0];
            if (e + 1 < n) p[e + 1] = beta * pv[k][1] + zv[k][1];
        }
    }
}

__global__ void k_dot_simple(uint32_t n, const double* __restrict__ a, const double* __restrict__ b,
                             double* partials, unsigned* ticket, double* out) {
    double part = 0;
    for (uint32_t i = blockIdx.x * RB + threadIdx.x; i < n; i += gridDim.x * RB) part += a[i] * b[i];
    part = block_sum(part);
    double tot;
    if (finish_reduce(part, partials, ticket, &tot) && threadIdx.x == 0) *out = tot;
}

const double* x0_device(uint32_t n, cudaStream_t s) {
    static std::mutex mu;
    static std::map<std::pair<int, uint32_t>, double*> cache;
    std::lock_guard<std::mutex> lk(mu);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    auto key = std::make_pair(dev, n);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    // generate_x0 (solvers.cc:9-21): srandom(3); 20*(random()-0.5*RAND_MAX)/RAND_MAX + 100.
    // random_r keeps glibc's generator without touching the process-wide state.
    std::vector<double> h(n);
    struct random_data rd;
    memset(&rd, 0, sizeof rd);
    char state[128];
    initstate_r(3, state, sizeof state, &rd);
    srandom_r(3, &rd);
    for (uint32_t i = 0; i < n; i++) {
        int32_t v;
        random_r(&rd, &v);
        h[i] = 20. * (v - 0.5 * RAND_MAX) / RAND_MAX + 100;
    }
    double* d = nullptr;
    CK(cudaMalloc(&d, (size_t)(n ? n : 1) * 8));
    CK(cudaMemcpyAsync(d, h.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    cache[key] = d;
    return d;
}

// ---------------------------------------------------------------------------
// Device-resident PCG: one solve is one graph launch.
// ---------------------------------------------------------------------------
__global__ void k_copy_d(uint32_t n, const double* __restrict__ a, double* __restrict__ b) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

__global__ void k_fill_d(uint32_t n, double* __restrict__ a, double v) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// Clears the PCG scalars (reduction tickets, status) at the start of a solve.
__global__ void k_zero_dev(PcgDev* d) {
    uint32_t* w = reinterpret_cast<uint32_t*>(d);
    for (uint32_t i = threadIdx.x; i < sizeof(PcgDev) / 4; i += blockDim.x) w[i] = 0;
}

// Start of the solve on the device: init = ||r0||, eps raised so that the
// absolute stop is >= 1e-14 (check_and_replace_eps, solvers.cc:49-58); no
// iteration when ||r0||/||r0|| > eps fails (the reference then throws "No need
// to iterate").
__global__ void k_pcg_start(PcgDev* d, const PcgParams* prm, cudaGraphConditionalHandle h) {
    double init = sqrt(d->rr);
    double eps = prm->eps;
    if (init * eps < 1e-14) eps = 1e-14 / init;
    d->init = init;
    d->eps = eps;
    d->it = 0;
    d->maxit = prm->maxit;
    d->status = isfinite(init) ? 0 : 2;
    if (!(init / init > eps) || d->status) cudaGraphSetConditional(h, 0u);
}

PcgWork::~PcgWork() {
    for (int k = 0; k < 6; k++) exec_release(full_key[k], full[k]);
}

static void pcg_work_alloc(Prec& P, uint32_t n) {
    PcgWork& W = P.pcg;
    if (W.n == n) return;
    for (int k = 0; k < 6; k++) {
        exec_release(W.full_key[k], W.full[k]);
        W.full[k] = nullptr;
    }
    W.n = n;
    W.xf.alloc(n); W.bf.alloc(n); W.p.alloc(n); W.Ap.alloc(n); W.rprev.alloc(n);
    W.bnat.alloc(n); W.xnat.alloc(n);
    unsigned G = (unsigned)std::max(1, std::min<int>((int)grid_for(n, RB), num_sms() * 4));
    W.partials.alloc(2 * (size_t)std::max<unsigned>(G, staged_grid(n)));
    W.d.alloc(1);
    W.prm.alloc(1);
}

// Records one PCG iteration (pcg.cc:46-75) on stream s.
static void record_iteration(Prec& P, const DCSR& Af, uint32_t n, bool flexible, cudaGraphConditionalHandle h,
                             cudaStream_t s) {
    PcgWork& W = P.pcg;
    PcgDev* d = W.d.p;
    double* r = P.fin_buf.p;
    double* z = P.fout_buf.p;
    unsigned G = (unsigned)std::max(1, std::min<int>((int)grid_for(n, RB), num_sms() * 4));
    bool staged = Af.tile_max && Af.tile_max <= ST_MAX_NNZ && n >= 4 * ST_ROWS;
    double avg = (double)Af.nnz / n;
    int lpr = avg <= 3 ? 2 : avg <= 6 ? 4 : avg <= 12 ? 8 : avg <= 24 ? 16 : 32;
    // programmatic dependent launches like the apply's kernels: each waits
    // for its predecessor before touching memory
    if (staged) {
        launch_pcg_spmv_dot_staged(n, Af, W.p.p, W.Ap.p, W.partials.p, d, s, true);
    } else switch (lpr) {
        case 2: launch_k(k_pcg_spmv_dot<2>, G, RB, 0, s, n, Af.ia.p, Af.ja.p, Af.a.p, W.p.p, W.Ap.p, W.partials.p, d); break;
        case 4: launch_k(k_pcg_spmv_dot<4>, G, RB, 0, s, n, Af.ia.p, Af.ja.p, Af.a.p, W.p.p, W.Ap.p, W.partials.p, d); break;
        case 8: launch_k(k_pcg_spmv_dot<8>, G, RB, 0, s, n, Af.ia.p, Af.ja.p, Af.a.p, W.p.p, W.Ap.p, W.partials.p, d); break;
        case 16: launch_k(k_pcg_spmv_dot<16>, G, RB, 0, s, n, Af.ia.p, Af.ja.p, Af.a.p, W.p.p, W.Ap.p, W.partials.p, d); break;
        default: launch_k(k_pcg_spmv_dot<32>, G, RB, 0, s, n, Af.ia.p, Af.ja.p, Af.a.p, W.p.p, W.Ap.p, W.partials.p, d); break;
    }
    // the (r, z) reduction with up to eight CTAs per SM (the partials hold
    // 2 * max(G, staged_grid(n)) slots: 6.4 against 7.3 us at 60x220x85; the
    // update measured slower so, 13.6 against 12.0 us)
    const unsigned Gv = std::max(G, std::min(staged_grid(n), (unsigned)grid_for((n + 1) / 2, RB)));
    launch_k(k_pcg_update, G, RB, 0, s, n, W.xf.p, r, (const double*)W.p.p, (const double*)W.Ap.p, W.partials.p, d,
             h, 1);
    P.plan.run(s);
    launch_k(k_pcg_dot_rz, Gv, RB, 0, s, n, (const double*)r, (const double*)z, (const double*)W.rprev.p,
             W.partials.p, d, flexible ? 1 : 0);
    launch_k(k_pcg_p, grid_for(((n + 1) / 2 + PCG_P_PAIRS - 1) / PCG_P_PAIRS, 256), 256, 0, s, n, W.p.p,
             (const double*)z, (const PcgDev*)d);
    if (flexible) k_copy_d<<<grid_for(n, 256), 256, 0, s>>>(n, r, W.rprev.p);
}

// Launches per loop iteration and per start (launch accounting).
static uint64_t iteration_launches(const Prec& P, bool flexible) {
    return 2 + P.plan.launches + 2 + (flexible ? 1 : 0);
}
static uint64_t start_launches(const Prec& P, bool flexible) {
    return 6 + P.plan.launches + 2 + (flexible ? 1 : 0) + 1;
}

// Appends one complete PCG solve (pcg.cc:8-102) of handle P to graph g:
// gather b and x0 into the frame, r = b - A x, the first apply, a conditional
// WHILE node whose body is one iteration, and the scatter of x back. The
// vectors live in P's PcgWork (b comes in through bnat, x leaves through xnat).
static std::vector<cudaGraphNode_t> append_pcg(cudaGraph_t g, Prec& P, uint32_t n, bool flexible, int x0m,
                                               cudaStream_t s, const std::vector<cudaGraphNode_t>& after = {}) {
    const Level& L0 = *P.H->lv[0];
    const DCSR& Af = L0.Af;
    PcgWork& W = P.pcg;
    PcgDev* d = W.d.p;
    double* r = P.fin_buf.p;
    double* z = P.fout_buf.p;
    unsigned G = (unsigned)std::max(1, std::min<int>((int)grid_for(n, RB), num_sms() * 4));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    const double* x0 = x0m == X0_GENERATE ? x0_device(n, s) : nullptr;
    // start
    CK(cudaStreamBeginCaptureToGraph(s, g, after.empty() ? nullptr : after.data(), nullptr, after.size(),
                                     cudaStreamCaptureModeThreadLocal));
    k_zero_dev<<<1, 32, 0, s>>>(d);
    CK(cudaPeekAtLastError());
    gather(n, L0.phi.p, W.bnat.p, W.bf.p, s);
    if (x0m == X0_ZERO) k_fill_d<<<grid_for(n, 256), 256, 0, s>>>(n, W.xf.p, 0.0);
    else gather(n, L0.phi.p, x0m == X0_GIVEN ? W.xnat.p : x0, W.xf.p, s);
    launch_spmv<double>(n, Af.nnz, Af.ia.p, Af.ja.p, Af.a.p, W.xf.p, r, W.bf.p, s, Af.tile_max);
    CK(cudaPeekAtLastError());
    k_dot_simple<<<G, RB, 0, s>>>(n, r, r, W.partials.p, &d->ticket[1], &d->rr);
    CK(cudaPeekAtLastError());
    P.plan.run(s);
    CK(cudaPeekAtLastError());
    k_copy_d<<<grid_for(n, 256), 256, 0, s>>>(n, z, W.p.p);
    k_dot_simple<<<G, RB, 0, s>>>(n, r, z, W.partials.p, &d->ticket[2], &d->rz0);
    if (flexible) k_copy_d<<<grid_for(n, 256), 256, 0, s>>>(n, r, W.rprev.p);
    k_pcg_start<<<1, 1, 0, s>>>(d, W.prm.p, h);
    cudaError_t le = cudaGetLastError();
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &ndeps));
    std::vector<cudaGraphNode_t> dv(deps, deps + ndeps);
    cudaGraph_t got;
    CK(cudaStreamEndCapture(s, &got));
    if (le != cudaSuccess) MLP_THROW(ERR_CUDA, cudaGetErrorString(le));
    // loop
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, g, dv.data(), dv.size(), &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    record_iteration(P, Af, n, flexible, h, s);
    le = cudaGetLastError();
    CK(cudaStreamEndCapture(s, &got));
    if (le != cudaSuccess) MLP_THROW(ERR_CUDA, cudaGetErrorString(le));
    // tail
    CK(cudaStreamBeginCaptureToGraph(s, g, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
    scatter(n, L0.phi.p, W.xf.p, W.xnat.p, s);
    le = cudaGetLastError();
    CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &ndeps));
    std::vector<cudaGraphNode_t> tail(deps, deps + ndeps);
    CK(cudaStreamEndCapture(s, &got));
    if (le != cudaSuccess) MLP_THROW(ERR_CUDA, cudaGetErrorString(le));
    return tail;
}

static cudaGraphExec_t instantiate(cudaGraph_t g) {
    cudaGraphExec_t ex = nullptr;
    cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) MLP_THROW(ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    return ex;
}

static cudaGraphExec_t full_graph(Prec& P, uint32_t n, bool flexible, int x0m, cudaStream_t s) {
    const int k = (flexible ? 1 : 0) * 3 + x0m;
    cudaGraphExec_t& ex = P.pcg.full[k];
    if (ex) return ex;
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    try {
        append_pcg(g, P, n, flexible, x0m, s);
    } catch (...) {
        cudaGraphDestroy(g);
        throw;
    }
    P.pcg.full_key[k] = plan_key(P, "pcg|" + std::to_string(n) + "|" + std::to_string(k));
    ex = exec_for(P.pcg.full_key[k], g);
    return ex;
}

static void read_stats(const PcgDev& h, PcgStats& st, int& rc, std::string& msg) {
    st.niter = h.it;
    st.init_norm = h.init;
    st.final_norm = std::sqrt(h.rr);
    st.final_rel = st.final_norm / h.init;
    st.napply = h.it + 1;
    rc = OK;
    if (h.status & 1) { rc = ERR_CURVATURE; msg = "<Ap, p> = " + std::to_string(h.app); }
    else if (h.status & 2) { rc = ERR_NOT_FINITE; msg = "non-finite value in PCG scalars"; }
    else if (h.maxit && h.it >= h.maxit && st.final_rel > h.eps) { rc = ERR_MAXIT; msg = "iteration cap reached"; }
    else if (h.it == 0) { rc = ERR_NO_ITER; msg = "No need to iterate"; }
}

static thread_local int t_x0_mode = X0_GENERATE;
void set_pcg_x0_mode(int mode) { t_x0_mode = mode; }
static int take_x0_mode() {
    int m = t_x0_mode;
    t_x0_mode = X0_GENERATE;
    return m;
}

// PCGSolver (pcg.cc:8-102) as one graph launch: start, loop and scatter run on
// the device; the host waits once, for the statistics.
int pcg_solve(const DCSR& A, const double* b, Prec& P, double* x, double eps, uint32_t maxit, bool flexible,
              PcgStats& st, cudaStream_t s) {
    if (maxit == 0) maxit = PCG_DEFAULT_MAXIT;
    const Level& L0 = *P.H->lv[0];
    uint32_t n = A.nrow;
    if (n != L0.N) MLP_THROW(ERR_ARG, "matrix and preconditioner sizes differ");
    if (!n) MLP_THROW(ERR_ARG, "empty system");
    int x0m = take_x0_mode();
    pcg_work_alloc(P, n);
    PcgWork& W = P.pcg;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    cudaGraphExec_t ex = full_graph(P, n, flexible, x0m, s);
    CK(cudaEventRecord(e0, s));
    PcgParams prm{eps, maxit};
    CK(cudaMemcpyAsync(W.prm.p, &prm, sizeof prm, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(W.bnat.p, b, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    if (x0m == X0_GIVEN) CK(cudaMemcpyAsync(W.xnat.p, x, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaGraphLaunch(ex, s));
    CK(cudaMemcpyAsync(x, W.xnat.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaEventRecord(e1, s));
    PcgDev h;
    CK(cudaMemcpyAsync(&h, W.d.p, sizeof(PcgDev), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    count_launches(start_launches(P, flexible) + (uint64_t)h.it * iteration_launches(P, flexible));
    check_persist(P, s);
    int rc;
    std::string msg;
    read_stats(h, st, rc, msg);
    st.t_total_ms = ms;
    if (rc != OK) set_last_error(msg);
    return rc;
}

std::vector<std::pair<std::string, double>> timeline_pcg(const DCSR& A, const double* b, Prec& P, double* x,
                                                         double eps, bool flexible, cudaStream_t s) {
    const size_t nops = P.plan.ops.size(), per = nops + 4;
    // the solve's kernels that pass a dependent-launch wait: the start's
    // residual SpMV and first application, then per iteration the SpMV with
    // (Ap, p), the update, the application, the (r, z) reduction and p
    DBuf<unsigned long long> buf;
    tl_begin(buf, 1 + nops + (size_t)PCG_DEFAULT_MAXIT * per + 64, s);
    PcgStats st;
    int rc = OK;
    try {
        rc = pcg_solve(A, b, P, x, eps, 0, flexible, st, s);
    } catch (...) {
        unsigned g = 0;
        tl_end(buf, g, s);
        throw;
    }
    unsigned got = 0;
    std::vector<unsigned long long> t = tl_end(buf, got, s);
    if (rc != OK && rc != ERR_NO_ITER) MLP_THROW(rc, "timeline: the solve failed");
    const size_t want = 1 + nops + (size_t)st.niter * per;
    if (got != want || st.niter < 2)
        MLP_THROW(ERR_INTERNAL, "timeline: " + std::to_string(got) + " stamps where the solve's launches give " +
                                    std::to_string(want));
    // an iteration from the end, with the next one's first stamp after it
    const size_t k = st.niter >= 3 ? st.niter - 3 : 0, base = 1 + nops + k * per;
    std::vector<std::pair<std::string, double>> out;
    std::vector<std::string> names{"pcg spmv_dot", "pcg update"};
    names.insert(names.end(), P.plan.names.begin(), P.plan.names.end());
    names.push_back("pcg dot_rz");
    names.push_back("pcg p");
    for (size_t i = 0; i < per; i++) out.emplace_back(names[i], (double)(t[base + i + 1] - t[base + i]) / 1e3);
    return out;
}

// ---------------------------------------------------------------------------
// SymPrec (modules/prec/sym/sym_prec.cc:8-40): the preconditioner is a PCG
// solve (eps 1e-14) with the uh_cheb preconditioner of the matrix's symmetric
// part. Its construction symmetrizes the matrix on the device; the solver
// around it is the PCG loop below, driven from the host one iteration at a
// time because each application is itself a whole device-resident solve.
// ---------------------------------------------------------------------------
// a_ij = max(a_ij, a_ji) off the diagonal, a missing a_ji counting as 0
// (sym_prec.cc:28-33; the reference's in-place row loop gives the same
// values, each pair's maximum, whatever the row order)
__global__ void k_symmetrize(uint32_t n, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                             const double* __restrict__ a, double* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t rs = ia[i], re = ia[i + 1];
    out[rs] = a[rs];
    for (uint32_t j_ = rs + 1; j_ < re; j_++) {
        uint32_t j = ja[j_];
        uint32_t lo = ia[j] + 1, hi = ia[j + 1];
        while (lo < hi) {
            uint32_t mid = (lo + hi) / 2;
            if (ja[mid] < i) lo = mid + 1;
            else hi = mid;
        }
        double d = (lo < ia[j + 1] && ja[lo] == i) ? a[lo] : 0.0;
        double v = a[j_];
        out[j_] = d > v ? d : v;
    }
}

void symmetrize(const DCSR& A, DCSR& S, cudaStream_t s) {
    S.alloc(A.nrow, A.ncol, A.nnz);
    CK(cudaMemcpyAsync(S.ia.p, A.ia.p, ((size_t)A.nrow + 1) * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(S.ja.p, A.ja.p, (size_t)A.nnz * 4, cudaMemcpyDeviceToDevice, s));
    if (A.nrow) {
        k_symmetrize<<<grid_for(A.nrow, 256), 256, 0, s>>>(A.nrow, A.ia.p, A.ja.p, A.a.p, S.a.p);
        CK_LAUNCH();
    }
    csr_tile_stats(S, s);
}

// PCGSolver (pcg.cc:8-102) on natural-order device vectors with the
// preconditioner given as a call z = B r (each call may run whole device
// solves); one host round trip per iteration, the same kernels as the
// device-resident loop.
int pcg_solve_cb(const DCSR& A, const double* b, const std::function<void(const double*, double*)>& apply,
                 double* x, double eps, uint32_t maxit, bool flexible, PcgStats& st, cudaStream_t s) {
    if (maxit == 0) maxit = PCG_DEFAULT_MAXIT;
    uint32_t n = A.nrow;
    if (!n) MLP_THROW(ERR_ARG, "empty system");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
    DBuf<double> r(n), z(n), p(n), Ap(n), rprev(flexible ? n : 1);
    unsigned G = (unsigned)std::max(1, std::min<int>((int)grid_for(n, RB), num_sms() * 4));
    bool staged = A.tile_max && A.tile_max <= ST_MAX_NNZ && n >= 4 * ST_ROWS;
    DBuf<double> partials(2 * (size_t)std::max<unsigned>(G, staged_grid(n)));
    DBuf<PcgDev> dd(1);
    dd.zero(s);
    PcgDev* d = dd.p;
    CK(cudaMemcpyAsync(x, x0_device(n, s), (size_t)n * 8, cudaMemcpyDeviceToDevice, s));  // generate_x0
    launch_spmv<double>(n, A.nnz, A.ia.p, A.ja.p, A.a.p, x, r.p, b, s, A.tile_max);
    CK_LAUNCH();
    k_dot_simple<<<G, RB, 0, s>>>(n, r.p, r.p, partials.p, &d->ticket[1], &d->rr);
    CK_LAUNCH();
    auto fetch = [&]() -> PcgDev {
        PcgDev h;
        CK(cudaMemcpyAsync(&h, d, sizeof(PcgDev), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return h;
    };
    apply(r.p, z.p);
    CK(cudaMemcpyAsync(p.p, z.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    k_dot_simple<<<G, RB, 0, s>>>(n, r.p, z.p, partials.p, &d->ticket[2], &d->rz0);
    CK_LAUNCH();
    if (flexible) CK(cudaMemcpyAsync(rprev.p, r.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    PcgDev h = fetch();
    double norm = std::sqrt(h.rr), init = norm;
    st.init_norm = init;
    int rc = OK;
    std::string msg;
    if (!std::isfinite(init)) { rc = ERR_NOT_FINITE; msg = "non-finite initial residual norm"; }
    if (init * eps < 1e-14) eps = 1e-14 / init;  // check_and_replace_eps, solvers.cc:49-58
    uint32_t it = 0, napply = 1;
    int lpr = pick_lpr(n, A.nnz);
    if (lpr < 2) lpr = 2;
    while (rc == OK && norm / init > eps) {
        if (maxit && it >= maxit) { rc = ERR_MAXIT; msg = "iteration cap reached"; break; }
        if (staged) {
            launch_pcg_spmv_dot_staged(n, A, p.p, Ap.p, partials.p, d, s);
        } else switch (lpr) {
            case 2: k_pcg_spmv_dot<2><<<G, RB, 0, s>>>(n, A.ia.p, A.ja.p, A.a.p, p.p, Ap.p, partials.p, d); break;
            case 4: k_pcg_spmv_dot<4><<<G, RB, 0, s>>>(n, A.ia.p, A.ja.p, A.a.p, p.p, Ap.p, partials.p, d); break;
            case 8: k_pcg_spmv_dot<8><<<G, RB, 0, s>>>(n, A.ia.p, A.ja.p, A.a.p, p.p, Ap.p, partials.p, d); break;
            case 16: k_pcg_spmv_dot<16><<<G, RB, 0, s>>>(n, A.ia.p, A.ja.p, A.a.p, p.p, Ap.p, partials.p, d); break;
            default: k_pcg_spmv_dot<32><<<G, RB, 0, s>>>(n, A.ia.p, A.ja.p, A.a.p, p.p, Ap.p, partials.p, d); break;
        }
        k_pcg_update<<<G, RB, 0, s>>>(n, x, r.p, p.p, Ap.p, partials.p, d, 0, 0);
        count_launches(2);
        CK_LAUNCH();
        h = fetch();
        if (h.status & 1) { rc = ERR_CURVATURE; msg = "<Ap, p> = " + std::to_string(h.app); break; }
        if (h.status & 2) { rc = ERR_NOT_FINITE; msg = "non-finite value in PCG scalars"; break; }
        norm = std::sqrt(h.rr);
        it++;
        if (!(norm / init > eps)) break;
        apply(r.p, z.p);
        napply++;
        k_pcg_dot_rz<<<G, RB, 0, s>>>(n, r.p, z.p, rprev.p, partials.p, d, flexible ? 1 : 0);
        k_pcg_p<<<grid_for(((n + 1) / 2 + PCG_P_PAIRS - 1) / PCG_P_PAIRS, 256), 256, 0, s>>>(n, p.p, z.p, d);
        count_launches(2);
        if (flexible) CK(cudaMemcpyAsync(rprev.p, r.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
        CK_LAUNCH();
    }
    CK(cudaEventRecord(e1, s));
    CK(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st.niter = it;
    st.final_norm = norm;
    st.final_rel = norm / init;
    st.t_total_ms = ms;
    st.napply = napply;
    if (rc == OK && it == 0) { rc = ERR_NO_ITER; msg = "No need to iterate"; }
    if (rc != OK) set_last_error(msg);
    return rc;
}

// ---------------------------------------------------------------------------
// ChebSolver (modules/solvers/cheb.cc:9-100): the Chebyshev iteration as the
// outer solver, for a preconditioner with known spectral bounds (uh_cheb's
// level-0 lmin / lmax). Like PCG it runs as one graph: start, the first step,
// a conditional WHILE loop of steps, scatter. The recurrence coefficients
// cheb(eta, k) (misc.cc:232-242) are tabulated on the host for every step the
// cap allows, so they are the reference's values; the two state vectors of
// the three-term recurrence alternate roles by the parity of the step count
// (the new iterate overwrites the oldest one element by element), and the
// current iterate is also written to one fixed vector for the residual.
// Element arithmetic keeps the reference's separate multiplies and adds.
// ---------------------------------------------------------------------------
struct ChebDev {
    double rr, init, eps;
    unsigned ticket;
    int status;      // 2: not finite
    uint32_t niter;  // the reference's niter (1 at the start, 2 after step 1)
    uint32_t maxit;
};

__global__ void k_cheb_start(ChebDev* d, double eps, uint32_t maxit) {
    double init = sqrt(d->rr);
    if (init * eps < 1e-14) eps = 1e-14 / init;  // check_and_replace_eps, solvers.cc:49-58
    d->init = init;
    d->eps = eps;
    d->niter = 1;
    d->maxit = maxit;
    d->status = isfinite(init) ? 0 : 2;
}

// Step 1 (cheb.cc:38-46): u1 = x; x = alpha B r + u1 (dscal, then daxpy).
__global__ void k_cheb_first(uint32_t n, double alpha, int scale, const double* __restrict__ z,
                             double* __restrict__ u1, double* __restrict__ x, double* __restrict__ xcur) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x0 = x[i];
    u1[i] = x0;
    double v = scale ? __dmul_rn(alpha, z[i]) : z[i];
    v = __dadd_rn(v, x0);
    x[i] = v;
    xcur[i] = v;
}

// Steps 2+ (cheb.cc:58-72): x = u1 + alpha B r + beta (u1 - u0) with
// alpha = 4/(lmax-lmin) T(k-1)/T(k), beta = T(k-2)/T(k), k = niter. The new
// iterate goes to U[k % 2] (the oldest state vector, read first), the newest
// is U[(k + 1) % 2].
__global__ void k_cheb_step(uint32_t n, const ChebDev* __restrict__ d, const double* __restrict__ T, double c4,
                            const double* __restrict__ z, double* U0, double* U1, double* __restrict__ xcur) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k = d->niter;
    double alpha = c4 * T[k - 1] / T[k];
    double beta = T[k - 2] / T[k];
    double* unew = (k & 1) ? U1 : U0;
    const double* u1 = (k & 1) ? U0 : U1;
    double a1 = u1[i], a0 = unew[i];
    double v = __dadd_rn(__dadd_rn(a1, __dmul_rn(alpha, z[i])), __dmul_rn(beta, __dsub_rn(a1, a0)));
    unew[i] = v;
    xcur[i] = v;
}

// norm of the new residual, niter++ (cheb.cc:74-78), and the loop condition.
__global__ void k_cheb_check(ChebDev* d, cudaGraphConditionalHandle h) {
    double norm = sqrt(d->rr);
    if (!isfinite(norm)) d->status |= 2;
    d->niter++;
    bool go = norm / d->init > d->eps && d->status == 0 && (d->niter - 1) < d->maxit;
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

int cheb_solve(const DCSR& A, const double* b, Prec& P, double* x, double lmin, double lmax, double eps,
               uint32_t maxit, PcgStats& st, cudaStream_t s) {
    if (maxit == 0) maxit = PCG_DEFAULT_MAXIT;
    const Level& L0 = *P.H->lv[0];
    const DCSR& Af = L0.Af;
    uint32_t n = A.nrow;
    if (n != L0.N) MLP_THROW(ERR_ARG, "matrix and preconditioner sizes differ");
    if (!n) MLP_THROW(ERR_ARG, "empty system");
    if (!(lmax > lmin) || !(lmin > 0)) MLP_THROW(ERR_ARG, "ChebSolver needs 0 < lmin < lmax");
    double eta = (lmax + lmin) / (lmax - lmin);
    // cheb(eta, k) for k = 0 .. maxit + 2, the reference's own formula (host libm)
    std::vector<double> Th(maxit + 3);
    for (uint32_t k = 0; k < Th.size(); k++) Th[k] = cheb_poly(eta, k);
    DBuf<double> T(Th.size()), xf(n), bf(n), U0(n), U1(n), xcur(n), bnat(n), xnat(n);
    unsigned G = (unsigned)std::max(1, std::min<int>((int)grid_for(n, RB), num_sms() * 4));
    DBuf<double> partials(G);
    DBuf<ChebDev> d(1);
    T.upload(Th.data(), Th.size(), s);
    d.zero(s);
    CK(cudaMemcpyAsync(bnat.p, b, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    double* r = P.fin_buf.p;
    double* z = P.fout_buf.p;
    const double* x0 = x0_device(n, s);
    double alpha1 = 2 / (lmax + lmin);
    int scale1 = std::fabs(alpha1 - 1.0) <= 2.220446049250313e-16 ? 0 : 1;  // dscal skips alpha = 1
    double c4 = 4 / (lmax - lmin);
    ChebDev* dd = d.p;
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphExec_t ex = nullptr;
    try {
        cudaGraphConditionalHandle h;
        CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        CK(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        gather(n, L0.phi.p, bnat.p, bf.p, s);
        gather(n, L0.phi.p, x0, U1.p, s);  // x = generate_x0
        launch_spmv<double>(n, Af.nnz, Af.ia.p, Af.ja.p, Af.a.p, U1.p, r, bf.p, s, Af.tile_max);
        k_dot_simple<<<G, RB, 0, s>>>(n, r, r, partials.p, &dd->ticket, &dd->rr);
        k_cheb_start<<<1, 1, 0, s>>>(dd, eps, maxit);
        P.plan.run(s);  // z = B r
        k_cheb_first<<<grid_for(n, 256), 256, 0, s>>>(n, alpha1, scale1, z, U0.p, U1.p, xcur.p);
        launch_spmv<double>(n, Af.nnz, Af.ia.p, Af.ja.p, Af.a.p, xcur.p, r, bf.p, s, Af.tile_max);
        k_dot_simple<<<G, RB, 0, s>>>(n, r, r, partials.p, &dd->ticket, &dd->rr);
        k_cheb_check<<<1, 1, 0, s>>>(dd, h);
        cudaError_t le = cudaGetLastError();
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &ndeps));
        std::vector<cudaGraphNode_t> dv(deps, deps + ndeps);
        cudaGraph_t got;
        CK(cudaStreamEndCapture(s, &got));
        if (le != cudaSuccess) MLP_THROW(ERR_CUDA, cudaGetErrorString(le));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        CK(cudaGraphAddNode(&cnode, g, dv.data(), dv.size(), &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        P.plan.run(s);  // z = B r
        k_cheb_step<<<grid_for(n, 256), 256, 0, s>>>(n, dd, T.p, c4, z, U0.p, U1.p, xcur.p);
        launch_spmv<double>(n, Af.nnz, Af.ia.p, Af.ja.p, Af.a.p, xcur.p, r, bf.p, s, Af.tile_max);
        k_dot_simple<<<G, RB, 0, s>>>(n, r, r, partials.p, &dd->ticket, &dd->rr);
        k_cheb_check<<<1, 1, 0, s>>>(dd, h);
        le = cudaGetLastError();
        CK(cudaStreamEndCapture(s, &got));
        if (le != cudaSuccess) MLP_THROW(ERR_CUDA, cudaGetErrorString(le));
        CK(cudaStreamBeginCaptureToGraph(s, g, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
        scatter(n, L0.phi.p, xcur.p, xnat.p, s);
        le = cudaGetLastError();
        CK(cudaStreamEndCapture(s, &got));
        if (le != cudaSuccess) MLP_THROW(ERR_CUDA, cudaGetErrorString(le));
    } catch (...) {
        cudaGraphDestroy(g);
        throw;
    }
    ex = instantiate(g);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
    cudaError_t lerr = cudaGraphLaunch(ex, s);
    CK(cudaEventRecord(e1, s));
    ChebDev hd;
    CK(cudaMemcpyAsync(&hd, d.p, sizeof hd, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(x, xnat.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
    cudaGraphExecDestroy(ex);
    if (lerr != cudaSuccess) MLP_THROW(ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(lerr));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_persist(P, s);
    uint32_t steps = hd.niter >= 2 ? hd.niter - 1 : 0;  // cheb.cc:84 niter--
    count_launches(8 + P.plan.launches + (uint64_t)(steps ? steps - 1 : 0) * (4 + P.plan.launches));
    st.niter = steps;
    st.napply = steps;
    st.init_norm = hd.init;
    st.final_norm = std::sqrt(hd.rr);
    st.final_rel = st.final_norm / hd.init;
    st.t_total_ms = ms;
    int rc = OK;
    if (hd.status & 2) { rc = ERR_NOT_FINITE; set_last_error("non-finite residual norm in ChebSolver"); }
    else if (steps >= maxit && st.final_rel > hd.eps) { rc = ERR_MAXIT; set_last_error("iteration cap reached"); }
    return rc;
}

// ---------------------------------------------------------------------------
// Ensemble form: many independent solves (uneven sizes) as parallel branches
// of one graph, launched once.
// ---------------------------------------------------------------------------
Ensemble::~Ensemble() {
    if (exec) cudaGraphExecDestroy(exec);
}

std::unique_ptr<Ensemble> make_ensemble(const std::vector<Prec*>& members, bool flexible, int x0m,
                                        cudaStream_t s) {
    auto E = std::unique_ptr<Ensemble>(new Ensemble());
    E->members = members;
    E->flexible = flexible;
    E->x0m = x0m;
    PdlOff no_pdl;  // the members' branches run concurrently
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    try {
        for (Prec* P : members) {
            uint32_t n = P->H->lv[0]->N;
            pcg_work_alloc(*P, n);
            append_pcg(g, *P, n, flexible, x0m, s);
        }
    } catch (...) {
        cudaGraphDestroy(g);
        throw;
    }
    E->exec = instantiate(g);
    return E;
}

// dJ/dp of J = 0.5 sum_k (p[obs_k] - pobs_k)^2: zero, then the observed cells.
__global__ void k_misfit_rhs(uint32_t nobs, const uint32_t* __restrict__ obs, const double* __restrict__ pobs,
                             const double* __restrict__ p, double* __restrict__ g) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nobs) g[obs[k]] = p[obs[k]] - pobs[k];
}

__global__ void k_copy_pcgdev(const PcgDev* __restrict__ a, PcgDev* __restrict__ b) {
    const uint32_t* s = reinterpret_cast<const uint32_t*>(a);
    uint32_t* d = reinterpret_cast<uint32_t*>(b);
    for (uint32_t i = threadIdx.x; i < sizeof(PcgDev) / 4; i += blockDim.x) d[i] = s[i];
}

// Gradient form of the ensemble: each member's branch of the one graph runs
// the forward solve A p = b (zero start), forms the misfit gradient dJ/dp at
// the observation cells, runs the adjoint solve A lambda = dJ/dp (zero start,
// same hierarchy: A is symmetric) and the dT/dlogK gradient kernel; so one
// launch gives every member's p, lambda and dJ/dlnK.
std::unique_ptr<Ensemble> make_ensemble_gradient(const std::vector<Prec*>& members,
                                                 const std::vector<GradMember>& gm, bool flexible,
                                                 cudaStream_t s) {
    if (gm.size() != members.size()) MLP_THROW(ERR_ARG, "one gradient description per member");
    auto E = std::unique_ptr<Ensemble>(new Ensemble());
    E->members = members;
    E->flexible = flexible;
    E->x0m = X0_ZERO;
    E->gradient = true;
    E->fwd.resize(members.size());
    PdlOff no_pdl;  // the members' branches run concurrently
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    try {
        for (size_t i = 0; i < members.size(); i++) {
            Prec& P = *members[i];
            const GradMember& m = gm[i];
            uint32_t n = P.H->lv[0]->N;
            if (m.nx * m.ny * m.nz != n) MLP_THROW(ERR_ARG, "member mesh and preconditioner sizes differ");
            pcg_work_alloc(P, n);
            E->fwd[i].alloc(1);
            std::vector<cudaGraphNode_t> t = append_pcg(g, P, n, flexible, X0_ZERO, s);
            PcgWork& W = P.pcg;
            CK(cudaStreamBeginCaptureToGraph(s, g, t.data(), nullptr, t.size(), cudaStreamCaptureModeThreadLocal));
            k_copy_pcgdev<<<1, 32, 0, s>>>(W.d.p, E->fwd[i].p);
            k_copy_d<<<grid_for(n, 256), 256, 0, s>>>(n, W.xnat.p, m.p);
            k_fill_d<<<grid_for(n, 256), 256, 0, s>>>(n, W.bnat.p, 0.0);
            if (m.nobs) k_misfit_rhs<<<grid_for(m.nobs, 256), 256, 0, s>>>(m.nobs, m.obs, m.pobs, m.p, W.bnat.p);
            cudaError_t le = cudaGetLastError();
            cudaStreamCaptureStatus cs;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &ndeps));
            std::vector<cudaGraphNode_t> mid(deps, deps + ndeps);
            cudaGraph_t got;
            CK(cudaStreamEndCapture(s, &got));
            if (le != cudaSuccess) MLP_THROW(ERR_CUDA, cudaGetErrorString(le));
            t = append_pcg(g, P, n, flexible, X0_ZERO, s, mid);
            CK(cudaStreamBeginCaptureToGraph(s, g, t.data(), nullptr, t.size(), cudaStreamCaptureModeThreadLocal));
            k_copy_d<<<grid_for(n, 256), 256, 0, s>>>(n, W.xnat.p, m.lam);
            spe_grad_logk(m.nx, m.ny, m.nz, m.kx, m.ky, m.kz, m.dirichlet, m.p, m.lam, m.grad, s);
            le = cudaGetLastError();
            CK(cudaStreamEndCapture(s, &got));
            if (le != cudaSuccess) MLP_THROW(ERR_CUDA, cudaGetErrorString(le));
        }
    } catch (...) {
        cudaGraphDestroy(g);
        throw;
    }
    E->exec = instantiate(g);
    return E;
}

int ensemble_solve(Ensemble& E, const std::vector<const double*>& b, const std::vector<double*>& x, double eps,
                   uint32_t maxit, std::vector<PcgStats>& st, double& ms_out, cudaStream_t s) {
    if (maxit == 0) maxit = PCG_DEFAULT_MAXIT;
    size_t K = E.members.size();
    if (b.size() != K || (!E.gradient && x.size() != K)) MLP_THROW(ERR_ARG, "one b and one x per ensemble member");
    PcgParams prm{eps, maxit};
    for (size_t i = 0; i < K; i++) {
        Prec& P = *E.members[i];
        uint32_t n = P.pcg.n;
        CK(cudaMemcpyAsync(P.pcg.prm.p, &prm, sizeof prm, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(P.pcg.bnat.p, b[i], (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
        if (E.x0m == X0_GIVEN && !E.gradient)
            CK(cudaMemcpyAsync(P.pcg.xnat.p, x[i], (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
    CK(cudaGraphLaunch(E.exec, s));
    CK(cudaEventRecord(e1, s));
    std::vector<PcgDev> hs(K), hf(E.gradient ? K : 0);
    for (size_t i = 0; i < K; i++) {
        Prec& P = *E.members[i];
        if (!E.gradient) CK(cudaMemcpyAsync(x[i], P.pcg.xnat.p, (size_t)P.pcg.n * 8, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(&hs[i], P.pcg.d.p, sizeof(PcgDev), cudaMemcpyDeviceToHost, s));
        if (E.gradient) CK(cudaMemcpyAsync(&hf[i], E.fwd[i].p, sizeof(PcgDev), cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    for (Prec* P : E.members) check_persist(*P, s);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ms_out = ms;
    st.resize(E.gradient ? 2 * K : K);
    int rc_all = OK;
    std::string msg_all;
    for (size_t i = 0; i < K; i++) {
        // gradient form: entry i is member i's forward solve, entry K + i its adjoint solve
        for (int pass = 0; pass < (E.gradient ? 2 : 1); pass++) {
            const PcgDev& h = (E.gradient && pass == 0) ? hf[i] : hs[i];
            PcgStats& so = st[(E.gradient && pass == 1) ? K + i : i];
            int rc;
            std::string msg;
            read_stats(h, so, rc, msg);
            so.t_total_ms = ms;
            count_launches(start_launches(*E.members[i], E.flexible) +
                           (uint64_t)h.it * iteration_launches(*E.members[i], E.flexible));
            if (rc != OK && rc_all == OK) { rc_all = rc; msg_all = "member " + std::to_string(i) + ": " + msg; }
        }
        if (E.gradient) count_launches(6);
    }
    if (rc_all != OK) set_last_error(msg_all);
    return rc_all;
}

// Host-driven form of pcg_solve (one host round trip per iteration), kept as
// the reference point of the device loop in the tests.
int pcg_solve_hostloop(const DCSR& A, const double* b, Prec& P, double* x, double eps, uint32_t maxit,
                       bool flexible, PcgStats& st, cudaStream_t s) {
    if (maxit == 0) maxit = PCG_DEFAULT_MAXIT;
    Hierarchy& H = *P.H;
    const Level& L0 = *H.lv[0];
    const DCSR& Af = L0.Af;
    uint32_t n = A.nrow;
    if (n != L0.N) MLP_THROW(ERR_ARG, "matrix and preconditioner sizes differ");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
    DBuf<double> xf(n), bf(n), p(n), Ap(n), rprev(flexible ? n : 1);
    double* r = P.fin_buf.p;
    double* z = P.fout_buf.p;
    unsigned G = (unsigned)std::max(1, std::min<int>((int)grid_for(n, RB), num_sms() * 4));
    DBuf<double> partials(2 * (size_t)G);
    DBuf<PcgDev> dd(1);
    dd.zero(s);
    PcgDev* d = dd.p;
    gather(n, L0.phi.p, b, bf.p, s);
    int x0m = take_x0_mode();
    if (x0m == X0_ZERO) xf.zero(s);
    else gather(n, L0.phi.p, x0m == X0_GIVEN ? x : x0_device(n, s), xf.p, s);
    // r = b - A x
    launch_spmv<double>(n, Af.nnz, Af.ia.p, Af.ja.p, Af.a.p, xf.p, r, bf.p, s, Af.tile_max);
    CK_LAUNCH();
    double* hpin = nullptr;
    CK(cudaMallocHost(&hpin, sizeof(PcgDev)));
    auto fetch = [&]() -> PcgDev {
        CK(cudaMemcpyAsync(hpin, d, sizeof(PcgDev), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        PcgDev h;
        memcpy(&h, hpin, sizeof h);
        return h;
    };
    k_dot_simple<<<G, RB, 0, s>>>(n, r, r, partials.p, &d->ticket[1], &d->rr);
    CK_LAUNCH();
    prec_apply_frame(P, s);
    CK(cudaMemcpyAsync(p.p, z, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    k_dot_simple<<<G, RB, 0, s>>>(n, r, z, partials.p, &d->ticket[2], &d->rz0);
    CK_LAUNCH();
    if (flexible) CK(cudaMemcpyAsync(rprev.p, r, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    PcgDev h = fetch();
    double norm = std::sqrt(h.rr), init = norm;
    st.init_norm = init;
    if (init * eps < 1e-14) eps = 1e-14 / init;  // check_and_replace_eps, solvers.cc:49-58
    uint32_t it = 0;
    uint32_t napply = 1;
    double avg = (double)Af.nnz / n;
    int lpr = avg <= 3 ? 2 : avg <= 6 ? 4 : avg <= 12 ? 8 : avg <= 24 ? 16 : 32;
    int rc = OK;
    std::string msg;
    if (!std::isfinite(init)) { rc = ERR_NOT_FINITE; msg = "non-finite initial residual norm"; }
    bool staged = Af.tile_max && Af.tile_max <= ST_MAX_NNZ && n >= 4 * ST_ROWS;
    unsigned Gs = staged_grid(n);
    if (staged && 2 * (size_t)Gs > partials.n) partials.alloc(2 * (size_t)Gs);
    while (rc == OK && norm / init > eps) {
        if (maxit && it >= maxit) { rc = ERR_MAXIT; msg = "iteration cap reached"; break; }
        if (staged) {
            launch_pcg_spmv_dot_staged(n, Af, p.p, Ap.p, partials.p, d, s);
        } else switch (lpr) {
            case 2: k_pcg_spmv_dot<2><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p.p, Ap.p, partials.p, d); break;
            case 4: k_pcg_spmv_dot<4><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p.p, Ap.p, partials.p, d); break;
            case 8: k_pcg_spmv_dot<8><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p.p, Ap.p, partials.p, d); break;
            case 16: k_pcg_spmv_dot<16><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p.p, Ap.p, partials.p, d); break;
            default: k_pcg_spmv_dot<32><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p.p, Ap.p, partials.p, d); break;
        }
        k_pcg_update<<<G, RB, 0, s>>>(n, xf.p, r, p.p, Ap.p, partials.p, d, 0, 0);
        count_launches(1);
        CK_LAUNCH();
        h = fetch();
        if (h.status & 1) { rc = ERR_CURVATURE; msg = "<Ap, p> = " + std::to_string(h.app); break; }
        if (h.status & 2) { rc = ERR_NOT_FINITE; msg = "non-finite value in PCG scalars"; break; }
        norm = std::sqrt(h.rr);
        it++;
        if (!(norm / init > eps)) break;  // the reference's last apply cannot change x
        prec_apply_frame(P, s);
        napply++;
        k_pcg_dot_rz<<<G, RB, 0, s>>>(n, r, z, rprev.p, partials.p, d, flexible ? 1 : 0);
        k_pcg_p<<<grid_for(((n + 1) / 2 + PCG_P_PAIRS - 1) / PCG_P_PAIRS, 256), 256, 0, s>>>(n, p.p, z, d);
        count_launches(2);
        if (flexible) CK(cudaMemcpyAsync(rprev.p, r, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
        CK_LAUNCH();
    }
    scatter(n, L0.phi.p, xf.p, x, s);
    CK(cudaEventRecord(e1, s));
    CK(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeHost(hpin);
    check_persist(P, s);
    st.niter = it;
    st.final_norm = norm;
    st.final_rel = norm / init;
    st.t_total_ms = ms;
    st.napply = napply;
    if (rc == OK && it == 0) { rc = ERR_NO_ITER; msg = "No need to iterate"; }
    if (rc != OK) set_last_error(msg);
    return rc;
}

}  // namespace mlp

namespace mlp {

// ---------------------------------------------------------------------------
// PCG without device allocation.
//
// Some host applications cannot let a library call cudaMalloc while they
// solve: their device memory is owned by their own allocator (a framework's
// caching allocator that has reserved the device, or a process held to a fixed
// device-memory budget), so an allocation from inside this library would fail
// or break the host's accounting. They use this variant of pcg_solve. The
// solver's own vectors, its reduction scratch and the start vector live in the
// file-scope array below instead of buffers from cudaMalloc; the matrix and
// the preconditioner handle were built beforehand (those calls allocate). The
// array holds up to NOALLOC_MAX_N unknowns; every GPU that loads the library
// holds it (about 6 MB) until the process exits.
// ---------------------------------------------------------------------------
static constexpr uint32_t NOALLOC_MAX_N = 131072;
static constexpr uint32_t NOALLOC_GRID = 1024;  // largest reduction grid used
static constexpr size_t NOALLOC_HDR = 16;       // doubles reserved for PcgDev
static constexpr size_t NOALLOC_DOUBLES = NOALLOC_HDR + 2 * (size_t)NOALLOC_GRID + 6 * (size_t)NOALLOC_MAX_N;
static_assert(sizeof(PcgDev) <= NOALLOC_HDR * sizeof(double), "PcgDev must fit the header");

static __device__ __align__(256) double g_pcg_scratch[NOALLOC_DOUBLES];

// Device address of g_pcg_scratch on the current device. In host code the
// array's name is only a stand-in, so every call looks the address up with
// cudaGetSymbolAddress while the caller's device is current (the lookup
// allocates nothing once the library's device code is loaded on the device);
// a context recreated after cudaDeviceReset therefore gets the array's new
// address rather than a stale one.
static double* noalloc_scratch() {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
    if (e != cudaSuccess) MLP_THROW(ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return (double*)p;
}

// generate_x0 (solvers.cc:9-21) for NOALLOC_MAX_N unknowns, made once on the
// host: srandom(3) with a fixed sequence, so the start vector of a system of n
// unknowns is the first n entries.
static const std::vector<double>& noalloc_x0_host() {
    static std::once_flag once;
    static std::vector<double> h;
    std::call_once(once, [] {
        h.resize(NOALLOC_MAX_N);
        struct random_data rd;
        memset(&rd, 0, sizeof rd);
        char state[128];
        initstate_r(3, state, sizeof state, &rd);
        srandom_r(3, &rd);
        for (uint32_t i = 0; i < NOALLOC_MAX_N; i++) {
            int32_t v;
            random_r(&rd, &v);
            h[i] = 20. * (v - 0.5 * RAND_MAX) / RAND_MAX + 100;
        }
    });
    return h;
}

uint32_t pcg_noalloc_max_n() { return NOALLOC_MAX_N; }

int pcg_solve_noalloc(const DCSR& A, const double* b, Prec& P, double* x, double eps, uint32_t maxit,
                      bool flexible, PcgStats& st, cudaStream_t s) {
    if (maxit == 0) maxit = PCG_DEFAULT_MAXIT;
    Hierarchy& H = *P.H;
    const Level& L0 = *H.lv[0];
    const DCSR& Af = L0.Af;
    uint32_t n = A.nrow;
    if (n != L0.N) MLP_THROW(ERR_ARG, "matrix and preconditioner sizes differ");
    if (n > NOALLOC_MAX_N)
        MLP_THROW(ERR_LIMIT, "the allocation-free PCG holds at most " + std::to_string(NOALLOC_MAX_N) +
                                 " unknowns; this system has " + std::to_string(n));
    unsigned G = (unsigned)std::max(1, std::min<int>((int)grid_for(n, RB), num_sms() * 4));
    if (G > NOALLOC_GRID) MLP_THROW(ERR_LIMIT, "reduction grid exceeds the static scratch");
    auto t0 = std::chrono::steady_clock::now();
    double* base = noalloc_scratch();
    PcgDev* d = reinterpret_cast<PcgDev*>(base);
    double* partials = base + NOALLOC_HDR;
    double* xf = partials + 2 * (size_t)NOALLOC_GRID;
    double* bf = xf + NOALLOC_MAX_N;
    double* p = bf + NOALLOC_MAX_N;
    double* Ap = p + NOALLOC_MAX_N;
    double* rprev = Ap + NOALLOC_MAX_N;
    double* x0 = rprev + NOALLOC_MAX_N;
    double* r = P.fin_buf.p;
    double* z = P.fout_buf.p;
    // the array keeps the previous call's contents: the reduction tickets and
    // status flags must start at zero
    CK(cudaMemsetAsync(d, 0, sizeof(PcgDev), s));
    // x0 of generate_x0 in natural order, then permuted into the frame like b
    CK(cudaMemcpyAsync(x0, noalloc_x0_host().data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
    gather(n, L0.phi.p, b, bf, s);
    gather(n, L0.phi.p, x0, xf, s);
    launch_spmv<double>(n, Af.nnz, Af.ia.p, Af.ja.p, Af.a.p, xf, r, bf, s, Af.tile_max);
    CK_LAUNCH();
    auto fetch = [&]() -> PcgDev {
        PcgDev h;
        CK(cudaMemcpyAsync(&h, d, sizeof(PcgDev), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return h;
    };
    k_dot_simple<<<G, RB, 0, s>>>(n, r, r, partials, &d->ticket[1], &d->rr);
    CK_LAUNCH();
    prec_apply_frame(P, s);
    CK(cudaMemcpyAsync(p, z, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    k_dot_simple<<<G, RB, 0, s>>>(n, r, z, partials, &d->ticket[2], &d->rz0);
    CK_LAUNCH();
    if (flexible) CK(cudaMemcpyAsync(rprev, r, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    PcgDev h = fetch();
    double norm = std::sqrt(h.rr), init = norm;
    st.init_norm = init;
    if (init * eps < 1e-14) eps = 1e-14 / init;  // check_and_replace_eps, solvers.cc:49-58
    uint32_t it = 0, napply = 1;
    double avg = (double)Af.nnz / n;
    int lpr = avg <= 3 ? 2 : avg <= 6 ? 4 : avg <= 12 ? 8 : avg <= 24 ? 16 : 32;
    int rc = OK;
    std::string msg;
    if (!std::isfinite(init)) { rc = ERR_NOT_FINITE; msg = "non-finite initial residual norm"; }
    bool staged = Af.tile_max && Af.tile_max <= ST_MAX_NNZ && n >= 4 * ST_ROWS;
    unsigned Gs = staged_grid(n);
    if (staged && Gs > 2 * NOALLOC_GRID) MLP_THROW(ERR_LIMIT, "reduction grid exceeds the static scratch");
    while (rc == OK && norm / init > eps) {
        if (maxit && it >= maxit) { rc = ERR_MAXIT; msg = "iteration cap reached"; break; }
        if (staged) {
            launch_pcg_spmv_dot_staged(n, Af, p, Ap, partials, d, s);
        } else switch (lpr) {
            case 2: k_pcg_spmv_dot<2><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p, Ap, partials, d); break;
            case 4: k_pcg_spmv_dot<4><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p, Ap, partials, d); break;
            case 8: k_pcg_spmv_dot<8><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p, Ap, partials, d); break;
            case 16: k_pcg_spmv_dot<16><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p, Ap, partials, d); break;
            default: k_pcg_spmv_dot<32><<<G, RB, 0, s>>>(n, Af.ia.p, Af.ja.p, Af.a.p, p, Ap, partials, d); break;
        }
        k_pcg_update<<<G, RB, 0, s>>>(n, xf, r, p, Ap, partials, d, 0, 0);
        count_launches(1);
        CK_LAUNCH();
        h = fetch();
        if (h.status & 1) { rc = ERR_CURVATURE; msg = "<Ap, p> = " + std::to_string(h.app); break; }
        if (h.status & 2) { rc = ERR_NOT_FINITE; msg = "non-finite value in PCG scalars"; break; }
        norm = std::sqrt(h.rr);
        it++;
        if (!(norm / init > eps)) break;
        prec_apply_frame(P, s);
        napply++;
        k_pcg_dot_rz<<<G, RB, 0, s>>>(n, r, z, rprev, partials, d, flexible ? 1 : 0);
        k_pcg_p<<<grid_for(((n + 1) / 2 + PCG_P_PAIRS - 1) / PCG_P_PAIRS, 256), 256, 0, s>>>(n, p, z, d);
        count_launches(2);
        if (flexible) CK(cudaMemcpyAsync(rprev, r, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
        CK_LAUNCH();
    }
    scatter(n, L0.phi.p, xf, x, s);
    CK(cudaStreamSynchronize(s));
    check_persist(P, s);
    st.niter = it;
    st.final_norm = norm;
    st.final_rel = norm / init;
    st.t_total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    st.napply = napply;
    if (rc == OK && it == 0) { rc = ERR_NO_ITER; msg = "No need to iterate"; }
    if (rc != OK) set_last_error(msg);
    return rc;
}

}  // namespace mlp
