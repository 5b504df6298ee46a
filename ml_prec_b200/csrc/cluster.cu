// k_cluster_level: one cluster-resident level call (cluster.cuh).
//
// Work split: the rows of a matrix step are partitioned like the matrix (CTA
// b takes rows [b << shift, (b + 1) << shift)), and inside a CTA each warp
// takes 32 / LPR consecutive rows per pass, lane l of a row adding the row's
// entries l, l + LPR, ... in order with a fused multiply-add before the xor
// butterfly, exactly as the separate row kernels do; a dense product takes a
// warp per row across the cluster. Elementwise steps stride over the cluster's
// threads. Only the assignment of rows to warps differs from the separate
// kernels, which changes no row's arithmetic.
//
// Memory: matrix partitions and constant arrays are read from this CTA's own
// shared memory with ordinary loads; vector elements go through the cluster
// window (mapa + ld/st.shared::cluster, the owner may be any CTA). The
// cluster barrier (arrive.release / wait.acquire) between steps orders every
// step's stores before the next step's loads in all CTAs.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

#include "cluster.cuh"

namespace mlp {

namespace {

__device__ __forceinline__ double fmadd_c(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmadd_c(float a, float b, float c) { return __fmaf_rn(a, b, c); }

__device__ __forceinline__ uint32_t cl_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cl_sync() {
    asm volatile(
        "barrier.cluster.arrive.release.aligned;\n\t"
        "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t cl_map(uint32_t a, uint32_t cta) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(cta));
    return r;
}

template <class T>
__device__ __forceinline__ T dsm_ld(uint32_t a);
template <>
__device__ __forceinline__ double dsm_ld<double>(uint32_t a) {
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a));
    return v;
}
template <>
__device__ __forceinline__ float dsm_ld<float>(uint32_t a) {
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void dsm_st(uint32_t a, double v) {
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void dsm_st(uint32_t a, float v) {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}

// A vector operand: element i of array A at element offset o.
template <class T>
struct VRef {
    uint32_t base, shift, mask, o;  // base: shared-window address of the array's chunk in this CTA
    __device__ __forceinline__ VRef(const CArr& A, uint32_t sm_base, uint32_t off)
        : base(sm_base + A.off), shift(A.shift), mask((1u << A.shift) - 1u), o(off) {}
    __device__ __forceinline__ uint32_t addr(uint32_t i) const {
        uint32_t k = o + i;
        return cl_map(base + (k & mask) * (uint32_t)sizeof(T), k >> shift);
    }
    __device__ __forceinline__ T ld(uint32_t i) const { return dsm_ld<T>(addr(i)); }
    __device__ __forceinline__ void st(uint32_t i, T v) const { dsm_st(addr(i), v); }
};

template <class T, int LPR, class Val, class Out>
__device__ __forceinline__ void cl_rows(const CMat& m, const uint8_t* sm, uint32_t rank, Val val, Out out) {
    constexpr uint32_t RPW = 32 / LPR;
    const uint32_t r0 = rank << m.shift;
    if (r0 >= m.rows) return;
    const uint32_t r1 = min(m.rows, r0 + (1u << m.shift));
    const uint32_t* ia = reinterpret_cast<const uint32_t*>(sm + m.ia_off);
    const uint32_t* ja = reinterpret_cast<const uint32_t*>(sm + m.ja_off);
    const T* a = reinterpret_cast<const T*>(sm + m.a_off);
    const uint32_t j00 = ia[0];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t base = r0 + warp * RPW; base < r1; base += (CL_THREADS / 32) * RPW) {
        const uint32_t row = base + lane / LPR;
        const bool act = row < r1;
        const int sub = (int)(lane % LPR);
        T s = 0;
        if (act) {
            const uint32_t e = ia[row - r0 + 1] - j00;
            for (uint32_t j = ia[row - r0] - j00 + sub; j < e; j += LPR) s = fmadd_c(a[j], val(ja[j]), s);
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (act && sub == 0) out(row, s);
    }
}

template <class T, int LPR>
__device__ __forceinline__ void cl_row_step(const CStep<T>& st, const CArr* arr, const CMat* mat, const uint8_t* sm,
                                            uint32_t smb, uint32_t rank) {
    const CMat& m = mat[st.mat];
    switch (st.op) {
        case PS_PHASE1: {
            const VRef<T> src(arr[st.arr[0]], smb, st.off[0]), w(arr[st.arr[1]], smb, st.off[1]);
            cl_rows<T, LPR>(m, sm, rank, [&](uint32_t c) { return src.ld(c); }, [&](uint32_t row, T s) { w.st(row, s); });
            break;
        }
        case PS_PHASE2: {
            const uint32_t M = st.n0;
            const VRef<T> w(arr[st.arr[0]], smb, st.off[0]), out(arr[st.arr[1]], smb, st.off[1]);
            cl_rows<T, LPR>(m, sm, rank, [&](uint32_t c) { return c < M ? w.ld(c) : out.ld(c); },
                            [&](uint32_t row, T s) { out.st(row, s); });
            break;
        }
        case PS_UPDATE: {
            const VRef<T> u0(arr[st.arr[0]], smb, st.off[0]), x(arr[st.arr[1]], smb, st.off[1]),
                r(arr[st.arr[2]], smb, st.off[2]);
            cl_rows<T, LPR>(m, sm, rank, [&](uint32_t c) { return u0.ld(c); }, [&](uint32_t row, T s) {
                x.st(row, x.ld(row) + u0.ld(row));
                r.st(row, r.ld(row) - s);
            });
            break;
        }
        case PS_RESID: {
            const VRef<T> x(arr[st.arr[0]], smb, st.off[0]), y(arr[st.arr[1]], smb, st.off[1]),
                f(arr[st.arr[2]], smb, st.off[2]);
            cl_rows<T, LPR>(m, sm, rank, [&](uint32_t c) { return x.ld(c); },
                            [&](uint32_t row, T s) { y.st(row, f.ld(row) - s); });
            break;
        }
        default:
            break;
    }
}

template <class T, class CT>
__device__ __forceinline__ void cl_dense(uint32_t n, const CT* __restrict__ C, const VRef<T>& f, const VRef<T>& x,
                                         uint32_t rank, uint32_t cs) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t W = cs * (CL_THREADS / 32);
    for (uint32_t row = rank * (CL_THREADS / 32) + (threadIdx.x >> 5); row < n; row += W) {
        const CT* c = C + (size_t)row * n;
        CT s = 0;
        for (uint32_t j = lane; j < n; j += 32) s = fmadd_c(__ldg(c + j), (CT)f.ld(j), s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) x.st(row, (T)s);
    }
}

template <class T>
__device__ void cl_step(const CStep<T>& st, const CArr* arr, const CMat* mat, const uint8_t* sm, uint32_t smb,
                        uint32_t rank, uint32_t cs) {
    const uint32_t nthr = cs * CL_THREADS, tid = rank * CL_THREADS + threadIdx.x;
    switch (st.op) {
        case PS_PHASE1:
        case PS_PHASE2:
        case PS_UPDATE:
        case PS_RESID:
            if (st.op == PS_UPDATE && st.mode == 0) {
                // the last correction of a level call: x += u0
                const VRef<T> u0(arr[st.arr[0]], smb, st.off[0]), x(arr[st.arr[1]], smb, st.off[1]);
                for (uint32_t i = tid; i < st.n0; i += nthr) x.st(i, x.ld(i) + u0.ld(i));
                break;
            }
            switch (st.lpr) {
                case 1: cl_row_step<T, 1>(st, arr, mat, sm, smb, rank); break;
                case 2: cl_row_step<T, 2>(st, arr, mat, sm, smb, rank); break;
                case 4: cl_row_step<T, 4>(st, arr, mat, sm, smb, rank); break;
                case 8: cl_row_step<T, 8>(st, arr, mat, sm, smb, rank); break;
                case 16: cl_row_step<T, 16>(st, arr, mat, sm, smb, rank); break;
                default: cl_row_step<T, 32>(st, arr, mat, sm, smb, rank); break;
            }
            if (st.op == PS_PHASE1 && st.n1 > st.n0) {
                // diagonal rows [R, N): out = dval * src; dval element k = q - R
                // lives in this CTA's chunk of its constant array
                const uint32_t R = st.n0;
                const CArr& D = arr[st.dval];
                const T* dv = reinterpret_cast<const T*>(sm + D.off);
                const VRef<T> src(arr[st.arr[0]], smb, st.off[0]), out(arr[st.arr[2]], smb, st.off[2]);
                const uint32_t k0 = rank << D.shift, k1 = min(st.n1 - R, k0 + (1u << D.shift));
                for (uint32_t k = k0 + threadIdx.x; k < k1; k += CL_THREADS) out.st(R + k, dv[k - k0] * src.ld(R + k));
            }
            break;
        case PS_DENSE: {
            const VRef<T> f(arr[st.arr[0]], smb, st.off[0]), x(arr[st.arr[1]], smb, st.off[1]);
            if (st.mode == 1) cl_dense<T, double>(st.n0, static_cast<const double*>(st.C), f, x, rank, cs);
            else cl_dense<T, T>(st.n0, static_cast<const T*>(st.C), f, x, rank, cs);
            break;
        }
        default:
            break;
    }
}

template <class T>
__global__ void __launch_bounds__(CL_THREADS, 1) k_cluster_level(const CProg<T>* __restrict__ prog) {
    extern __shared__ __align__(16) uint8_t sm[];
    __shared__ CArr s_arr[CL_MAX_ARR];
    __shared__ CMat s_mat[CL_MAX_MAT];
    constexpr uint32_t NW = sizeof(CStep<T>) / 4;
    __shared__ __align__(16) uint32_t sbuf[2][NW];
    const uint32_t rank = cl_rank();
    const uint32_t tid = threadIdx.x;
    const CProg<T> P = *prog;
    if (tid < P.narr) s_arr[tid] = P.arrs[tid];
    if (tid < P.nmat) s_mat[tid] = P.mats[tid];
    const uint32_t* gsrc = reinterpret_cast<const uint32_t*>(P.steps);
    if (tid < NW) sbuf[0][tid] = __ldg(gsrc + tid);
    // constant partitions: independent of the preceding kernel, copied before
    // waiting for it
    uint32_t* smw = reinterpret_cast<uint32_t*>(sm);
    for (uint32_t k = __ldg(P.copy_first + rank), ke = __ldg(P.copy_first + rank + 1); k < ke; k++) {
        const CCopy c = P.copies[k];
        const uint32_t* src = c.src;
        uint32_t* dst = smw + c.dst / 4;
        for (uint32_t i = tid; i < c.words; i += CL_THREADS) dst[i] = __ldg(src + i);
    }
    pdl_wait();
    pdl_trigger();
    __syncthreads();
    {
        // this CTA's chunk of the input vector (written by the preceding kernels)
        const CArr& F = s_arr[P.f_arr];
        const uint32_t lo = rank << F.shift, hi = min(P.n, lo + (1u << F.shift));
        T* fl = reinterpret_cast<T*>(sm + F.off);
        for (uint32_t i = lo + tid; i < hi; i += CL_THREADS) fl[i - lo] = P.f[i];
    }
    const uint32_t smb = (uint32_t)__cvta_generic_to_shared(sm);
    cl_sync();
    int cur = 0;
    for (uint32_t pc = 0; pc < P.nsteps; pc++) {
        if (pc + 1 < P.nsteps && tid < NW) sbuf[cur ^ 1][tid] = __ldg(gsrc + (size_t)(pc + 1) * NW + tid);
        const CStep<T>& st = *reinterpret_cast<const CStep<T>*>(sbuf[cur]);
        cl_step<T>(st, s_arr, s_mat, sm, smb, rank, P.cs);
        // every CTA's stores of this step before any CTA's loads of the next;
        // the barrier also publishes the prefetched descriptor within the CTA
        cl_sync();
        cur ^= 1;
    }
    {
        // no CTA touches another's shared memory after the last barrier: write
        // this CTA's chunk of the output vector back
        const CArr& X = s_arr[P.x_arr];
        const uint32_t lo = rank << X.shift, hi = min(P.n, lo + (1u << X.shift));
        const T* xl = reinterpret_cast<const T*>(sm + X.off);
        for (uint32_t i = lo + tid; i < hi; i += CL_THREADS) P.x[i] = xl[i - lo];
    }
}

template <class T>
cudaLaunchConfig_t level_cfg(unsigned cs, uint32_t smem, cudaStream_t s, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(CL_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 2 : 1;
    return cfg;
}

}  // namespace

template <class T>
unsigned cluster_level_size(uint32_t smem) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    auto k = k_cluster_level<T>;
    static bool attr_set = false;
    if (!attr_set) {
        CK(cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CL_SMEM_BUDGET));
        attr_set = true;
    }
    static std::map<uint32_t, unsigned> fits;  // by smem rounded up to 8 KB
    uint32_t key = (smem + 8191u) & ~8191u;
    auto it = fits.find(key);
    if (it != fits.end()) return it->second;
    cudaLaunchAttribute attr[2];
    cudaLaunchConfig_t cfg = level_cfg<T>(16, key, 0, attr);
    int n = 0;
    unsigned cs = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) == cudaSuccess && n >= 1) cs = 16;
    cudaGetLastError();
    fits[key] = cs;
    return cs;
}

template <class T>
void launch_cluster_level(const CProg<T>* prog, uint32_t cs, uint32_t smem, cudaStream_t s) {
    cudaLaunchAttribute attr[2];
    cudaLaunchConfig_t cfg = level_cfg<T>(cs, smem, s, attr);
    CK(cudaLaunchKernelEx(&cfg, k_cluster_level<T>, prog));
}

template <class T>
bool cluster_prog_build(const std::vector<PStep<T>>& steps, const T* f, T* x, uint32_t n,
                        const std::vector<ClusterVec>& vecs, DBuf<uint8_t>& out, uint32_t& cs_out, uint32_t& smem_out,
                        cudaStream_t s) {
    const uint32_t cs = 16;
    auto chunk_shift = [&](uint32_t len) {
        uint32_t per = (len + cs - 1) / cs, sh = 0;
        while ((1u << sh) < per) sh++;
        return sh;
    };
    struct Arr {
        const char* base;
        uint32_t n;
        const T* src;  // constant data copied in (dval), else nullptr (a vector)
        uint32_t shift, off;
    };
    std::vector<Arr> arrs;
    auto add_vec = [&](const void* p, uint32_t len) {
        arrs.push_back({static_cast<const char*>(p), len, nullptr, chunk_shift(len), 0});
    };
    add_vec(f, n);  // array 0: the call's input
    add_vec(x, n);  // array 1: the call's output
    for (const ClusterVec& v : vecs)
        if (v.p && v.n) add_vec(v.p, v.n);
    // operand at p with `extent` elements -> (array, element offset)
    auto find_vec = [&](const void* p, uint32_t extent, uint32_t& id, uint32_t& off) -> bool {
        if (!extent) {
            id = 0;
            off = 0;
            return true;
        }
        const char* c = static_cast<const char*>(p);
        for (uint32_t i = 0; i < arrs.size(); i++) {
            const Arr& a = arrs[i];
            if (a.src || c < a.base || c >= a.base + (size_t)a.n * sizeof(T)) continue;
            size_t d = (size_t)(c - a.base);
            if (d % sizeof(T)) return false;
            off = (uint32_t)(d / sizeof(T));
            if ((uint64_t)off + extent > a.n) return false;
            id = i;
            return true;
        }
        return false;
    };
    auto const_arr = [&](const T* p, uint32_t len) -> uint32_t {
        for (uint32_t i = 0; i < arrs.size(); i++)
            if (arrs[i].src == p && arrs[i].n == len) return i;
        arrs.push_back({reinterpret_cast<const char*>(p), len, p, chunk_shift(len), 0});
        return (uint32_t)arrs.size() - 1;
    };
    struct Mat {
        const uint32_t* ia;
        const uint32_t* ja;
        const T* a;
        uint32_t rows, shift, nnz_max, ia_off, ja_off, a_off;
        std::vector<uint32_t> iah;
    };
    std::vector<Mat> mats;
    auto find_mat = [&](const PStep<T>& p, uint32_t rows, uint32_t& id) -> bool {
        for (uint32_t i = 0; i < mats.size(); i++)
            if (mats[i].ia == p.ia) {
                if (mats[i].rows != rows || mats[i].ja != p.ja || mats[i].a != p.a) return false;
                id = i;
                return true;
            }
        Mat m{p.ia, p.ja, p.a, rows, chunk_shift(rows), 0, 0, 0, 0, {}};
        m.iah.resize((size_t)rows + 1);
        CK(cudaMemcpyAsync(m.iah.data(), p.ia, ((size_t)rows + 1) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (uint32_t b = 0; b < cs; b++) {
            uint32_t r0 = b << m.shift;
            if (r0 >= rows) break;
            uint32_t r1 = std::min(rows, r0 + (1u << m.shift));
            m.nnz_max = std::max(m.nnz_max, m.iah[r1] - m.iah[r0]);
        }
        mats.push_back(std::move(m));
        id = (uint32_t)mats.size() - 1;
        return true;
    };

    std::vector<CStep<T>> cst;
    cst.reserve(steps.size());
    for (const PStep<T>& p : steps) {
        CStep<T> c;
        memset(&c, 0, sizeof c);
        c.op = p.op;
        c.lpr = p.lpr;
        c.n0 = p.n0;
        c.n1 = p.n1;
        c.mode = p.mode;
        bool ok = true;
        switch (p.op) {
            case PS_PHASE1: {  // src N, w R, out N; P1 has R rows
                const uint32_t R = p.n0, N = p.n1;
                ok = find_mat(p, R, c.mat) && find_vec(p.v[0], N, c.arr[0], c.off[0]) &&
                     find_vec(p.v[1], R, c.arr[1], c.off[1]) && find_vec(p.v[2], N, c.arr[2], c.off[2]);
                if (ok && N > R) c.dval = const_arr(p.dval, N - R);
                break;
            }
            case PS_PHASE2:  // w M, out N (columns past M read it); G has M rows
                ok = p.n1 != 0 && find_mat(p, p.n0, c.mat) && find_vec(p.v[0], p.n0, c.arr[0], c.off[0]) &&
                     find_vec(p.v[1], p.n1, c.arr[1], c.off[1]);
                break;
            case PS_UPDATE:  // u0, x (and r) N
                ok = find_vec(p.v[0], p.n0, c.arr[0], c.off[0]) && find_vec(p.v[1], p.n0, c.arr[1], c.off[1]);
                if (ok && p.mode == 1) ok = find_mat(p, p.n0, c.mat) && find_vec(p.v[2], p.n0, c.arr[2], c.off[2]);
                break;
            case PS_RESID:  // x, y, f N
                ok = find_mat(p, p.n0, c.mat) && find_vec(p.v[0], p.n0, c.arr[0], c.off[0]) &&
                     find_vec(p.v[1], p.n0, c.arr[1], c.off[1]) && find_vec(p.v[2], p.n0, c.arr[2], c.off[2]);
                break;
            case PS_DENSE:  // f, x n; the operator stays in global memory
                ok = find_vec(p.v[0], p.n0, c.arr[0], c.off[0]) && find_vec(p.v[1], p.n0, c.arr[1], c.off[1]);
                c.C = p.mode == 1 ? p.v[2] : static_cast<const void*>(p.a);
                break;
            default:
                ok = false;
        }
        if (!ok) return false;
        cst.push_back(c);
    }
    if (cst.empty() || arrs.size() > CL_MAX_ARR || mats.size() > CL_MAX_MAT) return false;

    // shared-memory layout, the same in every CTA
    uint32_t used = 0;
    auto take = [&](uint64_t bytes) {
        uint32_t o = used;
        uint64_t e = (uint64_t)used + ((bytes + 15) & ~(uint64_t)15);
        used = e > 0xffffffffu ? 0xffffffffu : (uint32_t)e;
        return o;
    };
    for (Arr& a : arrs) a.off = take((uint64_t)(1u << a.shift) * sizeof(T));
    for (Mat& m : mats) {
        m.ia_off = take(((uint64_t)(1u << m.shift) + 1) * 4);
        m.ja_off = take((uint64_t)m.nnz_max * 4);
        m.a_off = take((uint64_t)m.nnz_max * sizeof(T));
    }
    if (used > CL_SMEM_BUDGET) return false;
    if (cluster_level_size<T>(used) != cs) return false;

    // per-CTA copies of the constant partitions
    std::vector<uint32_t> first(cs + 1, 0);
    std::vector<CCopy> copies;
    for (uint32_t b = 0; b < cs; b++) {
        first[b] = (uint32_t)copies.size();
        for (const Arr& a : arrs) {
            if (!a.src) continue;
            uint32_t lo = b << a.shift;
            if (lo >= a.n) continue;
            uint32_t hi = std::min(a.n, lo + (1u << a.shift));
            copies.push_back({reinterpret_cast<const uint32_t*>(a.src + lo), a.off,
                              (uint32_t)((hi - lo) * sizeof(T) / 4)});
        }
        for (const Mat& m : mats) {
            uint32_t r0 = b << m.shift;
            if (r0 >= m.rows) continue;
            uint32_t r1 = std::min(m.rows, r0 + (1u << m.shift));
            uint32_t j0 = m.iah[r0], j1 = m.iah[r1];
            copies.push_back({m.ia + r0, m.ia_off, r1 - r0 + 1});
            if (j1 > j0) {
                copies.push_back({m.ja + j0, m.ja_off, j1 - j0});
                copies.push_back({reinterpret_cast<const uint32_t*>(m.a + j0), m.a_off,
                                  (uint32_t)((size_t)(j1 - j0) * sizeof(T) / 4)});
            }
        }
    }
    first[cs] = (uint32_t)copies.size();

    // one device buffer: header, arrays, matrices, steps, copy index, copies
    auto al = [](size_t v) { return (v + 15) & ~(size_t)15; };
    size_t o_arr = al(sizeof(CProg<T>));
    size_t o_mat = al(o_arr + arrs.size() * sizeof(CArr));
    size_t o_st = al(o_mat + mats.size() * sizeof(CMat));
    size_t o_first = al(o_st + cst.size() * sizeof(CStep<T>));
    size_t o_cp = al(o_first + first.size() * 4);
    size_t total = al(o_cp + copies.size() * sizeof(CCopy));
    out.alloc(total);
    std::vector<uint8_t> img(total, 0);
    uint8_t* d = out.p;
    CProg<T> h;
    memset(&h, 0, sizeof h);
    h.nsteps = (uint32_t)cst.size();
    h.narr = (uint32_t)arrs.size();
    h.nmat = (uint32_t)mats.size();
    h.cs = cs;
    h.smem = used;
    h.f_arr = 0;
    h.x_arr = 1;
    h.n = n;
    h.f = f;
    h.x = x;
    h.arrs = reinterpret_cast<const CArr*>(d + o_arr);
    h.mats = reinterpret_cast<const CMat*>(d + o_mat);
    h.steps = reinterpret_cast<const CStep<T>*>(d + o_st);
    h.copy_first = reinterpret_cast<const uint32_t*>(d + o_first);
    h.copies = reinterpret_cast<const CCopy*>(d + o_cp);
    memcpy(img.data(), &h, sizeof h);
    for (size_t i = 0; i < arrs.size(); i++) {
        CArr a{arrs[i].off, arrs[i].shift, arrs[i].n, 0};
        memcpy(img.data() + o_arr + i * sizeof(CArr), &a, sizeof a);
    }
    for (size_t i = 0; i < mats.size(); i++) {
        CMat m{mats[i].ia_off, mats[i].ja_off, mats[i].a_off, mats[i].shift, mats[i].rows, {0, 0, 0}};
        memcpy(img.data() + o_mat + i * sizeof(CMat), &m, sizeof m);
    }
    memcpy(img.data() + o_st, cst.data(), cst.size() * sizeof(CStep<T>));
    memcpy(img.data() + o_first, first.data(), first.size() * 4);
    if (!copies.empty()) memcpy(img.data() + o_cp, copies.data(), copies.size() * sizeof(CCopy));
    CK(cudaMemcpy(out.p, img.data(), total, cudaMemcpyHostToDevice));
    cs_out = cs;
    smem_out = used;
    return true;
}

template unsigned cluster_level_size<double>(uint32_t);
template unsigned cluster_level_size<float>(uint32_t);
template void launch_cluster_level<double>(const CProg<double>*, uint32_t, uint32_t, cudaStream_t);
template void launch_cluster_level<float>(const CProg<float>*, uint32_t, uint32_t, cudaStream_t);
template bool cluster_prog_build<double>(const std::vector<PStep<double>>&, const double*, double*, uint32_t,
                                         const std::vector<ClusterVec>&, DBuf<uint8_t>&, uint32_t&, uint32_t&,
                                         cudaStream_t);
template bool cluster_prog_build<float>(const std::vector<PStep<float>>&, const float*, float*, uint32_t,
                                        const std::vector<ClusterVec>&, DBuf<uint8_t>&, uint32_t&, uint32_t&,
                                        cudaStream_t);

}  // namespace mlp
