// Shared-memory-resident solve of the small coarse levels (small.cuh).
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "small.cuh"

namespace mlp {

// ---------------------------------------------------------------------------
// Device side. Every helper is executed by the whole CTA and ends with a
// barrier, so the recursion below keeps all threads in step.
// ---------------------------------------------------------------------------
template <class P>
__device__ __forceinline__ P* at(uint8_t* sm, uint32_t off) {
    return reinterpret_cast<P*>(sm + off);
}

template <class T>
__device__ void s_lsolve(const SLevel& L, uint8_t* sm, const T* src, T* w) {
    const uint32_t* lwo = at<uint32_t>(sm, L.o_lwo);
    const uint32_t* ia = at<uint32_t>(sm, L.o_Lia);
    const uint32_t* ja = at<uint32_t>(sm, L.o_Lja);
    const T* a = at<T>(sm, L.o_La);
    for (uint32_t d = 0; d < L.nwl; d++) {
        for (uint32_t q = lwo[d] + threadIdx.x; q < lwo[d + 1]; q += blockDim.x) {
            T s = src[q];
            for (uint32_t j = ia[q]; j < ia[q + 1]; j++) s -= a[j] * w[ja[j]];
            w[q] = s;
        }
        __syncthreads();
    }
}

template <class T>
__device__ void s_coarse_diag(const SLevel& L, uint8_t* sm, const T* src, T* w, T* out) {
    const uint32_t* ia = at<uint32_t>(sm, L.o_Lia);
    const uint32_t* ja = at<uint32_t>(sm, L.o_Lja);
    const T* a = at<T>(sm, L.o_La);
    const T* dv = at<T>(sm, L.o_dval);
    uint32_t R = L.N - L.Md;
    for (uint32_t q = L.M + threadIdx.x; q < L.N; q += blockDim.x) {
        if (q < R) {
            T s = src[q];
            for (uint32_t j = ia[q]; j < ia[q + 1]; j++) s -= a[j] * w[ja[j]];
            w[q] = s;
        } else {
            out[q] = dv[q - R] * src[q];
        }
    }
    __syncthreads();
}

template <class T>
__device__ void s_usolve(const SLevel& L, uint8_t* sm, const T* w, T* out) {
    const uint32_t* uwo = at<uint32_t>(sm, L.o_uwo);
    const uint32_t* rows = at<uint32_t>(sm, L.o_uwr);
    const uint32_t* ia = at<uint32_t>(sm, L.o_Uia);
    const uint32_t* ja = at<uint32_t>(sm, L.o_Uja);
    const T* a = at<T>(sm, L.o_Ua);
    for (uint32_t d = 0; d < L.nwu; d++) {
        for (uint32_t t = uwo[d] + threadIdx.x; t < uwo[d + 1]; t += blockDim.x) {
            uint32_t q = rows[t];
            uint32_t rs = ia[q];
            T z = w[q];
            for (uint32_t j = rs + 1; j < ia[q + 1]; j++) z -= a[j] * out[ja[j]];
            out[q] = z / a[rs];
        }
        __syncthreads();
    }
}

// r = f - A x (A given by offsets)
template <class T>
__device__ void s_resid(uint32_t n, uint8_t* sm, uint32_t oia, uint32_t oja, uint32_t oa, const T* f, const T* x,
                        T* r) {
    const uint32_t* ia = at<uint32_t>(sm, oia);
    const uint32_t* ja = at<uint32_t>(sm, oja);
    const T* a = at<T>(sm, oa);
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        T s = 0;
        for (uint32_t j = ia[i]; j < ia[i + 1]; j++) s += a[j] * x[ja[j]];
        r[i] = f[i] - s;
    }
    __syncthreads();
}

template <class T>
__device__ void s_dense(const SLevel& L, uint8_t* sm, const T* f, T* x) {
    const T* C = at<T>(sm, L.o_cinv);
    uint32_t n = L.N;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        T s = 0;
        for (uint32_t j = 0; j < n; j++) s += C[(size_t)i * n + j] * f[j];
        x[i] = s;
    }
    __syncthreads();
}

// MultiSplitPrec::solve(level, f, x) (multi_split_solve.cc:59-157)
template <class T>
__device__ void s_ms(const SBlob& D, uint8_t* sm, uint32_t l, const T* f, T* x) {
    const SLevel& L = D.lv[l];
    if (L.direct) { s_dense(L, sm, f, x); return; }
    T* w = at<T>(sm, L.o_w);
    bool next = l + 1 < D.nlev && L.n;
    s_lsolve(L, sm, f, w);
    s_coarse_diag(L, sm, f, w, x);
    if (next) s_ms(D, sm, l + 1, w + L.M, x + L.M);
    s_usolve(L, sm, w, x);
    if (L.niter < 2) return;
    T* r = at<T>(sm, L.o_r);
    T* u0 = at<T>(sm, L.o_u0);
    for (uint32_t it = 2; it <= L.niter; it++) {
        s_resid(L.N, sm, L.o_Aia, L.o_Aja, L.o_Aa, f, x, r);
        s_lsolve(L, sm, r, w);
        s_coarse_diag(L, sm, r, w, u0);
        if (next) s_ms(D, sm, l + 1, w + L.M, u0 + L.M);
        s_usolve(L, sm, w, u0);
        for (uint32_t i = threadIdx.x; i < L.N; i += blockDim.x) x[i] += u0[i];
        __syncthreads();
    }
}

// Prec::solve(level, f, x) (cheb_solve.cc:13-123). The residual is formed as
// F - A u1 and the sign folded into ch_alpha (the operator is linear).
template <class T>
__device__ void s_ch(const SBlob& D, uint8_t* sm, uint32_t l, const T* f, T* x) {
    const SLevel& L = D.lv[l];
    T* w = at<T>(sm, L.o_w);
    s_lsolve(L, sm, f, w);
    s_coarse_diag(L, sm, f, w, x);
    if (l + 1 < D.nlev) {
        const SLevel& Ln = D.lv[l + 1];
        uint32_t n = Ln.N, nch = L.ncheb;
        const T* F = w + L.M;
        T* u0 = at<T>(sm, L.o_cu0);
        T* u1 = at<T>(sm, L.o_cu1);
        T* x2 = at<T>(sm, L.o_cx2);
        T* tmp = at<T>(sm, L.o_ctmp);
        T a1 = (T)L.ch_a1;
        T* first = nch > 1 ? u1 : x2;
        s_ch(D, sm, l + 1, F, first);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) first[i] *= a1;
        __syncthreads();
        if (nch > 1) {
            s_resid(n, sm, Ln.o_Sia, Ln.o_Sja, Ln.o_Sa, F, u1, tmp);
            s_ch(D, sm, l + 1, tmp, x2);
            T al = (T)L.ch_alpha[2], c = (T)L.ch_beta[2];
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) x2[i] = x2[i] * al + c * u1[i];
            __syncthreads();
        }
        for (uint32_t k = 3; k <= nch; k++) {
            T* t = u0; u0 = u1; u1 = x2; x2 = t;
            s_resid(n, sm, Ln.o_Sia, Ln.o_Sja, Ln.o_Sa, F, u1, tmp);
            s_ch(D, sm, l + 1, tmp, x2);
            T al = (T)L.ch_alpha[k], be = (T)L.ch_beta[k];
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
                x2[i] = u1[i] - al * x2[i] + be * (u1[i] - u0[i]);
            __syncthreads();
        }
        T* xo = x + L.M;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) xo[i] = x2[i];
        __syncthreads();
    }
    s_usolve(L, sm, w, x);
}

template <class T>
__global__ void __launch_bounds__(SMALL_THREADS) k_small(const SBlob* __restrict__ gdesc,
                                                         const uint8_t* __restrict__ gblob,
                                                         const T* __restrict__ f, T* __restrict__ x) {
    extern __shared__ __align__(16) uint8_t sm[];
    __shared__ __align__(16) SBlob D;
    pdl_wait();
    pdl_trigger();
    {
        const int4* src = reinterpret_cast<const int4*>(gdesc);
        int4* dst = reinterpret_cast<int4*>(&D);
        for (uint32_t i = threadIdx.x; i < sizeof(SBlob) / 16; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    {
        const int4* src = reinterpret_cast<const int4*>(gblob);
        int4* dst = reinterpret_cast<int4*>(sm);
        uint32_t n16 = D.bytes_static / 16;
        for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
        T* sf = at<T>(sm, D.o_f);
        for (uint32_t i = threadIdx.x; i < D.lv[0].N; i += blockDim.x) sf[i] = f[i];
    }
    __syncthreads();
    T* sx = at<T>(sm, D.o_x);
    if (D.kind == PREC_MSPLIT) s_ms<T>(D, sm, 0, at<T>(sm, D.o_f), sx);
    else s_ch<T>(D, sm, 0, at<T>(sm, D.o_f), sx);
    for (uint32_t i = threadIdx.x; i < D.lv[0].N; i += blockDim.x) x[i] = sx[i];
}

// Tabulates the small solve: block j solves with e_j and writes column j of
// the N0 x N0 row-major operator.
template <class T>
__global__ void __launch_bounds__(SMALL_THREADS) k_small_columns(const SBlob* __restrict__ gdesc,
                                                                 const uint8_t* __restrict__ gblob,
                                                                 T* __restrict__ S) {
    extern __shared__ __align__(16) uint8_t sm[];
    __shared__ __align__(16) SBlob D;
    {
        const int4* src = reinterpret_cast<const int4*>(gdesc);
        int4* dst = reinterpret_cast<int4*>(&D);
        for (uint32_t i = threadIdx.x; i < sizeof(SBlob) / 16; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    uint32_t n = D.lv[0].N, col = blockIdx.x;
    {
        const int4* src = reinterpret_cast<const int4*>(gblob);
        int4* dst = reinterpret_cast<int4*>(sm);
        uint32_t n16 = D.bytes_static / 16;
        for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
        T* sf = at<T>(sm, D.o_f);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sf[i] = (i == col) ? T(1) : T(0);
    }
    __syncthreads();
    T* sx = at<T>(sm, D.o_x);
    if (D.kind == PREC_MSPLIT) s_ms<T>(D, sm, 0, at<T>(sm, D.o_f), sx);
    else s_ch<T>(D, sm, 0, at<T>(sm, D.o_f), sx);
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) S[(size_t)i * n + col] = sx[i];
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
uint32_t small_smem_limit() {
    static int lim = -1;
    if (lim < 0) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    }
    return (uint32_t)lim;
}

static bool is_eq1(double a) { return std::fabs(a - 1.0) <= 2.220446049250313e-16; }

template <class T>
static const T* tvals(const DCSR& m);
template <>
const double* tvals<double>(const DCSR& m) { return m.a.p; }
template <>
const float* tvals<float>(const DCSR& m) { return m.a32.p; }

namespace {
struct Packer {
    uint32_t cur = 0;
    struct Item { uint32_t off; const void* src; size_t bytes; };
    std::vector<Item> items;
    uint32_t add(const void* src, size_t bytes) {
        cur = (cur + 15u) & ~15u;
        uint32_t off = cur;
        if (src && bytes) items.push_back({off, src, bytes});
        cur += (uint32_t)bytes;
        return off;
    }
    uint32_t reserve(size_t bytes) { return add(nullptr, bytes); }
};
}  // namespace

template <class T>
static bool pack(Hierarchy& H, uint32_t first, SmallPlan<T>& sp, uint32_t budget, bool dry,
                 std::vector<DBuf<uint32_t>>& keep, cudaStream_t s) {
    uint32_t nl = H.nlevels - first;
    if (nl > (uint32_t)SMALL_MAXLEV) return false;
    SBlob h;
    memset(&h, 0, sizeof h);
    h.kind = H.kind;
    h.nlev = nl;
    Packer pk;
    const size_t sT = sizeof(T);
    for (uint32_t k = 0; k < nl; k++) {
        Level& L = *H.lv[first + k];
        SLevel& d = h.lv[k];
        d.N = L.N; d.M = L.M; d.Md = L.Md; d.n = L.n; d.niter = L.niter; d.ncheb = L.ncheb;
        d.direct = L.direct;
        if (L.direct) {
            if ((size_t)L.N * L.N * sT > budget) return false;
            const T* C = std::is_same<T, double>::value ? (const T*)L.cinv.p : (const T*)L.cinv32.p;
            d.o_cinv = pk.add(C, (size_t)L.N * L.N * sT);
            continue;
        }
        uint32_t R = L.N - L.Md;
        if (H.kind == PREC_MSPLIT && L.niter >= 2) {
            d.o_Aia = pk.add(L.Af.ia.p, ((size_t)L.N + 1) * 4);
            d.o_Aja = pk.add(L.Af.ja.p, (size_t)L.Af.nnz * 4);
            d.o_Aa = pk.add(tvals<T>(L.Af), (size_t)L.Af.nnz * sT);
        }
        if (H.kind == PREC_CHEB && k > 0) {
            d.o_Sia = pk.add(L.As.ia.p, ((size_t)L.N + 1) * 4);
            d.o_Sja = pk.add(L.As.ja.p, (size_t)L.As.nnz * 4);
            d.o_Sa = pk.add(tvals<T>(L.As), (size_t)L.As.nnz * sT);
        }
        d.o_Lia = pk.add(L.Lf.ia.p, ((size_t)R + 1) * 4);
        d.o_Lja = pk.add(L.Lf.ja.p, (size_t)L.Lf.nnz * 4);
        d.o_La = pk.add(tvals<T>(L.Lf), (size_t)L.Lf.nnz * sT);
        if (L.M) {
            d.o_Uia = pk.add(L.Uf.ia.p, ((size_t)L.M + 1) * 4);
            d.o_Uja = pk.add(L.Uf.ja.p, (size_t)L.Uf.nnz * 4);
            d.o_Ua = pk.add(tvals<T>(L.Uf), (size_t)L.Uf.nnz * sT);
        }
        const T* dv = std::is_same<T, double>::value ? (const T*)L.dval.p : (const T*)L.dval32.p;
        d.o_dval = pk.add(dv, (size_t)L.Md * sT);
        d.nwl = L.lw_off.empty() ? 0 : (uint32_t)L.lw_off.size() - 1;
        d.nwu = L.uw_off.empty() ? 0 : (uint32_t)L.uw_off.size() - 1;
        // wavefront offsets live on the host: stage them on the device for the copy
        if (!dry) {
            keep.emplace_back(L.lw_off.size() + 1);
            if (!L.lw_off.empty()) keep.back().upload(L.lw_off.data(), L.lw_off.size(), s);
            d.o_lwo = pk.add(keep.back().p, L.lw_off.size() * 4);
            keep.emplace_back(L.uw_off.size() + 1);
            if (!L.uw_off.empty()) keep.back().upload(L.uw_off.data(), L.uw_off.size(), s);
            d.o_uwo = pk.add(keep.back().p, L.uw_off.size() * 4);
        } else {
            d.o_lwo = pk.reserve(L.lw_off.size() * 4);
            d.o_uwo = pk.reserve(L.uw_off.size() * 4);
        }
        if (L.M) d.o_uwr = pk.add(L.uw_rows.p, (size_t)L.M * 4);
        // Chebyshev coefficients (cheb_solve.cc:51-100), computed exactly as the plan does
        if (H.kind == PREC_CHEB && first + k + 1 < H.nlevels) {
            if (L.ncheb > (uint32_t)SMALL_MAXCHEB) return false;
            Level& Ln = *H.lv[first + k + 1];
            double lmin = Ln.lmin, lmax = Ln.lmax;
            double eta = (lmax + lmin) / (lmax - lmin);
            double alpha = 2 / (lmax + lmin);
            d.ch_a1 = is_eq1(alpha) ? 1.0 : alpha;
            if (L.ncheb > 1) {
                alpha = 4 / (lmax - lmin) * cheb_poly(eta, 1) / cheb_poly(eta, 2);
                double beta = cheb_poly(eta, 0) / cheb_poly(eta, 2);
                d.ch_alpha[2] = alpha;
                d.ch_beta[2] = is_eq1(1 + beta) ? 1.0 : 1 + beta;
            }
            for (uint32_t i = 3; i <= L.ncheb; i++) {
                d.ch_alpha[i] = -(4 / (lmax - lmin) * cheb_poly(eta, i - 1) / cheb_poly(eta, i));
                d.ch_beta[i] = cheb_poly(eta, i - 2) / cheb_poly(eta, i);
            }
        }
    }
    h.bytes_static = (pk.cur + 15u) & ~15u;
    // work vectors
    for (uint32_t k = 0; k < nl; k++) {
        Level& L = *H.lv[first + k];
        SLevel& d = h.lv[k];
        if (L.direct) continue;
        d.o_w = pk.reserve((size_t)(L.N - L.Md) * sT);
        if (H.kind == PREC_MSPLIT && L.niter >= 2) {
            d.o_r = pk.reserve((size_t)L.N * sT);
            d.o_u0 = pk.reserve((size_t)L.N * sT);
        }
        if (H.kind == PREC_CHEB && first + k + 1 < H.nlevels) {
            size_t n = L.n;
            d.o_cu0 = pk.reserve(n * sT);
            d.o_cu1 = pk.reserve(n * sT);
            d.o_cx2 = pk.reserve(n * sT);
            d.o_ctmp = pk.reserve(n * sT);
        }
    }
    uint32_t N0 = H.lv[first]->N;
    h.o_f = pk.reserve((size_t)N0 * sT);
    h.o_x = pk.reserve((size_t)N0 * sT);
    h.bytes_total = (pk.cur + 15u) & ~15u;
    if (h.bytes_total > budget) return false;
    if (dry) return true;
    sp.blob.alloc(h.bytes_static ? h.bytes_static : 16);
    sp.blob.zero(s);
    for (auto& it : pk.items)
        CK(cudaMemcpyAsync(sp.blob.p + it.off, it.src, it.bytes, cudaMemcpyDeviceToDevice, s));
    sp.desc.alloc(1);
    CK(cudaMemcpyAsync(sp.desc.p, &h, sizeof h, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    sp.h = h;
    sp.first = first;
    sp.N0 = N0;
    return true;
}

template <class T>
void build_small(Hierarchy& H, SmallPlan<T>& sp, uint32_t budget, cudaStream_t s) {
    std::vector<DBuf<uint32_t>> keep;
    uint32_t limit = small_smem_limit();
    uint32_t stat = (uint32_t)sizeof(SBlob) + 1024;
    if (limit <= stat) return;
    budget = std::min(budget, limit - stat);
    // deepest-first search for the largest sub-hierarchy that fits
    int best = -1;
    for (int l = (int)H.nlevels - 1; l >= 0; l--) {
        if (H.lv[l]->N > 16384) break;
        if (pack<T>(H, (uint32_t)l, sp, budget, true, keep, s)) best = l;
        else break;
    }
    if (best < 0) return;
    if (!pack<T>(H, (uint32_t)best, sp, budget, false, keep, s)) return;
    // The attribute belongs to the kernel, not to this plan: several plans (of
    // different sizes) live in one process, so it is set once to the largest
    // size any plan may use and never lowered.
    static int set_for[2] = {0, 0};
    int& done = set_for[std::is_same<T, double>::value ? 0 : 1];
    if (!done) {
        int mx = (int)(limit - stat);
        CK(cudaFuncSetAttribute(k_small<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
        CK(cudaFuncSetAttribute(k_small_columns<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
        done = 1;
    }
    // The recursive solve nests one call per level (about 150 bytes of stack
    // each); raise the per-thread stack limit when the default is too small.
    size_t need = 256 + (size_t)(sp.h.nlev + 2) * 256, cur = 0;
    CK(cudaDeviceGetLimit(&cur, cudaLimitStackSize));
    if (cur < need) CK(cudaDeviceSetLimit(cudaLimitStackSize, need));
    // tabulate the operator when it is small (MLP_DENSE_OP_MAX overrides the
    // largest size, 0 turns tabulation off)
    uint32_t dmax = 2048;
    if (const char* e = getenv("MLP_DENSE_OP_MAX")) dmax = (uint32_t)strtoul(e, nullptr, 10);
    if (sp.N0 && sp.N0 <= dmax) {
        sp.dense.alloc((size_t)sp.N0 * sp.N0);
        k_small_columns<T><<<sp.N0, SMALL_THREADS, sp.h.bytes_total, s>>>(sp.desc.p, sp.blob.p, sp.dense.p);
        CK_LAUNCH();
        CK(cudaStreamSynchronize(s));
    }
}

template <class T>
void launch_small(const SmallPlan<T>& sp, const T* f, T* x, cudaStream_t s) {
    launch_k(k_small<T>, 1, SMALL_THREADS, sp.h.bytes_total, s, (const SBlob*)sp.desc.p,
             (const uint8_t*)sp.blob.p, f, x);
}

template void build_small<double>(Hierarchy&, SmallPlan<double>&, uint32_t, cudaStream_t);
template void build_small<float>(Hierarchy&, SmallPlan<float>&, uint32_t, cudaStream_t);
template void launch_small<double>(const SmallPlan<double>&, const double*, double*, cudaStream_t);
template void launch_small<float>(const SmallPlan<float>&, const float*, float*, cudaStream_t);

}  // namespace mlp
