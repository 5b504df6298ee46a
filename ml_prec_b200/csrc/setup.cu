// Hierarchy construction kernels (marking, ordering, sparse Schur elimination,
// matrix assembly). Compiled with -fmad=false: every floating-point expression
// rounds exactly as the reference's x86-64 SSE2 build does (no contraction into
// FMA), so every integer decision taken on a floating-point comparison (which
// link is dropped, the node ordering, the coarse sparsity pattern) and every
// factor value come out bit-identical to the reference.
#include "setup.cuh"
#include "solve.cuh"

namespace mlp {

// ---------------------------------------------------------------------------
// SPE 7-point assembly (spe.cc:69-131, XYZ order). Row i = (x, y, z) has the
// diagonal first (initialised to c) followed by the existing neighbours in the
// order -z, -y, -x, +x, +y, +z; each link value v = 2/(1/k_i + 1/k_j)/(h*h) is
// stored as -v and added to the diagonal in that order. The permeability field
// is addressed like SPEMesh::index_k (mesh.h:57-59), i.e. modulo 60x220x85.
// Dirichlet x-faces (benchmark problem): diag += 2*kx/hx^2 at x = 0 and
// x = nx-1 (in that order), b = that value at x = 0 (p = 1), 0 elsewhere.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t kidx(uint32_t i, uint32_t j, uint32_t k) {
    return (k * 13200u + j * 60u + i) % 1122000u;
}

__global__ void k_spe_rowlen(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t* len) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t N = nx * ny * nz;
    if (r >= N) return;
    uint32_t i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
    len[r] = 1 + (k > 0) + (j > 0) + (i > 0) + (i + 1 < nx) + (j + 1 < ny) + (k + 1 < nz);
}

__device__ __forceinline__ double spe_link(const double* K, uint32_t a, uint32_t b, double h) {
    return 2 / (1 / K[a] + 1 / K[b]) / (h * h);
}

__global__ void k_spe_fill(uint32_t nx, uint32_t ny, uint32_t nz, const double* __restrict__ kx,
                           const double* __restrict__ ky, const double* __restrict__ kz, double c,
                           int dirichlet, const uint32_t* __restrict__ ia, uint32_t* __restrict__ ja,
                           double* __restrict__ a, double* __restrict__ b) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t N = nx * ny * nz;
    if (r >= N) return;
    const double hx = 20, hy = 10, hz = 2;
    uint32_t i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
    uint32_t p = ia[r];
    uint32_t dind = p;
    uint32_t me = kidx(i, j, k);
    double diag = c;
    ja[p++] = r;
    if (k) { double v = spe_link(kz, me, kidx(i, j, k - 1), hz); ja[p] = r - nx * ny; a[p++] = -v; diag += v; }
    if (j) { double v = spe_link(ky, me, kidx(i, j - 1, k), hy); ja[p] = r - nx; a[p++] = -v; diag += v; }
    if (i) { double v = spe_link(kx, me, kidx(i - 1, j, k), hx); ja[p] = r - 1; a[p++] = -v; diag += v; }
    if (i + 1 < nx) { double v = spe_link(kx, me, kidx(i + 1, j, k), hx); ja[p] = r + 1; a[p++] = -v; diag += v; }
    if (j + 1 < ny) { double v = spe_link(ky, me, kidx(i, j + 1, k), hy); ja[p] = r + nx; a[p++] = -v; diag += v; }
    if (k + 1 < nz) { double v = spe_link(kz, me, kidx(i, j, k + 1), hz); ja[p] = r + nx * ny; a[p++] = -v; diag += v; }
    double bb = 0;
    if (dirichlet) {
        double tD = 2 * kx[me] / (hx * hx);
        if (i == 0) { diag += tD; bb += tD * 1.0; }
        if (i == nx - 1) diag += tD;
    }
    a[dind] = diag;
    if (b) b[r] = bb;
}

void spe_assemble(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx, const double* ky,
                  const double* kz, double c, int dirichlet, DCSR& A, double* b, cudaStream_t s) {
    ArenaScope arena;
    uint32_t N = nx * ny * nz;
    Tmp<uint32_t> len(N);
    k_spe_rowlen<<<grid_for(N, 256), 256, 0, s>>>(nx, ny, nz, len.p);
    CK_LAUNCH();
    A.ia.alloc((size_t)N + 1);
    uint32_t nnz = exclusive_scan_u32(len.p, A.ia.p, N, s);
    A.nrow = A.ncol = N;
    A.nnz = nnz;
    A.ja.alloc(nnz);
    A.a.alloc(nnz);
    k_spe_fill<<<grid_for(N, 256), 256, 0, s>>>(nx, ny, nz, kx, ky, kz, c, dirichlet, A.ia.p, A.ja.p,
                                               A.a.p, b);
    CK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Marking.
// Stable ascending order of a row's off-diagonals by |a| (the insertion sort of
// multi_split_constr.cc:26-36 / cheb_constr.cc:155-165: strict '>' keeps equal
// magnitudes in ja order). Rows are short (7-point stencil and its Schur
// complements), so each thread sorts its row in a local array of MAXR entries;
// longer rows set the overflow flag and the host reports ERR_LIMIT.
// ---------------------------------------------------------------------------
static constexpr int MAXR = 64;

__device__ __forceinline__ int sort_row(const double* __restrict__ a, uint32_t rs, uint32_t nrz,
                                        uint8_t* idx) {
    if (nrz > MAXR) return -1;
    for (uint32_t t = 0; t < nrz; t++) {
        double v = fabs(a[rs + 1 + t]);
        int j = (int)t - 1;
        while (j >= 0 && fabs(a[rs + 1 + idx[j]]) > v) { idx[j + 1] = idx[j]; j--; }
        idx[j + 1] = (uint8_t)t;
    }
    return 0;
}

// Multi-split q-threshold link dropping (multi_split_constr.cc:65-113):
// aux = a_ii + sum_j a_ij (ja order); s = q/(1-q)*aux; walk the off-diagonals by
// increasing |a|, dropping link (i,j) while -a_ij <= s (s -= -a_ij); then
// aux *= 1/(1-q). keep[j_] = 0 for dropped links; nout = kept links of the row;
// nin[j] = number of kept links pointing to j.
__global__ void k_mark_msplit(uint32_t N, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                              const double* __restrict__ a, double q, uint8_t* __restrict__ keep,
                              int* __restrict__ nout, int* __restrict__ nin, double* __restrict__ aux,
                              int* __restrict__ err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint32_t rs = ia[i], re = ia[i + 1], nrz = re - rs - 1;
    double ax = a[rs];
    for (uint32_t j_ = rs + 1; j_ < re; j_++) ax += a[j_];
    uint8_t idx[MAXR];
    if (sort_row(a, rs, nrz, idx)) { atomicOr(err, 1); return; }
    uint64_t drop = 0;
    int no = (int)nrz;
    double s = q / (1 - q) * ax;
    for (uint32_t t = 0; t < nrz; t++) {
        uint32_t j_ = rs + 1 + idx[t];
        double aij = -a[j_];
        if (aij <= s) {
            drop |= 1ull << idx[t];
            no--;
            s -= aij;
        } else
            break;
    }
    keep[rs] = 1;
    for (uint32_t t = 0; t < nrz; t++) {
        uint32_t j_ = rs + 1 + t;
        bool kp = !((drop >> t) & 1ull);
        keep[j_] = kp;
        if (kp) atomicAdd(&nin[ja[j_]], 1);
    }
    nout[i] = no;
    aux[i] = ax * (1. / (1 - q));
}

// uh_cheb two-ended marking (cheb_constr.cc:191-232 with to_remove,
// cheb_prec.h:57-85): aux = sum of the row (diagonal first, ja order); walk the
// off-diagonals by increasing |a| accumulating t = -2v/(aux*(beta-1)) while
// s + t <= 1; each such link is marked from this end (want[j_] = 1). A link is
// removed when both of its ends marked it (LinkTypeCheb::mark, cheb_misc.h:73).
__global__ void k_mark_cheb(uint32_t N, const uint32_t* __restrict__ ia, const double* __restrict__ a,
                            double beta, uint8_t* __restrict__ want, double* __restrict__ aux,
                            int* __restrict__ err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint32_t rs = ia[i], re = ia[i + 1], nrz = re - rs - 1;
    double ax = 0.0;
    for (uint32_t j_ = rs; j_ < re; j_++) ax += a[j_];
    uint8_t idx[MAXR];
    if (sort_row(a, rs, nrz, idx)) { atomicOr(err, 1); return; }
    for (uint32_t j_ = rs; j_ < re; j_++) want[j_] = 0;
    double s = 0.;
    for (uint32_t t = 0; t < nrz; t++) {
        double v = a[rs + 1 + idx[t]];
        double tt = -2 * v / (ax * (beta - 1));
        if (s + tt > 1) break;
        s += tt;
        want[rs + 1 + idx[t]] = 1;
    }
    aux[i] = ax;
}

// Transpose position of every off-diagonal: tpos[j_] = position of (j, i) in
// row j (binary search over the sorted off-diagonal part, skyline.cc:15-28).
__global__ void k_transpose_pos(uint32_t N, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                                uint32_t* __restrict__ tpos, int* __restrict__ err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    for (uint32_t j_ = ia[i] + 1; j_ < ia[i + 1]; j_++) {
        uint32_t j = ja[j_];
        uint32_t lo = ia[j] + 1, hi = ia[j + 1];
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (ja[mid] < i) lo = mid + 1; else hi = mid;
        }
        if (lo < ia[j + 1] && ja[lo] == i) tpos[j_] = lo;
        else { tpos[j_] = 0xffffffffu; atomicOr(err, 2); }
    }
}

// Link state after the two-ended marking: keep = not marked from both ends;
// nlinks = kept links of the row; slot[j_] = upper-triangle position of the link
// (where LinkTypeCheb keeps its counter).
__global__ void k_cheb_links(uint32_t N, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                             const uint8_t* __restrict__ want, const uint32_t* __restrict__ tpos,
                             uint8_t* __restrict__ keep, int* __restrict__ nlinks, uint32_t* __restrict__ slot) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int nl = 0;
    keep[ia[i]] = 1;
    for (uint32_t j_ = ia[i] + 1; j_ < ia[i + 1]; j_++) {
        uint32_t t = tpos[j_];
        bool removed = want[j_] && want[t];
        keep[j_] = !removed;
        nl += !removed;
        slot[j_] = ja[j_] > i ? j_ : t;
    }
    nlinks[i] = nl;
}

// ---------------------------------------------------------------------------
// Stable bucket partition (the node orderings). Every node gets a bucket id
// (< NB, or NONE to skip it); nodes are written bucket by bucket, keeping index
// order inside a bucket, or reversed order for buckets flagged in rev_mask
// (the reference fills the diagonal group from the end: map[eind--]).
// ---------------------------------------------------------------------------
static constexpr int PT = 1024;  // nodes per partition tile

__global__ void k_part_count(uint32_t N, const uint8_t* __restrict__ bucket, int NB, uint32_t ntile,
                             uint32_t* __restrict__ counts) {
    __shared__ uint32_t c[8];
    if (threadIdx.x < 8) c[threadIdx.x] = 0;
    __syncthreads();
    uint32_t i = blockIdx.x * PT + threadIdx.x;
    if (i < N && bucket[i] < NB) atomicAdd(&c[bucket[i]], 1u);
    __syncthreads();
    if (threadIdx.x < (unsigned)NB) counts[threadIdx.x * ntile + blockIdx.x] = c[threadIdx.x];
}

__global__ void k_part_scatter(uint32_t N, const uint8_t* __restrict__ bucket, int NB, uint32_t ntile,
                               const uint32_t* __restrict__ offs, uint32_t base, uint32_t rev_mask,
                               const uint32_t* __restrict__ bucket_total_start, uint32_t* __restrict__ map) {
    __shared__ uint32_t wcnt[8][PT / 32];
    uint32_t i = blockIdx.x * PT + threadIdx.x;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int b = (i < N) ? bucket[i] : 255;
    uint32_t myrank = 0;
    for (int v = 0; v < NB; v++) {
        unsigned m = __ballot_sync(0xffffffffu, b == v);
        if (b == v) myrank = __popc(m & ((1u << lane) - 1));
        if (lane == 0) wcnt[v][w] = __popc(m);
    }
    __syncthreads();
    if (b < NB) {
        uint32_t before = 0;
        for (int ww = 0; ww < w; ww++) before += wcnt[b][ww];
        uint32_t r = offs[b * ntile + blockIdx.x] + before + myrank;  // rank over all nodes
        uint32_t bstart = bucket_total_start[b];                       // start of bucket b
        uint32_t bend = bucket_total_start[b + 1];
        uint32_t inb = r - bstart;
        uint32_t pos = ((rev_mask >> b) & 1u) ? (bend - 1 - inb) : r;
        map[base + pos] = i;
    }
}

__global__ void k_bucket_starts(const uint32_t* offs, uint32_t ntile, int NB, uint32_t total, uint32_t* starts) {
    if (threadIdx.x == 0) {
        for (int v = 0; v < NB; v++) starts[v] = offs[v * ntile];
        starts[NB] = total;
    }
}

// Writes map[base + ...] for every node whose bucket < NB; returns the count of
// each bucket (host side, synchronises).
std::vector<uint32_t> stable_partition(uint32_t N, const uint8_t* bucket, int NB, uint32_t rev_mask,
                                       uint32_t* map, uint32_t base, cudaStream_t s) {
    uint32_t ntile = (N + PT - 1) / PT;
    if (!ntile) ntile = 1;
    Tmp<uint32_t> counts((size_t)NB * ntile + 1), offs((size_t)NB * ntile + 1), starts(NB + 1);
    counts.zero(s);
    k_part_count<<<ntile, PT, 0, s>>>(N, bucket, NB, ntile, counts.p);
    CK_LAUNCH();
    uint32_t total = exclusive_scan_u32(counts.p, offs.p, NB * ntile, s);
    k_bucket_starts<<<1, 32, 0, s>>>(offs.p, ntile, NB, total, starts.p);
    CK_LAUNCH();
    k_part_scatter<<<ntile, PT, 0, s>>>(N, bucket, NB, ntile, offs.p, base, rev_mask, starts.p, map);
    CK_LAUNCH();
    std::vector<uint32_t> st = starts.download(s);
    std::vector<uint32_t> cnt(NB);
    for (int v = 0; v < NB; v++) cnt[v] = st[v + 1] - st[v];
    return cnt;
}

// Bucket ids of order_simple_1 (multi_split_mark.cc:156-191):
// 0: out = 0 and in != 0, 1: out = 1, 2: out = 2, 3: out > 2, 4: out = 0 and in = 0.
__global__ void k_bucket_simple1(uint32_t N, const int* __restrict__ nout, const int* __restrict__ nin,
                                 uint8_t* __restrict__ bucket) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int o = nout[i];
    uint8_t b;
    if (o == 0) b = nin[i] != 0 ? 0 : 4;
    else b = o <= 2 ? (uint8_t)o : 3;
    bucket[i] = b;
}

// Bucket ids of order_none (multi_split_mark.cc:8-25): 0 linked, 1 isolated.
__global__ void k_bucket_none(uint32_t N, const int* __restrict__ nout, const int* __restrict__ nin,
                              uint8_t* __restrict__ bucket) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    bucket[i] = (nin[i] == 0 && nout[i] == 0) ? 1 : 0;
}

// Buckets of order_original after its tail group (multi_split_mark.cc:120-151):
// 0: group 2 (in <= 2 or out <= 2, index order), 1: still linked (index
// order), 2: no links (reversed); marked tail nodes are skipped.
__global__ void k_bucket_original(uint32_t N, const int* __restrict__ nout, const int* __restrict__ nin,
                                  const uint8_t* __restrict__ marked, uint8_t* __restrict__ bucket) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint8_t b;
    if (marked[i]) b = 255;
    else if (nin[i] <= 2 || nout[i] <= 2) b = 0;
    else b = (nin[i] == 0 && nout[i] == 0) ? 2 : 1;
    bucket[i] = b;
}

// order_block (multi_split_mark.cc:193-252) on the 60x220x85 mesh: the inner
// nodes of the 5x5x5 blocks (i, j, k not on a block face) that keep a link,
// block after block (K, J, I) and inside a block in (k, j, i) order. Thread p
// takes the p-th inner position of that order and flags whether it is taken;
// a scan of the flags gives each taken node its place in map.
constexpr uint32_t BLK_NX = 60, BLK_NY = 220, BLK_NZ = 85, BLK_B = 5;
constexpr uint32_t BLK_IN = BLK_B - 2;  // inner nodes per block side
constexpr uint32_t BLK_NI = BLK_NX / BLK_B, BLK_NJ = BLK_NY / BLK_B, BLK_NK = BLK_NZ / BLK_B;
constexpr uint32_t BLK_POS = BLK_NI * BLK_NJ * BLK_NK * BLK_IN * BLK_IN * BLK_IN;
static_assert(BLK_NX % BLK_B == 0 && BLK_NY % BLK_B == 0 && BLK_NZ % BLK_B == 0, "whole blocks");

__device__ __forceinline__ uint32_t block_pos_node(uint32_t p) {
    uint32_t t = p % BLK_IN;  // i - I - 1
    uint32_t q = p / BLK_IN;
    uint32_t u = q % BLK_IN;  // j - J - 1
    q /= BLK_IN;
    uint32_t v = q % BLK_IN;  // k - K - 1
    q /= BLK_IN;
    uint32_t I = q % BLK_NI;
    q /= BLK_NI;
    uint32_t J = q % BLK_NJ;
    uint32_t K = q / BLK_NJ;
    uint32_t i = I * BLK_B + 1 + t, j = J * BLK_B + 1 + u, k = K * BLK_B + 1 + v;
    return (k * BLK_NY + j) * BLK_NX + i;
}
__global__ void k_block_flags(const int* __restrict__ nout, const int* __restrict__ nin, uint32_t* __restrict__ flag) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= BLK_POS) return;
    uint32_t id = block_pos_node(p);
    flag[p] = (nin[id] || nout[id]) ? 1u : 0u;
}
__global__ void k_block_place(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                              uint32_t* __restrict__ map, uint8_t* __restrict__ marked) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= BLK_POS || !flag[p]) return;
    uint32_t id = block_pos_node(p);
    map[pos[p]] = id;
    marked[id] = 1;
}
// The remaining nodes of order_block: 0 linked (index order), 1 no links (reversed).
__global__ void k_bucket_rest(uint32_t N, const int* __restrict__ nout, const int* __restrict__ nin,
                              const uint8_t* __restrict__ marked, uint8_t* __restrict__ bucket) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    bucket[i] = marked[i] ? 255 : ((nin[i] == 0 && nout[i] == 0) ? 1 : 0);
}

// Remaining nodes after the uh_cheb tail group (cheb_mark.cc:177-189):
// 0 = still linked (coarse, index order), 1 = no links (diagonal, reversed),
// marked nodes are skipped.
__global__ void k_bucket_cheb_rest(uint32_t N, const int* __restrict__ nlinks, const uint8_t* __restrict__ marked,
                                   uint8_t* __restrict__ bucket) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    bucket[i] = marked[i] ? 255 : (nlinks[i] == 0 ? 1 : 0);
}

__global__ void k_bucket_deg1(uint32_t N, const int* __restrict__ nlinks, uint8_t* __restrict__ bucket) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    bucket[i] = nlinks[i] == 1 ? 0 : 255;
}

// uh_cheb tail group (cheb_mark.cc:121-162). A tail starts at a node with one
// remaining link and follows it while the next node is left with exactly one
// link. Only nodes that start with one link can ever be found with exactly one
// link by the outer scan (a walk that leaves a node with one link continues
// through it), so the scan runs over that candidate list in index order. The
// walk is one ordered greedy pass (each step changes the link counts the next
// reads), so it runs on the host over the marking kernels' link slots: an L2
// round trip per step would make one GPU thread far slower at 1.12 M cells.
// Returns the eliminated nodes in order; nlinks and marked are updated.
static std::vector<uint32_t> cheb_tails(const std::vector<uint32_t>& ia, const std::vector<uint32_t>& ja,
                                        const std::vector<uint32_t>& slot, std::vector<uint8_t> state,
                                        std::vector<int>& nlinks, const std::vector<uint32_t>& cand,
                                        std::vector<uint8_t>& marked) {
    std::vector<uint32_t> order;
    for (uint32_t i0 : cand) {
        if (nlinks[i0] != 1) continue;
        do {
            order.push_back(i0);
            marked[i0] = 1;
            uint32_t j_ = ia[i0] + 1, e = ia[i0 + 1];
            for (; j_ < e; j_++)
                if (state[slot[j_]]) break;
            if (j_ == e) MLP_THROW(ERR_INTERNAL, "Could not find remaining link");
            uint32_t i1 = ja[j_];
            state[slot[j_]] = 0;
            nlinks[i0] = -1;
            nlinks[i1]--;
            i0 = i1;
        } while (nlinks[i0] == 1);
        if (nlinks[i0] == 0) {
            order.push_back(i0);
            marked[i0] = 1;
            nlinks[i0] = -1;
        }
    }
    return order;
}

__global__ void k_rmap(uint32_t N, const uint32_t* __restrict__ map, uint32_t* __restrict__ rmap) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) rmap[map[i]] = i;
}

// ---------------------------------------------------------------------------
// Sparse Schur elimination (construct_sparse_lu, sparse_lu.cc:6-133).
// Each permuted row i < N-Md is processed by one thread in its own slot of
// `cap` (column, value) pairs kept sorted by column. The row is loaded as the
// diagonal aux[map[i]] minus the kept links scaled by 1/beta (ja order), then
// the slot's columns k < min(i, M) are eliminated in increasing order with
// l_ik = w_k / U_kk and the k-th U row's updates, fill allowed. l_ik overwrites
// the value of column k; after the loop the slot holds the L entries first and
// the U row (i < M) or next-level row (i >= M) after them.
// Rows i < M depend on the U rows of the columns they eliminate, so they are
// processed in rounds: a row is finished in round r only if every U row it
// reads finished in an earlier round, otherwise it records the blocking column
// and retries. done[i] (the round number) is therefore one plus the largest
// round among its dependencies: the level schedule of the L solve. Rows >= M
// depend on U rows only and are processed in one pass afterwards.
// ---------------------------------------------------------------------------
struct LUArgs {
    const uint32_t* Aia;
    const uint32_t* Aja;
    const double* Aa;
    const uint8_t* keep;
    const double* aux;
    const uint32_t* map;
    const uint32_t* rmap;
    uint32_t M, R;  // R = N - Md rows are factored
    double beta;
    uint32_t cap;
    uint32_t* scol;
    double* sval;
    uint32_t* slen;
    uint32_t* sldiv;
    int* done;
    uint32_t* wait;
    int* flags;  // bit 0: overflow
};

// 1 = finished, 0 = blocked, -1 = slot overflow
__device__ int lu_row(const LUArgs& g, uint32_t i, int round) {
    const uint32_t cap = g.cap;
    uint32_t* wc = g.scol + (size_t)i * cap;
    double* wv = g.sval + (size_t)i * cap;
    uint32_t arow = g.map[i];
    uint32_t wn = 1;
    wc[0] = i;
    double diag = g.aux[arow];
    for (uint32_t j_ = g.Aia[arow] + 1; j_ < g.Aia[arow + 1]; j_++) {
        if (!g.keep[j_]) continue;
        uint32_t nj = g.rmap[g.Aja[j_]];
        double z = g.Aa[j_] / g.beta;
        if (wn == cap) return -1;
        uint32_t p = wn;
        while (p > 0 && wc[p - 1] > nj) { wc[p] = wc[p - 1]; wv[p] = wv[p - 1]; p--; }
        wc[p] = nj; wv[p] = z; wn++;
        diag -= z;
    }
    for (uint32_t t = 0; t < wn; t++)
        if (wc[t] == i) { wv[t] = diag; break; }
    uint32_t m = i < g.M ? i : g.M;
    uint32_t t = 0;
    for (; t < wn && wc[t] < m; t++) {
        uint32_t k = wc[t];
        int dk = g.done[k];
        if (dk == 0 || dk >= round) { g.wait[i] = k; return 0; }
        const uint32_t* kc = g.scol + (size_t)k * cap;
        const double* kv = g.sval + (size_t)k * cap;
        uint32_t ks = g.sldiv[k], ke = g.slen[k];
        double lik = wv[t] / kv[ks];
        wv[t] = lik;
        uint32_t pos = t + 1;  // columns of U row k are > k and sorted: merge forward
        for (uint32_t u = ks + 1; u < ke; u++) {
            uint32_t j = kc[u];
            double uv = kv[u];
            while (pos < wn && wc[pos] < j) pos++;
            if (pos < wn && wc[pos] == j) {
                wv[pos] = wv[pos] - lik * uv;
            } else {
                if (wn == cap) return -1;
                for (uint32_t q = wn; q > pos; q--) { wc[q] = wc[q - 1]; wv[q] = wv[q - 1]; }
                wc[pos] = j;
                wv[pos] = -lik * uv;
                wn++;
            }
            pos++;
        }
    }
    g.slen[i] = wn;
    g.sldiv[i] = t;
    return 1;
}

// Rounds run back to back as programmatic dependent launches; of three
// counters the round reads one (the rows left by the previous round), adds to
// the next and clears the third, which the following round will add to.
__global__ void k_lu_round(LUArgs g, const uint32_t* __restrict__ pin, const uint32_t* __restrict__ npin,
                           uint32_t* __restrict__ pout, uint32_t* __restrict__ npout, uint32_t* __restrict__ nclear,
                           int round) {
    pdl_wait();
    pdl_trigger();
    if (blockIdx.x == 0 && threadIdx.x == 0) *nclear = 0;
    uint32_t n = *npin;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        uint32_t i = pin[idx];
        uint32_t k = g.wait[i];
        if (k != 0xffffffffu) {
            int dk = g.done[k];
            if (dk == 0 || dk >= round) { pout[atomicAdd(npout, 1u)] = i; continue; }
        }
        int r = lu_row(g, i, round);
        if (r == 1) g.done[i] = round;
        else if (r == 0) pout[atomicAdd(npout, 1u)] = i;
        else atomicOr(g.flags, 1);
    }
}

__global__ void k_lu_coarse(LUArgs g) {
    uint32_t i = g.M + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.R) return;
    int r = lu_row(g, i, 0x7fffffff);
    if (r != 1) atomicOr(g.flags, r < 0 ? 1 : 8);
}

__global__ void k_iota(uint32_t n, uint32_t* __restrict__ v) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

// counts for the compaction: L (R rows), U (M rows), next-level (R-M rows)
__global__ void k_lu_counts(uint32_t R, uint32_t M, const uint32_t* __restrict__ slen,
                            const uint32_t* __restrict__ sldiv, uint32_t* __restrict__ lc,
                            uint32_t* __restrict__ uc, uint32_t* __restrict__ nc) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R) return;
    lc[i] = sldiv[i];
    if (i < M) uc[i] = slen[i] - sldiv[i];
    else nc[i - M] = slen[i] - sldiv[i];
}

__global__ void k_lu_emit(uint32_t R, uint32_t M, uint32_t cap, const uint32_t* __restrict__ scol,
                          const double* __restrict__ sval, const uint32_t* __restrict__ slen,
                          const uint32_t* __restrict__ sldiv, const uint32_t* __restrict__ Lia,
                          uint32_t* __restrict__ Lja, double* __restrict__ La, const uint32_t* __restrict__ Uia,
                          uint32_t* __restrict__ Uja, double* __restrict__ Ua, const uint32_t* __restrict__ nia,
                          uint32_t* __restrict__ nja, double* __restrict__ na) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R) return;
    const uint32_t* c = scol + (size_t)i * cap;
    const double* v = sval + (size_t)i * cap;
    uint32_t ld = sldiv[i], wn = slen[i];
    uint32_t p = Lia[i];
    for (uint32_t t = 0; t < ld; t++) { Lja[p] = c[t]; La[p] = v[t]; p++; }
    if (i < M) {
        p = Uia[i];
        for (uint32_t t = ld; t < wn; t++) { Uja[p] = c[t]; Ua[p] = v[t]; p++; }
    } else {
        p = nia[i - M];
        for (uint32_t t = ld; t < wn; t++)
            if (c[t] == i) { nja[p] = i - M; na[p] = v[t]; p++; break; }
        for (uint32_t t = ld; t < wn; t++)
            if (c[t] != i) { nja[p] = c[t] - M; na[p] = v[t]; p++; }
    }
}

__global__ void k_dval(uint32_t Md, uint32_t base, const uint32_t* __restrict__ map, const double* __restrict__ aux,
                       double* __restrict__ dval) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Md) dval[i] = 1. / aux[map[base + i]];
}

}  // namespace mlp

// ===========================================================================
// Host orchestration of the hierarchy build.
// ===========================================================================
namespace mlp {

double cheb_poly(double x, uint32_t k) {  // misc.cc:232-242
    switch (k) {
        case 0: return 1;
        case 1: return x;
        case 2: return 2 * x * x - 1;
        case 3: return x * (4 * x * x - 3);
        default: return cosh(k * acosh(x));
    }
}

static int read_flag(const int* d, cudaStream_t s) {
    int h = 0;
    CK(cudaMemcpyAsync(&h, d, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return h;
}
static uint32_t read_u32(const uint32_t* d, cudaStream_t s) {
    uint32_t h = 0;
    CK(cudaMemcpyAsync(&h, d, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return h;
}

// ---- frame construction kernels -----------------------------------------
// pi(q): frame position -> permuted index; phi(q) = map[pi(q)].
__global__ void k_frame_phi(uint32_t N, uint32_t M, uint32_t n, const uint32_t* __restrict__ eperm,
                            const uint32_t* __restrict__ phi_next, const uint32_t* __restrict__ map,
                            uint32_t* __restrict__ pi, uint32_t* __restrict__ phi) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N) return;
    uint32_t p;
    if (q < M) p = eperm[q];
    else if (q < M + n) p = M + phi_next[q - M];
    else p = q;
    pi[q] = p;
    phi[q] = map[p];
}

__global__ void k_invert(uint32_t N, const uint32_t* __restrict__ perm, uint32_t* __restrict__ inv) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < N) inv[perm[q]] = q;
}

__global__ void k_row_len_perm(uint32_t R, const uint32_t* __restrict__ src_row, const uint32_t* __restrict__ ia,
                               uint32_t* __restrict__ len) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= R) return;
    uint32_t r = src_row ? src_row[q] : q;
    len[q] = ia[r + 1] - ia[r];
}

// Copies rows src_row[q] of (ia, ja, a) to row q of the output, relabelling the
// columns through colmap (identity when null).
__global__ void k_gather_rows(uint32_t R, const uint32_t* __restrict__ src_row, const uint32_t* __restrict__ ia,
                              const uint32_t* __restrict__ ja, const double* __restrict__ a,
                              const uint32_t* __restrict__ colmap, const uint32_t* __restrict__ oia,
                              uint32_t* __restrict__ oja, double* __restrict__ oa) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= R) return;
    uint32_t r = src_row ? src_row[q] : q;
    uint32_t o = oia[q];
    for (uint32_t j = ia[r]; j < ia[r + 1]; j++, o++) {
        oja[o] = colmap ? colmap[ja[j]] : ja[j];
        oa[o] = a[j];
    }
}

// Relabel map for U/L columns given in permuted indexing: E columns go through
// einv, coarse columns through M + iphi_next, diagonal columns stay.
__global__ void k_perm_to_frame(uint32_t N, uint32_t M, uint32_t n, const uint32_t* __restrict__ einv,
                                const uint32_t* __restrict__ iphi_next, uint32_t* __restrict__ out) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    if (p < M) out[p] = einv[p];
    else if (p < M + n) out[p] = M + iphi_next[p - M];
    else out[p] = p;
}

// uh_cheb sym_multiply operator (skyline.cc:115-155) as a full matrix: entries
// on and below the diagonal come from the row itself, entries above it from the
// mirrored lower entry of the other row.
__global__ void k_sym_values(uint32_t N, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                             const double* __restrict__ a, const uint32_t* __restrict__ tpos,
                             double* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[ia[i]] = a[ia[i]];
    for (uint32_t j_ = ia[i] + 1; j_ < ia[i + 1]; j_++) out[j_] = ja[j_] < i ? a[j_] : a[tpos[j_]];
}

// Level schedule of a triangular DAG given as CSR dependencies (diagonal entry
// skipped when it equals the row): level[i] = 1 + max level of its
// dependencies, computed in rounds like the elimination.
// Counters as k_lu_round.
__global__ void k_dag_round(uint32_t R, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                            uint32_t depmax, int* __restrict__ lev, const uint32_t* __restrict__ pin,
                            const uint32_t* __restrict__ npin, uint32_t* __restrict__ pout,
                            uint32_t* __restrict__ npout, uint32_t* __restrict__ nclear, int round) {
    pdl_wait();
    pdl_trigger();
    if (blockIdx.x == 0 && threadIdx.x == 0) *nclear = 0;
    uint32_t n = *npin;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        uint32_t i = pin[idx];
        bool ok = true;
        for (uint32_t j = ia[i]; j < ia[i + 1]; j++) {
            uint32_t k = ja[j];
            if (k == i || k >= depmax) continue;
            int lk = lev[k];
            if (lk == 0 || lk >= round) { ok = false; break; }
        }
        if (ok) lev[i] = round;
        else pout[atomicAdd(npout, 1u)] = i;
    }
}

// ---- dense inverse of the coarsest level (Gauss-Jordan, no pivoting) -----
__global__ void k_dense_from_csr(uint32_t n, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                                 const double* __restrict__ a, double* __restrict__ D) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint32_t j = ia[i]; j < ia[i + 1]; j++) D[(size_t)i * n + ja[j]] = a[j];
}
__global__ void k_gj_pivot(uint32_t n, uint32_t k, double* __restrict__ D, double* __restrict__ col,
                           int* __restrict__ err) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    double p = D[(size_t)k * n + k];
    if (p == 0.0) { if (t == 0) atomicOr(err, 16); return; }
    if (t < n) col[t] = D[(size_t)t * n + k];  // column k before the update
}
__global__ void k_gj_update(uint32_t n, uint32_t k, double* __restrict__ D, const double* __restrict__ col) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = blockIdx.y;
    if (j >= n) return;
    double piv = 1 / col[k];
    double rkj = (j == k) ? piv : D[(size_t)k * n + j] * piv;
    if (i == k) return;
    double f = col[i];
    double v = (j == k) ? 0.0 : D[(size_t)i * n + j];
    D[(size_t)i * n + j] = v - f * rkj;
}
__global__ void k_gj_rowk(uint32_t n, uint32_t k, double* __restrict__ D, const double* __restrict__ col) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double piv = 1 / col[k];
    D[(size_t)k * n + j] = (j == k) ? piv : D[(size_t)k * n + j] * piv;
}


// ---- explicit triangular solves ------------------------------------------
// Rows are built as Row(q) = base(q) + sum_k c_qk Row(k) with the rows k
// finished in an earlier wavefront. Each row is a sorted (column, value) list
// in its own slot of `cap` pairs.
__device__ __forceinline__ bool slot_merge(uint32_t* wc, double* wv, uint32_t& wn, uint32_t cap,
                                           const uint32_t* kc, const double* kv, uint32_t kn, double c) {
    uint32_t pos = 0;
    for (uint32_t u = 0; u < kn; u++) {
        uint32_t j = kc[u];
        while (pos < wn && wc[pos] < j) pos++;
        if (pos < wn && wc[pos] == j) {
            wv[pos] += c * kv[u];
        } else {
            if (wn == cap) return false;
            for (uint32_t t = wn; t > pos; t--) { wc[t] = wc[t - 1]; wv[t] = wv[t - 1]; }
            wc[pos] = j;
            wv[pos] = c * kv[u];
            wn++;
        }
        pos++;
    }
    return true;
}

// P1 rows q in [r0, r1): Row(q) = e_q - sum_k l_qk Row(k).
__global__ void k_p1_rows(uint32_t r0, uint32_t r1, const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                          const double* __restrict__ a, uint32_t cap, uint32_t* scol, double* sval,
                          uint32_t* slen, int* flags) {
    uint32_t q = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= r1) return;
    uint32_t* wc = scol + (size_t)q * cap;
    double* wv = sval + (size_t)q * cap;
    uint32_t wn = 1;
    wc[0] = q;
    wv[0] = 1.0;
    for (uint32_t j = ia[q]; j < ia[q + 1]; j++) {
        uint32_t k = ja[j];
        if (!slot_merge(wc, wv, wn, cap, scol + (size_t)k * cap, sval + (size_t)k * cap, slen[k], -a[j])) {
            atomicOr(flags, 1);
            return;
        }
    }
    slen[q] = wn;
}

// G rows (E rows listed by U wavefront): Row(q) = (e_q - sum_C u_qc e_c
// - sum_E u_qj Row(j)) / u_qq.
__global__ void k_g_rows(uint32_t cnt, const uint32_t* __restrict__ rows, uint32_t M,
                         const uint32_t* __restrict__ ia, const uint32_t* __restrict__ ja,
                         const double* __restrict__ a, uint32_t cap, uint32_t* scol, double* sval, uint32_t* slen,
                         int* flags) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    uint32_t q = rows[t];
    uint32_t rs = ia[q], re = ia[q + 1];
    double inv = 1 / a[rs];
    uint32_t* wc = scol + (size_t)q * cap;
    double* wv = sval + (size_t)q * cap;
    uint32_t wn = 1;
    wc[0] = q;
    wv[0] = inv;
    for (uint32_t j = rs + 1; j < re; j++) {
        uint32_t c = ja[j];
        if (c < M) continue;
        uint32_t one = c;
        double v = 1.0;
        if (!slot_merge(wc, wv, wn, cap, &one, &v, 1, -a[j] * inv)) { atomicOr(flags, 1); return; }
    }
    for (uint32_t j = rs + 1; j < re; j++) {
        uint32_t k = ja[j];
        if (k >= M) continue;
        if (!slot_merge(wc, wv, wn, cap, scol + (size_t)k * cap, sval + (size_t)k * cap, slen[k], -a[j] * inv)) {
            atomicOr(flags, 1);
            return;
        }
    }
    slen[q] = wn;
}

__global__ void k_slots_emit(uint32_t R, uint32_t cap, const uint32_t* __restrict__ scol,
                             const double* __restrict__ sval, const uint32_t* __restrict__ ia,
                             uint32_t* __restrict__ ja, double* __restrict__ a) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= R) return;
    uint32_t o = ia[q], n = ia[q + 1] - o;
    for (uint32_t t = 0; t < n; t++) {
        ja[o + t] = scol[(size_t)q * cap + t];
        a[o + t] = sval[(size_t)q * cap + t];
    }
}

// ---- per-level construction ------------------------------------------------

struct Scratch {
    Tmp<uint8_t> keep, want, bucket, marked, state;
    Tmp<int> nout, nin, nlinks, flag;
    Tmp<double> aux;
    Tmp<uint32_t> rmap, tpos, slot, cand, cnt;
};

// First slot capacity for `rows` rows: as large as a 2 GB slot area allows
// (at most 256 entries; never below what the previously built, coarser level
// needed: rows get longer towards the fine levels), so that the usual rows
// never overflow and the build is not repeated. The slots are scratch of the
// build, and the rows computed do not depend on the capacity.
static uint32_t slot_cap0(uint32_t rows, uint32_t prev) {
    uint64_t fit = ((uint64_t)1 << 31) / ((uint64_t)(rows ? rows : 1) * 12);
    uint32_t cap = 16;
    while (cap < 256 && (uint64_t)cap * 2 <= fit) cap *= 2;
    return std::max(cap, prev);
}

static void sparse_lu_level(Level& li, Level& ln, const uint8_t* keep, const double* aux, const uint32_t* rmap,
                            double beta, cudaStream_t s) {
    const DCSR& A = li.A;
    uint32_t N = li.N, M = li.M, Md = li.Md, R = N - Md;
    li.done.alloc(M ? M : 1);
    li.done.zero(s);
    Tmp<uint32_t> slen(R ? R : 1), sldiv(R ? R : 1), wait(R ? R : 1);
    Tmp<int> flags(1);
    uint32_t cap = slot_cap0(R, 32);
    for (int attempt = 0;; attempt++) {
        Tmp<uint32_t> scol((size_t)R * cap + 1);
        Tmp<double> sval((size_t)R * cap + 1);
        flags.zero(s);
        li.done.zero(s);
        CK(cudaMemsetAsync(wait.p, 0xff, wait.n * 4, s));
        LUArgs g{A.ia.p, A.ja.p, A.a.p, keep, aux, li.map.p, rmap, M, R, beta, cap,
                 scol.p, sval.p, slen.p, sldiv.p, li.done.p, wait.p, flags.p};
        // E rows in rounds
        int rounds = 0;
        if (M) {
            Tmp<uint32_t> pa(M), pb(M), cnt(3);
            cnt.zero(s);
            k_iota<<<grid_for(M, 256), 256, 0, s>>>(M, pa.p);
            CK_LAUNCH();
            CK(cudaMemcpyAsync(cnt.p, &M, 4, cudaMemcpyHostToDevice, s));
            uint32_t* pin = pa.p; uint32_t* pout = pb.p;
            unsigned grid = (unsigned)std::min<size_t>(grid_for(M, 256), (size_t)num_sms() * 8);
            uint32_t prev_left = M;
            for (;;) {
                for (int b = 0; b < 16; b++) {
                    rounds++;
                    launch_k(k_lu_round, grid, 256, 0, s, g, (const uint32_t*)pin,
                             (const uint32_t*)(cnt.p + (rounds - 1) % 3), pout, cnt.p + rounds % 3,
                             cnt.p + (rounds + 1) % 3, rounds);
                    CK_LAUNCH();
                    std::swap(pin, pout);
                }
                std::vector<uint32_t> h =
                    read_words({cnt.p + rounds % 3, reinterpret_cast<const uint32_t*>(flags.p)}, s);
                uint32_t left = h[0];
                if ((h[1] & 1) || left == 0) break;
                // every round finishes at least the rows whose dependencies are
                // done; no progress over sixteen rounds means a cycle
                if (left >= prev_left) MLP_THROW(ERR_INTERNAL, "elimination makes no progress");
                prev_left = left;
            }
        }
        // k_lu_coarse runs also after an overflow (its rows then fail fast
        // on the flag); one read of the flags decides
        if (R > M) {
            k_lu_coarse<<<grid_for(R - M, 128), 128, 0, s>>>(g);
            CK_LAUNCH();
        }
        int fl = read_flag(flags.p, s);
        if (fl & 1) {  // an overflow (the coarse rows may then also have met unfinished rows)
            if (cap >= 4096) MLP_THROW(ERR_LIMIT, "elimination row exceeds 4096 entries");
            cap *= 2;
            continue;
        }
        if (fl & 8) MLP_THROW(ERR_INTERNAL, "coarse row met an unfinished U row");
        // compaction
        Tmp<uint32_t> lc(R + 1), uc(M + 1), nc(R - M + 1);
        k_lu_counts<<<grid_for(R, 256), 256, 0, s>>>(R, M, slen.p, sldiv.p, lc.p, uc.p, nc.p);
        CK_LAUNCH();
        li.L.ia.alloc((size_t)R + 1);
        li.U.ia.alloc((size_t)M + 1);
        ln.A.ia.alloc((size_t)(R - M) + 1);
        std::vector<uint32_t> tot = exclusive_scans_u32({{lc.p, li.L.ia.p, R}, {uc.p, li.U.ia.p, M},
                                                         {nc.p, ln.A.ia.p, R - M}}, s);
        uint32_t lnnz = tot[0], unnz = tot[1], nnnz = tot[2];
        li.L.nrow = li.L.ncol = R; li.L.nnz = lnnz;
        li.L.ja.alloc(lnnz ? lnnz : 1); li.L.a.alloc(lnnz ? lnnz : 1);
        li.U.nrow = M; li.U.ncol = R; li.U.nnz = unnz;
        li.U.ja.alloc(unnz ? unnz : 1); li.U.a.alloc(unnz ? unnz : 1);
        ln.A.nrow = ln.A.ncol = R - M; ln.A.nnz = nnnz;
        ln.A.ja.alloc(nnnz ? nnnz : 1); ln.A.a.alloc(nnnz ? nnnz : 1);
        if (R) {
            k_lu_emit<<<grid_for(R, 128), 128, 0, s>>>(R, M, cap, scol.p, sval.p, slen.p, sldiv.p, li.L.ia.p,
                                                      li.L.ja.p, li.L.a.p, li.U.ia.p, li.U.ja.p, li.U.a.p,
                                                      ln.A.ia.p, ln.A.ja.p, ln.A.a.p);
            CK_LAUNCH();
        }
        li.nwave_l = (uint32_t)rounds;  // upper bound, refined by the frame build
        break;
    }
}

// The tail group of order_original (multi_split_mark.cc:41-113). Starting at
// every node (index order) that keeps one outgoing and at most one incoming
// link, the walk eliminates the node when its only links join it to the node
// its outgoing link points to, removes those links and moves on to that node;
// a node left with no links at the end of a walk is eliminated too. Each walk
// changes the link counts that the next start test and the next walk read, so
// the group is one ordered pass: it runs on the host (one pass over the level's
// links, a few milliseconds at 1.12 M nodes, where one GPU thread would spend
// an L2 round trip per step), on the link flags and counts of the marking
// kernel, and returns the eliminated nodes in order. nin / nout are updated in
// place as the reference updates them.
static std::vector<uint32_t> original_tails(uint32_t N, const std::vector<uint32_t>& ia,
                                            const std::vector<uint32_t>& ja, std::vector<uint8_t> keep,
                                            std::vector<int>& nin, std::vector<int>& nout,
                                            std::vector<uint8_t>& marked) {
    std::vector<uint32_t> order;
    auto find_col = [&](uint32_t row, uint32_t col) -> int64_t {
        // column col among row's off-diagonal entries (sorted after the diagonal)
        uint32_t lo = ia[row] + 1, hi = ia[row + 1];
        while (lo < hi) {
            uint32_t mid = (lo + hi) / 2;
            if (ja[mid] < col) lo = mid + 1;
            else hi = mid;
        }
        return (lo < ia[row + 1] && ja[lo] == col) ? (int64_t)lo : -1;
    };
    for (uint32_t i = 0; i < N; i++) {
        if (!(nout[i] == 1 && nin[i] <= 1)) continue;
        uint32_t i0 = i;
        for (;;) {
            if (nout[i0] != 1) break;
            uint32_t j_ = ia[i0] + 1;
            while (j_ < ia[i0 + 1] && !keep[j_]) j_++;
            if (j_ == ia[i0 + 1])
                MLP_THROW(ERR_INTERNAL, "Row " + std::to_string(i0) + ": remaining link was not found");
            uint32_t i1 = ja[j_];
            int64_t back = find_col(i1, i0);
            bool aji = back >= 0 && keep[back];
            if (!(nin[i0] == 0 || (nin[i0] == 1 && aji))) break;
            order.push_back(i0);
            marked[i0] = 1;
            keep[j_] = 0;
            if (aji) {
                keep[back] = 0;
                nin[i0]--;
                nout[i1]--;
            }
            nout[i0] = -1;
            nin[i1]--;
            i0 = i1;
        }
        if (nout[i0] == 0 && nin[i0] == 0) {
            order.push_back(i0);
            marked[i0] = 1;
            nout[i0] = -1;
        }
    }
    return order;
}

static void build_level_msplit(Hierarchy& H, const BuildCfg& cfg, uint32_t level, Scratch& S, cudaStream_t s) {
    Level& li = *H.lv[level];
    const DCSR& A = li.A;
    li.N = A.nrow;
    li.nnz = A.nnz;
    if (li.N <= H.coarse_n || level == H.nlevels - 1) {
        H.nlevels = level + 1;
        H.coarse_n = li.N;
        li.direct = true;
        return;
    }
    uint32_t N = li.N;
    S.keep.alloc(A.nnz ? A.nnz : 1);
    S.nout.alloc(N); S.nin.alloc(N); S.aux.alloc(N); S.flag.alloc(1);
    S.nin.zero(s); S.flag.zero(s);
    k_mark_msplit<<<grid_for(N, 128), 128, 0, s>>>(N, A.ia.p, A.ja.p, A.a.p, li.q, S.keep.p, S.nout.p, S.nin.p,
                                                  S.aux.p, S.flag.p);
    CK_LAUNCH();
    if (read_flag(S.flag.p, s)) MLP_THROW(ERR_LIMIT, "a row has more than 64 off-diagonal entries");
    li.map.alloc(N);
    S.bucket.alloc(N);
    li.M = 0;
    if (cfg.order == ORDER_SIMPLE_1) {
        k_bucket_simple1<<<grid_for(N, 256), 256, 0, s>>>(N, S.nout.p, S.nin.p, S.bucket.p);
        CK_LAUNCH();
        std::vector<uint32_t> cnt = stable_partition(N, S.bucket.p, 5, 0, li.map.p, 0, s);
        uint32_t acc = cnt[0];
        for (uint32_t d = 1; d <= 3; d++) {
            acc += cnt[d];
            if (d == cfg.degree_max) li.M = acc;
        }
        li.Md = cnt[4];
    } else if (cfg.order == ORDER_NONE) {
        k_bucket_none<<<grid_for(N, 256), 256, 0, s>>>(N, S.nout.p, S.nin.p, S.bucket.p);
        CK_LAUNCH();
        std::vector<uint32_t> cnt = stable_partition(N, S.bucket.p, 2, 2u, li.map.p, 0, s);
        li.M = 0;
        li.Md = cnt[1];
    } else if (cfg.order == ORDER_ORIGINAL) {
        // order_original (multi_split_mark.cc:27-154): tails (host pass), then
        // group 2 and the remaining nodes on the device
        S.marked.alloc(N);
        uint32_t ntail = 0;
        if (cfg.use_tails) {
            std::vector<uint32_t> ia = A.ia.download(s, (size_t)N + 1), ja = A.ja.download(s, A.nnz);
            std::vector<uint8_t> keep = S.keep.download(s, A.nnz);
            std::vector<int> nin = S.nin.download(s, N), nout = S.nout.download(s, N);
            std::vector<uint8_t> marked(N, 0);
            std::vector<uint32_t> tails = original_tails(N, ia, ja, std::move(keep), nin, nout, marked);
            ntail = (uint32_t)tails.size();
            if (ntail) CK(cudaMemcpyAsync(li.map.p, tails.data(), (size_t)ntail * 4, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(S.marked.p, marked.data(), N, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(S.nin.p, nin.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(S.nout.p, nout.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s));
            CK(cudaStreamSynchronize(s));  // the host vectors go out of scope
        } else {
            S.marked.zero(s);
        }
        k_bucket_original<<<grid_for(N, 256), 256, 0, s>>>(N, S.nout.p, S.nin.p, S.marked.p, S.bucket.p);
        CK_LAUNCH();
        std::vector<uint32_t> cnt = stable_partition(N, S.bucket.p, 3, 4u, li.map.p, ntail, s);
        li.M = ntail + cnt[0];
        li.Md = cnt[2];
    } else if (cfg.order == ORDER_BLOCK) {
        // order_block (multi_split_mark.cc:193-252): only the 60x220x85 mesh
        if (N != BLK_NX * BLK_NY * BLK_NZ)
            MLP_THROW(ERR_CONFIG, "Wrong mesh size: " + std::to_string(N) + " (expected 1122000)");
        S.marked.alloc(N);
        S.marked.zero(s);
        Tmp<uint32_t> flag(BLK_POS), pos((size_t)BLK_POS + 1);
        k_block_flags<<<grid_for(BLK_POS, 256), 256, 0, s>>>(S.nout.p, S.nin.p, flag.p);
        CK_LAUNCH();
        uint32_t nb = exclusive_scan_u32(flag.p, pos.p, BLK_POS, s);
        k_block_place<<<grid_for(BLK_POS, 256), 256, 0, s>>>(flag.p, pos.p, li.map.p, S.marked.p);
        CK_LAUNCH();
        k_bucket_rest<<<grid_for(N, 256), 256, 0, s>>>(N, S.nout.p, S.nin.p, S.marked.p, S.bucket.p);
        CK_LAUNCH();
        std::vector<uint32_t> cnt = stable_partition(N, S.bucket.p, 2, 2u, li.map.p, nb, s);
        li.M = nb;
        li.Md = cnt[1];
    } else {
        MLP_THROW(ERR_CONFIG, "unknown elim_order");
    }
    S.rmap.alloc(N);
    k_rmap<<<grid_for(N, 256), 256, 0, s>>>(N, li.map.p, S.rmap.p);
    CK_LAUNCH();
    H.lv.emplace_back(new Level());
    Level& ln = *H.lv[level + 1];
    Level& lc = *H.lv[level];  // re-fetch: emplace_back may move unique_ptrs (not the objects)
    trace(("ms mark+order L" + std::to_string(level)).c_str());
    sparse_lu_level(lc, ln, S.keep.p, S.aux.p, S.rmap.p, 1.0, s);
    trace(("ms sparse lu L" + std::to_string(level) + " (" + std::to_string(lc.nwave_l) + " rounds)").c_str());
    lc.n = N - lc.M - lc.Md;
    lc.dval.alloc(lc.Md ? lc.Md : 1);
    if (lc.Md) {
        k_dval<<<grid_for(lc.Md, 256), 256, 0, s>>>(lc.Md, N - lc.Md, lc.map.p, S.aux.p, lc.dval.p);
        CK_LAUNCH();
    }
    if (lc.n) {
        ln.q = level + 1 < cfg.q.size() ? cfg.q[level + 1] : cfg.q.back();
        // multi_split_constr.cc:256-264: a fixed count, or with dynamic inner
        // iterations an eps (niter keeps the Level() default 0 then)
        if (!cfg.eps.empty()) ln.eps = level + 1 < cfg.eps.size() ? cfg.eps[level + 1] : cfg.eps.back();
        else ln.niter = level + 1 < cfg.niter.size() ? cfg.niter[level + 1] : cfg.niter.back();
        build_level_msplit(H, cfg, level + 1, S, s);
    } else {
        H.lv.pop_back();
        H.nlevels = level + 1;
    }
}

static void build_level_cheb(Hierarchy& H, const BuildCfg& cfg, uint32_t level, Scratch& S, cudaStream_t s) {
    Level& li = *H.lv[level];
    const DCSR& A = li.A;
    uint32_t N = A.nrow, nnz = A.nnz;
    li.N = N;
    li.nnz = nnz;
    S.want.alloc(nnz ? nnz : 1); S.keep.alloc(nnz ? nnz : 1); S.aux.alloc(N); S.flag.alloc(1);
    S.tpos.alloc(nnz ? nnz : 1); S.slot.alloc(nnz ? nnz : 1); S.nlinks.alloc(N);
    S.flag.zero(s);
    k_mark_cheb<<<grid_for(N, 128), 128, 0, s>>>(N, A.ia.p, A.a.p, li.beta, S.want.p, S.aux.p, S.flag.p);
    CK_LAUNCH();
    k_transpose_pos<<<grid_for(N, 128), 128, 0, s>>>(N, A.ia.p, A.ja.p, S.tpos.p, S.flag.p);
    CK_LAUNCH();
    int fl = read_flag(S.flag.p, s);
    if (fl & 1) MLP_THROW(ERR_LIMIT, "a row has more than 64 off-diagonal entries");
    if (fl & 2) MLP_THROW(ERR_ARG, "uh_cheb needs a structurally symmetric matrix");
    k_cheb_links<<<grid_for(N, 128), 128, 0, s>>>(N, A.ia.p, A.ja.p, S.want.p, S.tpos.p, S.keep.p, S.nlinks.p,
                                                 S.slot.p);
    CK_LAUNCH();
    // sym operator values for the Chebyshev steps that use this level's matrix
    if (level > 0) {
        li.As.nrow = li.As.ncol = N; li.As.nnz = nnz;
        li.As.a.alloc(nnz ? nnz : 1);
        k_sym_values<<<grid_for(N, 128), 128, 0, s>>>(N, A.ia.p, A.ja.p, A.a.p, S.tpos.p, li.As.a.p);
        CK_LAUNCH();
    }
    li.map.alloc(N);
    S.marked.alloc(N);
    S.marked.zero(s);
    uint32_t M = 0;
    if (cfg.use_tails) {
        S.bucket.alloc(N);
        S.cand.alloc(N ? N : 1);
        k_bucket_deg1<<<grid_for(N, 256), 256, 0, s>>>(N, S.nlinks.p, S.bucket.p);
        CK_LAUNCH();
        std::vector<uint32_t> c1 = stable_partition(N, S.bucket.p, 1, 0, S.cand.p, 0, s);
        std::vector<uint32_t> ia = A.ia.download(s, (size_t)N + 1), ja = A.ja.download(s, nnz);
        std::vector<uint32_t> slot = S.slot.download(s, nnz), cand = S.cand.download(s, c1[0]);
        std::vector<uint8_t> state = S.keep.download(s, nnz), marked(N, 0);  // the walk works on a copy
        std::vector<int> nlinks = S.nlinks.download(s, N);
        std::vector<uint32_t> tails = cheb_tails(ia, ja, slot, std::move(state), nlinks, cand, marked);
        M = (uint32_t)tails.size();
        if (M) CK(cudaMemcpyAsync(li.map.p, tails.data(), (size_t)M * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(S.marked.p, marked.data(), N, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(S.nlinks.p, nlinks.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));  // the host vectors go out of scope
    }
    S.bucket.alloc(N);
    k_bucket_cheb_rest<<<grid_for(N, 256), 256, 0, s>>>(N, S.nlinks.p, S.marked.p, S.bucket.p);
    CK_LAUNCH();
    std::vector<uint32_t> cnt = stable_partition(N, S.bucket.p, 2, 2u, li.map.p, M, s);
    li.M = M;
    li.Md = cnt[1];
    S.rmap.alloc(N);
    k_rmap<<<grid_for(N, 256), 256, 0, s>>>(N, li.map.p, S.rmap.p);
    CK_LAUNCH();
    H.lv.emplace_back(new Level());
    Level& ln = *H.lv[level + 1];
    Level& lc = *H.lv[level];
    sparse_lu_level(lc, ln, S.keep.p, S.aux.p, S.rmap.p, lc.beta, s);
    lc.n = N - lc.M - lc.Md;
    lc.dval.alloc(lc.Md ? lc.Md : 1);
    if (lc.Md) {
        k_dval<<<grid_for(lc.Md, 256), 256, 0, s>>>(lc.Md, N - lc.Md, lc.map.p, S.aux.p, lc.dval.p);
        CK_LAUNCH();
    }
    if (lc.n) {
        if (level + 1 >= H.nlevels) MLP_THROW(ERR_LEVELS, "Too many levels: " + std::to_string(level + 1));
        ln.alpha = 1.0;
        ln.beta = level + 1 < cfg.sigma.size() ? cfg.sigma[level + 1] : cfg.sigma.back();
        build_level_cheb(H, cfg, level + 1, S, s);
    } else {
        H.lv.pop_back();
        H.nlevels = level + 1;
    }
}

// Host counting sort of rows by level value (1-based), stable in row index.
static void counting_sort(const std::vector<int>& lev, uint32_t nrows, std::vector<uint32_t>& off,
                          std::vector<uint32_t>& rows) {
    int maxl = 0;
    for (uint32_t i = 0; i < nrows; i++) maxl = std::max(maxl, lev[i]);
    off.assign((size_t)maxl + 1, 0);
    for (uint32_t i = 0; i < nrows; i++) off[lev[i]]++;  // lev >= 1
    uint32_t acc = 0;
    for (int d = 0; d <= maxl; d++) { uint32_t c = off[d]; off[d] = acc; acc += c; }
    std::vector<uint32_t> pos(off);
    rows.resize(nrows);
    for (uint32_t i = 0; i < nrows; i++) rows[pos[lev[i]]++] = i;
    // off[d] is the start of level d (levels start at 1); drop level 0 slot
    off.erase(off.begin());
    off.push_back(nrows);
}


// ---- the same sort on the device --------------------------------------------
// Rows in blocks of KS_BLOCK: per-block bin counts (bin-major, so one scan of
// them gives every block's start in every bin), then each block scatters its
// rows; within a block a row's place is the rows of its bin in earlier warps
// plus its rank among the lanes of its warp with the same key, so the order
// within a bin is the index order (a stable sort, as counting_sort).
constexpr uint32_t KS_BLOCK = 1024;
constexpr uint32_t KS_MAXK = 64;

__global__ void __launch_bounds__(KS_BLOCK) k_key_hist(const int* __restrict__ key, uint32_t n, uint32_t K,
                                                       uint32_t nblk, uint32_t* __restrict__ bcnt,
                                                       int* __restrict__ bad) {
    __shared__ uint32_t h[KS_MAXK];
    for (uint32_t t = threadIdx.x; t < K; t += blockDim.x) h[t] = 0;
    __syncthreads();
    uint32_t i = blockIdx.x * KS_BLOCK + threadIdx.x;
    if (i < n) {
        int k = key[i];
        if (k >= 1 && (uint32_t)k <= K) atomicAdd(&h[k - 1], 1u);
        else atomicOr(bad, 1);
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < K; t += blockDim.x) bcnt[(size_t)t * nblk + blockIdx.x] = h[t];
}

__global__ void __launch_bounds__(KS_BLOCK) k_key_scatter(const int* __restrict__ key, uint32_t n, uint32_t K,
                                                          uint32_t nblk, const uint32_t* __restrict__ bpos,
                                                          uint32_t* __restrict__ rows) {
    __shared__ uint32_t wc[KS_BLOCK / 32][KS_MAXK];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    for (uint32_t t = threadIdx.x; t < (KS_BLOCK / 32) * KS_MAXK; t += blockDim.x) (&wc[0][0])[t] = 0;
    __syncthreads();
    const uint32_t i = blockIdx.x * KS_BLOCK + threadIdx.x;
    const bool act = i < n;
    int k = act ? key[i] - 1 : -1;
    if (act && (k < 0 || (uint32_t)k >= K)) k = -1;  // reported by k_key_hist; placed nowhere
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    if (k >= 0 && lane == (uint32_t)(__ffs(peers) - 1)) wc[w][k] = __popc(peers);
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < K; t += blockDim.x) {
        uint32_t acc = 0;
        for (uint32_t v = 0; v < KS_BLOCK / 32; v++) {
            uint32_t c = wc[v][t];
            wc[v][t] = acc;
            acc += c;
        }
    }
    __syncthreads();
    if (k >= 0) rows[bpos[(size_t)k * nblk + blockIdx.x] + wc[w][k] + rank] = i;
}

// off[d] = start of bin d (bpos of block 0), off[K] = n; off[K + 1] = the bad flag
__global__ void k_key_offsets(uint32_t n, uint32_t K, uint32_t nblk, const uint32_t* __restrict__ bpos,
                              const int* __restrict__ bad, uint32_t* __restrict__ off) {
    uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < K) off[d] = bpos[(size_t)d * nblk];
    if (d == K) off[K] = n;
    if (d == K + 1) off[K + 1] = (uint32_t)*bad;
}

// counting_sort of the device keys key[0, n) (each in [1, K]) into rows_out on
// the device and off on the host; false (nothing written) when K is above
// KS_MAXK or a key is out of range, and the caller sorts on the host.
static bool device_key_sort(const int* key, uint32_t n, uint32_t K, uint32_t* rows_out, std::vector<uint32_t>& off,
                            cudaStream_t s) {
    if (!n || !K || K > KS_MAXK) return false;
    const uint32_t nblk = (n + KS_BLOCK - 1) / KS_BLOCK;
    Tmp<uint32_t> bcnt((size_t)K * nblk + 1), bpos((size_t)K * nblk + 1), offs(K + 2);
    Tmp<int> bad(1);
    bad.zero(s);
    k_key_hist<<<nblk, KS_BLOCK, 0, s>>>(key, n, K, nblk, bcnt.p, bad.p);
    CK_LAUNCH();
    exclusive_scan_u32_async(bcnt.p, bpos.p, K * nblk, s);
    k_key_offsets<<<1, 128, 0, s>>>(n, K, nblk, bpos.p, bad.p, offs.p);
    CK_LAUNCH();
    std::vector<uint32_t> h(K + 2);
    CK(cudaMemcpyAsync(h.data(), offs.p, (K + 2) * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h[K + 1]) return false;
    k_key_scatter<<<nblk, KS_BLOCK, 0, s>>>(key, n, K, nblk, bpos.p, rows_out);
    CK_LAUNCH();
    // counting_sort's offsets: bins up to the last non-empty one, then n
    off.assign(h.begin(), h.begin() + K + 1);
    while (off.size() > 1 && off[off.size() - 2] == n) off.pop_back();
    return true;
}

// Explicit forms of the level's triangular solves (P1 and G, setup.cuh).
static void build_explicit(Level& li, cudaStream_t s, uint32_t& p1_cap, uint32_t& g_cap) {
    uint32_t M = li.M, R = li.N - li.Md;
    Tmp<int> flags(1);
    const uint32_t* flag_word = reinterpret_cast<const uint32_t*>(flags.p);
    // P1
    for (uint32_t cap = slot_cap0(R, p1_cap);; cap *= 2) {
        if (cap > 65536) MLP_THROW(ERR_LIMIT, "explicit L solve row exceeds 65536 entries");
        Tmp<uint32_t> scol((size_t)R * cap + 1), slen(R + 1);
        Tmp<double> sval((size_t)R * cap + 1);
        flags.zero(s);
        for (size_t d = 0; d + 1 < li.lw_off.size(); d++) {
            uint32_t r0 = li.lw_off[d], r1 = li.lw_off[d + 1];
            if (r1 > r0) k_p1_rows<<<grid_for(r1 - r0, 128), 128, 0, s>>>(r0, r1, li.Lf.ia.p, li.Lf.ja.p, li.Lf.a.p,
                                                                         cap, scol.p, sval.p, slen.p, flags.p);
        }
        if (R > M)
            k_p1_rows<<<grid_for(R - M, 128), 128, 0, s>>>(M, R, li.Lf.ia.p, li.Lf.ja.p, li.Lf.a.p, cap, scol.p,
                                                         sval.p, slen.p, flags.p);
        CK_LAUNCH();
        // the row pointers are scanned before the overflow flag is known, so
        // that one read brings back both
        li.P1.ia.alloc((size_t)R + 1);
        exclusive_scan_u32_async(slen.p, li.P1.ia.p, R, s);
        std::vector<uint32_t> h = read_words({flag_word, li.P1.ia.p + R}, s);
        if (h[0]) continue;
        uint32_t z = h[1];
        li.P1.nrow = R; li.P1.ncol = R; li.P1.nnz = z;
        li.P1.ja.alloc(z ? z : 1); li.P1.a.alloc(z ? z : 1);
        if (R) k_slots_emit<<<grid_for(R, 128), 128, 0, s>>>(R, cap, scol.p, sval.p, li.P1.ia.p, li.P1.ja.p, li.P1.a.p);
        CK_LAUNCH();
        p1_cap = cap;
        trace(("  explicit: P1 (" + std::to_string(li.lw_off.size() - 1) + " waves, slot " + std::to_string(cap) +
               ")").c_str());
        break;
    }
    // G
    li.G.nrow = M; li.G.ncol = R; li.G.nnz = 0;
    if (!M) { li.G.ia.alloc(1); li.G.ia.zero(s); li.G.ja.alloc(1); li.G.a.alloc(1); return; }
    for (uint32_t cap = slot_cap0(M, g_cap);; cap *= 2) {
        if (cap > 65536) MLP_THROW(ERR_LIMIT, "explicit U solve row exceeds 65536 entries");
        Tmp<uint32_t> scol((size_t)M * cap + 1), slen(M + 1);
        Tmp<double> sval((size_t)M * cap + 1);
        flags.zero(s);
        for (size_t d = 0; d + 1 < li.uw_off.size(); d++) {
            uint32_t o0 = li.uw_off[d], o1 = li.uw_off[d + 1];
            if (o1 > o0) k_g_rows<<<grid_for(o1 - o0, 128), 128, 0, s>>>(o1 - o0, li.uw_rows.p + o0, M, li.Uf.ia.p,
                                                                        li.Uf.ja.p, li.Uf.a.p, cap, scol.p, sval.p,
                                                                        slen.p, flags.p);
        }
        CK_LAUNCH();
        li.G.ia.alloc((size_t)M + 1);
        exclusive_scan_u32_async(slen.p, li.G.ia.p, M, s);
        std::vector<uint32_t> h = read_words({flag_word, li.G.ia.p + M}, s);
        if (h[0]) continue;
        uint32_t z = h[1];
        li.G.nnz = z;
        li.G.ja.alloc(z ? z : 1); li.G.a.alloc(z ? z : 1);
        k_slots_emit<<<grid_for(M, 128), 128, 0, s>>>(M, cap, scol.p, sval.p, li.G.ia.p, li.G.ja.p, li.G.a.p);
        CK_LAUNCH();
        g_cap = cap;
        trace(("  explicit: G (" + std::to_string(li.uw_off.size() - 1) + " waves, slot " + std::to_string(cap) +
               ")").c_str());
        break;
    }
}

// Builds the frame-order operators of every level, bottom-up.
static void build_frames(Hierarchy& H, cudaStream_t s) {
    uint32_t p1_cap = 16, g_cap = 16;
    for (int l = (int)H.nlevels - 1; l >= 0; l--) {
        Level& li = *H.lv[l];
        uint32_t N = li.N;
        li.phi.alloc(N ? N : 1);
        li.iphi.alloc(N ? N : 1);
        if (li.direct) {
            k_iota<<<grid_for(N, 256), 256, 0, s>>>(N, li.phi.p);
            CK_LAUNCH();
            k_iota<<<grid_for(N, 256), 256, 0, s>>>(N, li.iphi.p);
            CK_LAUNCH();
        }
        uint32_t M = li.M, n = li.n, R = N - li.Md;
        if (!li.direct) {
        // E block order: by L wavefront (elimination round), then permuted index
        std::vector<uint32_t> off;
        li.eperm.alloc(M ? M : 1);
        if (!device_key_sort(li.done.p, M, li.nwave_l, li.eperm.p, off, s)) {
            std::vector<int> done = li.done.download(s, M);
            std::vector<uint32_t> rows;
            counting_sort(done, M, off, rows);
            if (M) li.eperm.upload(rows.data(), M, s);
        }
        li.lw_off = off;
        li.nwave_l = (uint32_t)off.size() - 1;
        li.lw_off_d.alloc(off.size());
        li.lw_off_d.upload(off.data(), off.size(), s);
        Tmp<uint32_t> pi(N), einv(M ? M : 1), p2f(N);
        const uint32_t* phi_next = (l + 1 < (int)H.nlevels) ? H.lv[l + 1]->phi.p : nullptr;
        const uint32_t* iphi_next = (l + 1 < (int)H.nlevels) ? H.lv[l + 1]->iphi.p : nullptr;
        k_frame_phi<<<grid_for(N, 256), 256, 0, s>>>(N, M, n, li.eperm.p, phi_next, li.map.p, pi.p, li.phi.p);
        CK_LAUNCH();
        k_invert<<<grid_for(N, 256), 256, 0, s>>>(N, li.phi.p, li.iphi.p);
        CK_LAUNCH();
        if (M) {
            k_invert<<<grid_for(M, 256), 256, 0, s>>>(M, li.eperm.p, einv.p);
            CK_LAUNCH();
        }
        k_perm_to_frame<<<grid_for(N, 256), 256, 0, s>>>(N, M, n, einv.p, iphi_next, p2f.p);
        CK_LAUNCH();
        trace("  frame: E order + maps");
        // Lf: rows pi(q), q < R; columns (E, permuted) -> frame
        {
            Tmp<uint32_t> len(R + 1);
            k_row_len_perm<<<grid_for(R, 256), 256, 0, s>>>(R, pi.p, li.L.ia.p, len.p);
            CK_LAUNCH();
            li.Lf.ia.alloc((size_t)R + 1);
            // the rows are L's, permuted: the total is known (checked below)
            exclusive_scan_u32_async(len.p, li.Lf.ia.p, R, s);
            uint32_t z = li.L.nnz;
            li.Lf.nrow = R; li.Lf.ncol = M; li.Lf.nnz = z;
            li.Lf.ja.alloc(z ? z : 1); li.Lf.a.alloc(z ? z : 1);
            k_gather_rows<<<grid_for(R, 256), 256, 0, s>>>(R, pi.p, li.L.ia.p, li.L.ja.p, li.L.a.p, p2f.p,
                                                         li.Lf.ia.p, li.Lf.ja.p, li.Lf.a.p);
            CK_LAUNCH();
        }
        // Uf: rows eperm[q], columns -> frame
        if (M) {
            Tmp<uint32_t> len(M + 1);
            k_row_len_perm<<<grid_for(M, 256), 256, 0, s>>>(M, li.eperm.p, li.U.ia.p, len.p);
            CK_LAUNCH();
            li.Uf.ia.alloc((size_t)M + 1);
            exclusive_scan_u32_async(len.p, li.Uf.ia.p, M, s);
            uint32_t z = li.U.nnz;
            li.Uf.nrow = M; li.Uf.ncol = R; li.Uf.nnz = z;
            li.Uf.ja.alloc(z ? z : 1); li.Uf.a.alloc(z ? z : 1);
            k_gather_rows<<<grid_for(M, 256), 256, 0, s>>>(M, li.eperm.p, li.U.ia.p, li.U.ja.p, li.U.a.p, p2f.p,
                                                         li.Uf.ia.p, li.Uf.ja.p, li.Uf.a.p);
            CK_LAUNCH();
            // U-solve wavefronts: row q depends on the E columns of its row
            Tmp<int> lev(M);
            lev.zero(s);
            Tmp<uint32_t> pa(M), pb(M), cnt(3);
            cnt.zero(s);
            k_iota<<<grid_for(M, 256), 256, 0, s>>>(M, pa.p);
            CK_LAUNCH();
            CK(cudaMemcpyAsync(cnt.p, &M, 4, cudaMemcpyHostToDevice, s));
            uint32_t *pin = pa.p, *pout = pb.p;
            int round = 0;
            uint32_t prev_left = M;
            unsigned grid = (unsigned)std::min<size_t>(grid_for(M, 256), (size_t)num_sms() * 8);
            for (;;) {
                for (int b = 0; b < 16; b++) {
                    round++;
                    launch_k(k_dag_round, grid, 256, 0, s, M, (const uint32_t*)li.Uf.ia.p, (const uint32_t*)li.Uf.ja.p,
                             M, lev.p, (const uint32_t*)pin, (const uint32_t*)(cnt.p + (round - 1) % 3), pout,
                             cnt.p + round % 3, cnt.p + (round + 1) % 3, round);
                    CK_LAUNCH();
                    std::swap(pin, pout);
                }
                uint32_t left = read_u32(cnt.p + round % 3, s);
                if (left == 0) break;
                if (left >= prev_left) MLP_THROW(ERR_INTERNAL, "U schedule makes no progress");
                prev_left = left;
            }
            trace(("  frame: Lf, Uf, U schedule (" + std::to_string(round) + " rounds)").c_str());
            std::vector<uint32_t> uoff;
            li.uw_rows.alloc(M);
            if (!device_key_sort(lev.p, M, (uint32_t)round, li.uw_rows.p, uoff, s)) {
                std::vector<int> ul = lev.download(s, M);
                std::vector<uint32_t> urows;
                counting_sort(ul, M, uoff, urows);
                li.uw_rows.upload(urows.data(), M, s);
            }
            li.uw_off = uoff;
            li.uw_off_d.alloc(uoff.size());
            li.uw_off_d.upload(uoff.data(), uoff.size(), s);
        }
        }  // !direct
        // Af: rows phi(q), columns -> iphi
        {
            const DCSR& A = li.A;
            Tmp<uint32_t> len(N + 1);
            k_row_len_perm<<<grid_for(N, 256), 256, 0, s>>>(N, li.phi.p, A.ia.p, len.p);
            CK_LAUNCH();
            li.Af.ia.alloc((size_t)N + 1);
            exclusive_scan_u32_async(len.p, li.Af.ia.p, N, s);
            uint32_t z = A.nnz;
            li.Af.nrow = li.Af.ncol = N; li.Af.nnz = z;
            li.Af.ja.alloc(z ? z : 1); li.Af.a.alloc(z ? z : 1);
            k_gather_rows<<<grid_for(N, 256), 256, 0, s>>>(N, li.phi.p, A.ia.p, A.ja.p, A.a.p, li.iphi.p,
                                                         li.Af.ia.p, li.Af.ja.p, li.Af.a.p);
            CK_LAUNCH();
            if (H.kind == PREC_CHEB && l > 0) {
                // symmetric operator with the same pattern, frame order
                li.As.ia.alloc((size_t)N + 1);
                CK(cudaMemcpyAsync(li.As.ia.p, li.Af.ia.p, ((size_t)N + 1) * 4, cudaMemcpyDeviceToDevice, s));
                DBuf<double> av(z ? z : 1);
                DBuf<uint32_t> jv(z ? z : 1);
                k_gather_rows<<<grid_for(N, 256), 256, 0, s>>>(N, li.phi.p, A.ia.p, A.ja.p, li.As.a.p, li.iphi.p,
                                                             li.As.ia.p, jv.p, av.p);
                CK_LAUNCH();
                li.As.ja = std::move(jv);
                li.As.a = std::move(av);
                li.As.nrow = li.As.ncol = N; li.As.nnz = z;
            }
        }
        trace(("frame operators L" + std::to_string(l)).c_str());
        if (!li.direct) build_explicit(li, s, p1_cap, g_cap);
        // tile statistics of the level's operators and the check of the
        // permuted row pointers' totals, in one read
        std::vector<DCSR*> ms{&li.Af};
        std::vector<const uint32_t*> ends{li.Af.ia.p + N};
        std::vector<uint32_t> want{li.A.nnz};
        if (H.kind == PREC_CHEB && l > 0) ms.push_back(&li.As);
        if (!li.direct) {
            ms.push_back(&li.P1);
            ms.push_back(&li.G);
            ends.push_back(li.Lf.ia.p + R);
            want.push_back(li.L.nnz);
            if (M) {
                ends.push_back(li.Uf.ia.p + M);
                want.push_back(li.U.nnz);
            }
        }
        std::vector<uint32_t> got;
        csr_tile_stats_batch(ms, ends, got, s);
        if (got != want) MLP_THROW(ERR_INTERNAL, "permuted operator has the wrong number of entries");
        trace(("explicit solves L" + std::to_string(l)).c_str());
    }
}

static void build_direct(Level& li, cudaStream_t s) {
    uint32_t n = li.N;
    li.cinv.alloc((size_t)n * n + 1);
    li.cinv.zero(s);
    if (!n) return;
    k_dense_from_csr<<<grid_for(n, 128), 128, 0, s>>>(n, li.A.ia.p, li.A.ja.p, li.A.a.p, li.cinv.p);
    CK_LAUNCH();
    Tmp<double> col(n);
    Tmp<int> err(1);
    err.zero(s);
    dim3 g2(grid_for(n, 256), n);
    for (uint32_t k = 0; k < n; k++) {
        k_gj_pivot<<<grid_for(n, 256), 256, 0, s>>>(n, k, li.cinv.p, col.p, err.p);
        k_gj_update<<<g2, 256, 0, s>>>(n, k, li.cinv.p, col.p);
        k_gj_rowk<<<grid_for(n, 256), 256, 0, s>>>(n, k, li.cinv.p, col.p);
    }
    CK_LAUNCH();
    if (read_flag(err.p, s)) MLP_THROW(ERR_INTERNAL, "zero pivot in the coarse-level inverse");
}

std::unique_ptr<Hierarchy> build_hierarchy(const DCSR& A0, const BuildCfg& cfg, cudaStream_t s) {
    ArenaScope arena;
    trace("build start");
    auto H = std::unique_ptr<Hierarchy>(new Hierarchy());
    H->kind = cfg.kind;
    H->lv.emplace_back(new Level());
    Level& l0 = *H->lv[0];
    // level 0 keeps its own copy of A (the caller may release its matrix)
    l0.A.alloc(A0.nrow, A0.ncol, A0.nnz);
    CK(cudaMemcpyAsync(l0.A.ia.p, A0.ia.p, ((size_t)A0.nrow + 1) * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(l0.A.ja.p, A0.ja.p, (size_t)A0.nnz * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(l0.A.a.p, A0.a.p, (size_t)A0.nnz * 8, cudaMemcpyDeviceToDevice, s));
    Scratch S;
    if (cfg.kind == PREC_MSPLIT) {
        // multi_split_constr.cc:252-275
        if (cfg.max_levels == 0 || cfg.q.empty() || cfg.niter.empty())
            MLP_THROW(ERR_CONFIG, "max_levels, q and level_niter must be non-empty");
        H->nlevels = cfg.max_levels;
        H->coarse_n = cfg.coarse_n;
        l0.q = cfg.q[0];
        l0.niter = 1;
        build_level_msplit(*H, cfg, 0, S, s);
        Level& last = *H->lv[H->nlevels - 1];
        if (last.M == 0) { last.niter = 0; last.eps = 0; last.q = 0; }
    } else {
        // cheb_constr.cc:292-365
        if (cfg.sigma.empty() || cfg.ncheb.empty()) MLP_THROW(ERR_CONFIG, "sigmas and niters must be non-empty");
        H->nlevels = 30;
        l0.alpha = 1.0;
        l0.beta = cfg.sigma[0];
        build_level_cheb(*H, cfg, 0, S, s);
        for (uint32_t l = 0; l < H->nlevels; l++)
            H->lv[l]->ncheb = l < cfg.ncheb.size() ? cfg.ncheb[l] : cfg.ncheb.back();
        Level& last = *H->lv[H->nlevels - 1];
        last.lmin = last.alpha;
        last.lmax = last.beta;
        for (int l = (int)H->nlevels - 2; l >= 0; l--) {
            Level& a = *H->lv[l];
            Level& b = *H->lv[l + 1];
            double cs = cheb_poly((b.lmax + b.lmin) / (b.lmax - b.lmin), a.ncheb);
            a.lmin = a.alpha * (1 - 1 / cs);
            a.lmax = a.beta * (1 + 1 / cs);
        }
    }
    H->lv.resize(H->nlevels);
    Level& last = *H->lv[H->nlevels - 1];
    if (H->kind == PREC_MSPLIT && H->coarse_n && !last.direct) {
        // a configured coarse_n makes the last level a direct solve even when
        // the hierarchy ended on its own (multi_split_solve.cc:77-83)
        last.direct = true;
    }
    if (last.direct) {
        if (last.N > cfg.dense_max)
            MLP_THROW(ERR_LIMIT, "coarsest level has " + std::to_string(last.N) +
                                     " unknowns, more than the dense direct solve allows (" +
                                     std::to_string(cfg.dense_max) + ")");
        build_direct(last, s);
        trace("dense coarse inverse");
    }
    build_frames(*H, s);
    CK(cudaStreamSynchronize(s));
    return H;
}

}  // namespace mlp
