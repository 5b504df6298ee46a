/*
 * CPU restatement of the ml_prec hot path. TEST INFRASTRUCTURE ONLY: the parity
 * tests, the golden-fixture script and bench.py's CPU-baseline leg use it as the
 * checker; the product library never links or calls it.
 *
 * Built with -ffp-contract=off: no fused multiply-add, so each expression rounds
 * exactly like the reference compiled for x86-64 SSE2 (g++ -O3, no -march).
 * File:line citations are into the ml_prec source tree.
 */
#define _DEFAULT_SOURCE
#include "mlp_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define KNX 60u
#define KNY 220u
#define KNZ 85u
#define KN (KNX * KNY * KNZ)

void or_csr_free(or_csr* A) {
    free(A->ia); free(A->ja); free(A->a);
    memset(A, 0, sizeof *A);
}

static void csr_alloc(or_csr* A, uint32_t nrow, uint32_t ncol, uint32_t nnz) {
    A->nrow = nrow; A->ncol = ncol;
    A->ia = (uint32_t*)calloc((size_t)nrow + 1, 4);
    A->ja = (uint32_t*)malloc((size_t)(nnz ? nnz : 1) * 4);
    A->a = (double*)malloc((size_t)(nnz ? nnz : 1) * 8);
}

/* ------------------------------------------------------------------------- */
/* Assembly: SPEMesh::construct_matrix, spe.cc:69-131 (XYZ order, mesh.h:50-77).
 * Row = diagonal first (initialised to c), then neighbours -z,-y,-x,+x,+y,+z
 * (spe.cc:109-115); each link value v = 2/(1/k_i + 1/k_j)/(h*h) (spe.cc:84),
 * stored as -v and added to the diagonal in that order (spe.cc:85-86). The
 * permeability index wraps modulo the 60x220x85 field (mesh.h:57-59).
 * Dirichlet x-faces (benchmark problem, not reference behaviour): after the
 * stencil, diag += 2*kx/hx^2 on i=0 and i=nx-1; b += that value on i=0 (p=1). */
int or_assemble(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx, const double* ky,
                const double* kz, double c, int dirichlet, or_csr* A, double* b) {
    const double hx = 20, hy = 10, hz = 2;
    uint32_t N = nx * ny * nz;
    size_t cap = 7 * (size_t)N;
    csr_alloc(A, N, N, (uint32_t)cap);
    uint32_t pos = 0;
    A->ia[0] = 0;
#define IDX(i, j, k) ((k) * ny * nx + (j) * nx + (i))
#define IDXK(i, j, k) (((k) * KNY * KNX + (j) * KNX + (i)) % KN)
#define LINK(di, dj, dk, K, H)                                                   \
    do {                                                                         \
        uint32_t i1 = IDX(i + (di), j + (dj), k + (dk));                          \
        double v = 2 / (1 / K[IDXK(i, j, k)] + 1 / K[IDXK(i + (di), j + (dj), k + (dk))]) / (H * H); \
        A->ja[pos] = i1; A->a[pos] = -v; pos++;                                  \
        A->a[dind] += v;                                                         \
    } while (0)
    for (uint32_t k = 0; k < nz; k++)
        for (uint32_t j = 0; j < ny; j++)
            for (uint32_t i = 0; i < nx; i++) {
                uint32_t i0 = IDX(i, j, k);
                uint32_t dind = pos;
                A->ja[pos] = i0; A->a[pos] = c; pos++;
                if (k) LINK(0, 0, -1, kz, hz);
                if (j) LINK(0, -1, 0, ky, hy);
                if (i) LINK(-1, 0, 0, kx, hx);
                if (i < nx - 1) LINK(+1, 0, 0, kx, hx);
                if (j < ny - 1) LINK(0, +1, 0, ky, hy);
                if (k < nz - 1) LINK(0, 0, +1, kz, hz);
                A->ia[i0 + 1] = pos;
            }
    if (b) memset(b, 0, 8 * (size_t)N);
    if (dirichlet) {
        for (uint32_t k = 0; k < nz; k++)
            for (uint32_t j = 0; j < ny; j++)
                for (int f = 0; f < 2; f++) {
                    uint32_t i = f ? nx - 1 : 0;
                    uint32_t row = IDX(i, j, k);
                    double tD = 2 * kx[IDXK(i, j, k)] / (hx * hx);
                    A->a[A->ia[row]] += tD;
                    if (f == 0 && b) b[row] += tD * 1.0;
                }
    }
#undef LINK
#undef IDX
#undef IDXK
    return 0;
}

/* y = A x, row loop in ja order (csrmatrix.cc:260-274). */
void or_spmv(const or_csr* A, const double* x, double* y) {
    for (uint32_t i = 0; i < A->nrow; i++) {
        double s = 0;
        for (uint32_t j = A->ia[i]; j < A->ia[i + 1]; j++) s += A->a[j] * x[A->ja[j]];
        y[i] = s;
    }
}

/* generate_x0, solvers.cc:9-21: srandom(3); x_i = 20*(random()-0.5*RAND_MAX)/RAND_MAX + 100. */
void or_generate_x0(double* x, uint32_t n) {
    srandom(3);
    for (uint32_t i = 0; i < n; i++) x[i] = 20. * (random() - 0.5 * RAND_MAX) / RAND_MAX + 100;
}

static int is_equal(double x, double y) { return fabs(x - y) <= DBL_EPSILON; } /* tools.h:28-30 */

static double ddot(const double* x, const double* y, uint32_t n) { /* blas.cc:41-46 */
    double s = 0.;
    for (uint32_t i = 0; i < n; i++) s += x[i] * y[i];
    return s;
}
static void daxpy(double alpha, const double* x, double* y, uint32_t n) { /* blas.cc:27-34 */
    if (!is_equal(alpha, 1.))
        for (uint32_t i = 0; i < n; i++) y[i] += alpha * x[i];
    else
        for (uint32_t i = 0; i < n; i++) y[i] += x[i];
}
static void dscal(double alpha, double* x, uint32_t n) { /* blas.cc:36-39, vector wrapper :61-66 */
    if (n && !is_equal(alpha, 1.))
        for (uint32_t i = 0; i < n; i++) x[i] *= alpha;
}

/* Stable insertion sort of off-diagonals by |a| (multi_split_constr.cc:26-36,
 * cheb_constr.cc:155-165): strict '>' keeps equal values in ja order. */
static void psort(const double* a, uint32_t n, uint32_t* sorted) {
    if (!n) return;
    sorted[0] = 0;
    for (uint32_t i = 1; i < n; i++) {
        double v = fabs(a[i]);
        int j;
        for (j = (int)i - 1; j >= 0 && fabs(a[sorted[j]]) > v; j--) sorted[j + 1] = sorted[j];
        sorted[j + 1] = i;
    }
}

/* Dense LU without pivoting (right-looking), row-major. The coarsest-level
 * direct-solver hook (multi_split_solve.cc:77-83) solves A_c x = f exactly; the
 * multi-split coarse matrix is not symmetric, so an LU stands in for UMFPACK. */
int or_dense_lu(double* a, uint32_t n) {
    for (uint32_t k = 0; k < n; k++) {
        double p = a[(size_t)k * n + k];
        if (p == 0.0) return -1;
        for (uint32_t i = k + 1; i < n; i++) {
            double l = a[(size_t)i * n + k] / p;
            a[(size_t)i * n + k] = l;
            if (l != 0.0)
                for (uint32_t j = k + 1; j < n; j++) a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
        }
    }
    return 0;
}
void or_dense_lu_solve(const double* lu, uint32_t n, const double* b, double* x) {
    for (uint32_t i = 0; i < n; i++) {
        double s = b[i];
        for (uint32_t j = 0; j < i; j++) s -= lu[(size_t)i * n + j] * x[j];
        x[i] = s;
    }
    for (int i = (int)n - 1; i >= 0; i--) {
        double s = x[i];
        for (uint32_t j = i + 1; j < n; j++) s -= lu[(size_t)i * n + j] * x[j];
        x[i] = s / lu[(size_t)i * n + i];
    }
}

/* ------------------------------------------------------------------------- */
/* Growable arrays for the factor build. */
typedef struct { uint32_t* p; size_t n, cap; } vu32;
typedef struct { double* p; size_t n, cap; } vf64;
static void pu(vu32* v, uint32_t x) {
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 64; v->p = (uint32_t*)realloc(v->p, v->cap * 4); }
    v->p[v->n++] = x;
}
static void pf(vf64* v, double x) {
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 64; v->p = (double*)realloc(v->p, v->cap * 8); }
    v->p[v->n++] = x;
}

/* Row-wise sparse elimination (sparse_lu.cc:6-133, Saad pp. 310-312).
 * keep[j_] != 0 marks links present after dropping. For every permuted row
 * i < N-Md: load the diagonal aux[map[i]] and the kept links scaled by 1/beta
 * (each subtracted from the diagonal in ja order, :51-74), then eliminate the
 * buffered columns k < min(i, M) in increasing order, l_ik = w_k / U_kk, with the
 * k-th U row's updates (fill allowed, :77-104). Rows i < M become U rows (diag
 * first, then sorted columns >= i), rows >= M become rows of the next-level
 * matrix (diag first, then sorted columns >= M other than i, shifted by -M). */
static void sparse_lu(const or_csr* A, const uint32_t* map, const uint32_t* rmap, uint32_t Md,
                      uint32_t M, const unsigned char* keep, double beta, const double* aux,
                      or_csr* nA, or_csr* U, or_csr* L) {
    uint32_t N = A->nrow, n = N - M - Md;
    vu32 Lja = {0}, Uja = {0}, nja = {0};
    vf64 La = {0}, Ua = {0}, na = {0};
    uint32_t* Lia = (uint32_t*)malloc(((size_t)(N - Md) + 1) * 4);
    uint32_t* Uia = (uint32_t*)malloc(((size_t)M + 1) * 4);
    uint32_t* nia = (uint32_t*)malloc(((size_t)n + 1) * 4);
    Lia[0] = Uia[0] = nia[0] = 0;
    /* working row: sorted column list with values */
    size_t wcap = 64;
    uint32_t* wc = (uint32_t*)malloc(wcap * 4);
    double* wv = (double*)malloc(wcap * 8);
    for (uint32_t i = 0; i < N - Md; i++) {
        uint32_t arow = map[i], wn = 0;
        /* insert keeping columns sorted; values follow */
#define WINS(col, val)                                                            \
        do {                                                                      \
            if (wn == wcap) { wcap *= 2; wc = (uint32_t*)realloc(wc, wcap * 4); wv = (double*)realloc(wv, wcap * 8); } \
            uint32_t p_ = wn;                                                     \
            while (p_ > 0 && wc[p_ - 1] > (col)) { wc[p_] = wc[p_ - 1]; wv[p_] = wv[p_ - 1]; p_--; } \
            wc[p_] = (col); wv[p_] = (val); wn++;                                 \
        } while (0)
        double diag = aux[arow];
        /* the diagonal slot is updated as links are read; insert it first */
        WINS(i, 0.0);
        for (uint32_t j_ = A->ia[arow] + 1; j_ < A->ia[arow + 1]; j_++) {
            if (!keep[j_]) continue;
            uint32_t nj = rmap[A->ja[j_]];
            double z = A->a[j_] / beta;
            WINS(nj, z);
            diag -= z;
        }
        for (uint32_t t = 0; t < wn; t++) if (wc[t] == i) wv[t] = diag;
        uint32_t m = i < M ? i : M;
        /* eliminate in increasing column order; inserted columns are > k */
        for (uint32_t t = 0; t < wn && wc[t] < m; t++) {
            uint32_t k = wc[t];
            double ukk = Ua.p[Uia[k]];
            double lik = wv[t] / ukk;
            pu(&Lja, k); pf(&La, lik);
            for (uint32_t u = Uia[k] + 1; u < Uia[k + 1]; u++) {
                uint32_t j = Uja.p[u];
                double uv = Ua.p[u];
                /* find j in the working row (sorted) */
                uint32_t lo = 0, hi = wn;
                while (lo < hi) { uint32_t mid = (lo + hi) / 2; if (wc[mid] < j) lo = mid + 1; else hi = mid; }
                if (lo < wn && wc[lo] == j) wv[lo] -= lik * uv;
                else WINS(j, -lik * uv);
            }
        }
        Lia[i + 1] = (uint32_t)Lja.n;
        if (i < M) {
            for (uint32_t t = 0; t < wn; t++)
                if (wc[t] >= i) { pu(&Uja, wc[t]); pf(&Ua, wv[t]); }
            Uia[i + 1] = (uint32_t)Uja.n;
        } else {
            double dv = 0; for (uint32_t t = 0; t < wn; t++) if (wc[t] == i) dv = wv[t];
            pu(&nja, i - M); pf(&na, dv);
            for (uint32_t t = 0; t < wn; t++)
                if (wc[t] >= M && wc[t] != i) { pu(&nja, wc[t] - M); pf(&na, wv[t]); }
            nia[i - M + 1] = (uint32_t)nja.n;
        }
#undef WINS
    }
    free(wc); free(wv);
    L->nrow = L->ncol = N - Md; L->ia = Lia; L->ja = Lja.p; L->a = La.p;
    U->nrow = M; U->ncol = N - Md; U->ia = Uia; U->ja = Uja.p; U->a = Ua.p;
    nA->nrow = nA->ncol = n; nA->ia = nia; nA->ja = nja.p; nA->a = na.p;
    if (!L->ja) { L->ja = (uint32_t*)malloc(4); L->a = (double*)malloc(8); }
    if (!U->ja) { U->ja = (uint32_t*)malloc(4); U->a = (double*)malloc(8); }
    if (!nA->ja) { nA->ja = (uint32_t*)malloc(4); nA->a = (double*)malloc(8); }
}

static void csr_copy(or_csr* dst, const or_csr* src) {
    uint32_t nnz = src->ia[src->nrow];
    csr_alloc(dst, src->nrow, src->ncol, nnz);
    memcpy(dst->ia, src->ia, ((size_t)src->nrow + 1) * 4);
    memcpy(dst->ja, src->ja, (size_t)nnz * 4);
    memcpy(dst->a, src->a, (size_t)nnz * 8);
}

/* ---- multi-split level construction -------------------------------------- */
/* Marking (multi_split_constr.cc:60-113). */
static void ms_mark(const or_csr* A, double q, unsigned char* keep, int* nout, int* nin, double* aux) {
    uint32_t N = A->nrow;
    uint32_t* sorted = (uint32_t*)malloc(10000 * 4);
    for (uint32_t i = 0; i < N; i++) nin[i] = 0;
    memset(keep, 1, A->ia[N]);
    for (uint32_t i = 0; i < N; i++) {
        uint32_t rs = A->ia[i], re = A->ia[i + 1], nrz = re - rs - 1;
        nout[i] = (int)nrz;
        aux[i] = A->a[rs];
        for (uint32_t j_ = rs + 1; j_ < re; j_++) { nin[A->ja[j_]]++; aux[i] += A->a[j_]; }
        psort(A->a + rs + 1, nrz, sorted);
        double s = q / (1 - q) * aux[i];
        for (uint32_t k = 0; k < nrz; k++) {
            uint32_t j_ = rs + 1 + sorted[k];
            double aij = -A->a[j_];
            if (aij <= s) {
                keep[j_] = 0;
                nout[i]--;
                nin[A->ja[j_]]--;
                s -= aij;
            } else
                break;
        }
        aux[i] *= 1. / (1 - q);
    }
    free(sorted);
}

/* order_none (multi_split_mark.cc:8-25): diagonal nodes last, in reverse. */
static void ms_order_none(uint32_t N, const int* nin, const int* nout, uint32_t* Md, uint32_t* M, uint32_t* map) {
    uint32_t pind = 0, eind = N - 1;
    *M = 0;
    for (uint32_t i = 0; i < N; i++)
        if (nin[i] == 0 && nout[i] == 0) map[eind--] = i; else map[pind++] = i;
    *Md = N - pind;
}

/* order_simple_1 (multi_split_mark.cc:156-191): buckets by kept out-degree
 * [out=0 & in!=0 | 1 | 2 | >2], M after bucket degree_max, then out=0 & in=0. */
static void ms_order_simple_1(uint32_t N, const int* nin, const int* nout, uint32_t degree_max,
                              uint32_t* Md, uint32_t* M, uint32_t* map) {
    uint32_t pind = 0;
    for (uint32_t i = 0; i < N; i++) if (nout[i] == 0 && nin[i] != 0) map[pind++] = i;
    for (int d = 1; d <= 3; d++) {
        for (uint32_t i = 0; i < N; i++) {
            int b = nout[i] <= 2 ? nout[i] : 3;
            if (b == d) map[pind++] = i;
        }
        if ((uint32_t)d == degree_max) *M = pind;
    }
    uint32_t start = pind;
    for (uint32_t i = 0; i < N; i++) if (nout[i] == 0 && nin[i] == 0) map[pind++] = i;
    *Md = N - start;
}

/* order_original (multi_split_mark.cc:27-154) with the tail group enabled when
 * use_tails != 0. keep is modified on a copy (the reference copies ltype). */
static int ms_order_original(const or_csr* A, const unsigned char* keep0, int* nin, int* nout, int use_tails,
                             uint32_t* Md, uint32_t* M, uint32_t* map) {
    uint32_t N = A->nrow, pind = 0;
    uint32_t nnz = A->ia[N];
    unsigned char* keep = (unsigned char*)malloc(nnz ? nnz : 1);
    memcpy(keep, keep0, nnz);
    unsigned char* marked = (unsigned char*)calloc(N ? N : 1, 1);
    if (use_tails) {
        for (uint32_t i = 0; i < N; i++) {
            if (!(nout[i] == 1 && nin[i] <= 1)) continue;
            uint32_t i0 = i, i1;
            for (;;) {
                if (nout[i0] != 1) break;
                uint32_t j_;
                for (j_ = A->ia[i0] + 1; j_ < A->ia[i0 + 1]; j_++) if (keep[j_]) break;
                if (j_ == A->ia[i0 + 1]) { free(keep); free(marked); return -1; }
                i1 = A->ja[j_];
                /* stat(i1, i0): binary search of column i0 in row i1 (skyline.cc:15-28) */
                int aji = 0; uint32_t aji_pos = 0;
                {
                    uint32_t lo = A->ia[i1] + 1, hi = A->ia[i1 + 1];
                    while (lo < hi) { uint32_t mid = (lo + hi) / 2; if (A->ja[mid] < i0) lo = mid + 1; else hi = mid; }
                    if (lo < A->ia[i1 + 1] && A->ja[lo] == i0) { aji_pos = lo; aji = keep[lo] ? 1 : 0; }
                }
                if (!(nin[i0] == 0 || (nin[i0] == 1 && aji))) break;
                map[pind++] = i0;
                marked[i0] = 1;
                keep[j_] = 0;
                if (aji) { keep[aji_pos] = 0; nin[i0]--; nout[i1]--; }
                nout[i0] = -1;
                nin[i1]--;
                i0 = i1;
            }
            if (nout[i0] == 0 && nin[i0] == 0) { map[pind++] = i0; marked[i0] = 1; nout[i0] = -1; }
        }
    }
    for (uint32_t i = 0; i < N; i++)
        if (!marked[i] && (nin[i] <= 2 || nout[i] <= 2)) {
            map[pind++] = i; nin[i] = 0; nout[i] = -1; marked[i] = 1;
        }
    *M = pind;
    uint32_t eind = N - 1;
    for (uint32_t i = 0; i < N; i++)
        if (!marked[i]) {
            if (nin[i] == 0 && nout[i] == 0) map[eind--] = i; else map[pind++] = i;
        }
    *Md = N - pind;
    free(keep); free(marked);
    return 0;
}

static void set_err(char* err, int errlen, const char* msg) {
    if (err && errlen > 0) { strncpy(err, msg, errlen - 1); err[errlen - 1] = 0; }
}

/* MultiSplitPrec::construct_level (multi_split_constr.cc:39-168) with the
 * direct-solver hook compiled in (HAVE_UMFPACK): a level becomes the coarsest
 * (solved directly) when N <= coarse_n or it is the last allowed level. */
static int ms_construct(or_prec* P, const or_prec_cfg* cfg, uint32_t level, char* err, int errlen) {
    or_level* li = &P->levels[level];
    const or_csr* A = &li->A;
    li->N = A->nrow;
    li->nnz = A->ia[A->nrow];
    if (li->N <= P->coarse_n || level == P->nlevels - 1) {
        P->nlevels = level + 1;
        P->coarse_n = li->N;
        return 0;
    }
    uint32_t N = li->N, nnz = li->nnz;
    unsigned char* keep = (unsigned char*)malloc(nnz ? nnz : 1);
    int* nout = (int*)malloc((size_t)N * sizeof(int));
    int* nin = (int*)malloc((size_t)N * sizeof(int));
    double* aux = (double*)malloc((size_t)N * 8);
    ms_mark(A, li->q, keep, nout, nin, aux);
    li->map = (uint32_t*)malloc((size_t)N * 4);
    li->M = 0; li->Md = 0;
    switch (cfg->order) {
        case OR_ORDER_NONE: ms_order_none(N, nin, nout, &li->Md, &li->M, li->map); break;
        case OR_ORDER_SIMPLE_1: ms_order_simple_1(N, nin, nout, cfg->degree_max, &li->Md, &li->M, li->map); break;
        case OR_ORDER_ORIGINAL:
            if (ms_order_original(A, keep, nin, nout, cfg->use_tails, &li->Md, &li->M, li->map)) {
                set_err(err, errlen, "remaining link was not found");
                return -1;
            }
            break;
        default: set_err(err, errlen, "unsupported elim_order"); return -1;
    }
    li->rmap = (uint32_t*)malloc((size_t)N * 4);
    for (uint32_t i = 0; i < N; i++) li->rmap[li->map[i]] = i;
    or_level* ln = &P->levels[level + 1];
    sparse_lu(A, li->map, li->rmap, li->Md, li->M, keep, 1.0, aux, &ln->A, &li->U, &li->L);
    li->dval = (double*)malloc(((size_t)li->Md + 1) * 8);
    for (uint32_t i = 0; i < li->Md; i++) li->dval[i] = 1. / aux[li->map[i + (N - li->Md)]];
    free(keep); free(nout); free(nin); free(aux);
    if (ln->A.nrow) return ms_construct(P, cfg, level + 1, err, errlen);
    or_csr_free(&ln->A);
    P->nlevels = level + 1;
    return 0;
}

/* ---- uh_cheb level construction (cheb_constr.cc:167-290) ------------------ */
/* Undirected link state (cheb_misc.h:15-96): one counter per link, stored at the
 * upper-triangle position; 2 = present, decremented by mark() from each end,
 * 0 = removed. upos[j_] maps every stored position to its upper-triangle slot. */
static uint32_t sky_index(const or_csr* A, uint32_t i, uint32_t j) { /* skyline.cc:15-28 */
    if (i == j) return A->ia[i];
    uint32_t lo = A->ia[i] + 1, hi = A->ia[i + 1];
    while (lo < hi) { uint32_t mid = (lo + hi) / 2; if (A->ja[mid] < j) lo = mid + 1; else hi = mid; }
    if (lo < A->ia[i + 1] && A->ja[lo] == j) return lo;
    return (uint32_t)-1;
}

double or_cheb(double x, uint32_t k) { /* misc.cc:232-242 */
    switch (k) {
        case 0: return 1;
        case 1: return x;
        case 2: return 2 * x * x - 1;
        case 3: return x * (4 * x * x - 3);
        default: return cosh(k * acosh(x));
    }
}

static int ch_construct(or_prec* P, const or_prec_cfg* cfg, uint32_t level, char* err, int errlen) {
    or_level* li = &P->levels[level];
    const or_csr* A = &li->A;
    uint32_t N = A->nrow, nnz = A->ia[N];
    li->N = N; li->nnz = nnz;
    int* nlinks = (int*)calloc(N ? N : 1, sizeof(int));
    unsigned char* cnt = (unsigned char*)malloc(nnz ? nnz : 1); /* counters at upper slots */
    uint32_t* upos = (uint32_t*)malloc((size_t)(nnz ? nnz : 1) * 4);
    for (uint32_t i = 0; i < N; i++)
        for (uint32_t j_ = A->ia[i] + 1; j_ < A->ia[i + 1]; j_++) {
            uint32_t j = A->ja[j_];
            if (j < i) upos[j_] = sky_index(A, j, i); else { upos[j_] = j_; cnt[j_] = 2; }
        }
    double* aux = (double*)malloc((size_t)(N ? N : 1) * 8);
    uint32_t* sorted = (uint32_t*)malloc(1000 * 4);
    for (uint32_t i = 0; i < N; i++) {
        uint32_t rs = A->ia[i], re = A->ia[i + 1], nrz = re - rs - 1;
        nlinks[i] += (int)nrz;
        aux[i] = 0.0;
        for (uint32_t j_ = rs; j_ < re; j_++) aux[i] += A->a[j_];
        psort(A->a + rs + 1, nrz, sorted);
        double s = 0.;
        for (uint32_t t = 0; t < nrz; t++) {
            double v = A->a[rs + 1 + sorted[t]];
            /* to_remove (cheb_prec.h:57-85, dynamic variant) */
            double tt = -2 * v / (aux[i] * (li->beta - 1));
            if (s + tt > 1) break;
            s += tt;
            uint32_t j_ = rs + 1 + sorted[t];
            uint32_t j = A->ja[j_];
            if (--cnt[upos[j_]] == 0) { nlinks[i]--; nlinks[j]--; }
        }
    }
    free(sorted);
    /* construct_permutation (cheb_mark.cc:8-92) on a copy of the link state */
    unsigned char* c2 = (unsigned char*)malloc(nnz ? nnz : 1);
    memcpy(c2, cnt, nnz);
    unsigned char* marked = (unsigned char*)calloc(N ? N : 1, 1);
    li->map = (uint32_t*)malloc((size_t)(N ? N : 1) * 4);
    uint32_t pind = 0;
    if (cfg->use_tails) {
        for (uint32_t i = 0; i < N; i++) {
            if (nlinks[i] != 1) continue;
            uint32_t i0 = i, i1 = (uint32_t)-1;
            do {
                li->map[pind++] = i0;
                marked[i0] = 1;
                uint32_t j_;
                for (j_ = A->ia[i0] + 1; j_ < A->ia[i0 + 1]; j_++)
                    if (c2[upos[j_]]) { i1 = A->ja[j_]; break; }
                if (j_ == A->ia[i0 + 1]) { set_err(err, errlen, "Could not find remaining link"); return -1; }
                c2[upos[j_]] = 0;  /* remove(i0, i1) */
                nlinks[i0] = -1;
                nlinks[i1]--;
                i0 = i1;
            } while (nlinks[i0] == 1);
            if (nlinks[i0] == 0) { li->map[pind++] = i0; marked[i0] = 1; nlinks[i0] = -1; }
        }
    }
    li->M = pind;
    uint32_t eind = N - 1;
    for (uint32_t i = 0; i < N; i++)
        if (!marked[i]) { if (nlinks[i] == 0) li->map[eind--] = i; else li->map[pind++] = i; }
    li->Md = N - pind;
    free(c2); free(marked);
    li->rmap = (uint32_t*)malloc((size_t)(N ? N : 1) * 4);
    for (uint32_t i = 0; i < N; i++) li->rmap[li->map[i]] = i;
    /* present links for the elimination: counter != 0 */
    unsigned char* keep = (unsigned char*)malloc(nnz ? nnz : 1);
    for (uint32_t i = 0; i < N; i++) {
        keep[A->ia[i]] = 1;
        for (uint32_t j_ = A->ia[i] + 1; j_ < A->ia[i + 1]; j_++) keep[j_] = cnt[upos[j_]] != 0;
    }
    or_level* ln = &P->levels[level + 1];
    sparse_lu(A, li->map, li->rmap, li->Md, li->M, keep, li->beta, aux, &ln->A, &li->U, &li->L);
    li->dval = (double*)malloc(((size_t)li->Md + 1) * 8);
    for (uint32_t i = 0; i < li->Md; i++) li->dval[i] = 1. / aux[li->map[i + (N - li->Md)]];
    free(keep); free(cnt); free(upos); free(aux); free(nlinks);
    if (ln->A.nrow) {
        if (level + 1 >= P->nlevels) { set_err(err, errlen, "Too many levels"); return -1; }
        return ch_construct(P, cfg, level + 1, err, errlen);
    }
    or_csr_free(&ln->A);
    P->nlevels = level + 1;
    return 0;
}

/* ---- build / free ------------------------------------------------------- */
/* SymPrec::SymPrec (sym_prec.cc:19-40): a_ij = max(a_ij, a_ji) off the
 * diagonal (a missing a_ji counts as 0; the rows' order does not matter, the
 * in-place loop gives the same result), then the uh_cheb Prec of it. */
static or_prec* sym_build(const or_csr* A, const or_prec_cfg* cfg, char* err, int errlen) {
    or_prec* P = (or_prec*)calloc(1, sizeof *P);
    P->kind = OR_PREC_SYM;
    csr_copy(&P->Asym, A);
    or_csr* S = &P->Asym;
    for (uint32_t i = 0; i < S->nrow; i++)
        for (uint32_t j_ = S->ia[i] + 1; j_ < S->ia[i + 1]; j_++) {
            uint32_t j = S->ja[j_];
            uint32_t lo = S->ia[j] + 1, hi = S->ia[j + 1];
            while (lo < hi) { uint32_t mid = (lo + hi) / 2; if (S->ja[mid] < i) lo = mid + 1; else hi = mid; }
            double d = (lo < S->ia[j + 1] && S->ja[lo] == i) ? S->a[lo] : 0.0; /* Asym(j, i) */
            if (d > S->a[j_]) S->a[j_] = d;
        }
    or_prec_cfg c1 = *cfg;
    c1.kind = OR_PREC_CHEB;
    P->inner = or_prec_build(S, &c1, err, errlen);
    if (!P->inner) { or_csr_free(S); free(P); return NULL; }
    P->nlevels = ((or_prec*)P->inner)->nlevels;
    P->levels = NULL;
    return P;
}

or_prec* or_prec_build(const or_csr* A, const or_prec_cfg* cfg, char* err, int errlen) {
    if (cfg->kind == OR_PREC_SYM) return sym_build(A, cfg, err, errlen);
    or_prec* P = (or_prec*)calloc(1, sizeof *P);
    P->kind = cfg->kind;
    int rc = 0;
    if (cfg->kind == OR_PREC_MSPLIT) {
        /* multi_split_constr.cc:252-275 */
        P->nlevels = cfg->max_levels;
        P->coarse_n = cfg->coarse_n;
        if (P->nlevels == 0 || cfg->nq == 0) { set_err(err, errlen, "bad config"); free(P); return NULL; }
        P->levels = (or_level*)calloc(P->nlevels + 1, sizeof(or_level));
        for (uint32_t l = 0; l < P->nlevels; l++) {
            P->levels[l].q = l >= cfg->nq ? cfg->q[cfg->nq - 1] : cfg->q[l];
            /* multi_split_constr.cc:256-264: level 0 always one iteration; the
             * others a fixed count or, with dynamic inner iterations, an eps
             * (niter keeps the Level() default 0 then) */
            if (l == 0) P->levels[l].niter = 1;
            else if (cfg->neps) P->levels[l].eps = l >= cfg->neps ? cfg->level_eps[cfg->neps - 1] : cfg->level_eps[l];
            else P->levels[l].niter = l >= cfg->nnit ? cfg->niter[cfg->nnit - 1] : cfg->niter[l];
        }
        csr_copy(&P->levels[0].A, A);
        rc = ms_construct(P, cfg, 0, err, errlen);
        if (rc == 0 && P->levels[P->nlevels - 1].M == 0) {
            P->levels[P->nlevels - 1].niter = 0;
            P->levels[P->nlevels - 1].eps = 0;
            P->levels[P->nlevels - 1].q = 0;
        }
    } else {
        /* cheb_constr.cc:292-365 */
        P->nlevels = 30;
        P->coarse_n = 0;
        P->levels = (or_level*)calloc(P->nlevels + 1, sizeof(or_level));
        for (uint32_t l = 0; l < P->nlevels; l++) {
            P->levels[l].alpha = 1.0;
            P->levels[l].beta = l < cfg->nsig ? cfg->sigma[l] : cfg->sigma[cfg->nsig - 1];
        }
        csr_copy(&P->levels[0].A, A);
        rc = ch_construct(P, cfg, 0, err, errlen);
        if (rc == 0) {
            for (uint32_t l = 0; l < P->nlevels; l++)
                P->levels[l].ncheb = l >= cfg->nch ? cfg->ncheb[cfg->nch - 1] : cfg->ncheb[l];
            or_level* last = &P->levels[P->nlevels - 1];
            last->lmin = last->alpha;
            last->lmax = last->beta;
            for (int l = (int)P->nlevels - 2; l >= 0; l--) {
                or_level* a = &P->levels[l];
                or_level* b = &P->levels[l + 1];
                double cs = or_cheb((b->lmax + b->lmin) / (b->lmax - b->lmin), a->ncheb);
                a->lmin = a->alpha * (1 - 1 / cs);
                a->lmax = a->beta * (1 + 1 / cs);
            }
        }
    }
    if (rc) { or_prec_free(P); return NULL; }
    if (P->kind == OR_PREC_MSPLIT && P->coarse_n) {
        or_level* c = &P->levels[P->nlevels - 1];
        uint32_t n = c->A.nrow;
        c->lu = (double*)calloc((size_t)n * n + 1, 8);
        for (uint32_t i = 0; i < n; i++)
            for (uint32_t j = c->A.ia[i]; j < c->A.ia[i + 1]; j++) c->lu[(size_t)i * n + c->A.ja[j]] = c->A.a[j];
        if (or_dense_lu(c->lu, n)) { set_err(err, errlen, "zero pivot in coarse LU"); or_prec_free(P); return NULL; }
    }
    size_t tot = 0;
    for (uint32_t l = 0; l < P->nlevels; l++) tot += 6 * (size_t)P->levels[l].N + 8;
    P->work = (double*)calloc(tot, 8);
    return P;
}

void or_prec_free(or_prec* P) {
    if (!P) return;
    if (P->kind == OR_PREC_SYM) {
        or_prec_free((or_prec*)P->inner);
        or_csr_free(&P->Asym);
        free(P);
        return;
    }
    for (uint32_t l = 0; l <= P->nlevels && P->levels; l++) {
        or_level* li = &P->levels[l];
        or_csr_free(&li->A); or_csr_free(&li->L); or_csr_free(&li->U);
        free(li->map); free(li->rmap); free(li->dval); free(li->lu);
    }
    free(P->levels); free(P->work); free(P);
}

uint32_t or_prec_nlevels(const or_prec* P) { return P->nlevels; }
const or_level* or_prec_level(const or_prec* P, uint32_t l) {
    if (P->kind == OR_PREC_SYM) return &((const or_prec*)P->inner)->levels[l];
    return &P->levels[l];
}

/* ---- apply -------------------------------------------------------------- */
static double* level_work(const or_prec* P, uint32_t level) {
    size_t off = 0;
    for (uint32_t l = 0; l < level; l++) off += 6 * (size_t)P->levels[l].N + 8;
    return P->work + off;
}

/* solve_L (multi_split_solve.cc:25-36): w_i = f[map i] - sum L_ik w_k. */
static void solve_L(const or_level* li, const double* f, double* w) {
    uint32_t R = li->N - li->Md;
    for (uint32_t i = 0; i < R; i++) {
        w[i] = f[li->map[i]];
        for (uint32_t j = li->L.ia[i]; j < li->L.ia[i + 1]; j++) w[i] -= li->L.a[j] * w[li->L.ja[j]];
    }
}
/* solve_U (multi_split_solve.cc:39-53). */
static void solve_U(const or_level* li, const double* w, double* x) {
    for (int i = (int)li->M - 1; i >= 0; i--) {
        double z = w[i];
        for (uint32_t j = li->U.ia[i] + 1; j < li->U.ia[i + 1]; j++) z -= li->U.a[j] * x[li->map[li->U.ja[j]]];
        x[li->map[i]] = z / li->U.a[li->U.ia[i]];
    }
}
/* solve_diagonal (multi_split_solve.cc:12-22). */
static void solve_diag(const or_level* li, const double* f, double* x) {
    for (uint32_t i = 0; i < li->Md; i++) {
        uint32_t j = li->map[(li->N - li->Md) + i];
        x[j] = li->dval[i] * f[j];
    }
}

static double or_dnrm2(const double* x, uint32_t n) {
    double s = 0; /* blas.cc:52-54: sqrt(ddot(x, x)), a sequential sum */
    for (uint32_t i = 0; i < n; i++) s += x[i] * x[i];
    return sqrt(s);
}

/* Sweeps of one dynamic level call before the oracle gives up (the reference
 * has no cap and would loop for ever). */
#define OR_LEVEL_SWEEP_CAP 100000u

/* MultiSplitPrec::solve(level, f, x) (multi_split_solve.cc:59-157): fixed inner
 * iterations, or with li->eps != 0 sweeps until ||f - A x|| / ||f|| < eps. */
static void ms_solve(or_prec* P, uint32_t level, const double* f, double* x) {
    const or_level* li = &P->levels[level];
    uint32_t N = li->N, M = li->M;
    uint32_t n = level < P->nlevels - 1 ? P->levels[level + 1].N : 0;
    if (level == P->nlevels - 1 && P->coarse_n) {
        or_dense_lu_solve(li->lu, N, f, x);
        return;
    }
    double* wk = level_work(P, level);
    double *r = wk, *w = wk + N, *u0 = wk + 2 * (size_t)N, *x2 = wk + 3 * (size_t)N, *F = wk + 4 * (size_t)N;
    memcpy(r, f, 8 * (size_t)N);
    double init_norm = li->eps != 0 ? or_dnrm2(r, N) : 0;
    solve_L(li, r, w);
    if (level < P->nlevels - 1) {
        memcpy(F, w + M, 8 * (size_t)n);
        ms_solve(P, level + 1, F, x2);
        for (uint32_t i = 0; i < n; i++) x[li->map[i + M]] = x2[i];
    }
    solve_U(li, w, x);
    solve_diag(li, r, x);
    for (uint32_t it = 2; li->eps != 0 || it <= li->niter; it++) {
        or_spmv(&li->A, x, r);
        for (uint32_t i = 0; i < N; i++) r[i] = f[i] - r[i];
        if (li->eps != 0) {
            if (or_dnrm2(r, N) / init_norm < li->eps) break;
            if (it > OR_LEVEL_SWEEP_CAP) { P->apply_err = 1; break; }
        }
        solve_L(li, r, w);
        if (level < P->nlevels - 1) {
            memcpy(F, w + M, 8 * (size_t)n);
            ms_solve(P, level + 1, F, x2);
            for (uint32_t i = 0; i < n; i++) u0[li->map[i + M]] = x2[i];
        }
        solve_U(li, w, u0);
        solve_diag(li, r, u0);
        daxpy(1., u0, x, N);
    }
}

/* sym_multiply (skyline.cc:115-155): lower half incl. diagonal, mirrored. */
static void sym_spmv(const or_csr* A, const double* v, double* res) {
    uint32_t N = A->nrow;
    memset(res, 0, 8 * (size_t)N);
    for (uint32_t i = 0; i < N; i++) {
        uint32_t s = A->ia[i], e = A->ia[i + 1];
        res[i] += A->a[s] * v[i];
        for (uint32_t j_ = s + 1; j_ < e; j_++) {
            uint32_t j = A->ja[j_];
            if (j > i) break; /* columns after the diagonal are sorted */
            res[i] += A->a[j_] * v[j];
            res[j] += A->a[j_] * v[i];
        }
    }
}

/* Prec::solve(level, f, x) (cheb_solve.cc:13-123). */
static void ch_solve(const or_prec* P, uint32_t level, const double* f, double* x) {
    const or_level* li = &P->levels[level];
    uint32_t N = li->N, M = li->M;
    double* wk = level_work(P, level);
    double* w = wk;
    solve_L(li, f, w);
    if (level < P->nlevels - 1) {
        const or_level* ln = &P->levels[level + 1];
        uint32_t n = ln->N, nch = li->ncheb;
        double *F = wk + N, *tmp = wk + 2 * (size_t)N, *x2 = wk + 3 * (size_t)N, *u1 = wk + 4 * (size_t)N,
               *u0 = wk + 5 * (size_t)N;
        memcpy(F, w + M, 8 * (size_t)n);
        double lmin = ln->lmin, lmax = ln->lmax;
        double eta = (lmax + lmin) / (lmax - lmin);
        memcpy(tmp, F, 8 * (size_t)n);
        double alpha = 2 / (lmax + lmin), beta;
        if (nch > 1) { ch_solve(P, level + 1, tmp, u1); dscal(alpha, u1, n); }
        else { ch_solve(P, level + 1, tmp, x2); dscal(alpha, x2, n); }
        if (nch > 1) {
            alpha = 4 / (lmax - lmin) * or_cheb(eta, 1) / or_cheb(eta, 2);
            beta = or_cheb(eta, 0) / or_cheb(eta, 2);
            sym_spmv(&ln->A, u1, tmp);
            daxpy(-1, F, tmp, n);
            ch_solve(P, level + 1, tmp, x2);
            dscal(-alpha, x2, n);
            daxpy(1 + beta, u1, x2, n);
        }
        for (uint32_t i = 3; i <= nch; i++) {
            double* t = u0; u0 = u1; u1 = x2; x2 = t;  /* swaps at cheb_solve.cc:87-89 */
            alpha = 4 / (lmax - lmin) * or_cheb(eta, i - 1) / or_cheb(eta, i);
            beta = or_cheb(eta, i - 2) / or_cheb(eta, i);
            sym_spmv(&ln->A, u1, tmp);
            daxpy(-1, F, tmp, n);
            ch_solve(P, level + 1, tmp, x2);
            for (uint32_t k = 0; k < n; k++) x2[k] = u1[k] - alpha * x2[k] + beta * (u1[k] - u0[k]);
        }
        for (uint32_t i = 0; i < n; i++) x[li->map[i + M]] = x2[i];
    }
    solve_U(li, w, x);
    solve_diag(li, f, x);
}

void or_prec_apply(const or_prec* P, const double* f, double* x) {
    if (P->kind == OR_PREC_MSPLIT) ms_solve((or_prec*)P, 0, f, x);  /* apply_err is the only write */
    else if (P->kind == OR_PREC_SYM) {
        /* SymPrec::solve (sym_prec.cc:8-17): PCGSolver(Asym, f, B, x, 1e-14) from generate_x0 */
        uint32_t it;
        double rel;
        int rc = or_pcg_ex(&P->Asym, f, (const or_prec*)P->inner, x, 1e-14, &it, &rel, 0, 0);
        if (rc != 0) ((or_prec*)P)->apply_err = 1;
    } else ch_solve(P, 0, f, x);
}

/* ---- ChebSolver (cheb.cc:9-100) -------------------------------------------- */
int or_cheb_solve(const or_csr* A, const double* b, const or_prec* P, double lmin, double lmax, double* x_out,
                  double eps, uint32_t* niter_out, double* final_rel, uint32_t maxit) {
    uint32_t n = A->nrow;
    double* r = (double*)malloc(8 * (size_t)n);
    double* buf[3];
    for (int k = 0; k < 3; k++) buf[k] = (double*)malloc(8 * (size_t)n);
    double *x = buf[0], *u1 = buf[1], *u0 = buf[2];
    double eta = (lmax + lmin) / (lmax - lmin);
    or_generate_x0(x, n);
    or_spmv(A, x, r);
    for (uint32_t i = 0; i < n; i++) r[i] = b[i] - r[i];
    double norm = sqrt(ddot(r, r, n)), init_norm = norm;
    uint32_t niter = 1;
    if (init_norm * eps < 1e-14) eps = 1e-14 / init_norm; /* solvers.cc:49-58 */
    /* step 1: u1 = x; x = alpha B r + u1 */
    double alpha = 2 / (lmax + lmin), beta;
    memcpy(u1, x, 8 * (size_t)n);
    or_prec_apply(P, r, x);
    dscal(alpha, x, n);
    daxpy(1, u1, x, n);
    or_spmv(A, x, r);
    for (uint32_t i = 0; i < n; i++) r[i] = b[i] - r[i];
    norm = sqrt(ddot(r, r, n));
    niter++;
    if (maxit == 0) maxit = 100000; /* the checker must always return */
    int rc = 0;
    while (norm / init_norm > eps) {
        if (niter - 1 >= maxit) { rc = -3; break; }
        double* t = u0; u0 = x; x = t; /* u0.swap(x) */
        t = u1; u1 = u0; u0 = t;       /* u1.swap(u0) */
        alpha = 4 / (lmax - lmin) * or_cheb(eta, niter - 1) / or_cheb(eta, niter);
        beta = or_cheb(eta, niter - 2) / or_cheb(eta, niter);
        or_prec_apply(P, r, x);
        for (uint32_t k = 0; k < n; k++) x[k] = u1[k] + alpha * x[k] + beta * (u1[k] - u0[k]);
        or_spmv(A, x, r);
        for (uint32_t i = 0; i < n; i++) r[i] = b[i] - r[i];
        norm = sqrt(ddot(r, r, n));
        niter++;
    }
    niter--; /* cheb.cc:84 */
    memcpy(x_out, x, 8 * (size_t)n);
    *niter_out = niter;
    *final_rel = norm / init_norm;
    free(r);
    for (int k = 0; k < 3; k++) free(buf[k]);
    if (rc == 0 && P->apply_err) rc = -4;
    return rc;
}

/* ---- PCG (pcg.cc:8-102) ---------------------------------------------------- */
int or_pcg(const or_csr* A, const double* b, const or_prec* P, double* x, double eps,
           uint32_t* niter_out, double* final_rel, uint32_t maxit) {
    return or_pcg_ex(A, b, P, x, eps, niter_out, final_rel, maxit, 0);
}

int or_pcg_ex(const or_csr* A, const double* b, const or_prec* P, double* x, double eps,
              uint32_t* niter_out, double* final_rel, uint32_t maxit, int x0_mode) {
    uint32_t n = A->nrow;
    double* r = (double*)malloc(8 * (size_t)n);
    double* z = (double*)malloc(8 * (size_t)n);
    double* p = (double*)malloc(8 * (size_t)n);
    double* Ap = (double*)malloc(8 * (size_t)n);
    if (x0_mode == 1) memset(x, 0, 8 * (size_t)n);
    else or_generate_x0(x, n);
    or_spmv(A, x, r);
    for (uint32_t i = 0; i < n; i++) r[i] = b[i] - r[i];
    double norm = sqrt(ddot(r, r, n)), init_norm = norm;
    or_prec_apply(P, r, z);
    memcpy(p, z, 8 * (size_t)n);
    double rz0 = ddot(r, z, n);
    if (init_norm * eps < 1e-14) eps = 1e-14 / init_norm; /* solvers.cc:49-58 */
    if (maxit == 0) maxit = 100000; /* the checker must always return */
    uint32_t it = 0;
    int rc = 0;
    while (norm / init_norm > eps) {
        if (maxit && it >= maxit) { rc = -3; break; }
        or_spmv(A, p, Ap);
        double app = ddot(Ap, p, n);
        if (app <= 0) { rc = -1; break; }
        double alpha = rz0 / app;
        daxpy(alpha, p, x, n);
        daxpy(-alpha, Ap, r, n);
        norm = sqrt(ddot(r, r, n));
        or_prec_apply(P, r, z);
        double rz1 = ddot(r, z, n);
        double beta = rz1 / rz0;
        dscal(beta, p, n);
        daxpy(1, z, p, n);
        rz0 = rz1;
        it++;
    }
    if (rc == 0 && it == 0) rc = -2;
    if (rc == 0 && P->apply_err) rc = -4; /* a dynamic level iteration hit its cap */
    *niter_out = it;
    *final_rel = norm / init_norm;
    free(r); free(z); free(p); free(Ap);
    return rc;
}

/* ---- differentiation form ------------------------------------------------
 * dT/dtheta_i = 2 k_i k_j^2 / (h^2 (k_i + k_j)^2) for the harmonic-mean link of
 * spe.cc:84 with k = K * (axis scale); dtD/dtheta = tD for the Dirichlet faces.
 * g_c = -sum_j dT_cj (lam_c - lam_j)(p_c - p_j) - face: tD lam_c (p_c - p_D). */
static double dT_dtheta(double ki, double kj, double h) {
    double s = ki + kj;
    return 2 * ki * kj * kj / (h * h * s * s);
}

void or_grad_logk(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx, const double* ky, const double* kz,
                  int dirichlet, const double* p, const double* lam, double* g) {
    const double hx = 20, hy = 10, hz = 2;
#define IDXK2(i, j, k) (((k) * KNY * KNX + (j) * KNX + (i)) % KN)
#define TERM(cond, K, H, o, ii, jj, kk) \
    if (cond) acc += dT_dtheta(K[me], K[IDXK2(ii, jj, kk)], H) * (lam[r] - lam[o]) * (p[r] - p[o]);
    for (uint32_t k = 0; k < nz; k++)
        for (uint32_t j = 0; j < ny; j++)
            for (uint32_t i = 0; i < nx; i++) {
                uint32_t r = (k * ny + j) * nx + i, me = IDXK2(i, j, k);
                double acc = 0;
                TERM(k > 0, kz, hz, r - nx * ny, i, j, k - 1)
                TERM(j > 0, ky, hy, r - nx, i, j - 1, k)
                TERM(i > 0, kx, hx, r - 1, i - 1, j, k)
                TERM(i + 1 < nx, kx, hx, r + 1, i + 1, j, k)
                TERM(j + 1 < ny, ky, hy, r + nx, i, j + 1, k)
                TERM(k + 1 < nz, kz, hz, r + nx * ny, i, j, k + 1)
                if (dirichlet) {
                    double tD = 2 * kx[me] / (hx * hx);
                    if (i == 0) acc += tD * lam[r] * (p[r] - 1.0);
                    if (i == nx - 1) acc += tD * lam[r] * p[r];
                }
                g[r] = -acc;
            }
#undef TERM
#undef IDXK2
}
