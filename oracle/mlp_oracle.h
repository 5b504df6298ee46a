/*
 * CPU restatement of the ml_prec hot path. TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker the parity tests (and bench.py's CPU-baseline leg)
 * compare the CUDA path against. It is never linked into, loaded by or called
 * from the product library. Each function cites the reference file:line whose
 * behaviour it restates; arithmetic keeps the reference's operation order and is
 * compiled without FMA contraction so that every integer decision that depends on
 * a floating-point comparison (link dropping, hierarchy shape) comes out identical.
 *
 * Parity of this restatement is pinned against the reference itself, compiled
 * from its own sources by oracle/Makefile (target "ref"), through the golden
 * fixtures under tests/golden/ that tests/golden/make_golden.py writes.
 */
#ifndef MLP_ORACLE_H
#define MLP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CSR matrix, 32-bit indices, FP64 values; "skyline" rows keep the diagonal first
 * (modules/matrix/matrix.h:187-291). */
typedef struct {
    uint32_t nrow, ncol;
    uint32_t* ia; /* nrow+1 */
    uint32_t* ja; /* nnz */
    double* a;    /* nnz */
} or_csr;

void or_csr_free(or_csr* A);

/* 7-point SPE stencil (spe.cc:69-131) plus the benchmark's Dirichlet x-faces. */
int or_assemble(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx, const double* ky,
                const double* kz, double c, int dirichlet, or_csr* A, double* b);

/* y = A x (csrmatrix.cc:260-274). */
void or_spmv(const or_csr* A, const double* x, double* y);

/* x0 of generate_x0 (solvers.cc:9-21): srandom(3), glibc random(). */
void or_generate_x0(double* x, uint32_t n);

/* ---- multilevel preconditioners ---------------------------------------- */
enum { OR_ORDER_NONE = 0, OR_ORDER_ORIGINAL = 1, OR_ORDER_BLOCK = 2, OR_ORDER_SIMPLE_1 = 3 };
enum { OR_PREC_MSPLIT = 0, OR_PREC_CHEB = 1, OR_PREC_SYM = 2 };

typedef struct {
    int kind;              /* OR_PREC_MSPLIT / OR_PREC_CHEB */
    /* multi-split (multi_split_constr.cc:170-268) */
    uint32_t nq;    const double* q;      /* per-level q, last one repeats */
    uint32_t nnit;  const uint32_t* niter;/* per-level inner iterations, index 0 ignored */
    uint32_t coarse_n, max_levels, degree_max;
    int order;
    int use_tails;         /* elim_order=original tail group */
    /* uh_cheb (cheb_constr.cc:292-365) */
    uint32_t nsig;  const double* sigma;  /* beta per level */
    uint32_t nch;   const uint32_t* ncheb;/* Chebyshev degree per level */
    /* multi-split inner_iter = dynamic (multi_split_constr.cc:198-203): level_eps
     * per level, index 0 ignored, last one repeats; neps = 0 keeps fixed niter */
    uint32_t neps;  const double* level_eps;
} or_prec_cfg;

typedef struct {
    uint32_t N, nnz, M, Md, niter;
    double q;
    double eps;        /* dynamic inner iterations: stop when ||r|| / ||f|| < eps */
    or_csr A;          /* level matrix (level 0: copy of the input) */
    or_csr L, U;       /* factors (multi_split_prec.h:31-33) */
    uint32_t* map;     /* permuted -> original */
    uint32_t* rmap;    /* original -> permuted */
    double* dval;      /* reciprocal diagonal of the Md block */
    /* uh_cheb */
    double alpha, beta, lmin, lmax;
    uint32_t ncheb;
    /* coarsest-level dense LU (direct-solver hook) */
    double* lu;        /* row-major n*n, unit-lower L below, U on/above diagonal */
} or_level;

typedef struct {
    int kind;
    uint32_t nlevels;
    uint32_t coarse_n;  /* != 0 => coarsest level is solved directly */
    or_level* levels;
    double* work;       /* scratch for apply */
    char err[256];
    int apply_err;      /* set when a dynamic level iteration hit its cap */
    /* SymPrec (sym_prec.cc:8-40): the uh_cheb preconditioner of the symmetric
     * part, applied as a PCG solve to eps = 1e-14 */
    or_csr Asym;
    void* inner;        /* or_prec* of the symmetric part */
} or_prec;

or_prec* or_prec_build(const or_csr* A, const or_prec_cfg* cfg, char* err, int errlen);
void or_prec_apply(const or_prec* P, const double* f, double* x);
void or_prec_free(or_prec* P);

/* accessors for ctypes */
uint32_t or_prec_nlevels(const or_prec* P);
const or_level* or_prec_level(const or_prec* P, uint32_t l);

/* ---- PCG (pcg.cc:8-102) --------------------------------------------------- */
/* Returns 0 on success; x holds the solution; *niter the iteration count;
 * *final_rel the last relative residual. Throws (returns <0) like the reference:
 * -1 non-positive curvature, -2 "No need to iterate". */
int or_pcg(const or_csr* A, const double* b, const or_prec* P, double* x, double eps,
           uint32_t* niter, double* final_rel, uint32_t maxit);

/* or_pcg with a choice of start: x0_mode 0 = generate_x0, 1 = zero. */
int or_pcg_ex(const or_csr* A, const double* b, const or_prec* P, double* x, double eps,
              uint32_t* niter, double* final_rel, uint32_t maxit, int x0_mode);

/* ChebSolver (cheb.cc:9-100) with the preconditioner's spectral bounds;
 * *niter as the reference reports it. Returns 0, or -3 at the cap. */
int or_cheb_solve(const or_csr* A, const double* b, const or_prec* P, double lmin, double lmax, double* x,
                  double eps, uint32_t* niter, double* final_rel, uint32_t maxit);

/* Differentiation form (no reference counterpart): dJ/d(ln K) per cell for
 * the SPE matrix with Dirichlet x-faces, given p (A p = b) and lambda
 * (A lambda = dJ/dp); the same formula as the CUDA kernel, in FP64 on the CPU. */
void or_grad_logk(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx, const double* ky, const double* kz,
                  int dirichlet, const double* p, const double* lam, double* g);

/* Dense LU without pivoting, in place (row-major n x n) and its solve. */
int or_dense_lu(double* a, uint32_t n);
void or_dense_lu_solve(const double* lu, uint32_t n, const double* b, double* x);

#ifdef __cplusplus
}
#endif
#endif
