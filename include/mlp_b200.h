/*
 * ml_prec_b200 — C ABI of the B200 (sm_100a) implementation of ml_prec's hot
 * path: PCG on the 7-point reservoir-pressure matrix preconditioned by the
 * multilevel multi-split or Chebyshev ("uh_cheb") preconditioner.
 *
 * Every function returns an int status (MLP_OK = 0); on failure
 * mlp_last_error() returns a message for the calling thread. Pointers named
 * *_host are host memory; pointers named *_dev are device memory of the
 * current CUDA device. Handles are not thread-safe: use one per thread/stream
 * (the reference's solve() mutates `mutable` scratch the same way,
 * multi_split_prec.h:40-41).
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the ml_prec source tree).
 */
#ifndef MLP_B200_H
#define MLP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MLP_OK 0
#define MLP_ERR_ARG 1         /* invalid argument or size                            */
#define MLP_ERR_CONFIG 2      /* bad preconditioner configuration (ConfigFile keys)  */
#define MLP_ERR_LEVELS 3      /* "Too many levels" (cheb_constr.cc:282-283)          */
#define MLP_ERR_CURVATURE 4   /* <Ap, p> <= 0 (pcg.cc:51-55)                         */
#define MLP_ERR_NOT_FINITE 5  /* NaN / Inf in a PCG scalar                           */
#define MLP_ERR_MAXIT 6       /* iteration cap reached                               */
#define MLP_ERR_CUDA 7        /* CUDA runtime error                                  */
#define MLP_ERR_NO_ITER 8     /* "No need to iterate" (pcg.cc:94-96)                 */
#define MLP_ERR_LIMIT 9       /* a documented size limit was exceeded                */
#define MLP_ERR_INTERNAL 10   /* device-side consistency check failed                */

typedef struct mlp_matrix mlp_matrix; /* device-resident CSR, diagonal first per row */
typedef struct mlp_prec mlp_prec;     /* device-resident preconditioner hierarchy     */

/* Preconditioner kinds. */
#define MLP_PREC_MSPLIT 0 /* MultiSplitPrec, multi_split_prec.h:15-113 */
#define MLP_PREC_CHEB 1   /* Prec ("uh_cheb"), cheb_prec.h:13-127     */
#define MLP_PREC_SYM 2    /* SymPrec, sym_prec.h:13-27: the uh_cheb Prec of the symmetric
                             part (a_ij = max(a_ij, a_ji) off the diagonal), applied as a
                             PCG solve to 1e-14 from generate_x0 (sym_prec.cc:8-40); takes
                             the uh_cheb fields of mlp_prec_cfg. The outer mlp_pcg on such a
                             handle runs host-driven, one device solve per application. */

/* Node orderings (msplit.cfg key elim_order, multi_split_constr.cc:246-249). */
#define MLP_ORDER_NONE 0
#define MLP_ORDER_ORIGINAL 1
#define MLP_ORDER_BLOCK 2
#define MLP_ORDER_SIMPLE_1 3

/* Plain-old-data configuration, the parsed form of msplit.cfg / Config.
 * Replaces the ConfigFile reads of MultiSplitPrec::MultiSplitPrec
 * (multi_split_constr.cc:179-233) and the Config fields Prec reads
 * (cheb_constr.cc:292-365, project/config.h:54-86). */
typedef struct {
    int32_t kind;            /* MLP_PREC_MSPLIT or MLP_PREC_CHEB                      */
    uint32_t nq;             /* multi-split: q per level (last value repeats)         */
    const double* q;
    uint32_t nniter;         /* multi-split: level_niter per level (entry 0 ignored)  */
    const uint32_t* niter;
    uint32_t coarse_n;       /* coarsest-level size for the direct solve (0 = none)   */
    uint32_t max_levels;     /* multi-split max_levels                                */
    uint32_t degree_max;     /* multi-split simple_1 elimination bound                */
    int32_t order;           /* MLP_ORDER_*                                           */
    int32_t use_tails;       /* tail elimination (Config::use_tails): uh_cheb, and the
                                tail group of multi-split elim_order = original      */
    uint32_t nsigma;         /* uh_cheb sigma (= beta) per level                      */
    const double* sigma;
    uint32_t nncheb;         /* uh_cheb Chebyshev degree per level                    */
    const uint32_t* ncheb;
    int32_t fp32;            /* 1: store and apply the hierarchy in FP32              */
    int32_t autotune;        /* 1: time the row kernels' launch shapes (lanes per row,
                                block size) on each level at build and keep the
                                fastest (cached per level shape); 0: fixed heuristic */
    uint32_t neps;           /* multi-split inner_iter = dynamic (msplit.cfg level_eps,
                                multi_split_constr.cc:198-203, 256-264): per-level eps,
                                entry 0 ignored, last value repeats; each level call
                                sweeps until ||f - A x|| / ||f|| < eps
                                (multi_split_solve.cc:119-134), at most 1,000 sweeps
                                per level call and 100,000 per apply (the reference
                                has no cap; reaching one returns MLP_ERR_MAXIT).
                                neps = 0: the fixed niter.                           */
    const double* level_eps;
} mlp_prec_cfg;

/* Solver statistics, the fields of SolverStats (solvers.h:15-28) plus the
 * quantities the GPU path reports. */
typedef struct {
    uint32_t niter;
    uint32_t napply;
    double init_norm;
    double final_norm;
    double final_rel;
    double t_solve_ms;   /* device time of the whole PCG call              */
    double t_setup_ms;   /* device time of the preconditioner construction */
} mlp_stats;

/* Per-level summary, the fields printed by operator<< for MultiSplitPrec::Level
 * (multi_split_misc.cc:228-240) and Prec::Level (cheb_misc.cc:61-74). */
typedef struct {
    uint32_t N, nnz, M, Md, n;
    uint32_t niter, ncheb;
    int32_t direct;            /* 1 if the level is solved with the dense inverse */
    double q, alpha, beta, lmin, lmax;
    uint32_t L_nnz, U_nnz;
    uint32_t nwave_l, nwave_u; /* wavefronts of the level-scheduled L / U solves  */
    uint32_t P1_nnz, G_nnz;    /* explicit triangular factors of the sweeps       */
    double eps;                /* dynamic inner iterations: the level's eps (0 = fixed niter) */
} mlp_level_info;

const char* mlp_last_error(void);
int mlp_version(void);
int mlp_device_count(int* count);
int mlp_set_device(int device);

/* ---- matrices ------------------------------------------------------------
 * Replaces CSRMatrix / SkylineMatrix storage (matrix.h:187-291): uint32 ia
 * (n+1), ja and FP64 a (nnz), diagonal first in every row. The library keeps a
 * device copy; the host arrays may be released after the call. */
int mlp_matrix_create(uint32_t n, const uint32_t* ia_host, const uint32_t* ja_host, const double* a_host,
                      mlp_matrix** out);
/* SPEMesh(nx,ny,nz) + construct_matrix(A, c) (spe.cc:11-131) on the device,
 * from the SPE10-layout permeability blocks (1,122,000 values each, host).
 * dirichlet != 0 adds the benchmark's x-face Dirichlet terms; b_host (n values,
 * may be NULL) receives the matching right-hand side. */
int mlp_matrix_create_spe(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx_host, const double* ky_host,
                          const double* kz_host, double c, int32_t dirichlet, mlp_matrix** out, double* b_host);
int mlp_matrix_destroy(mlp_matrix* A);
int mlp_matrix_size(const mlp_matrix* A, uint32_t* n, uint32_t* nnz);
int mlp_matrix_download(const mlp_matrix* A, uint32_t* ia_host, uint32_t* ja_host, double* a_host);
/* y = A x (multiply(A, v, res, 'o'), csrmatrix.cc:260-274), device vectors. */
int mlp_spmv(const mlp_matrix* A, const double* x_dev, double* y_dev, void* stream);
/* Same with host vectors (copies in and out; the matrix's own stream). */
int mlp_spmv_host(const mlp_matrix* A, const double* x_host, double* y_host);

/* ---- preconditioners -------------------------------------------------------
 * mlp_prec_create replaces MultiSplitPrec(const SkylineMatrix&, const Config&)
 * (multi_split_prec.h:105) and Prec(const SkylineMatrix&, const Config&)
 * (cheb_prec.h:115); the hierarchy is built on the device. */
int mlp_prec_create(const mlp_matrix* A, const mlp_prec_cfg* cfg, mlp_prec** out);
int mlp_prec_destroy(mlp_prec* P);
/* x = B f (PrecBase::solve(Vector& f, Vector& x) const, prec_base.h:8-12),
 * device vectors in the matrix's natural order. */
int mlp_prec_apply(mlp_prec* P, const double* f_dev, double* x_dev, void* stream);
/* Same with host vectors (copies in and out). */
int mlp_prec_apply_host(mlp_prec* P, const double* f_host, double* x_host);
int mlp_prec_nlevels(const mlp_prec* P, uint32_t* nlevels);
int mlp_prec_level_info(const mlp_prec* P, uint32_t level, mlp_level_info* info);
/* Level data in the reference's indexing, for parity checks: map (N), L
 * (ia: N-Md+1, ja/a: L_nnz), U (ia: M+1, ja/a: U_nnz), the level matrix A
 * (ia: N+1, ja/a: nnz; level 0 is the input) and dval (Md). Any pointer may
 * be NULL to skip that array. */
int mlp_prec_level_export(const mlp_prec* P, uint32_t level, uint32_t* map, uint32_t* L_ia, uint32_t* L_ja,
                          double* L_a, uint32_t* U_ia, uint32_t* U_ja, double* U_a, uint32_t* A_ia,
                          uint32_t* A_ja, double* A_a, double* dval);
/* Algorithmic HBM bytes of one apply (the roofline numerator). */
int mlp_prec_bytes_per_apply(const mlp_prec* P, uint64_t* bytes);
/* Profiling aid without a reference counterpart: replays the apply (on the
 * vector of the last apply, in frame order) reps times launch by launch with
 * CUDA events between the launches and reports, per launch, its mean device
 * time (ms), its algorithmic bytes and its name ("phase1 L1", "persistent L1":
 * the step and the level whose call recorded it; names are written with
 * stride name_len). *nops receives the number of launches; at most cap
 * entries are written. */
int mlp_prec_profile(mlp_prec* P, uint32_t reps, uint32_t cap, uint32_t* nops, double* ms, uint64_t* bytes,
                     char* names, uint32_t name_len);
/* Profiling aid without a reference counterpart: replays the apply graph reps
 * (at least 2) times back to back and reports, per launch (the order and
 * names of mlp_prec_profile), its mean time inside the graph in us, from
 * %globaltimer stamps that each kernel writes as it passes its
 * dependent-launch wait (the launch lasts until the next one passes its
 * wait). Plans with launches of other kinds (the persistent or shared-memory
 * small-level kernels) return MLP_ERR_INTERNAL; no other apply may run on the
 * device meanwhile. */
int mlp_prec_timeline(mlp_prec* P, uint32_t reps, uint32_t cap, uint32_t* nops, double* us);
/* The same for a whole solve: one mlp_pcg_device-like solve (x0 from
 * generate_x0, stream of the handle) with the stamps on, and per launch of one
 * iteration near its end, in order (the SpMV with (Ap, p), the update, the
 * application's launches, the (r, z) reduction, the p update), its name and
 * time in us inside the graph. *n receives the number of launches; at most cap
 * entries are written. */
int mlp_pcg_timeline(const mlp_matrix* A, const double* b_dev, mlp_prec* P, double* x_dev, double eps,
                     int32_t flexible, uint32_t cap, uint32_t* n, double* us, char* names, uint32_t name_len);

/* ---- solver ----------------------------------------------------------------
 * PCGSolver(A, b, B, x, stats, eps, NORM_L2) (solvers.h:31-32, pcg.cc:8-102):
 * x0 from generate_x0 (solvers.cc:9-21), stop when ||r||/||r0|| <= eps (eps
 * raised so that the absolute stop is >= 1e-14, solvers.cc:49-58).
 * flexible != 0 uses the Polak-Ribiere beta (needed with an FP32 hierarchy).
 * maxit = 0 selects the library's cap of 10,000 iterations (the reference has
 * none; the iterations run on the device and must end); reaching the cap
 * returns MLP_ERR_MAXIT. */
int mlp_pcg(const mlp_matrix* A, const double* b_host, mlp_prec* P, double* x_host, double eps, uint32_t maxit,
            int32_t flexible, mlp_stats* stats);
int mlp_pcg_device(const mlp_matrix* A, const double* b_dev, mlp_prec* P, double* x_dev, double eps,
                   uint32_t maxit, int32_t flexible, mlp_stats* stats, void* stream);

/* mlp_pcg_device with a choice of start vector: x0_mode 0 = generate_x0 (the
 * reference's start, solvers.cc:9-21), 1 = zero, 2 = the values already in
 * x_dev. The zero start serves the adjoint solve of the differentiation form,
 * whose right-hand side is small next to A x0. */
int mlp_pcg_device_x0(const mlp_matrix* A, const double* b_dev, mlp_prec* P, double* x_dev, double eps,
                      uint32_t maxit, int32_t flexible, int32_t x0_mode, mlp_stats* stats, void* stream);

/* ChebSolver(A, lmin, lmax, b, B, x, eps, NORM_L2) (solvers.h:42-43,
 * modules/solvers/cheb.cc:9-100): the Chebyshev iteration with preconditioner
 * P, for spectral bounds lmin < lmax of the preconditioned operator (uh_cheb
 * level 0: mlp_level_info lmin / lmax, what project/main.cc:143-148 passes).
 * x0 from generate_x0; stops when ||r|| / ||r0|| <= eps (1e-14 absolute
 * floor); stats->niter counts the steps as the reference reports them. maxit
 * as for mlp_pcg. */
int mlp_cheb_solve(const mlp_matrix* A, const double* b_host, mlp_prec* P, double* x_host, double lmin,
                   double lmax, double eps, uint32_t maxit, mlp_stats* stats);
int mlp_cheb_solve_device(const mlp_matrix* A, const double* b_dev, mlp_prec* P, double* x_dev, double lmin,
                          double lmax, double eps, uint32_t maxit, mlp_stats* stats, void* stream);

/* Differentiation form (no reference counterpart: the reference has no
 * gradients). For a matrix made by mlp_matrix_create_spe, writes
 * grad[c] = dJ/d(ln K_c) = -lambda^T (dA/dtheta_c p - db/dtheta_c) per mesh cell,
 * where p solves A p = b and lambda solves A lambda = dJ/dp (A is symmetric);
 * K scales kx, ky and kz of the cell (kz = 0.1 K in the benchmark fields).
 * Uses the harmonic-mean transmissibility derivatives of the stencil of
 * spe.cc:81-87 plus the Dirichlet x-face terms. Device vectors of N entries. */
int mlp_matrix_grad_logk(const mlp_matrix* A, const double* p_dev, const double* lam_dev, double* grad_dev,
                         void* stream);

/* ---- ensemble form ----------------------------------------------------------
 * Independent PCG solves of several (matrix, preconditioner) pairs, e.g. an
 * ensemble of permeability realizations on meshes of different sizes, recorded
 * as parallel branches of ONE CUDA graph (each branch: start, a conditional
 * WHILE loop of iterations, scatter) and run with one launch. No reference
 * counterpart (the reference solves one system per process run). A handle may
 * belong to one ensemble at a time; the ensemble uses the handles' solver
 * vectors, so the handles must outlive it. */
typedef struct mlp_ensemble mlp_ensemble;
int mlp_ensemble_create(uint32_t count, mlp_prec* const* P, int32_t flexible, int32_t x0_mode, mlp_ensemble** out);
/* b_dev[i], x_dev[i]: member i's vectors (natural order); stats: count entries;
 * t_ms: device time of the launch. */
int mlp_ensemble_solve(mlp_ensemble* E, const double* const* b_dev, double* const* x_dev, double eps, uint32_t maxit,
                       mlp_stats* stats, double* t_ms, void* stream);
int mlp_ensemble_destroy(mlp_ensemble* E);

/* Gradient form of the ensemble (no reference counterpart): ONE graph whose
 * branch i runs member i's forward solve A_i p_i = b_i, the misfit gradient
 * dJ/dp at its observation cells (J = 0.5 sum_k (p[obs_k] - pobs_k)^2), the
 * adjoint solve A_i lambda_i = dJ/dp and the dJ/d(ln K) kernel of
 * mlp_matrix_grad_logk; both solves start from zero. A[i] must come from
 * mlp_matrix_create_spe. obs_dev / pobs_dev (nobs[i] entries) and the outputs
 * p_dev, lam_dev, grad_dev (device vectors of member i's cells) are bound at
 * creation and must outlive the handle. Run it with mlp_ensemble_solve
 * (x_dev may be NULL); stats then takes 2 * count entries: the forward solves,
 * then the adjoint solves. */
int mlp_ensemble_gradient_create(uint32_t count, const mlp_matrix* const* A, mlp_prec* const* P,
                                 const uint32_t* const* obs_dev, const uint32_t* nobs, const double* const* pobs_dev,
                                 double* const* p_dev, double* const* lam_dev, double* const* grad_dev,
                                 int32_t flexible, mlp_ensemble** out);

/* PCG that allocates no device memory. It has no counterpart in the
 * reference. It serves host applications that cannot let a library call
 * cudaMalloc while they solve: their device memory is owned by their own
 * allocator (a framework's caching allocator that has reserved the device, or
 * a process held to a fixed device-memory budget), so an allocation from
 * inside this library would fail or break the host's accounting. It computes
 * exactly what mlp_pcg_device computes, but the solver's vectors, reduction
 * scratch and start vector live in one file-scope device array of the
 * library, sized for at most 131072 unknowns (about 6 MB, held by every GPU
 * that loads the library until the process exits); larger systems are
 * rejected with MLP_ERR_LIMIT. The matrix and the preconditioner must have
 * been created beforehand (those calls allocate). Every call looks up the
 * array's address on the current device; the first call on a device (unless
 * an earlier call into the library on that device did it) loads the library's
 * device code there, which is what places the array. All calls share the one
 * array, which keeps the last call's contents: calls that overlap on the GPU
 * (other threads, other streams) race and must be serialised by the caller. The call waits on the
 * host for the device after every iteration. t_solve_ms is host wall time. */
int mlp_pcg_device_noalloc(const mlp_matrix* A, const double* b_dev, mlp_prec* P, double* x_dev, double eps,
                           uint32_t maxit, int32_t flexible, mlp_stats* stats, void* stream);

/* Number of kernels this library has launched in the process so far (graph
 * kernel nodes included); no reference counterpart, used for accounting. */
int mlp_launch_count(uint64_t* count);

/* generate_x0 (solvers.cc:9-21) on the host: srandom(3), glibc random(). */
int mlp_generate_x0(double* x_host, uint32_t n);

#ifdef __cplusplus
}
#endif
#endif
