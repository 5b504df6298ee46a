// Solve-phase objects: the preconditioner apply plan and the PCG driver.
#pragma once

#include <functional>

#include "persist.cuh"
#include "setup.cuh"

namespace mlp {

// Work vectors of one level for the apply (typed by the preconditioner's
// arithmetic: double for the plain path, float for the reduced-precision form).
template <class T>
struct LevelWork {
    DBuf<T> r, w, u0;            // multi-split: residual, L-solve output, correction
    DBuf<T> r2, u02;             // second residual / correction buffers of the merged sweeps
    DBuf<T> cu0, cu1, cx2, ctmp; // uh_cheb: Chebyshev vectors on the coarse slice
    // Folded coarse solve (launch plan): when the level below is one dense
    // operator C, the rows of G with coarse columns keep their product with C
    // (D = G_C C, FP64) so that phase 2 needs no separate coarse launch.
    DBuf<uint32_t> fold_rows;    // the rows of G with coarse columns, then the others
    DBuf<double> fold_D;         // fold_nf x n, row-major
    uint32_t fold_nf = 0;
    int fold_state = 0;          // 0 not tried, 1 built, -1 not applicable
};

// A recorded sequence of launches. Replaying it (directly or as a CUDA graph)
// applies the preconditioner z = B r, both vectors in level-0 frame order.
struct Plan {
    std::vector<std::function<void(cudaStream_t)>> ops;
    std::vector<std::string> names;      // per op: step and level ("phase1 L1", "persistent L1")
    std::vector<uint64_t> bytes_start;   // per op: algorithmic bytes of the apply before it
    uint64_t bytes_total = 0;
    size_t launches = 0;
    void run(cudaStream_t s) const;
};

// One timed replay of the apply, launch by launch (events between launches):
// per op its name, mean device time and algorithmic bytes.
struct OpProfile {
    std::string name;
    double ms = 0;
    uint64_t bytes = 0;
};
struct Prec;
std::vector<OpProfile> profile_apply(Prec& P, uint32_t reps, cudaStream_t s);
// Executable graphs of released handles, kept by shape and updated in place
// for the next handle of that shape (instantiation costs about a millisecond).
std::string plan_key(const Prec& P, const std::string& what);
void exec_release(const std::string& key, cudaGraphExec_t ex);
cudaGraphExec_t exec_for(const std::string& key, cudaGraph_t g);
void exec_cache_counts(uint64_t& updates, uint64_t& instantiations);
// Replays the apply graph reps (>= 2) times back to back with the in-graph
// timeline on; per launch of the plan its mean time inside the graph (us).
std::vector<double> timeline_apply(Prec& P, uint32_t reps, cudaStream_t s);
// One PCG solve (x0 from generate_x0) with the in-graph timeline on; per
// launch of one iteration near the end (its SpMV with (Ap, p), the update, the
// application's launches, the (r, z) reduction, the p update) its name and
// time in us.
std::vector<std::pair<std::string, double>> timeline_pcg(const DCSR& A, const double* b, Prec& P, double* x,
                                                         double eps, bool flexible, cudaStream_t s);

template <class T>
struct SmallPlan;
struct PcgDev;

struct PcgParams {
    double eps;
    uint32_t maxit;
};

// Device-resident PCG state of one preconditioner handle: the solver vectors
// and the whole-solve graphs (start, a conditional WHILE node whose body is one
// iteration, scatter), kept between solves of the same size.
struct PcgWork {
    uint32_t n = 0;
    DBuf<double> xf, bf, p, Ap, rprev, partials, bnat, xnat;
    DBuf<PcgDev> d;
    DBuf<PcgParams> prm;
    cudaGraphExec_t full[6] = {};  // [flexible * 3 + x0 mode]
    std::string full_key[6];       // their shape keys (released for reuse, see exec_for)
    ~PcgWork();
};

struct Prec {
    std::unique_ptr<Hierarchy> H;
    std::unique_ptr<SmallPlan<double>> sp64;
    std::unique_ptr<SmallPlan<float>> sp32;
    bool fp32 = false;  // hierarchy stored and applied in FP32
    std::vector<LevelWork<double>> w64;
    std::vector<LevelWork<float>> w32;
    DBuf<float> f32, z32;  // FP32 staging of the level-0 input/output
    DBuf<double> zin, zout; // frame-order staging for the natural-order apply entry point
    Plan plan;              // z = B r, frame order, on fin -> fout
    const double* fin = nullptr;
    double* fout = nullptr;
    DBuf<double> fin_buf, fout_buf;
    cudaGraphExec_t graph = nullptr;
    std::string graph_key;  // its shape key (released for reuse)
    cudaStream_t stream = nullptr;
    uint64_t bytes_per_apply = 0;  // algorithmic bytes of one apply
    // persistent regions of the plan: step descriptors and the grid barrier
    std::vector<DBuf<uint8_t>> pdesc;
    DBuf<PBar> pbar;
    uint32_t persist_regions = 0, persist_steps = 0;
    PcgWork pcg;
    Prec();
    ~Prec();
};

std::unique_ptr<Prec> make_prec(const DCSR& A, const BuildCfg& cfg, bool fp32, cudaStream_t s);
void prec_apply_frame(Prec& P, cudaStream_t s);  // fout = B fin
// Throws ERR_INTERNAL (and clears the flag) when a grid barrier of a
// persistent region gave up waiting since the last check; synchronises s.
void check_persist(Prec& P, cudaStream_t s);

// Records the largest nnz of a 256-row tile (decides the staged SpMV).
void csr_tile_stats(DCSR& m, cudaStream_t s);
// The same for several matrices with one host synchronisation; the device
// words `extra` are read back in the same copy (into extra_out).
void csr_tile_stats_batch(const std::vector<DCSR*>& ms, const std::vector<const uint32_t*>& extra,
                          std::vector<uint32_t>& extra_out, cudaStream_t s);

// y = A x for a CSR matrix (any level, frame or natural order).
void spmv(const DCSR& A, const double* x, double* y, cudaStream_t s);

void gather(uint32_t n, const uint32_t* idx, const double* src, double* dst, cudaStream_t s);
void scatter(uint32_t n, const uint32_t* idx, const double* src, double* dst, cudaStream_t s);

struct PcgStats {
    uint32_t niter = 0;
    double init_norm = 0, final_norm = 0, final_rel = 0;
    double t_total_ms = 0, t_prec_ms = 0, t_spmv_ms = 0;
    uint32_t napply = 0;
};

// PCGSolver (pcg.cc:8-102) with x0 of generate_x0; b and x are device
// vectors in natural order. flexible = Polak-Ribiere beta (needed when the
// preconditioner is applied in reduced precision).
int pcg_solve(const DCSR& A, const double* b, Prec& P, double* x, double eps, uint32_t maxit, bool flexible,
              PcgStats& st, cudaStream_t s);

// SymPrec support: S = A with a_ij = max(a_ij, a_ji) off the diagonal
// (sym_prec.cc:19-40), and PCGSolver on natural-order device vectors with the
// preconditioner given as a call z = B r.
void symmetrize(const DCSR& A, DCSR& S, cudaStream_t s);
int pcg_solve_cb(const DCSR& A, const double* b, const std::function<void(const double*, double*)>& apply,
                 double* x, double eps, uint32_t maxit, bool flexible, PcgStats& st, cudaStream_t s);

// ChebSolver (cheb.cc:9-100) with x0 of generate_x0, b and x device vectors in
// natural order, spectral bounds lmin < lmax of the preconditioned operator.
int cheb_solve(const DCSR& A, const double* b, Prec& P, double* x, double lmin, double lmax, double eps,
               uint32_t maxit, PcgStats& st, cudaStream_t s);

// pcg_solve with every solver vector and reduction scratch in a static device
// array instead of allocations (at most pcg_noalloc_max_n() unknowns).
int pcg_solve_noalloc(const DCSR& A, const double* b, Prec& P, double* x, double eps, uint32_t maxit,
                      bool flexible, PcgStats& st, cudaStream_t s);
uint32_t pcg_noalloc_max_n();

// Start vector of pcg_solve: the reference's generate_x0 (default), zero, or
// the values already in x.
enum X0Mode : int { X0_GENERATE = 0, X0_ZERO = 1, X0_GIVEN = 2 };
void set_pcg_x0_mode(int mode);  // per thread, consumed by the next pcg_solve

int pcg_solve_hostloop(const DCSR& A, const double* b, Prec& P, double* x, double eps, uint32_t maxit,
                       bool flexible, PcgStats& st, cudaStream_t s);

// Ensemble form: independent solves of several handles in one graph launch.
struct Ensemble {
    std::vector<Prec*> members;
    bool flexible = false;
    int x0m = 0;
    bool gradient = false;             // forward, misfit, adjoint and gradient per member
    std::vector<DBuf<PcgDev>> fwd;     // gradient form: the forward solves' scalars
    cudaGraphExec_t exec = nullptr;
    ~Ensemble();
};

// Gradient form of one member: its mesh and permeability field (device), the
// observation cells and observed pressures (device), and where p, lambda and
// dJ/dlnK go (device vectors of the mesh's cells, natural order).
struct GradMember {
    uint32_t nx = 0, ny = 0, nz = 0;
    const double *kx = nullptr, *ky = nullptr, *kz = nullptr;
    int dirichlet = 1;
    const uint32_t* obs = nullptr;
    uint32_t nobs = 0;
    const double* pobs = nullptr;
    double *p = nullptr, *lam = nullptr, *grad = nullptr;
};
std::unique_ptr<Ensemble> make_ensemble_gradient(const std::vector<Prec*>& members,
                                                 const std::vector<GradMember>& gm, bool flexible,
                                                 cudaStream_t s);
std::unique_ptr<Ensemble> make_ensemble(const std::vector<Prec*>& members, bool flexible, int x0m, cudaStream_t s);
int ensemble_solve(Ensemble& E, const std::vector<const double*>& b, const std::vector<double*>& x, double eps,
                   uint32_t maxit, std::vector<PcgStats>& st, double& ms, cudaStream_t s);

// Gradient of J with respect to ln K per cell (adjoint.cu).
void spe_grad_logk(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx, const double* ky, const double* kz,
                   int dirichlet, const double* p, const double* lam, double* g, cudaStream_t s);

// Cached x0 (generate_x0 depends only on n).
const double* x0_device(uint32_t n, cudaStream_t s);

}  // namespace mlp
