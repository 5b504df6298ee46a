// Declarations shared between the hierarchy construction (setup.cu, compiled
// without FMA contraction) and the solve-phase code.
#pragma once

#include <memory>

#include "common.cuh"

namespace mlp {

enum PrecKind : int { PREC_MSPLIT = 0, PREC_CHEB = 1 };
enum Order : int { ORDER_NONE = 0, ORDER_ORIGINAL = 1, ORDER_BLOCK = 2, ORDER_SIMPLE_1 = 3 };

struct BuildCfg {
    int kind = PREC_MSPLIT;
    std::vector<double> q{0.8};          // multi-split q per level (last repeats)
    std::vector<uint32_t> niter{5};      // inner iterations per level (entry 0 ignored)
    std::vector<double> eps;             // inner_iter = dynamic: level_eps per level (entry 0
                                         // ignored); empty = the fixed niter
    uint32_t coarse_n = 0, max_levels = 15, degree_max = 2;
    int order = ORDER_SIMPLE_1;
    int use_tails = 1;
    std::vector<double> sigma{3.0};      // uh_cheb beta per level
    std::vector<uint32_t> ncheb{2};      // uh_cheb Chebyshev degree per level
    uint32_t dense_max = 8192;           // largest coarsest level solved directly
    int autotune = 0;                    // time the row kernels' launch shapes at build
};

// One level of the hierarchy. Two indexings are kept:
//  * the reference's: map (permuted -> level-natural), L and U with permuted
//    column indices, the next level's matrix in the order construct_sparse_lu
//    emits it. These are what the parity tests compare.
//  * the solve "frame": positions [0, M) hold the eliminated block sorted by
//    the L-solve wavefront, [M, M+n) hold the coarse block in the NEXT level's
//    frame order, [M+n, N) the diagonal block. With every level in its frame,
//    the next level's vectors are plain slices of this level's vectors and no
//    gather or scatter happens between levels.
struct Level {
    // parameters
    double q = 0;
    uint32_t niter = 0;
    double eps = 0;  // dynamic inner iterations: sweep until ||f - A x|| / ||f|| < eps
    double alpha = 1, beta = 1, lmin = 0, lmax = 0;
    uint32_t ncheb = 0;
    // sizes
    uint32_t N = 0, nnz = 0, M = 0, Md = 0, n = 0;
    bool direct = false;  // coarsest level solved with the dense inverse
    // reference indexing
    DCSR A;                 // level matrix in its natural order
    DCSR L, U;              // factors (L: N-Md rows, U: M rows)
    DBuf<uint32_t> map;     // permuted -> natural
    DBuf<double> dval;      // reciprocal diagonal of the Md block
    DBuf<int> done;         // elimination round of each E row (1-based)
    uint32_t nwave_l = 0;   // L-solve wavefronts
    // frame indexing
    DBuf<uint32_t> eperm;   // frame E position -> permuted index
    DBuf<uint32_t> phi;     // frame -> natural
    DBuf<uint32_t> iphi;    // natural -> frame
    DCSR Af;                // A in frame order (residual sweeps)
    DCSR Lf;                // L rows in frame order (R = N-Md rows, columns < M)
    DCSR Uf;                // U rows (M) with frame columns
    DCSR As;                // uh_cheb: full matrix mirrored from the lower half, frame order
    // Triangular solves in explicit form (frame order):
    //  P1 (rows [0, R), columns [0, R)): w = P1 s solves the L system of the
    //     eliminated and coarse rows at once, P1 = (I + L)^{-1} restricted to them;
    //  G  (rows [0, M), columns [0, M+n)): x_E = G [w_E; x_C] solves the U system.
    DCSR P1, G;
    std::vector<uint32_t> lw_off;  // L wavefront d covers E rows [lw_off[d], lw_off[d+1])
    std::vector<uint32_t> uw_off;  // U wavefront d covers uw_rows[uw_off[d] .. uw_off[d+1])
    DBuf<uint32_t> uw_rows;
    DBuf<uint32_t> lw_off_d, uw_off_d;  // device copies of the wavefront offsets
    // direct coarsest level
    DBuf<double> cinv;      // dense inverse, row-major N x N
    DBuf<float> cinv32;
    // FP32 copies for the reduced-precision form
    DBuf<float> dval32;
};

struct Hierarchy {
    int kind = PREC_MSPLIT;
    uint32_t nlevels = 0;
    uint32_t coarse_n = 0;
    std::vector<std::unique_ptr<Level>> lv;
    double setup_ms = 0;
};

// Builds the hierarchy of A (natural order, diagonal-first rows, on the device).
std::unique_ptr<Hierarchy> build_hierarchy(const DCSR& A, const BuildCfg& cfg, cudaStream_t s);

// SPE assembly on the device; b may be null.
void spe_assemble(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx, const double* ky,
                  const double* kz, double c, int dirichlet, DCSR& A, double* b, cudaStream_t s);

std::vector<uint32_t> stable_partition(uint32_t N, const uint8_t* bucket, int NB, uint32_t rev_mask,
                                       uint32_t* map, uint32_t base, cudaStream_t s);

double cheb_poly(double x, uint32_t k);

}  // namespace mlp
