// Shared-memory-resident solve of the small coarse levels.
//
// The multilevel apply recurses with niter (multi-split) or ncheb (uh_cheb)
// calls per level, so the coarsest levels are entered thousands of times per
// outer iteration while holding only a few hundred unknowns. Launching one
// kernel per wavefront there is pure latency. Instead, the sub-hierarchy from
// level Ls down is packed into one contiguous blob; a single 1024-thread CTA
// copies it into shared memory and runs the whole recursive solve of level Ls
// (all sweeps, all deeper levels) with __syncthreads between phases.
#pragma once

#include "solve.cuh"

namespace mlp {

static constexpr int SMALL_MAXLEV = 16;
static constexpr int SMALL_MAXCHEB = 16;
static constexpr int SMALL_THREADS = 1024;

// Offsets are bytes from the start of dynamic shared memory.
struct SLevel {
    uint32_t N, M, Md, n, niter, ncheb;
    int32_t direct;
    uint32_t nwl, nwu;
    uint32_t o_Aia, o_Aja, o_Aa;  // A in frame order (multi-split residual sweeps)
    uint32_t o_Sia, o_Sja, o_Sa;  // symmetric operator (uh_cheb, levels below the blob top)
    uint32_t o_Lia, o_Lja, o_La;
    uint32_t o_Uia, o_Uja, o_Ua;
    uint32_t o_dval, o_lwo, o_uwo, o_uwr, o_cinv;
    uint32_t o_w, o_r, o_u0, o_cu0, o_cu1, o_cx2, o_ctmp;
    double ch_a1;                       // step-1 scale (1.0 where the reference skips dscal)
    double ch_alpha[SMALL_MAXCHEB + 1];  // signed coefficient of the solve in step i
    double ch_beta[SMALL_MAXCHEB + 1];   // coefficient of u1 (step 2) / of (u1-u0) (step i>=3)
};

struct alignas(16) SBlob {
    int32_t kind;
    uint32_t nlev;
    uint32_t bytes_static;  // bytes copied from global memory (multiple of 16)
    uint32_t bytes_total;   // plus work vectors
    uint32_t o_f, o_x;      // top-level input / output
    SLevel lv[SMALL_MAXLEV];
};

// Host side: packed blob of levels [first, nlevels) of H.
template <class T>
struct SmallPlan {
    DBuf<uint8_t> blob;
    DBuf<SBlob> desc;
    SBlob h{};
    uint32_t first = 0xffffffffu;  // level where the small solve starts
    uint32_t N0 = 0;
    // The level solve is a fixed linear operator; when it is small enough it is
    // tabulated once (column j = the solve applied to e_j) and every later call
    // is one dense matrix-vector product.
    DBuf<T> dense;                  // N0 x N0, row-major; empty if not tabulated
    bool valid() const { return first != 0xffffffffu; }
};

// Chooses the first level whose sub-hierarchy fits the shared-memory budget
// and packs it; leaves the plan invalid if nothing fits.
template <class T>
void build_small(Hierarchy& H, SmallPlan<T>& sp, uint32_t smem_budget, cudaStream_t s);

// Records the single launch that solves level sp.first: x = B_first f.
template <class T>
void launch_small(const SmallPlan<T>& sp, const T* f, T* x, cudaStream_t s);

uint32_t small_smem_limit();

}  // namespace mlp
