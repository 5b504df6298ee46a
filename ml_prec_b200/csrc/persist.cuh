// Persistent apply: a run of preconditioner steps executed by ONE cooperative
// kernel launch instead of one launch per step.
//
// The multilevel apply below the finest level is a long chain of small,
// dependent sweep steps (phase 1, the coarse product, phase 2, the residual
// correction, Chebyshev updates): at 60x220x85 about a hundred per outer PCG
// iteration, each moving a few MB or less, so separate launches are bound by
// launch latency, not by HBM. The plan builder therefore records such a chain
// as an array of step descriptors (PStep) and k_persist runs them in order
// with a grid-wide barrier between consecutive steps. Every step repeats the
// arithmetic of the separate kernel it replaces (same products, lane split and
// butterfly order), so the two forms give bit-identical results.
#pragma once

#include "common.cuh"

namespace mlp {

enum PsOp : uint32_t {
    PS_PHASE1 = 0,  // k_phase1: w = P1 src on rows [0, R); out = dval src on [R, N)
    PS_PHASE2 = 1,  // k_phase2: out_q = sum_j G_qj (j < M ? w_j : out_j), q < M
    PS_UPDATE = 2,  // k_update: x += u0; r -= Af u0 (mode 1) or x += u0 only (mode 0)
    PS_RESID = 3,   // residual SpMV: y = f - A x
    PS_DENSE = 4,   // k_dense_gemv: x = C f, C dense n x n row-major
    PS_SCALE = 5,   // k_scale: v *= s0
    PS_CHEB2 = 6,   // k_cheb2: x2 = x2 * s0 + s1 * u1
    PS_CHEBK = 7,   // k_chebk: x2 = u1 - s0 x2 + s1 (u1 - u0)
    PS_COPY = 8,    // k_copy: dst = src
    PS_TOF32 = 9,   // k_to_f32: float dst = double src
    PS_TOF64 = 10,  // k_to_f64: double dst = float src
    // control flow of the dynamic inner iterations (multi_split_solve.cc:119-134)
    PS_NORM2 = 11,     // per-CTA partial sums of v_i^2 into the reduction buffer
    PS_LOOPTEST = 12,  // ||v|| from the partials; mode bit 8 set: record it as the
                       // loop's initial norm; else jump to target when ||v|| / init < s0
    PS_JUMP = 13,      // back to target; counts the loop's sweeps against its cap
};

// Loops (nested dynamic level calls) one program may hold; the sweeps of one
// level call, and of all level calls of one launch, before the apply gives up
// (the reference has no cap; nested loops multiply, so the total is capped too).
static constexpr uint32_t PK_MAXLOOP = 16;
static constexpr uint32_t PK_LOOP_CAP = 1000;
static constexpr uint32_t PK_TOTAL_CAP = 100000;

// One step. Fields not used by an op are zero.
template <class T>
struct alignas(16) PStep {
    uint32_t op;
    uint32_t lpr;    // lanes per row of the replaced kernel (1 = a serial row sum)
    uint32_t mode;   // PS_UPDATE: 1 = also r -= Af u0; loop ops: loop slot (+ 256 = record init)
    uint32_t target; // PS_LOOPTEST / PS_JUMP: step index to go to
    uint32_t n0, n1; // sizes (rows; second bound)
    uint32_t pad2[2];
    const uint32_t* ia;
    const uint32_t* ja;
    const T* a;      // matrix values (PS_DENSE: the dense operator)
    const T* dval;
    void* v[4];      // vector operands, in the order the op's comment lists them
    double s0, s1;   // scalar operands
};

// Grid barrier state of one persistent plan (device memory, zeroed once).
// count: arrivals (grows by the grid size per barrier, reset by the last CTA
// to leave the kernel); exitc: CTAs that left; err: 1 when a barrier wait ran
// out of its iteration limit, 2 when a dynamic level iteration reached
// PK_LOOP_CAP sweeps (the kernel then stops early and the host reports it).
// red: one partial sum per CTA for the norms of the dynamic iterations.
struct PBar {
    unsigned count;
    unsigned exitc;
    int err;
    unsigned pad;
    double red[2048];
};

// Threads per CTA of k_persist.
static constexpr int PK_THREADS = 512;

// Records the launch of k_persist<T> over steps[0, nsteps) on stream s (a
// cooperative launch: every CTA is resident at once, which the barrier needs).
template <class T>
void launch_persist(const PStep<T>* steps, uint32_t nsteps, PBar* bar, cudaStream_t s);

// CTAs of one launch (a multiple of the SM count).
template <class T>
unsigned persist_grid();

}  // namespace mlp
