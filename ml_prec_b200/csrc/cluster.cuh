// Cluster-resident level calls: one call of a small level (tens of thousands
// of rows) and everything below it, run by ONE thread-block cluster whose CTAs
// hold the level's vectors and matrices in their shared memory.
//
// The multi-split recursion calls the level below the finest one niter times
// per finest-level sweep, and every call is a chain of ~20 dependent sweep
// steps over a few hundred KB. As separate launches each step costs a launch
// latency; inside a grid-wide persistent kernel each costs a software grid
// barrier plus three dependent L2 round trips (row pointer, entries, vector
// values). Here the data sit in distributed shared memory (DSMEM): up to 16
// CTAs x ~200 KB on one GPC, the matrices partitioned by rows into the CTA
// that processes them, the vectors partitioned in power-of-two chunks and
// read or written through `mapa` + `ld/st.shared::cluster`, and consecutive
// steps separated by the hardware cluster barrier. A call copies its
// partitions in from global memory (L2-resident), runs all its steps, and
// writes its output vector back.
//
// The steps are the ones the plan builder records for the persistent forms
// (PStep), translated to array/offset operands. Each repeats the arithmetic
// of the kernel it replaces (lane split per row, fused multiply-adds in entry
// order, xor butterfly; a warp per dense row), so results are bit-identical to
// the launch-per-step plan.
#pragma once

#include "persist.cuh"

namespace mlp {

static constexpr int CL_THREADS = 1024;
static constexpr uint32_t CL_MAX_ARR = 64;
static constexpr uint32_t CL_MAX_MAT = 32;
// Dynamic shared memory a CTA may use for the level's data (B200: 227 KB per
// CTA; the rest holds the tables and descriptors).
static constexpr uint32_t CL_SMEM_BUDGET = 200 * 1024;

// A distributed array: element i lives in CTA i >> shift at byte offset
// off + (i & (2^shift - 1)) * element size of that CTA's shared memory.
struct CArr {
    uint32_t off, shift, n, pad;
};

// A CSR matrix partitioned by rows: CTA b holds rows [b << shift, (b + 1) << shift)
// (row pointers as stored, entries from the first row's start), at the same
// byte offsets in every CTA.
struct CMat {
    uint32_t ia_off, ja_off, a_off, shift;
    uint32_t rows, pad[3];
};

// One step: the PStep op with its vector operands as (array, element offset).
template <class T>
struct alignas(16) CStep {
    uint32_t op, lpr, n0, n1;
    uint32_t mat, dval, mode, pad;
    uint32_t arr[4], off[4];
    const void* C;  // PS_DENSE: the operator in global memory (T, or double when mode == 1)
    const void* pad2;
};

// A contiguous copy of 32-bit words from global memory into one CTA's shared
// memory (matrix partitions and constant arrays, read-only during the call).
struct CCopy {
    const uint32_t* src;
    uint32_t dst, words;
};

// Everything one launch reads, in one device buffer: this header, then the
// tables it points to.
template <class T>
struct CProg {
    uint32_t nsteps, narr, nmat, cs;
    uint32_t smem;          // dynamic shared memory per CTA (bytes)
    uint32_t f_arr, x_arr;  // the call's input and output arrays
    uint32_t n;             // their length
    const T* f;             // the call's input vector (global)
    T* x;                   // the call's output vector (global)
    const CArr* arrs;
    const CMat* mats;
    const CStep<T>* steps;
    const uint32_t* copy_first;  // cs + 1 entries: the copies of CTA b are [copy_first[b], copy_first[b + 1])
    const CCopy* copies;
};

// CTAs of the cluster for a launch that needs `smem` dynamic bytes per CTA:
// 16 when such a cluster fits on the device, else 0 (the call then takes
// another form).
template <class T>
unsigned cluster_level_size(uint32_t smem);

// Records the launch of one cluster-resident call on stream s. prog points to
// the device copy of a CProg<T> whose tables follow it.
template <class T>
void launch_cluster_level(const CProg<T>* prog, uint32_t cs, uint32_t smem, cudaStream_t s);

// A device vector the recorded steps may address (a level's work buffers).
struct ClusterVec {
    const void* p;
    uint32_t n;  // elements
};

// Translates the steps recorded for one level call (input f, output x, n
// elements each) into a cluster-resident program: every vector operand must
// lie inside f, x or one of vecs, every op must have a cluster form, and the
// partitions must fit the shared-memory budget of a 16-CTA cluster. On
// success the program is uploaded into `out` (its first bytes are the
// CProg<T>) and cs / smem give the launch shape; otherwise returns false and
// the call takes another form. Reads the row pointers of the matrices back
// from the device (stream s is synchronised).
template <class T>
bool cluster_prog_build(const std::vector<PStep<T>>& steps, const T* f, T* x, uint32_t n,
                        const std::vector<ClusterVec>& vecs, DBuf<uint8_t>& out, uint32_t& cs, uint32_t& smem,
                        cudaStream_t s);

}  // namespace mlp
