// Differentiation form: gradient of a pressure misfit with respect to the
// per-cell log-permeability, by the adjoint method.
//
// The SPE matrix (spe.cc:69-131) has, for each link (i, j) along axis a, the
// harmonic-mean transmissibility T = 2/(1/k_i + 1/k_j)/h_a^2 added to both
// diagonals and subtracted off the diagonal, and (benchmark problem) the
// Dirichlet x-face terms tD = 2 kx/hx^2 on the diagonal with tD * p_D in b.
// With theta = ln K per cell (kx = ky = K, kz = 0.1 K, so dk/dtheta = k on every
// axis):
//   dT_ij/dtheta_i = 2 k_i k_j^2 / (h^2 (k_i + k_j)^2),   dtD_i/dtheta_i = tD_i.
// For J(p(theta)) with A p = b and lambda solving A^T lambda = A lambda = dJ/dp
// (A is symmetric), dJ/dtheta_c = -lambda^T (dA/dtheta_c p - db/dtheta_c):
//   -sum_{j ~ c} dT_cj/dtheta_c (lambda_c - lambda_j)(p_c - p_j)
//   - [c on a Dirichlet face] tD_c lambda_c (p_c - p_D).
// The kernel gathers each cell's own terms from its (at most six) links, so the
// scatter of the transmissibility derivatives needs no atomics.
#include "solve.cuh"

namespace mlp {

__device__ __forceinline__ uint32_t gkidx(uint32_t i, uint32_t j, uint32_t k) {
    return (k * 13200u + j * 60u + i) % 1122000u;
}

__device__ __forceinline__ double dT_dtheta(double ki, double kj, double h) {
    double s = ki + kj;
    return 2 * ki * kj * kj / (h * h * s * s);
}

__global__ void k_grad_logk(uint32_t nx, uint32_t ny, uint32_t nz, const double* __restrict__ kx,
                            const double* __restrict__ ky, const double* __restrict__ kz, int dirichlet,
                            const double* __restrict__ p, const double* __restrict__ lam, double* __restrict__ g) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t N = nx * ny * nz;
    if (r >= N) return;
    const double hx = 20, hy = 10, hz = 2;
    uint32_t i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
    uint32_t me = gkidx(i, j, k);
    double pc = p[r], lc = lam[r], acc = 0;
    if (k > 0) { uint32_t o = r - nx * ny; acc += dT_dtheta(kz[me], kz[gkidx(i, j, k - 1)], hz) * (lc - lam[o]) * (pc - p[o]); }
    if (j > 0) { uint32_t o = r - nx; acc += dT_dtheta(ky[me], ky[gkidx(i, j - 1, k)], hy) * (lc - lam[o]) * (pc - p[o]); }
    if (i > 0) { uint32_t o = r - 1; acc += dT_dtheta(kx[me], kx[gkidx(i - 1, j, k)], hx) * (lc - lam[o]) * (pc - p[o]); }
    if (i + 1 < nx) { uint32_t o = r + 1; acc += dT_dtheta(kx[me], kx[gkidx(i + 1, j, k)], hx) * (lc - lam[o]) * (pc - p[o]); }
    if (j + 1 < ny) { uint32_t o = r + nx; acc += dT_dtheta(ky[me], ky[gkidx(i, j + 1, k)], hy) * (lc - lam[o]) * (pc - p[o]); }
    if (k + 1 < nz) { uint32_t o = r + nx * ny; acc += dT_dtheta(kz[me], kz[gkidx(i, j, k + 1)], hz) * (lc - lam[o]) * (pc - p[o]); }
    if (dirichlet) {
        double tD = 2 * kx[me] / (hx * hx);
        if (i == 0) acc += tD * lc * (pc - 1.0);
        if (i == nx - 1) acc += tD * lc * pc;
    }
    g[r] = -acc;
}

void spe_grad_logk(uint32_t nx, uint32_t ny, uint32_t nz, const double* kx, const double* ky, const double* kz,
                   int dirichlet, const double* p, const double* lam, double* g, cudaStream_t s) {
    uint32_t N = nx * ny * nz;
    if (!N) return;
    k_grad_logk<<<grid_for(N, 256), 256, 0, s>>>(nx, ny, nz, kx, ky, kz, dirichlet, p, lam, g);
    CK_LAUNCH();
}

}  // namespace mlp
