// poisson.cuh -- self-gravity potential of the collapsar model: red-black
// successive over-relaxation of the spherical Poisson equation
// (model/collapsar/src/custom.f90:489-620, coefficients
// model/collapsar/src/poisson.f90:6-64).
//
// Layout: the potential, the per-cell coefficients and the source term are
// stored split by colour, c = (j + k + l) & 1 (c = 0: the reference's red
// cells, (-1)**(j+k+l) > 0).  Cell (j, k, l), j,k,l = 0..n+1, lives in
// array c at h + hx * (k + (ny + 2) * l) with h = j >> 1 and hx = (nx + 3) / 2.
// A sweep over one colour then reads the other colour's array contiguously
// (its y and z neighbours sit at the same h in the neighbouring rows, its x
// neighbours at (j - 1) >> 1 and (j + 1) >> 1) and reads and writes its own
// contiguously: every access is coalesced, and no byte of a colour that a
// sweep does not touch is fetched.
#pragma once
#include <cuda_runtime.h>

namespace cumc {

struct SorDev {
    int nx, ny, nz, hx;
    double *phi[2];
    const double *clp1[2], *clm1[2], *epsc[2];  // per cell, colour-split (interior cells)
    double *src[2];                             // 4 pi rho_in per cell, colour-split
    const double *ajp1, *ajm1;                  // per j = 0..nx+1
    const double *bkp1, *bkm1;                  // per (j, k): j + (nx + 2) * k
    double omega;
    // loop state on the device: the iteration's max |dphi / phi_old| (bit
    // pattern of a non-negative double), [0] iterations taken, [1] 0 running /
    // 1 converged / 2 iteration limit, [2] the limit; the tolerance; the last
    // iteration's error
    unsigned long long *err;
    int *state;
    double *tol;
    double *err_last;
};

__host__ __device__ inline long long sor_index(const SorDev &s, int j, int k, int l) {
    return (long long)(j >> 1) + (long long)s.hx * (k + (long long)(s.ny + 2) * l);
}

// host side (poisson.cu)
void sor_coefficients(int nx, int ny, int nz, const double *x, const double *y, const double *z, double *ajp1,
                      double *ajm1, double *bkp1, double *bkm1, double *clp1, double *clm1, double *epsc);
void launch_sor_source(const SorDev &s, const double *rho, int NX, int NY, double rho_atm, cudaStream_t st);
void launch_sor_iteration(const SorDev &s, cudaStream_t st);
void launch_sor_reset(const SorDev &s, cudaStream_t st);

}  // namespace cumc
