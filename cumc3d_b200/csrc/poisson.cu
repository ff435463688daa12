// poisson.cu -- red-black SOR for the self-gravity potential of the collapsar
// model on a spherical grid (layout and state: poisson.cuh).  Compiled with
// --fmad=false: every expression rounds as the Fortran does.
//
// One iteration (model/collapsar/src/custom.f90:489-616) is three launches:
// the red sweep, the black sweep, and the ghost layers with the convergence
// check.
// The reference copies phi to phi_old before the sweeps and takes
// max |(phi - phi_old) / phi_old| afterwards; each interior cell is updated
// exactly once per iteration, so the sweep that updates a cell has both
// values at hand and takes the maximum itself (no copy).  The maximum of
// non-negative doubles is exact and independent of order, so the iteration
// count and every bit of phi match a sequential run of the same loops.
#include <cmath>

#include "poisson.cuh"

namespace cumc {

// poisson_coef (model/collapsar/src/poisson.f90:34-64) at every interior
// cell; x, y, z point at the centres of index 0 (valid for -1..n+2).
// Natural layouts: ajp1/ajm1 by j, bkp1/bkm1 by j + (nx+2) k, the rest by
// j + (nx+2) (k + (ny+2) l).
void sor_coefficients(int nx, int ny, int nz, const double *x, const double *y, const double *z, double *ajp1,
                      double *ajm1, double *bkp1, double *bkm1, double *clp1, double *clm1, double *epsc) {
    const long long px = nx + 2, py = (long long)(nx + 2) * (ny + 2);
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j)
            for (int k = 1; k <= nz; ++k) {
                const double xm1 = x[i - 1], xc = x[i], xp1 = x[i + 1];
                const double ym1 = y[j - 1], yc = y[j], yp1 = y[j + 1];
                const double zm1 = z[k - 1], zc = z[k], zp1 = z[k + 1];
                const double ty = std::tan(yc), sy = std::sin(yc);
                const long long c = i + px * j + py * k;
                epsc[c] = 2.0 * (xp1 + xm1 - 3.0 * xc) / xc / (xp1 - xc) / (xc - xm1) +
                          (yp1 + ym1 - 2.0 * yc - 2.0 * ty) / (xc * xc) / ty / (yp1 - yc) / (yc - ym1) -
                          2.0 / (xc * xc) / (sy * sy) / (zp1 - zc) / (zc - zm1);
                ajp1[i] = 2.0 * (2.0 * xc - xm1) / (xp1 - xm1) / (xp1 - xc) / xc;
                ajm1[i] = 2.0 * (2.0 * xc - xp1) / (xp1 - xm1) / (xc - xm1) / xc;
                bkp1[i + px * j] = (2.0 * ty + yc - ym1) / (xc * xc) / ty / (yp1 - yc) / (yp1 - ym1);
                bkm1[i + px * j] = (2.0 * ty + yc - yp1) / (xc * xc) / ty / (yp1 - ym1) / (yc - ym1);
                clp1[c] = 2.0 / (xc * xc) / (sy * sy) / (zp1 - zm1) / (zp1 - zc);
                clm1[c] = 2.0 / (xc * xc) / (sy * sy) / (zp1 - zm1) / (zc - zm1);
            }
}

// 4 pi rho_in per interior cell, rho_in = rho where rho exceeds the
// atmosphere density, else 0 (custom.f90:527-529).  rho in the engine's
// padded layout (index (j+2) + NX ((k+2) + NY (l+2))).
__global__ void k_sor_source(const SorDev s, const double *__restrict__ rho, int NX, int NY, double rho_atm,
                             double fourpi) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int l = blockIdx.z + 1;
    if (j > s.nx || k > s.ny) return;
    const double r = rho[(j + 2) + (long long)NX * ((k + 2) + (long long)NY * (l + 2))];
    const double diff = r - rho_atm;
    const double factor = diff > 0.0 ? 1.0 : 0.0;
    const double rho_in = factor * r;
    s.src[(j + k + l) & 1][sor_index(s, j, k, l)] = fourpi * rho_in;
}

// one colour: C = 0 red ((-1)**(j+k+l) > 0), 1 black; a 32 x 8 block covers
// 32 half-row cells (h) of RPT * 8 rows (k, every 8th row per thread) of
// plane l = blockIdx.z + 1, so a thread has the loads of RPT cells in flight
template <int C, int RPT>
__global__ void __launch_bounds__(256) k_sor_sweep(const SorDev s) {
    if (s.state[1]) return;
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.z + 1;
    const long long ys = s.hx, zs = (long long)s.hx * (s.ny + 2);
    unsigned long long e = 0ull;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int k = (blockIdx.y * RPT + r) * blockDim.y + threadIdx.y + 1;
        const int j = 2 * h + ((C + k + l) & 1);
        if (h < s.hx && k <= s.ny && j >= 1 && j <= s.nx) {
            const double *o = s.phi[1 - C];
            const long long row = (long long)s.hx * (k + (long long)(s.ny + 2) * l);
            const long long c = h + row;
            const double pE = o[((j + 1) >> 1) + row], pW = o[((j - 1) >> 1) + row];
            const double pN = o[c + ys], pS = o[c - ys], pU = o[c + zs], pD = o[c - zs];
            const long long b = j + (long long)(s.nx + 2) * k;
            double sum = s.ajp1[j] * pE + s.ajm1[j] * pW;
            sum = sum + s.bkp1[b] * pN;
            sum = sum + s.bkm1[b] * pS;
            sum = sum + s.clp1[C][c] * pU;
            sum = sum + s.clm1[C][c] * pD;
            const double rhs = (s.src[C][c] - sum) / s.epsc[C][c];
            const double old = s.phi[C][c];
            const double nw = (1.0 - s.omega) * old + s.omega * rhs;
            s.phi[C][c] = nw;
            // |x| of a double keeps the bit order of its magnitude (NaN above +inf)
            const unsigned long long v = (unsigned long long)__double_as_longlong(fabs((nw - old) / old));
            e = v > e ? v : e;
        }
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, e, m);
        e = v > e ? v : e;
    }
    __shared__ unsigned long long wmax[8];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if ((tid & 31) == 0) wmax[tid >> 5] = e;
    __syncthreads();
    if (tid == 0) {
        unsigned long long m = wmax[0];
        for (int w = 1; w < (int)(blockDim.x * blockDim.y) / 32; ++w) m = wmax[w] > m ? wmax[w] : m;
        if (m) atomicMax(s.err, m);
    }
}

// ghost layers (custom.f90:578-612): phi(0) = phi(1), phi(nx+1) = -1 along
// r; copies of the first and last row along theta; periodic along phi.  The
// three sets are disjoint and read interior cells only.  Thread 0 also takes
// the exit test (IF (abserror <= tolerance) EXIT) and the iteration limit:
// both sweeps have finished, so the iteration's maximum is complete; the
// error of the next iteration starts at 1e-50 as in the reference.  The
// ghost writes never skip: once the loop has ended, a replay recomputes the
// same values from the unchanged interior.
__global__ void k_sor_ghosts(const SorDev s) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0 && s.state[1] == 0) {
        const int it = s.state[0] + 1;
        s.state[0] = it;
        const double e = __longlong_as_double((long long)*s.err);
        *s.err_last = e;
        if (e <= *s.tol) s.state[1] = 1;
        else if (it >= s.state[2]) s.state[1] = 2;
        *s.err = (unsigned long long)__double_as_longlong(1.0e-50);
    }
    const long long nyz = (long long)s.ny * s.nz, nxz = (long long)s.nx * s.nz, nxy = (long long)s.nx * s.ny;
    auto at = [&](int j, int k, int l) -> double & { return s.phi[(j + k + l) & 1][sor_index(s, j, k, l)]; };
    if (t < nyz) {
        const int k = (int)(t % s.ny) + 1, l = (int)(t / s.ny) + 1;
        at(0, k, l) = at(1, k, l);
        at(s.nx + 1, k, l) = -1.0;
    } else if (t < nyz + nxz) {
        const long long u = t - nyz;
        const int j = (int)(u % s.nx) + 1, l = (int)(u / s.nx) + 1;
        at(j, 0, l) = at(j, 1, l);
        at(j, s.ny + 1, l) = at(j, s.ny, l);
    } else if (t < nyz + nxz + nxy) {
        const long long u = t - nyz - nxz;
        const int j = (int)(u % s.nx) + 1, k = (int)(u / s.nx) + 1;
        at(j, k, 0) = at(j, k, s.nz);
        at(j, k, s.nz + 1) = at(j, k, 1);
    }
}

__global__ void k_sor_reset(const SorDev s) {
    s.state[0] = 0;
    s.state[1] = 0;
    *s.err = (unsigned long long)__double_as_longlong(1.0e-50);
}

void launch_sor_source(const SorDev &s, const double *rho, int NX, int NY, double rho_atm, cudaStream_t st) {
    const double fourpi = 4.0 * (4.0 * std::atan(1.0));  // 4.0d0*pi, pi = 4.D0*DATAN(1.D0)
    const dim3 b(32, 8, 1), g((s.nx + 31) / 32, (s.ny + 7) / 8, s.nz);
    k_sor_source<<<g, b, 0, st>>>(s, rho, NX, NY, rho_atm, fourpi);
}

template <int RPT>
static void sweeps(const SorDev &s, cudaStream_t st) {
    const dim3 b(32, 8, 1), g((s.hx + 31) / 32, (s.ny + 8 * RPT - 1) / (8 * RPT), s.nz);
    k_sor_sweep<0, RPT><<<g, b, 0, st>>>(s);
    k_sor_sweep<1, RPT><<<g, b, 0, st>>>(s);
}

void launch_sor_iteration(const SorDev &s, cudaStream_t st) {
    sweeps<2>(s, st);  // two rows per thread: 0.185 vs 0.225 ms per iteration for one, 0.203 for four (384x192x192)
    const long long ng = (long long)s.ny * s.nz + (long long)s.nx * s.nz + (long long)s.nx * s.ny;
    k_sor_ghosts<<<(unsigned)((ng + 255) / 256), 256, 0, st>>>(s);
}

void launch_sor_reset(const SorDev &s, cudaStream_t st) { k_sor_reset<<<1, 1, 0, st>>>(s); }

}  // namespace cumc
