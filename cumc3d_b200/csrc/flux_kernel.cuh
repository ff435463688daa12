// flux_kernel.cuh -- fused reconstruction + face EOS + BUILDSTATES + Riemann
// solver + MHD_FLUX for one sweep direction.
//
// Replaces, per direction, the reference's chain of full-array passes
// {tvd,ppmc,weno}_recon{x,y,z} -> BUILDSTATES -> {LF,HLL,HLLC,HLLD}NM ->
// MHD_FLUX (solver/mhd/spatial.f90:33-63 and the modules it calls), which
// writes primL/primR/uL/uR/fluxL/fluxR (48 doubles per face) through HBM,
// with one kernel that keeps all of it on chip:
//
//   phase 1: one thread per cell of a tile along the sweep reads the 5-point
//            stencil of the 5 hydro primitives and the 2 transverse cell
//            fields and writes both edge values to shared memory;
//   phase 2: one thread per interior face of the tile combines the right edge
//            of cell f with the left edge of cell f+1, evaluates the face EOS,
//            the L/R conserved states and physical fluxes, and the Riemann
//            flux, then stores the 5 hydro fluxes and the 2 face EMFs.
//
// Tiles along the sweep overlap by one cell, so every face is produced by
// exactly one thread.
#pragma once
#include "engine.cuh"
#include "mhd_device.cuh"

namespace cumc {

// face EOS, model/riemann/src/getepsilon.f90:4-16 and soundspeed.f90:4-21
template <class T>
__device__ __forceinline__ T eos_eps(T rho, T p, T g) { return p / rho / (g - T(1)); }
template <class T>
__device__ __forceinline__ T eos_cs(T p, T rho, T e, T g) {
    T dpdden = e * (g - T(1));
    T dpdint = rho * (g - T(1));
    return dsqrt(dpdden + dpdint * p / (rho * rho));
}

template <class T> __device__ __forceinline__ const T *weights(const Dev &d, int dir);
template <> __device__ __forceinline__ const double *weights<double>(const Dev &d, int dir) {
    return dir == 0 ? d.wx : dir == 1 ? d.wy : d.wz;
}
template <> __device__ __forceinline__ const float *weights<float>(const Dev &d, int dir) {
    return dir == 0 ? d.wxf : dir == 1 ? d.wyf : d.wzf;
}

template <class T, int DIR, int REC, int RS>
__global__ void __launch_bounds__(256) k_flux(const Dev d) {
    if (d.S->done) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nthr = blockDim.x * blockDim.y;
    T *sVM = reinterpret_cast<T *>(smem_raw);
    T *sVP = sVM + 7 * nthr;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;

    int TS, ls, c, j, k, l, ns;
    bool tvalid;
    if (DIR == 0) {
        TS = blockDim.x; ls = threadIdx.x; c = blockIdx.x * (TS - 1) + ls;
        j = c; k = blockIdx.y * blockDim.y + threadIdx.y + 1; l = blockIdx.z + 1;
        ns = d.nx; tvalid = (k <= d.ny);
    } else if (DIR == 1) {
        TS = blockDim.y; ls = threadIdx.y; c = blockIdx.y * (TS - 1) + ls;
        k = c; j = blockIdx.x * blockDim.x + threadIdx.x + 1; l = blockIdx.z + 1;
        ns = d.ny; tvalid = (j <= d.nx);
    } else {
        TS = blockDim.y; ls = threadIdx.y; c = blockIdx.y * (TS - 1) + ls;
        l = c; j = blockIdx.x * blockDim.x + threadIdx.x + 1; k = blockIdx.z + 1;
        ns = d.nz; tvalid = (j <= d.nx);
    }
    const int st = (DIR == 0) ? 1 : (DIR == 1) ? d.NX : d.NX * d.NY;
    const bool rvalid = tvalid && (c <= ns + 1);
    const int ci = rvalid ? cidx(d, j, k, l) : 0;

    // transverse cell fields, in the reference's order (ppmc_module.f90:194-195, 263-264, 332-333)
    constexpr int tb1 = (DIR == 0) ? 1 : 0;  // bcell index 0..2
    constexpr int tb2 = (DIR == 2) ? 1 : 2;

    if (rvalid) {
        const T *wp = weights<T>(d, DIR) + (size_t)(c + 2) * 14;
        T w[14];
        constexpr int NW = (REC == REC_PPM) ? 14 : (REC == REC_WENO) ? 10 : 2;
#pragma unroll
        for (int m = 0; m < NW; ++m) w[m] = wp[m];
        bool fallback = false;
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            const double *src = (v < 5) ? d.P[v] : d.BC[v == 5 ? tb1 : tb2];
            T a0 = T(0), a4 = T(0);
            if (REC == REC_PPM || REC == REC_WENO) {
                a0 = (T)__ldg(src + ci - 2 * st);
                a4 = (T)__ldg(src + ci + 2 * st);
            }
            T a1 = (T)__ldg(src + ci - st);
            T a2 = (T)__ldg(src + ci);
            T a3 = (T)__ldg(src + ci + st);
            T vm, vp;
            recon_cell<T, REC>(w, a0, a1, a2, a3, a4, vm, vp);
            if (v == 4 && d.pos_fallback) {
                // first-order fallback when an edge density or pressure is not
                // positive (optional; the reference has no such guard)
                fallback = !(sVM[0 * nthr + tid] > T(0) && sVP[0 * nthr + tid] > T(0) && vm > T(0) && vp > T(0));
                if (fallback) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const T cv = (T)__ldg(d.P[u] + ci);
                        sVM[u * nthr + tid] = cv;
                        sVP[u * nthr + tid] = cv;
                    }
                }
            }
            if (fallback) vm = vp = a2;
            sVM[v * nthr + tid] = vm;
            sVP[v * nthr + tid] = vp;
        }
    }
    __syncthreads();
    if (!(rvalid && ls < TS - 1 && c <= ns)) return;

    using F = Frame<DIR>;
    const int tn = (DIR == 0) ? tid + 1 : tid + blockDim.x;
    T pl[9], pr[9];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        pl[1 + v] = sVP[v * nthr + tid];
        pr[1 + v] = sVM[v * nthr + tn];
    }
    pl[ibx + tb1] = sVP[5 * nthr + tid];
    pr[ibx + tb1] = sVM[5 * nthr + tn];
    pl[ibx + tb2] = sVP[6 * nthr + tid];
    pr[ibx + tb2] = sVM[6 * nthr + tn];
    const T bn = (T)d.P[F::ibn - 1][ci];  // face field at face c (ppmc_module.f90:198-199)
    pl[F::ibn] = bn;
    pr[F::ibn] = bn;
    const T g = (T)d.gamma;
    const T epsL = eos_eps(pl[irho], pl[itau], g);
    const T epsR = eos_eps(pr[irho], pr[itau], g);
    const T csL = eos_cs(pl[itau], pl[irho], epsL, g);
    const T csR = eos_cs(pr[itau], pr[irho], epsR, g);
    T fo[9];
    riemann_face<T, DIR, RS>(pl, pr, epsL, epsR, csL, csR, fo);

    double *const *FO = (DIR == 0) ? d.FX : (DIR == 1) ? d.FY : d.FZ;
#pragma unroll
    for (int v = 0; v < 5; ++v) FO[v][ci] = (double)fo[1 + v];
    // MHD_FLUX, solver/mhd/mhd_module.f90:229-270
    if (DIR == 0) {
        d.EF[e_yx][ci] = (double)fo[ibz];
        d.EF[e_zx][ci] = -(double)fo[iby];
    } else if (DIR == 1) {
        d.EF[e_xy][ci] = -(double)fo[ibz];
        d.EF[e_zy][ci] = (double)fo[ibx];
    } else {
        d.EF[e_xz][ci] = (double)fo[iby];
        d.EF[e_yz][ci] = -(double)fo[ibx];
    }
}

template <class T, int DIR, int REC>
static void launch_rs(const Dev &d, int rs, dim3 g, dim3 b, size_t sm, cudaStream_t s) {
    switch (rs) {
        case RS_LF: k_flux<T, DIR, REC, RS_LF><<<g, b, sm, s>>>(d); break;
        case RS_HLL: k_flux<T, DIR, REC, RS_HLL><<<g, b, sm, s>>>(d); break;
        case RS_HLLC: k_flux<T, DIR, REC, RS_HLLC><<<g, b, sm, s>>>(d); break;
        default: k_flux<T, DIR, REC, RS_HLLD><<<g, b, sm, s>>>(d); break;
    }
}
template <class T, int DIR>
static void launch_rec(const Dev &d, int rec, int rs, dim3 g, dim3 b, size_t sm, cudaStream_t s) {
    switch (rec) {
        case REC_TVD_MM: launch_rs<T, DIR, REC_TVD_MM>(d, rs, g, b, sm, s); break;
        case REC_TVD_VL: launch_rs<T, DIR, REC_TVD_VL>(d, rs, g, b, sm, s); break;
        case REC_TVD_MC: launch_rs<T, DIR, REC_TVD_MC>(d, rs, g, b, sm, s); break;
        case REC_PPM: launch_rs<T, DIR, REC_PPM>(d, rs, g, b, sm, s); break;
        default: launch_rs<T, DIR, REC_WENO>(d, rs, g, b, sm, s); break;
    }
}
template <class T>
static void launch_flux_t(const Dev &d, int dir, int rec, int rs, dim3 g, dim3 b, size_t sm, cudaStream_t s) {
    if (dir == 0) launch_rec<T, 0>(d, rec, rs, g, b, sm, s);
    else if (dir == 1) launch_rec<T, 1>(d, rec, rs, g, b, sm, s);
    else launch_rec<T, 2>(d, rec, rs, g, b, sm, s);
}

}  // namespace cumc
