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

// hydro face fluxes are stored in the precision of the flux arithmetic: FP64
// in the plain form, FP32 in the FP32 form (the RK accumulation that reads
// them stays FP64); the arrays are FP64-sized either way
template <class T> __device__ __forceinline__ void store_flux(double *a, int i, T v);
template <> __device__ __forceinline__ void store_flux<double>(double *a, int i, double v) { a[i] = v; }
template <> __device__ __forceinline__ void store_flux<float>(double *a, int i, float v) {
    reinterpret_cast<float *>(a)[i] = v;
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

    // stage the stencils of the tile in shared memory: every state value
    // loaded and converted once (2-cell halo along the sweep)
    const int SX = (DIR == 0) ? (int)blockDim.x + 4 : (int)blockDim.x;
    const int SR = (DIR == 0) ? (int)blockDim.y : (int)blockDim.y + 4;
    T *sS = sVP + 7 * nthr;  // [7][SR][SX]
    {
        const int c0 = (DIR == 0) ? (int)blockIdx.x * (TS - 1) : (int)blockIdx.y * (TS - 1);
        for (int idx = tid; idx < SR * SX; idx += nthr) {
            const int sr = idx / SX, sx = idx - sr * SX;
            int x, y, z;
            bool ok;
            if (DIR == 0) {
                x = c0 - 2 + sx; y = blockIdx.y * blockDim.y + sr + 1; z = blockIdx.z + 1;
                ok = x <= d.nx + 3 && y <= d.ny;
            } else if (DIR == 1) {
                x = blockIdx.x * blockDim.x + sx + 1; y = c0 - 2 + sr; z = blockIdx.z + 1;
                ok = x <= d.nx && y <= d.ny + 3;
            } else {
                x = blockIdx.x * blockDim.x + sx + 1; y = blockIdx.z + 1; z = c0 - 2 + sr;
                ok = x <= d.nx && z <= d.nz + 3;
            }
            if (ok) {
                const int cc = cidx(d, x, y, z);
#pragma unroll
                for (int v = 0; v < 7; ++v) {
                    const double *src = (v < 5) ? d.P[v] : d.BC[v == 5 ? tb1 : tb2];
                    sS[(v * SR + sr) * SX + sx] = (T)__ldg(src + cc);
                }
            }
        }
        __syncthreads();
    }
    // this cell's stencil c-2 .. c+2 in the staged tile
    const int sb = (DIR == 0) ? (int)threadIdx.y * SX + ls + 2 : (ls + 2) * SX + (int)threadIdx.x;
    const int sm = (DIR == 0) ? 1 : SX;

    if (rvalid) {
        const T *wp = weights<T>(d, DIR) + (size_t)(c + 2) * 14;
        T w[14];
        constexpr int NW = (REC == REC_PPM) ? 14 : (REC == REC_WENO) ? 10 : 2;
#pragma unroll
        for (int m = 0; m < NW; ++m) w[m] = wp[m];
        bool fallback = false;
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            const T *sv = sS + v * SR * SX + sb;
            T a0 = T(0), a4 = T(0);
            if (REC == REC_PPM || REC == REC_WENO) {
                a0 = sv[-2 * sm];
                a4 = sv[2 * sm];
            }
            T a1 = sv[-sm];
            T a2 = sv[0];
            T a3 = sv[sm];
            T vm, vp;
            recon_cell<T, REC>(w, a0, a1, a2, a3, a4, vm, vp);
            if (v == 4 && d.pos_fallback) {
                // first-order fallback when an edge density or pressure is not
                // positive (optional; the reference has no such guard)
                fallback = !(sVM[0 * nthr + tid] > T(0) && sVP[0 * nthr + tid] > T(0) && vm > T(0) && vp > T(0));
                // a cell shared by two tiles (ls = TS - 1 and 0 of the next) counts once
                if (fallback && d.fb_count && (ls < TS - 1 || c == ns + 1)) atomicAdd(d.fb_count, 1ull);
                if (fallback) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const T cv = sS[u * SR * SX + sb];
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
    for (int v = 0; v < 5; ++v) store_flux<T>(FO[v], ci, fo[1 + v]);
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

// ---------------------------------------------------------------------------
// split form: k_recon writes the face states, k_riemann consumes them.  The
// reconstruction (about 70% of the FP64 work, few registers) then runs at
// full occupancy instead of at the register-limited occupancy of HLLD.
// Face states: QL[v][f] = right edge of cell f, QR[v][f] = left edge of cell
// f+1, v = rho, vx, vy, vz, p, first and second transverse cell field.
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ T uni_w(const Dev &d, int dir, int m);
template <> __device__ __forceinline__ double uni_w<double>(const Dev &d, int dir, int m) { return d.wu[dir][m]; }
template <> __device__ __forceinline__ float uni_w<float>(const Dev &d, int dir, int m) { return d.wuf[dir][m]; }

// UNI = 1: every cell along the sweep has the same weights (uniform spacing
// along this axis, checked bit for bit on the host); they then come from the
// kernel parameters and live in uniform registers.
template <class T, int DIR, int REC, int UNI>
__global__ void __launch_bounds__(256) k_recon(const Dev d) {
    if (d.S->done) return;
    // one thread per reconstructed cell, enumerated x fastest with no tail
    // padding per row: x extent nx+2 (x sweep) or nx, then y, then z
    int c, j, k, l, ns;
    {
        const unsigned ex = (DIR == 0) ? d.nx + 2 : d.nx;
        const unsigned ey = (DIR == 1) ? d.ny + 2 : d.ny;
        const unsigned ez = (DIR == 2) ? d.nz + 2 : d.nz;
        const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= ex * ey * ez) return;
        int a, b, e;
        unflat3(t, ex, ey, a, b, e);
        if (DIR == 0) { c = a; j = c; k = b + 1; l = e + 1; ns = d.nx; }
        else if (DIR == 1) { c = b; k = c; j = a + 1; l = e + 1; ns = d.ny; }
        else { c = e; l = c; j = a + 1; k = b + 1; ns = d.nz; }
    }
    const int st = (DIR == 0) ? 1 : (DIR == 1) ? d.NX : d.NX * d.NY;
    const int ci = cidx(d, j, k, l);
    constexpr int tb1 = (DIR == 0) ? 1 : 0;
    constexpr int tb2 = (DIR == 2) ? 1 : 2;
    T w[14];
    constexpr int NW = (REC == REC_PPM) ? 14 : (REC == REC_WENO) ? 10 : 2;
    if (UNI) {
#pragma unroll
        for (int m = 0; m < NW; ++m) w[m] = uni_w<T>(d, DIR, m);
    } else {
        const T *wp = weights<T>(d, DIR) + (size_t)(c + 2) * 14;
#pragma unroll
        for (int m = 0; m < NW; ++m) w[m] = wp[m];
    }
    T *const *QL = reinterpret_cast<T *const *>(d.QL);
    T *const *QR = reinterpret_cast<T *const *>(d.QR);
    T vm_rho = T(0), vp_rho = T(0);
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
        if (v == 0) { vm_rho = vm; vp_rho = vp; }
        if (v == 4 && d.pos_fallback) {
            fallback = !(vm_rho > T(0) && vp_rho > T(0) && vm > T(0) && vp > T(0));
            if (fallback && d.fb_count) atomicAdd(d.fb_count, 1ull);
            if (fallback) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const T cv = (T)__ldg(d.P[u] + ci);
                    if (c <= ns) QL[u][ci] = cv;
                    if (c >= 1) QR[u][ci - st] = cv;
                }
            }
        }
        if (fallback) vm = vp = a2;
        if (c <= ns) QL[v][ci] = vp;       // left state of face c
        if (c >= 1) QR[v][ci - st] = vm;   // right state of face c-1
    }
}

template <class T, int DIR, int RS, int MINB>
__global__ void __launch_bounds__(128, MINB) k_riemann(const Dev d) {
    if (d.S->done) return;
    int f, j, k, l, ns;
    {
        const unsigned ex = (DIR == 0) ? d.nx + 1 : d.nx;
        const unsigned ey = (DIR == 1) ? d.ny + 1 : d.ny;
        const unsigned ez = (DIR == 2) ? d.nz + 1 : d.nz;
        const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= ex * ey * ez) return;
        int a, b, e;
        unflat3(t, ex, ey, a, b, e);
        if (DIR == 0) { f = a; j = f; k = b + 1; l = e + 1; ns = d.nx; }
        else if (DIR == 1) { f = b; k = f; j = a + 1; l = e + 1; ns = d.ny; }
        else { f = e; l = f; j = a + 1; k = b + 1; ns = d.nz; }
    }
    (void)ns;
    const int ci = cidx(d, j, k, l);
    constexpr int tb1 = (DIR == 0) ? 1 : 0;
    constexpr int tb2 = (DIR == 2) ? 1 : 2;
    using F = Frame<DIR>;
    const T *const *QL = reinterpret_cast<const T *const *>(d.QL);
    const T *const *QR = reinterpret_cast<const T *const *>(d.QR);
    T pl[9], pr[9];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        pl[1 + v] = QL[v][ci];
        pr[1 + v] = QR[v][ci];
    }
    pl[ibx + tb1] = QL[5][ci];
    pr[ibx + tb1] = QR[5][ci];
    pl[ibx + tb2] = QL[6][ci];
    pr[ibx + tb2] = QR[6][ci];
    const T bn = (T)d.P[F::ibn - 1][ci];
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
    for (int v = 0; v < 5; ++v) store_flux<T>(FO[v], ci, fo[1 + v]);
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

// The Riemann kernel with its loads taken off the critical path: CTAs of 128
// threads walk the faces of the sweep with a grid stride, and while a thread
// solves one face, asynchronous copies (cp.async, no registers held) bring
// the fourteen face states and the normal field of its next face into its
// own shared-memory slots; the solve then reads them from shared memory.
// Same faces, same arithmetic as k_riemann: the same bits.
__device__ __forceinline__ void cp_async_elem(void *smem, const void *gmem, int bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}

template <class T, int DIR, int RS, int MINB>
__global__ void __launch_bounds__(128, MINB) k_riemann_pf(const Dev d) {
    if (d.S->done) return;
    __shared__ T qb[2][14][128];
    __shared__ double bb[2][128];
    const int tid = threadIdx.x;
    const unsigned ex = (DIR == 0) ? d.nx + 1 : d.nx;
    const unsigned ey = (DIR == 1) ? d.ny + 1 : d.ny;
    const unsigned ez = (DIR == 2) ? d.nz + 1 : d.nz;
    const unsigned total = ex * ey * ez;
    const unsigned stride = gridDim.x * 128;
    using F = Frame<DIR>;
    constexpr int tb1 = (DIR == 0) ? 1 : 0;
    constexpr int tb2 = (DIR == 2) ? 1 : 2;
    const T *const *QL = reinterpret_cast<const T *const *>(d.QL);
    const T *const *QR = reinterpret_cast<const T *const *>(d.QR);
    auto face_index = [&](unsigned t) {
        int a, b, e;
        unflat3(t, ex, ey, a, b, e);
        if (DIR == 0) return cidx(d, a, b + 1, e + 1);
        if (DIR == 1) return cidx(d, a + 1, b, e + 1);
        return cidx(d, a + 1, b + 1, e);
    };
    auto issue = [&](unsigned t, int buf) {
        if (t < total) {
            const int ci = face_index(t);
#pragma unroll
            for (int v = 0; v < 7; ++v) {
                cp_async_elem(&qb[buf][v][tid], QL[v] + ci, (int)sizeof(T));
                cp_async_elem(&qb[buf][7 + v][tid], QR[v] + ci, (int)sizeof(T));
            }
            cp_async_elem(&bb[buf][tid], d.P[F::ibn - 1] + ci, 8);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    unsigned t = blockIdx.x * 128 + tid;
    issue(t, 0);
    for (int i = 0; t < total; ++i, t += stride) {
        issue(t + stride, (i + 1) & 1);
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        const int b = i & 1;
        const int ci = face_index(t);
        T pl[9], pr[9];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            pl[1 + v] = qb[b][v][tid];
            pr[1 + v] = qb[b][7 + v][tid];
        }
        pl[ibx + tb1] = qb[b][5][tid];
        pr[ibx + tb1] = qb[b][12][tid];
        pl[ibx + tb2] = qb[b][6][tid];
        pr[ibx + tb2] = qb[b][13][tid];
        const T bn = (T)bb[b][tid];
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
        for (int v = 0; v < 5; ++v) store_flux<T>(FO[v], ci, fo[1 + v]);
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
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// launch geometry of the split kernels: a flat 1D grid over the cells (or
// faces) of one sweep
static inline void split_dims(const Dev &d, int dir, bool recon, dim3 &g, dim3 &b) {
    const int extra = recon ? 2 : 1;  // cells 0..n+1 or faces 0..n along the sweep
    long long nx = d.nx, ny = d.ny, nz = d.nz;
    if (dir == 0) nx += extra;
    if (dir == 1) ny += extra;
    if (dir == 2) nz += extra;
    const int tpb = recon ? d.tpb_recon : d.tpb_riemann;
    const long long total = nx * ny * nz;
    b = dim3(tpb, 1, 1);
    g = dim3((unsigned)((total + tpb - 1) / tpb), 1, 1);
}

}  // namespace cumc
#include "recon_tile.cuh"
namespace cumc {

template <class T, int DIR, int UNI, int CPT, int MINB = 1>
static void launch_recon_tile_c(const Dev &d, int rec, cudaStream_t s) {
    const dim3 g = recon_tile_grid(d, DIR, CPT), b(32, 8, 1);
    switch (rec) {
        case REC_TVD_MM: k_recon_tile<T, DIR, REC_TVD_MM, UNI, CPT, 0, MINB><<<g, b, 0, s>>>(d); break;
        case REC_TVD_VL: k_recon_tile<T, DIR, REC_TVD_VL, UNI, CPT, 0, MINB><<<g, b, 0, s>>>(d); break;
        case REC_TVD_MC: k_recon_tile<T, DIR, REC_TVD_MC, UNI, CPT, 0, MINB><<<g, b, 0, s>>>(d); break;
        case REC_PPM: k_recon_tile<T, DIR, REC_PPM, UNI, CPT, 0, MINB><<<g, b, 0, s>>>(d); break;
        default: k_recon_tile<T, DIR, REC_WENO, UNI, CPT, 0, MINB><<<g, b, 0, s>>>(d); break;
    }
}
// recon_tile: 1, 2 staged tiles with 1 or 2 cells per thread; 4 one cell per
// thread at 64 registers (4 blocks per SM); 3 (TMA-staged) falls back to 1
// where no tensor maps are given
template <class T, int DIR, int UNI>
static void launch_recon_tile(const Dev &d, int rec, cudaStream_t s) {
    if (d.recon_tile == 2) launch_recon_tile_c<T, DIR, UNI, 2>(d, rec, s);
    else if (d.recon_tile == 4) launch_recon_tile_c<T, DIR, UNI, 1, 4>(d, rec, s);
    else launch_recon_tile_c<T, DIR, UNI, 1>(d, rec, s);
}

template <class T, int DIR, int UNI>
static void launch_recon_u(const Dev &d, int rec, dim3 g, dim3 b, cudaStream_t s) {
    if (d.recon_tile) {
        launch_recon_tile<T, DIR, UNI>(d, rec, s);
        return;
    }
    switch (rec) {
        case REC_TVD_MM: k_recon<T, DIR, REC_TVD_MM, UNI><<<g, b, 0, s>>>(d); break;
        case REC_TVD_VL: k_recon<T, DIR, REC_TVD_VL, UNI><<<g, b, 0, s>>>(d); break;
        case REC_TVD_MC: k_recon<T, DIR, REC_TVD_MC, UNI><<<g, b, 0, s>>>(d); break;
        case REC_PPM: k_recon<T, DIR, REC_PPM, UNI><<<g, b, 0, s>>>(d); break;
        default: k_recon<T, DIR, REC_WENO, UNI><<<g, b, 0, s>>>(d); break;
    }
}
// riemann_minb 14, 15, 16: the prefetching kernel at 4, 5, 6 blocks per SM
template <class T, int DIR, int MINB>
static void launch_riemann_pf(const Dev &d, int rs, cudaStream_t s) {
    const long long total = (long long)((DIR == 0) ? d.nx + 1 : d.nx) * ((DIR == 1) ? d.ny + 1 : d.ny) *
                            ((DIR == 2) ? d.nz + 1 : d.nz);
    long long nblk = (long long)d.num_sms * MINB * 2;
    const long long need = (total + 127) / 128;
    if (nblk > need) nblk = need;
    const dim3 g((unsigned)nblk), b(128);
    switch (rs) {
        case RS_LF: k_riemann_pf<T, DIR, RS_LF, MINB><<<g, b, 0, s>>>(d); break;
        case RS_HLL: k_riemann_pf<T, DIR, RS_HLL, MINB><<<g, b, 0, s>>>(d); break;
        case RS_HLLC: k_riemann_pf<T, DIR, RS_HLLC, MINB><<<g, b, 0, s>>>(d); break;
        default: k_riemann_pf<T, DIR, RS_HLLD, MINB><<<g, b, 0, s>>>(d); break;
    }
}
template <class T, int DIR, int MINB>
static void launch_riemann_m(const Dev &d, int rs, dim3 g, dim3 b, cudaStream_t s) {
    switch (rs) {
        case RS_LF: k_riemann<T, DIR, RS_LF, MINB><<<g, b, 0, s>>>(d); break;
        case RS_HLL: k_riemann<T, DIR, RS_HLL, MINB><<<g, b, 0, s>>>(d); break;
        case RS_HLLC: k_riemann<T, DIR, RS_HLLC, MINB><<<g, b, 0, s>>>(d); break;
        default: k_riemann<T, DIR, RS_HLLD, MINB><<<g, b, 0, s>>>(d); break;
    }
}
// the TMA-staged reconstruction: persistent CTAs, as many as fit on the GPU
template <int DIR, int REC, int UNI>
static void launch_recon_tma_r(const Dev &d, const TmaMaps &tm, cudaStream_t s) {
    static int per_sm = 0;  // resident CTAs per SM of this instantiation
    if (per_sm == 0) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_recon_tma<DIR, REC, UNI>, 256, TmaBox<DIR>::SMEM) !=
                cudaSuccess || n < 1)
            n = 1;
        per_sm = n;
    }
    const dim3 tg = recon_tile_grid(d, DIR, 1);
    const long long ntiles = (long long)tg.x * tg.y * tg.z;
    long long nblk = (long long)d.num_sms * per_sm;
    if (nblk > ntiles) nblk = ntiles;
    k_recon_tma<DIR, REC, UNI><<<(unsigned)nblk, dim3(32, 8, 1), TmaBox<DIR>::SMEM, s>>>(d, tm);
}
template <int DIR, int UNI>
static void launch_recon_tma(const Dev &d, int rec, const TmaMaps &tm, cudaStream_t s) {
    switch (rec) {
        case REC_TVD_MM: launch_recon_tma_r<DIR, REC_TVD_MM, UNI>(d, tm, s); break;
        case REC_TVD_VL: launch_recon_tma_r<DIR, REC_TVD_VL, UNI>(d, tm, s); break;
        case REC_TVD_MC: launch_recon_tma_r<DIR, REC_TVD_MC, UNI>(d, tm, s); break;
        case REC_PPM: launch_recon_tma_r<DIR, REC_PPM, UNI>(d, tm, s); break;
        default: launch_recon_tma_r<DIR, REC_WENO, UNI>(d, tm, s); break;
    }
}

template <class T, int DIR>
static void launch_split_dir(const Dev &d, int rec, int rs, cudaStream_t s, const TmaMaps *tma = nullptr) {
    dim3 g, b;
    split_dims(d, DIR, true, g, b);
    if constexpr (sizeof(T) == sizeof(double)) {
        if (d.recon_tile == 3 && tma) {
            if (d.wuni[DIR]) launch_recon_tma<DIR, 1>(d, rec, *tma, s);
            else launch_recon_tma<DIR, 0>(d, rec, *tma, s);
        } else if (d.wuni[DIR]) launch_recon_u<T, DIR, 1>(d, rec, g, b, s);
        else launch_recon_u<T, DIR, 0>(d, rec, g, b, s);
    } else {
        if (d.wuni[DIR]) launch_recon_u<T, DIR, 1>(d, rec, g, b, s);
        else launch_recon_u<T, DIR, 0>(d, rec, g, b, s);
    }
    split_dims(d, DIR, false, g, b);
    switch (d.riemann_minb) {
        case 4: launch_riemann_m<T, DIR, 4>(d, rs, g, b, s); break;
        case 5: launch_riemann_m<T, DIR, 5>(d, rs, g, b, s); break;
        case 6: launch_riemann_m<T, DIR, 6>(d, rs, g, b, s); break;
        case 14: launch_riemann_pf<T, DIR, 4>(d, rs, s); break;
        case 15: launch_riemann_pf<T, DIR, 5>(d, rs, s); break;
        case 16: launch_riemann_pf<T, DIR, 6>(d, rs, s); break;
        default: launch_riemann_m<T, DIR, 1>(d, rs, g, b, s); break;
    }
}
template <class T>
static void launch_split_t(const Dev &d, int dir, int rec, int rs, cudaStream_t s, const TmaMaps *tma = nullptr) {
    if (dir == 0) launch_split_dir<T, 0>(d, rec, rs, s, tma ? tma + 0 : nullptr);
    else if (dir == 1) launch_split_dir<T, 1>(d, rec, rs, s, tma ? tma + 1 : nullptr);
    else launch_split_dir<T, 2>(d, rec, rs, s, tma ? tma + 2 : nullptr);
}

template <class T, int DIR, int REC, int RS>
static void flux_smem(size_t sm) {
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_flux<T, DIR, REC, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
}
template <class T, int DIR, int REC>
static void launch_rs(const Dev &d, int rs, dim3 g, dim3 b, size_t sm, cudaStream_t s) {
    switch (rs) {
        case RS_LF: flux_smem<T, DIR, REC, RS_LF>(sm); break;
        case RS_HLL: flux_smem<T, DIR, REC, RS_HLL>(sm); break;
        case RS_HLLC: flux_smem<T, DIR, REC, RS_HLLC>(sm); break;
        default: flux_smem<T, DIR, REC, RS_HLLD>(sm); break;
    }
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
