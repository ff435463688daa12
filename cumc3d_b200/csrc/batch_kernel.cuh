// batch_kernel.cuh -- many independent 1D MHD problems of uneven size in one
// persistent launch.
//
// Each CTA takes problems from a global work counter (largest first) and runs
// INITIAL_UPDATE + the whole time loop (FINDDT, clamp, 3 RK stages) of one
// problem before taking the next, so a problem's per-step dt, its own t_end
// and its own step count never synchronise with any other problem.  Phases of
// a stage are separated by __syncthreads only.
//
// The reference's 1D configuration (n_dim = 1, ny = nz = 1, outflow on every
// side) keeps its arrays 7 x 7 wide in y and z; every y/z row is a copy of
// row (k,l) = (1,1) except the lower normal faces of y and z, which hold their
// initial values (boundary.f90 never fills them) and are RK-updated inside a
// stage.  This kernel carries exactly that reduced state per x-cell j:
//   hydro prims, eps, c_s, cell B (3), face Bx(j), the y face at k = 1 and
//   k = 0, the z face at l = 1 and l = 0, and their conserved copies,
// and evaluates every expression in the order the 3D path (and the Fortran)
// does, so results are bit-identical to the 3D engine on the same problem.
#pragma once
#include "../../include/cumc3d_gpu.h"
#include "engine.cuh"
#include "flux_kernel.cuh"
#include "mhd_device.cuh"

#include <cooperative_groups.h>

namespace cumc {
namespace cg = cooperative_groups;

struct BatchProblem {
    long long off;  // start of this problem's padded row in the packed arrays
    int n;          // interior zones
    int steps;      // output: steps taken
    double t_end;
    double t;       // output: time reached
    int status;     // output: 0 ok, CUMC_ESTATE
    int pad;
};

// packed arrays, all of length sum(n_i + 6); index off + (j + 2), j = -2..n+3
struct BatchDev {
    int nprob;
    int max_steps;
    double gamma, cfl;
    int floor_kind;
    int pos_fallback;
    int coop_min_n;        // problems of at most this many cells run on one CTA
    int *next;             // work counter
    const int *order;      // problem ids, largest first
    BatchProblem *prob;
    const double *dx, *w;  // per-cell dx, reconstruction weights (14 per cell)
    const float *wf;
    double *P[5];          // rho, vx, vy, vz, p
    double *EPS, *CS, *BC[3];
    double *BX, *BY1, *BZ1, *BY0, *BZ0;          // prim face fields
    double *U[5], *UBX, *UBY1, *UBZ1, *UBY0, *UBZ0;  // cons
    double *UBXb;          // second buffer of the cons x faces (stages alternate)
    double *O[5], *OBX, *OBY1, *OBZ1, *OBY0, *OBZ0;  // u_old
    void *QL[7], *QR[7];   // face states (T)
    double *F[5];          // x-face fluxes (hydro)
    double *EY, *EZ;       // edge EMFs per x-face
};

__device__ __forceinline__ double bmin_block(double v, double *red) {
    unsigned long long bits = (unsigned long long)__double_as_longlong(v);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
        bits = o < bits ? o : bits;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = __longlong_as_double((long long)bits);
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        unsigned long long b = lane < nw ? (unsigned long long)__double_as_longlong(red[lane]) : ~0ull;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            unsigned long long o = __shfl_xor_sync(0xffffffffu, b, off);
            b = o < b ? o : b;
        }
        if (lane == 0) red[0] = __longlong_as_double((long long)b);
    }
    __syncthreads();
    const double r = red[0];
    __syncthreads();
    return r;
}

// floors of model/riemann/src/custom.f90:103-127 (eps >= 0)
__device__ __forceinline__ void batch_floor(const BatchDev &b, double &e) {
    if (b.floor_kind == 1) e = dmax(e, 0.0);
}

constexpr int BATCH_THREADS = 256;
constexpr int BATCH_CLUSTER = 8;          // CTAs that share one large problem
constexpr int BATCH_COOP_MIN_N = 1024;    // default: problems of at most this many cells run on one CTA
constexpr int BATCH_COOP_MIN_N_FEW = 256; // the same when every problem can have a cluster of its own

struct BatchShared {
    unsigned long long part_dt;  // this CTA's FINDDT minimum (bit pattern)
    int part_bad;                // this CTA saw a bad state
    int pick;                    // problem index taken from the work counter
    int bad;                     // set by any thread of this CTA
    double red[32];
};

// one barrier of the group that runs a problem: the whole cluster, or one CTA
__device__ __forceinline__ void gsync(bool coop) {
    if (coop) cg::this_cluster().sync();
    else __syncthreads();
}

// INITIAL_UPDATE + the time loop of one problem.  The cells 0..n+1 are split
// in contiguous chunks over the `size` CTAs of the group (size 1: one CTA).
// Ghost cells (outflow: copies of cells 1 and n) are read through a clamped
// index instead of being refilled after every stage; they hold exactly the
// values the refill would store, so the arithmetic is unchanged.
template <class T, int REC, int RS>
__device__ __forceinline__ void batch_problem(const BatchDev &b, BatchShared &sh, int pid, bool coop, int rank, int size) {
    const double rk20 = 3.0 / 4.0, rk21 = 1.0 / 4.0, rk22 = 1.0 / 4.0;
    const double rk30 = 1.0 / 3.0, rk31 = 2.0 / 3.0, rk32 = 2.0 / 3.0;
    const double g1 = b.gamma - 1.0;
    T *const *QL = reinterpret_cast<T *const *>(b.QL);
    T *const *QR = reinterpret_cast<T *const *>(b.QR);
    const T *wts = (sizeof(T) == 8) ? reinterpret_cast<const T *>(b.w) : reinterpret_cast<const T *>(b.wf);
    const long long off = b.prob[pid].off + 2;  // X[off + j] is cell j
    const int n = b.prob[pid].n;
    const double t_end = b.prob[pid].t_end;
    // this CTA's share of the cell indices 0..n+1
    const int chunk = (n + 2 + size - 1) / size;
    const int lo = rank * chunk, hi = min(lo + chunk, n + 2);
    auto cl = [&](int j) { return off + (j < 1 ? 1 : (j > n ? n : j)); };
    if (threadIdx.x == 0) sh.bad = 0;
    __syncthreads();

    // FROMRVETOU + FINDPRESSURE of cell j; bxm = the recovered face j-1
    // (the values as stored: face fields bxf = BX[c], by1/by0, bz1/bz0 and the
    // primitives of cell c, passed in so that a caller that has just stored
    // them does not read them back)
    auto fromrvetou_v = [&](long long c, double bxf, double bxm, double by1, double by0, double bz1, double bz0,
                            double rho, double vx, double vy, double vz, double e) {
        const double bx = 0.5 * (bxf + bxm);
        const double by = 0.5 * (by1 + by0);
        const double bz = 0.5 * (bz1 + bz0);
        const double vsquare = vx * vx + vy * vy + vz * vz;
        const double bsquare = bx * bx + by * by + bz * bz;
        b.U[0][c] = rho;
        b.U[1][c] = vx * rho;
        b.U[2][c] = vy * rho;
        b.U[3][c] = vz * rho;
        b.U[4][c] = rho * (e + 0.5 * vsquare) + 0.5 * bsquare;
        b.BC[0][c] = bx;
        b.BC[1][c] = by;
        b.BC[2][c] = bz;
        const double p = rho * e * g1;
        b.P[4][c] = p;
        b.CS[c] = sqrt(e * g1 + rho * g1 * p / (rho * rho));
        if (!(rho > 0.0) || !isfinite(e) || !isfinite(p) || !isfinite(vx) || !isfinite(vy) || !isfinite(vz))
            sh.bad = 1;
    };
    auto fromrvetou = [&](int j, double bxm) {
        const long long c = off + j;
        fromrvetou_v(c, b.BX[c], bxm, b.BY1[c], b.BY0[c], b.BZ1[c], b.BZ0[c], b.P[0][c], b.P[1][c], b.P[2][c],
                     b.P[3][c], b.EPS[c]);
    };

    // -------- INITIAL_UPDATE (initial.f90:86-116) --------
    for (int j = max(lo, 1) + threadIdx.x; j < min(hi, n + 1); j += blockDim.x) {
        const long long c = off + j;
        double e = b.EPS[c];
        batch_floor(b, e);
        b.EPS[c] = e;
        fromrvetou(j, b.BX[c - 1]);
        b.UBX[c] = b.BX[c];
        b.UBY1[c] = b.BY1[c];
        b.UBZ1[c] = b.BZ1[c];
        b.UBY0[c] = b.BY0[c];  // the cons copy of the frozen lower faces
        b.UBZ0[c] = b.BZ0[c];
    }
    if (rank == 0 && threadIdx.x == 0) {
        b.UBX[off] = b.BX[off];
        b.UBY1[off] = b.BY1[off];
        b.UBZ1[off] = b.BZ1[off];
    }
    gsync(coop);

    double t = 0.0;
    int steps = 0;
    int ubp = 0;  // which buffer holds the cons x faces (INITIAL_UPDATE fills UBX)
    bool bad = false;
    while (true) {
        // -------- FINDDT (rungekutta.f90:221-332), 1D Cartesian --------
        double dtl = 1.0e5;
        for (int j = max(lo, 1) + threadIdx.x; j < min(hi, n + 1); j += blockDim.x) {
            const long long c = off + j;
            const double rho = b.P[0][c];
            const double a2 = b.CS[c] * b.CS[c];
            const double a4 = a2 * a2;
            const double bx = b.BC[0][c], by = b.BC[1][c], bz = b.BC[2][c];
            const double b2x = dv(bx * bx, rho), b2y = dv(by * by, rho), b2z = dv(bz * bz, rho);
            const double b2 = b2x + b2y + b2z;
            const double b4 = b2 * b2;
            const double cfx = sqrt(0.5 * (a2 + b2 + sqrt((a4 + 2.0 * a2 * b2 + b4) - 4.0 * a2 * b2x)));
            const double cfy = sqrt(0.5 * (a2 + b2 + sqrt((a4 + 2.0 * a2 * b2 + b4) - 4.0 * a2 * b2y)));
            const double cfz = sqrt(0.5 * (a2 + b2 + sqrt((a4 + 2.0 * a2 * b2 + b4) - 4.0 * a2 * b2z)));
            const double lambda = dmax3(fabs(b.P[1][c]) + cfx, fabs(b.P[2][c]) + cfy, fabs(b.P[3][c]) + cfz);
            double tt = b.dx[c];
            tt = tt * b.cfl / lambda;
            if (tt < dtl) dtl = tt;
        }
        double dt = bmin_block(dtl, sh.red);
        bad = sh.bad != 0;
        if (coop) {
            if (threadIdx.x == 0) {
                sh.part_dt = (unsigned long long)__double_as_longlong(dt);
                sh.part_bad = bad ? 1 : 0;
            }
            cg::cluster_group cluster = cg::this_cluster();
            cluster.sync();
            unsigned long long m = ~0ull;
            int anybad = 0;
            for (int r = 0; r < size; ++r) {
                const BatchShared *o = cluster.map_shared_rank(&sh, r);
                m = o->part_dt < m ? o->part_dt : m;
                anybad |= o->part_bad;
            }
            cluster.sync();
            dt = __longlong_as_double((long long)m);
            bad = anybad != 0;
        }
        if (bad || !(t < t_end) || steps >= b.max_steps) break;
        if (!(dt < 1.0e5)) dt = 1.0e5;
        if (t + dt > t_end) dt = t_end - t;

        for (int stage = 1; stage <= 3; ++stage) {
            // ---- A: reconstruction of cells 0..n+1 ----
            for (int c0 = lo + threadIdx.x; c0 < hi; c0 += blockDim.x) {
                const long long c = off + c0;
                const T *wp = wts + (size_t)c * 14;
                T w[14];
                constexpr int NW = (REC == REC_PPM) ? 14 : (REC == REC_WENO) ? 10 : 2;
#pragma unroll
                for (int m = 0; m < NW; ++m) w[m] = wp[m];
                const long long i0 = cl(c0 - 2), i1 = cl(c0 - 1), i2 = cl(c0), i3 = cl(c0 + 1), i4 = cl(c0 + 2);
                // every stencil value first: the face-state stores below may
                // alias the primitive arrays as far as the compiler knows, so
                // loads left between them would each wait a round trip
                T sv[7][5];
#pragma unroll
                for (int v = 0; v < 7; ++v) {
                    const double *src = (v < 5) ? b.P[v] : b.BC[v == 5 ? 1 : 2];
                    sv[v][0] = sv[v][4] = T(0);
                    if (REC == REC_PPM || REC == REC_WENO) { sv[v][0] = (T)src[i0]; sv[v][4] = (T)src[i4]; }
                    sv[v][1] = (T)src[i1];
                    sv[v][2] = (T)src[i2];
                    sv[v][3] = (T)src[i3];
                }
                bool fallback = false;
                T vm_rho = T(0), vp_rho = T(0);
#pragma unroll
                for (int v = 0; v < 7; ++v) {
                    const T a0 = sv[v][0], a1 = sv[v][1], a2 = sv[v][2], a3 = sv[v][3], a4 = sv[v][4];
                    T vm, vp;
                    recon_cell<T, REC>(w, a0, a1, a2, a3, a4, vm, vp);
                    if (v == 0) { vm_rho = vm; vp_rho = vp; }
                    if (v == 4 && b.pos_fallback) {
                        fallback = !(vm_rho > T(0) && vp_rho > T(0) && vm > T(0) && vp > T(0));
                        if (fallback) {
                            for (int u = 0; u < 4; ++u) {
                                const T cv = sv[u][2];  // (T)P[u][i2]
                                if (c0 <= n) QL[u][c] = cv;
                                if (c0 >= 1) QR[u][c - 1] = cv;
                            }
                        }
                    }
                    if (fallback) vm = vp = a2;
                    if (c0 <= n) QL[v][c] = vp;
                    if (c0 >= 1) QR[v][c - 1] = vm;
                }
            }
            gsync(coop);
            // ---- B: Riemann solve on faces 0..n, then the edge EMFs there ----
            for (int f = lo + threadIdx.x; f < min(hi, n + 1); f += blockDim.x) {
                const long long c = off + f;
                T pl[9], pr[9];
#pragma unroll
                for (int v = 0; v < 5; ++v) { pl[1 + v] = QL[v][c]; pr[1 + v] = QR[v][c]; }
                pl[iby] = QL[5][c]; pr[iby] = QR[5][c];
                pl[ibz] = QL[6][c]; pr[ibz] = QR[6][c];
                const T bn = (T)b.BX[c];
                pl[ibx] = bn;
                pr[ibx] = bn;
                const T g = (T)b.gamma;
                const T epsL = eos_eps(pl[irho], pl[itau], g), epsR = eos_eps(pr[irho], pr[itau], g);
                const T csL = eos_cs(pl[itau], pl[irho], epsL, g), csR = eos_cs(pr[itau], pr[irho], epsR, g);
                T fo[9];
                riemann_face<T, 0, RS>(pl, pr, epsL, epsR, csL, csR, fo);
#pragma unroll
                for (int v = 0; v < 5; ++v) b.F[v][c] = (double)fo[1 + v];
                // edge EMFs (mhd_module.f90:310-432 in 1D): face EMFs from the
                // flux, cell EMFs of the cells either side
                const double fyx = (double)fo[ibz];   // eface(iyx) = flux(ibz)
                const double fzx = -(double)fo[iby];  // eface(izx) = -flux(iby)
                const long long ca = cl(f), cb = cl(f + 1);
                const double ey_a = b.P[1][ca] * b.BC[2][ca] - b.P[3][ca] * b.BC[0][ca];
                const double ez_a = b.P[2][ca] * b.BC[0][ca] - b.P[1][ca] * b.BC[1][ca];
                const double ey_b = b.P[1][cb] * b.BC[2][cb] - b.P[3][cb] * b.BC[0][cb];
                const double ez_b = b.P[2][cb] * b.BC[0][cb] - b.P[1][cb] * b.BC[1][cb];
                b.EY[c] = 0.50 * (fyx + fyx + ey_a + ey_b) - 0.25 * (ey_a + ey_a + ey_b + ey_b);
                b.EZ[c] = 0.50 * (fzx + fzx + ez_a + ez_b) - 0.25 * (ez_a + ez_a + ez_b + ez_b);
            }
            gsync(coop);
            // ---- C + D: du/dt + Shu-Osher combination (j = 0..n), then on the
            // new values FROMUTORVE + floor, FROMRVETOU + FINDPRESSURE and the
            // index-0 layer of cons (j = 1..n), one phase.  The only operand a
            // cell takes from its neighbour is the updated x face below it; the
            // thread recomputes it (the same expression on the same values the
            // neighbour uses), reading the previous stage's faces from one
            // buffer while the new ones go to the other, so no barrier is needed
            // between the update and the recovery. ----
            double *const UBXo = ubp ? b.UBXb : b.UBX;  // this stage's input x faces
            double *const UBXn = ubp ? b.UBX : b.UBXb;  // its output
            for (int j = lo + threadIdx.x; j < min(hi, n + 1); j += blockDim.x) {
                const long long c = off + j;
                const double dxj = b.dx[c];
                double lr[5];
                if (j >= 1) {
#pragma unroll
                    for (int i = 0; i < 5; ++i) {
                        const double dflux = dv(b.F[i][c] - b.F[i][c - 1], dxj);
                        lr[i] = -dflux;
                        lr[i] = lr[i] + 0.0;  // + sc (no sources)
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 5; ++i) lr[i] = 0.0;
                }
                // spatial.f90:647-653; the y/z differences of the copied rows are
                // exactly zero, so their grid spacing does not enter
                const double zero = 0.0;
                const double lbx = -((zero) / 1.0 - (zero) / 1.0);
                const double ezd = (j >= 1) ? (b.EZ[c] - b.EZ[c - 1]) : 0.0;
                const double eyd = (j >= 1) ? (b.EY[c] - b.EY[c - 1]) : 0.0;
                const double lby = -((zero) / 1.0 - dv(ezd, dxj));
                const double lbz = -(dv(eyd, dxj) - (zero) / 1.0);
                // written with round-to-nearest intrinsics so that no build
                // (the FP32 form compiles with contraction) fuses it: the
                // recomputed face below must equal the one its owner stores
                auto combo = [&](double u, double o, double lrv) {
                    if (stage == 1) return __dadd_rn(u, __dmul_rn(dt, lrv));
                    if (stage == 2)
                        return __dadd_rn(__dadd_rn(__dmul_rn(rk20, o), __dmul_rn(rk21, u)), __dmul_rn(__dmul_rn(rk22, dt), lrv));
                    return __dadd_rn(__dadd_rn(__dmul_rn(rk30, o), __dmul_rn(rk31, u)), __dmul_rn(__dmul_rn(rk32, dt), lrv));
                };
                // every load first (a load after a store would wait its own
                // round trip: the compiler cannot tell that the arrays do not
                // alias), then the update and the recovery on the loaded values
                double *const Ua[10] = {b.U[0], b.U[1], b.U[2], b.U[3], b.U[4], UBXo, b.UBY1, b.UBZ1, b.UBY0, b.UBZ0};
                double *const Oa[10] = {b.O[0], b.O[1], b.O[2], b.O[3], b.O[4], b.OBX, b.OBY1, b.OBZ1, b.OBY0, b.OBZ0};
                const double lv[10] = {lr[0], lr[1], lr[2], lr[3], lr[4], lbx, lby, lbz, lby, lbz};
                const int nv = (j >= 1) ? 10 : 6;
                double uu[10], oo[10], un[10];
#pragma unroll
                for (int i = 0; i < 10; ++i) {
                    uu[i] = 0.0;
                    oo[i] = 0.0;
                    if (i < nv) {
                        uu[i] = Ua[i][c];
                        if (stage != 1) oo[i] = Oa[i][c];
                    }
                }
                double um = 0.0, om = 0.0, by0 = 0.0, bz0 = 0.0, by1_old = 0.0, bz1_old = 0.0, bx0 = 0.0;
                if (j >= 1) {
                    um = UBXo[c - 1];  // the face below, as the stage found it
                    if (stage != 1) om = b.OBX[c - 1];
                    by0 = b.BY0[c];
                    bz0 = b.BZ0[c];
                    if (j == 1) { by1_old = b.BY1[c]; bz1_old = b.BZ1[c]; bx0 = b.BX[off]; }
                }
#pragma unroll
                for (int i = 0; i < 10; ++i) {
                    un[i] = 0.0;
                    if (i >= nv) continue;
                    if (stage == 1) Oa[i][c] = uu[i];
                    un[i] = combo(uu[i], oo[i], lv[i]);
                }
                if (j == 0) {
                    // cell 0: the update only (its x face's final value is the
                    // prim face 0, written by the thread of cell 1)
#pragma unroll
                    for (int i = 0; i < 5; ++i) b.U[i][c] = un[i];
                    continue;
                }
                UBXn[c] = un[5];
                b.UBY1[c] = un[6];
                b.UBZ1[c] = un[7];
                // the recovery of cell j from its updated values (U, the y/z
                // faces) and the updated x face below (recomputed)
                const double ubxm = combo(um, om, lbx);
                const double ubx = un[5], uby1 = un[6], ubz1 = un[7], uby0 = un[8], ubz0 = un[9];
                const double u0 = un[0], u1 = un[1], u2 = un[2], u3 = un[3], u4 = un[4];
                const double bxu = 0.5 * (ubx + ubxm);
                const double byu = 0.5 * (uby1 + uby0);
                const double bzu = 0.5 * (ubz1 + ubz0);
                const double vx = dv(u1, u0), vy = dv(u2, u0), vz = dv(u3, u0);
                const double bsquare = bxu * bxu + byu * byu + bzu * bzu;
                const double vsquare = vx * vx + vy * vy + vz * vz;
                double e = (u4 - 0.5 * bsquare) / u0 - 0.5 * vsquare;
                batch_floor(b, e);
                if (stage == 3) batch_floor(b, e);
                b.P[0][c] = u0;
                b.P[1][c] = vx;
                b.P[2][c] = vy;
                b.P[3][c] = vz;
                b.EPS[c] = e;
                b.BX[c] = ubx;
                b.BY1[c] = uby1;
                b.BZ1[c] = ubz1;
                // face j-1 after recovery: the recovered cons face, or the
                // never-recovered face 0; FROMRVETOU also rewrites U of the cell
                fromrvetou_v(c, ubx, j == 1 ? bx0 : ubxm, uby1, by0, ubz1, bz0, u0, vx, vy, vz, e);
                b.UBY0[c] = by0;
                b.UBZ0[c] = bz0;
                if (j == 1) {
                    // cons layer 0 takes the prim faces of j = 0 as they stood
                    // before this recovery (the j = 0 ghosts of By, Bz copy cell 1)
                    UBXn[off] = bx0;
                    b.UBY1[off] = by1_old;
                    b.UBZ1[off] = bz1_old;
                }
            }
            ubp ^= 1;
            gsync(coop);
        }
        t = t + dt;
        steps += 1;
    }
    // BOUNDARY once at the end (outflow x; boundary.f90:439-505), so the
    // state read back carries its ghosts
    if (rank == 0 && threadIdx.x < 6) {
        const int g = threadIdx.x % 3 + 1;
        const bool inner = threadIdx.x < 3;
        const long long dst = off + (inner ? 1 - g : n + g), src = off + (inner ? 1 : n);
#pragma unroll
        for (int v = 0; v < 5; ++v) b.P[v][dst] = b.P[v][src];
#pragma unroll
        for (int v = 0; v < 3; ++v) b.BC[v][dst] = b.BC[v][src];
        b.EPS[dst] = b.EPS[src];
        b.CS[dst] = b.CS[src];
        b.BY1[dst] = b.BY1[src];
        b.BZ1[dst] = b.BZ1[src];
    }
    if (rank == 0 && threadIdx.x == 0) {
        b.prob[pid].t = t;
        b.prob[pid].steps = steps;
        b.prob[pid].status = bad ? CUMC_ESTATE : 0;
    }
    gsync(coop);
}

// Persistent kernel.  Launched in clusters of `size` CTAs: while the next
// problem (largest first) has more than b.coop_min_n cells, the whole
// cluster runs it; from the first smaller one on, every CTA takes problems on
// its own.
template <class T, int REC, int RS>
__global__ void __launch_bounds__(BATCH_THREADS, 2) k_batch(const BatchDev b) {
    __shared__ BatchShared sh;
    cg::cluster_group cluster = cg::this_cluster();
    const int size = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    bool coop = size > 1;
    while (true) {
        int pi;
        if (coop) {
            if (rank == 0 && threadIdx.x == 0) sh.pick = atomicAdd(b.next, 1);
            cluster.sync();
            pi = cluster.map_shared_rank(&sh, 0)->pick;
            cluster.sync();
            if (pi >= b.nprob) return;
            if (b.prob[b.order[pi]].n <= b.coop_min_n) {
                coop = false;  // from here on every CTA takes its own problems
                if (rank != 0) continue;
            }
        } else {
            if (threadIdx.x == 0) sh.pick = atomicAdd(b.next, 1);
            __syncthreads();
            pi = sh.pick;
            __syncthreads();
            if (pi >= b.nprob) return;
        }
        batch_problem<T, REC, RS>(b, sh, b.order[pi], coop, coop ? rank : 0, coop ? size : 1);
    }
}

template <class T, int REC, int RS>
static cudaError_t launch_batch_one(const BatchDev &b, int clusters, int cluster_size, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(clusters * cluster_size);
    cfg.blockDim = dim3(BATCH_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cluster_size > 8) {
        cudaError_t e = cudaFuncSetAttribute(k_batch<T, REC, RS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    if (clusters <= 0) {
        // size the persistent grid: as many clusters as can be resident
        int nc = 0;
        cfg.gridDim = dim3(cluster_size * 64);
        cudaError_t e = cudaOccupancyMaxActiveClusters(&nc, k_batch<T, REC, RS>, &cfg);
        if (e != cudaSuccess) return e;
        if (nc < 1) return cudaErrorInvalidConfiguration;
        cfg.gridDim = dim3(nc * cluster_size);
    }
    return cudaLaunchKernelEx(&cfg, k_batch<T, REC, RS>, b);
}

template <class T>
static cudaError_t launch_batch_t(const BatchDev &b, int rec, int rs, int clusters, int cluster_size, cudaStream_t s) {
#define CUMC_BATCH_RS(R)                                                                      \
    switch (rs) {                                                                             \
        case RS_LF: return launch_batch_one<T, R, RS_LF>(b, clusters, cluster_size, s);       \
        case RS_HLL: return launch_batch_one<T, R, RS_HLL>(b, clusters, cluster_size, s);     \
        case RS_HLLC: return launch_batch_one<T, R, RS_HLLC>(b, clusters, cluster_size, s);   \
        default: return launch_batch_one<T, R, RS_HLLD>(b, clusters, cluster_size, s);        \
    }
    switch (rec) {
        case REC_TVD_MM: CUMC_BATCH_RS(REC_TVD_MM);
        case REC_TVD_VL: CUMC_BATCH_RS(REC_TVD_VL);
        case REC_TVD_MC: CUMC_BATCH_RS(REC_TVD_MC);
        case REC_PPM: CUMC_BATCH_RS(REC_PPM);
        default: CUMC_BATCH_RS(REC_WENO);
    }
#undef CUMC_BATCH_RS
}

// clusters <= 0: as many clusters of cluster_size CTAs as fit on the device
cudaError_t launch_batch_fp64(const BatchDev &b, int rec, int rs, int clusters, int cluster_size, cudaStream_t s);
cudaError_t launch_batch_fp32(const BatchDev &b, int rec, int rs, int clusters, int cluster_size, cudaStream_t s);

}  // namespace cumc
