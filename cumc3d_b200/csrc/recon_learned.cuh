// recon_learned.cuh -- FP32 WENO reconstruction with the learned smooth-face
// flag (see learned.cuh).  Same cells, same enumeration and the same outputs
// (QL/QR face states) as k_recon<float, DIR, REC_WENO, UNI>.
//
// Stage 1 of every flag_interval-th RK step, k_recon_learned (a tile = 128
// consecutive cells of the flat enumeration; persistent CTAs walk the tiles):
//   1. each thread loads its cell's 7 stencils and builds the 35 features;
//   2. the MLP (tcgen05, BF16 operands, FP32 accumulators in TMEM) gives one
//      logit per cell; the flag (logit > threshold) is stored per cell;
//   3. a warp whose 32 cells are all flagged, in a tile not marked to fall
//      back, reconstructs with the linear optimal weights; every other warp
//      runs WENO-Z exactly as k_recon does;
//   4. every audit_interval steps all warps run WENO-Z (results identical to
//      the plain FP32 form), flagged cells also evaluate the linear values,
//      and the tile is marked to fall back until the next audit if any
//      flagged cell's relative face-value error exceeds audit_tol.
// All other stages, k_recon_tile<float, DIR, REC_WENO, UNI, CPT, 1>: the
// staged reconstruction, where the stored flags of the cell and of its
// neighbours within two cells along the sweep choose linear or WENO-Z per
// warp, without running the network.
//
// Cells next to the domain boundary along the sweep (c <= 1 or c >= n) always
// use WENO-Z: on a periodic axis face 0 and face n are one face, and their
// fluxes (hence the edge EMFs of constrained transport) must come out bit for
// bit equal from the identical stencils of cells 0/n and 1/n+1.
#pragma once
#include "flux_kernel.cuh"
#include "learned.cuh"

namespace cumc {

struct LearnedCell {
    int c, ns, st, ci;
    long long t;
    bool valid;
};

template <int DIR>
__device__ __forceinline__ LearnedCell learned_cell(const Dev &d, long long t0, long long total) {
    LearnedCell q;
    q.valid = t0 < total;
    q.t = q.valid ? t0 : total - 1;  // rows past the end load a real cell, store nothing
    const int ex = (DIR == 0) ? d.nx + 2 : d.nx;
    const int ey = (DIR == 1) ? d.ny + 2 : d.ny;
    int j, k, l;
    const int a = (int)(q.t % ex);
    const long long r = q.t / ex;
    const int b = (int)(r % ey);
    const int e = (int)(r / ey);
    if (DIR == 0) { q.c = a; j = q.c; k = b + 1; l = e + 1; q.ns = d.nx; }
    else if (DIR == 1) { q.c = b; q.ns = d.ny; k = q.c; j = a + 1; l = e + 1; }
    else { q.c = e; q.ns = d.nz; l = q.c; j = a + 1; k = b + 1; }
    q.st = (DIR == 0) ? 1 : (DIR == 1) ? d.NX : d.NX * d.NY;
    q.ci = cidx(d, j, k, l);
    return q;
}

template <int DIR, int UNI>
__device__ __forceinline__ void learned_weights(const Dev &d, int c, float *w) {
    if (UNI) {
#pragma unroll
        for (int m = 0; m < 10; ++m) w[m] = uni_w<float>(d, DIR, m);
    } else {
        const float *wp = weights<float>(d, DIR) + (size_t)(c + 2) * 14;
#pragma unroll
        for (int m = 0; m < 10; ++m) w[m] = wp[m];
    }
}

template <int DIR>
__device__ __forceinline__ void learned_stencils(const Dev &d, const LearnedCell &q, float a[LEARN_NV][5]) {
    constexpr int tb1 = (DIR == 0) ? 1 : 0;
    constexpr int tb2 = (DIR == 2) ? 1 : 2;
#pragma unroll
    for (int v = 0; v < LEARN_NV; ++v) {
        const double *src = (v < 5) ? d.P[v] : d.BC[v == 5 ? tb1 : tb2];
#pragma unroll
        for (int m = 0; m < 5; ++m) a[v][m] = (float)__ldg(src + q.ci + (m - 2) * q.st);
    }
}

// the 7 reconstructions of one cell and its stores (as k_recon); with audit,
// also the largest relative change the linear weights would make
__device__ __forceinline__ void learned_reconstruct(const Dev &d, const LearnedCell &q, const float *w,
                                                    float a[LEARN_NV][5], bool linear, bool audit_cell,
                                                    float &err) {
    float *const *QL = reinterpret_cast<float *const *>(d.QL);
    float *const *QR = reinterpret_cast<float *const *>(d.QR);
    float vm_rho = 0.0f, vp_rho = 0.0f;
    bool fallback = false;
#pragma unroll
    for (int v = 0; v < LEARN_NV; ++v) {
        float vm, vp;
        if (linear) {
            weno_linear<float>(w, a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], vm, vp);
        } else {
            weno<float>(w, a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], vm, vp);
            if (audit_cell) {
                float lm, lp;
                weno_linear<float>(w, a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], lm, lp);
                const float den = fabsf(a[v][2]) + 1.0e-30f;
                err = fmaxf(err, fmaxf(fabsf(lm - vm), fabsf(lp - vp)) / den);
            }
        }
        if (v == 0) { vm_rho = vm; vp_rho = vp; }
        if (v == 4 && d.pos_fallback) {
            fallback = !(vm_rho > 0.0f && vp_rho > 0.0f && vm > 0.0f && vp > 0.0f);
            if (fallback && q.valid && d.fb_count) atomicAdd(d.fb_count, 1ull);
            if (fallback && q.valid) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float cv = (float)__ldg(d.P[u] + q.ci);
                    if (q.c <= q.ns) QL[u][q.ci] = cv;
                    if (q.c >= 1) QR[u][q.ci - q.st] = cv;
                }
            }
        }
        if (fallback) vm = vp = a[v][2];
        if (q.valid) {
            if (q.c <= q.ns) QL[v][q.ci] = vp;
            if (q.c >= 1) QR[v][q.ci - q.st] = vm;
        }
    }
}

template <int DIR>
__device__ __forceinline__ long long learned_total(const Dev &d) {
    const long long ex = (DIR == 0) ? d.nx + 2 : d.nx;
    const long long ey = (DIR == 1) ? d.ny + 2 : d.ny;
    const long long ez = (DIR == 2) ? d.nz + 2 : d.nz;
    return ex * ey * ez;
}

// Steps on which the network runs: stage 1 of every flag_interval-th step
// (learned_refresh_stage, recon_tile.cuh).  Audits are taken there too: set
// audit_interval to a multiple of flag_interval.
__device__ __forceinline__ bool learned_audit(const Dev &d) {
    return d.audit_interval > 0 && (d.S->steps % d.audit_interval) == 0;
}

// Network + reconstruction, persistent: each CTA allocates tensor memory and
// loads the weights once, then walks tiles blockIdx.x, +gridDim.x, ...
// Runs on refresh stages only (uniform early exit otherwise).
// largest relative change the linear weights make to the 7 face pairs of a
// cell (FP32), for the audit of the flags-only network kernel
__device__ __forceinline__ float learned_linear_change(const float *w, float a[LEARN_NV][5]) {
    float err = 0.0f;
#pragma unroll
    for (int v = 0; v < LEARN_NV; ++v) {
        float vm, vp, lm, lp;
        weno<float>(w, a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], vm, vp);
        weno_linear<float>(w, a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], lm, lp);
        const float den = fabsf(a[v][2]) + 1.0e-30f;
        err = fmaxf(err, fmaxf(fabsf(lm - vm), fabsf(lp - vp)) / den);
    }
    return err;
}

// RECON = 1: the FP32 form (network + FP32 reconstruction of the refresh
// stage).  RECON = 0: flags (and the audit verdict) only, for the FP64 form,
// whose reconstruction runs in k_recon_tile<double, ..., LRN = 2>.
template <int DIR, int UNI, int RECON>
__global__ void __launch_bounds__(128, 4) k_recon_learned(const Dev d, int stage) {
    if (d.S->done || !learned_refresh_stage(d, stage)) return;
    __shared__ MlpTile tile;
    __shared__ float s_err[4];
    __shared__ int s_flag[4];
    const int tid = threadIdx.x;
    mlp_tile_setup(tile, reinterpret_cast<const MlpPacked *>(d.mlp));
    const long long total = learned_total<DIR>(d);
    const long long ntiles = (total + 127) / 128;
    const bool audit = learned_audit(d);
    uint32_t phase = 0;
    bool mma_ok = true;
    for (long long tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
        const LearnedCell q = learned_cell<DIR>(d, tl * 128 + tid, total);
        float w[14];
        learned_weights<DIR, UNI>(d, q.c, w);
        float a[LEARN_NV][5];
        learned_stencils<DIR>(d, q, a);
        float logit = -1.0e30f;
        {
            float x[LEARN_K];
#pragma unroll
            for (int v = 0; v < LEARN_NV; ++v)
                learn_var_features(a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], &x[4 * v], &x[4 * LEARN_NV + v]);
#pragma unroll
            for (int m = LEARN_NF; m < LEARN_K; ++m) x[m] = 0.0f;
            if (!mlp_tile_logit(tile, x, phase, logit) || !mma_ok) {
                // an MMA never completed: no cell is flagged, the error is reported
                logit = -1.0e30f;
                if (mma_ok && atomicCAS(&d.S->err_code, 0, LEARN_ERR_MMA) == 0) {
                    d.S->err_cell = (int)tl;
                    d.S->err_stage = -1;
                }
                mma_ok = false;
            }
        }
        const bool flag = q.valid && logit > d.learn_thr;
        if (q.valid) d.lflag[DIR][q.t] = flag ? 1 : 0;
        const bool inner = q.c >= 2 && q.c <= q.ns - 1;
        const bool warp_all = __all_sync(0xffffffffu, flag && inner);
        const bool linear = warp_all && !audit && d.lfb[DIR][tl] == 0;
        float err = 0.0f;
        if (RECON) learned_reconstruct(d, q, w, a, linear, audit && flag && inner, err);
        else if (audit && flag && inner) err = learned_linear_change(w, a);
        if (audit) {
            // tile verdict: the largest error of a flagged cell against the tolerance
            float e = err;
            int nf = (flag && inner) ? 1 : 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
                nf += __shfl_xor_sync(0xffffffffu, nf, o);
            }
            if ((tid & 31) == 0) {
                s_err[tid >> 5] = e;
                s_flag[tid >> 5] = nf;
            }
            __syncthreads();
            if (tid == 0) {
                const float te = fmaxf(fmaxf(s_err[0], s_err[1]), fmaxf(s_err[2], s_err[3]));
                const int tf = s_flag[0] + s_flag[1] + s_flag[2] + s_flag[3];
                const unsigned char fb = te > d.audit_tol ? 1 : 0;
                d.lfb[DIR][tl] = fb;
                const long long nvalid = total - tl * 128;
                // counters spread over 64 slots (summed on the host)
                unsigned long long *ls = d.lstats + (tl & (LEARN_STAT_SLOTS - 1)) * LEARN_STAT_FIELDS;
                atomicAdd(&ls[0], (unsigned long long)(nvalid < 128 ? nvalid : 128));
                atomicAdd(&ls[1], (unsigned long long)tf);
                atomicAdd(&ls[2], (unsigned long long)fb);
                if (tl == 0 && DIR == 0) atomicAdd(&ls[3], 1ull);
            }
            __syncthreads();
        }
    }
    mlp_tile_teardown(tile);
}

}  // namespace cumc
