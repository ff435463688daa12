// recon_learned.cuh -- FP32 WENO reconstruction with the learned smooth-face
// flag fused in (see learned.cuh).  Same cells, same enumeration and the same
// outputs (QL/QR face states) as k_recon<float, DIR, REC_WENO, UNI>.
//
// One CTA = 128 consecutive cells of the flat enumeration = one tile:
//   1. each thread loads its cell's 7 stencils and builds the 35 features;
//   2. the MLP (tcgen05, BF16 operands, FP32 accumulators in TMEM) gives one
//      logit per cell;
//   3. a warp whose 32 cells are all flagged, in a tile not marked to fall
//      back, reconstructs with the linear optimal weights; every other warp
//      runs WENO-Z exactly as k_recon does;
//   4. every audit_interval steps all warps run WENO-Z (results identical to
//      the plain FP32 form), flagged cells also evaluate the linear values,
//      and the tile is marked to fall back until the next audit if any
//      flagged cell's relative face-value error exceeds audit_tol.
#pragma once
#include "flux_kernel.cuh"
#include "learned.cuh"

namespace cumc {

template <int DIR, int UNI>
__global__ void __launch_bounds__(128, 4) k_recon_learned(const Dev d) {
    if (d.S->done) return;
    __shared__ MlpTile tile;
    __shared__ float s_err[4];
    __shared__ int s_flag[4];
    const int tid = threadIdx.x;
    mlp_tile_setup(tile, reinterpret_cast<const MlpPacked *>(d.mlp));

    const int ex = (DIR == 0) ? d.nx + 2 : d.nx;
    const int ey = (DIR == 1) ? d.ny + 2 : d.ny;
    const int ez = (DIR == 2) ? d.nz + 2 : d.nz;
    const long long total = (long long)ex * ey * ez;
    const long long t0 = (long long)blockIdx.x * 128 + tid;
    const bool valid = t0 < total;
    const long long t = valid ? t0 : total - 1;  // rows past the end load a real cell, store nothing
    int c, j, k, l, ns;
    {
        const int a = (int)(t % ex);
        const long long r = t / ex;
        const int b = (int)(r % ey);
        const int e = (int)(r / ey);
        if (DIR == 0) { c = a; j = c; k = b + 1; l = e + 1; ns = d.nx; }
        else if (DIR == 1) { c = b; k = c; j = a + 1; l = e + 1; ns = d.ny; }
        else { c = e; l = c; j = a + 1; k = b + 1; ns = d.nz; }
    }
    const int st = (DIR == 0) ? 1 : (DIR == 1) ? d.NX : d.NX * d.NY;
    const int ci = cidx(d, j, k, l);
    constexpr int tb1 = (DIR == 0) ? 1 : 0;
    constexpr int tb2 = (DIR == 2) ? 1 : 2;
    float w[14];
    if (UNI) {
#pragma unroll
        for (int m = 0; m < 10; ++m) w[m] = uni_w<float>(d, DIR, m);
    } else {
        const float *wp = weights<float>(d, DIR) + (size_t)(c + 2) * 14;
#pragma unroll
        for (int m = 0; m < 10; ++m) w[m] = wp[m];
    }
    float a[LEARN_NV][5];
#pragma unroll
    for (int v = 0; v < LEARN_NV; ++v) {
        const double *src = (v < 5) ? d.P[v] : d.BC[v == 5 ? tb1 : tb2];
#pragma unroll
        for (int m = 0; m < 5; ++m) a[v][m] = (float)__ldg(src + ci + (m - 2) * st);
    }
    float logit = -1.0e30f;
    {
        float x[LEARN_K];
#pragma unroll
        for (int v = 0; v < LEARN_NV; ++v)
            learn_var_features(a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], &x[4 * v], &x[4 * LEARN_NV + v]);
#pragma unroll
        for (int m = LEARN_NF; m < LEARN_K; ++m) x[m] = 0.0f;
        uint32_t phase = 0;
        if (!mlp_tile_logit(tile, x, phase, logit)) {
            // the MMA never completed: no cell is flagged, the error is reported
            logit = -1.0e30f;
            if (atomicCAS(&d.S->err_code, 0, LEARN_ERR_MMA) == 0) {
                d.S->err_cell = blockIdx.x;
                d.S->err_stage = -1;
            }
        }
    }
    const bool audit = d.audit_interval > 0 && (d.S->steps % d.audit_interval) == 0;
    const bool flag = valid && logit > d.learn_thr;
    const bool warp_all = __all_sync(0xffffffffu, flag);
    const bool linear = warp_all && !audit && d.lfb[DIR][blockIdx.x] == 0;

    float *const *QL = reinterpret_cast<float *const *>(d.QL);
    float *const *QR = reinterpret_cast<float *const *>(d.QR);
    float vm_rho = 0.0f, vp_rho = 0.0f;
    bool fallback = false;
    float err = 0.0f;
#pragma unroll
    for (int v = 0; v < LEARN_NV; ++v) {
        float vm, vp;
        if (linear) {
            weno_linear<float>(w, a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], vm, vp);
        } else {
            weno<float>(w, a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], vm, vp);
            if (audit && flag) {
                float lm, lp;
                weno_linear<float>(w, a[v][0], a[v][1], a[v][2], a[v][3], a[v][4], lm, lp);
                const float den = fabsf(a[v][2]) + 1.0e-30f;
                err = fmaxf(err, fmaxf(fabsf(lm - vm), fabsf(lp - vp)) / den);
            }
        }
        if (v == 0) { vm_rho = vm; vp_rho = vp; }
        if (v == 4 && d.pos_fallback) {
            fallback = !(vm_rho > 0.0f && vp_rho > 0.0f && vm > 0.0f && vp > 0.0f);
            if (fallback && valid) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float cv = (float)__ldg(d.P[u] + ci);
                    if (c <= ns) QL[u][ci] = cv;
                    if (c >= 1) QR[u][ci - st] = cv;
                }
            }
        }
        if (fallback) vm = vp = a[v][2];
        if (valid) {
            if (c <= ns) QL[v][ci] = vp;
            if (c >= 1) QR[v][ci - st] = vm;
        }
    }
    if (audit) {
        // tile verdict: the largest error of a flagged cell against the tolerance
        float e = err;
        int nf = flag ? 1 : 0;
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
            d.lfb[DIR][blockIdx.x] = fb;
            const long long nvalid = total - (long long)blockIdx.x * 128;
            // counters spread over 64 slots (summed on the host)
            unsigned long long *ls = d.lstats + (blockIdx.x & (LEARN_STAT_SLOTS - 1)) * LEARN_STAT_FIELDS;
            atomicAdd(&ls[0], (unsigned long long)(nvalid < 128 ? nvalid : 128));
            atomicAdd(&ls[1], (unsigned long long)tf);
            atomicAdd(&ls[2], (unsigned long long)fb);
            if (blockIdx.x == 0 && DIR == 0) atomicAdd(&ls[3], 1ull);
        }
    }
    mlp_tile_teardown(tile);
}

}  // namespace cumc
