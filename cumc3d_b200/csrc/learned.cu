// learned.cu -- harvesting, training and stand-alone inference of the learned
// smooth-face flag (learned.cuh).  Built with --fmad=false: the FP64 labels
// and the FP32 features of the harvest are plain IEEE arithmetic, as the CPU
// oracle computes them.
//
//   harvest   one row per sampled cell of a direction sweep: 35 FP32 features,
//             the relative face-value change that the linear optimal weights
//             would make (FP64 WENO-Z of the plain method), and the largest
//             deviation |omega_k - g_k| of the nonlinear weights;
//   training  binary cross-entropy of "face change < delta", forward and
//             backward in FP32 on the CUDA cores, gradients summed in a fixed
//             order (deterministic), Adam;
//   inference the BF16 tensor-core MLP of the reconstruction kernel, run on
//             given features (for checks and evaluation).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cumc3d_gpu.h"
#include "engine.cuh"
#include "flux_kernel.cuh"
#include "learned.cuh"
#include "mhd_device.cuh"

namespace cumc {

// ---------------------------------------------------------------------------
// harvest
// ---------------------------------------------------------------------------
template <int DIR>
__global__ void k_learn_harvest(const Dev d, long long stride, long long rows, float *out) {
    const long long row = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= rows) return;
    // interior cells 1..n along the sweep, x fastest (as the reconstruction enumerates)
    const int ex = d.nx, ey = d.ny;
    const long long t = row * stride;
    const int a = (int)(t % ex);
    const long long r = t / ex;
    const int b = (int)(r % ey);
    const int e = (int)(r / ey);
    const int j = a + 1, k = b + 1, l = e + 1;
    const int c = (DIR == 0) ? j : (DIR == 1) ? k : l;
    const int st = (DIR == 0) ? 1 : (DIR == 1) ? d.NX : d.NX * d.NY;
    const int ci = cidx(d, j, k, l);
    constexpr int tb1 = (DIR == 0) ? 1 : 0;
    constexpr int tb2 = (DIR == 2) ? 1 : 2;
    const double *wp = ((DIR == 0) ? d.wx : (DIR == 1) ? d.wy : d.wz) + (size_t)(c + 2) * 14;
    double w[14];
#pragma unroll
    for (int m = 0; m < 10; ++m) w[m] = wp[m];
    float *o = out + row * LEARN_ROW;
    double change = 0.0, wdev = 0.0;
    for (int v = 0; v < LEARN_NV; ++v) {
        const double *src = (v < 5) ? d.P[v] : d.BC[v == 5 ? tb1 : tb2];
        double s[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) s[m] = src[ci + (m - 2) * st];
        float f4[4], rv;
        learn_var_features((float)s[0], (float)s[1], (float)s[2], (float)s[3], (float)s[4], f4, &rv);
#pragma unroll
        for (int i = 0; i < 4; ++i) o[4 * v + i] = f4[i];
        o[4 * LEARN_NV + v] = rv;
        WenoParts<double> wp5;
        weno_parts<double>(w, s[0], s[1], s[2], s[3], s[4], wp5);
        double om[3];
        const double g[3] = {1.0 / 10.0, 6.0 / 10.0, 3.0 / 10.0};
        wenoz_weights<double>(wp5.Bp, om);
        const double vp_z = om[0] * wp5.Pp[0] + om[1] * wp5.Pp[1] + om[2] * wp5.Pp[2];
        for (int q = 0; q < 3; ++q) wdev = fmax(wdev, fabs(om[q] - g[q]));
        wenoz_weights<double>(wp5.Bm, om);
        const double vm_z = om[0] * wp5.Pm[0] + om[1] * wp5.Pm[1] + om[2] * wp5.Pm[2];
        for (int q = 0; q < 3; ++q) wdev = fmax(wdev, fabs(om[q] - g[q]));
        const double vp_l = g[0] * wp5.Pp[0] + g[1] * wp5.Pp[1] + g[2] * wp5.Pp[2];
        const double vm_l = g[0] * wp5.Pm[0] + g[1] * wp5.Pm[1] + g[2] * wp5.Pm[2];
        const double den = fabs(s[2]) + 1.0e-300;
        change = fmax(change, fmax(fabs(vp_l - vp_z), fabs(vm_l - vm_z)) / den);
    }
    o[LEARN_NF] = (float)change;
    o[LEARN_NF + 1] = (float)wdev;
}

// ---------------------------------------------------------------------------
// training
// ---------------------------------------------------------------------------
constexpr int TB = 128;  // samples per block of the gradient kernel

struct GradSmem {
    float P[LEARN_NP];
    float x[TB][LEARN_NF];
    float h1[TB][LEARN_H];
    float h2[TB][LEARN_H];
    float g1[TB][LEARN_H];
    float g2[TB][LEARN_H];
    float gz[TB];
    float loss[TB];
};

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void k_sample_idx(unsigned long long seed, unsigned long long step, long long n, int batch, long long *idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    idx[i] = (long long)(splitmix64(seed ^ (step * 0x632BE59BD9B4E019ull) ^ (unsigned long long)i) % (unsigned long long)n);
}

// Per block: forward + backward of TB samples, then the block's gradient sum
// (fixed sample order) -> partial[blockIdx.x][*], loss sum -> lpart[blockIdx.x].
// idx == nullptr: samples first + blockIdx.x * TB + tid (contiguous).
__global__ void __launch_bounds__(TB) k_mlp_grad(const float *__restrict__ params, const float *__restrict__ X,
                                                 const long long *__restrict__ idx, long long first, long long count,
                                                 float delta, float *__restrict__ partial,
                                                 float *__restrict__ lpart) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &S = *reinterpret_cast<GradSmem *>(smem_raw);
    const int tid = threadIdx.x;
    for (int p = tid; p < LEARN_NP; p += TB) S.P[p] = params[p];
    __syncthreads();
    const long long local = (long long)blockIdx.x * TB + tid;
    const bool valid = local < count;
    long long si = 0;
    if (valid) si = idx ? idx[local] : first + local;
    const float *row = X + si * LEARN_ROW;
    float x[LEARN_NF];
#pragma unroll
    for (int i = 0; i < LEARN_NF; ++i) x[i] = valid ? row[i] : 0.0f;
    const float y = (valid && row[LEARN_NF] < delta) ? 1.0f : 0.0f;
    float h1[LEARN_H], h2[LEARN_H];
    for (int o = 0; o < LEARN_H; ++o) {
        float acc = S.P[LP_B1 + o];
        const float *wr = &S.P[LP_W1 + o * LEARN_K];
#pragma unroll
        for (int i = 0; i < LEARN_NF; ++i) acc += wr[i] * x[i];
        h1[o] = fmaxf(acc, 0.0f);
    }
    for (int o = 0; o < LEARN_H; ++o) {
        float acc = S.P[LP_B2 + o];
        const float *wr = &S.P[LP_W2 + o * LEARN_H];
#pragma unroll
        for (int i = 0; i < LEARN_H; ++i) acc += wr[i] * h1[i];
        h2[o] = fmaxf(acc, 0.0f);
    }
    float z = S.P[LP_B3];
#pragma unroll
    for (int i = 0; i < LEARN_H; ++i) z += S.P[LP_W3 + i] * h2[i];
    // binary cross-entropy with logits: max(z,0) - y z + log(1 + exp(-|z|))
    const float loss = fmaxf(z, 0.0f) - y * z + log1pf(expf(-fabsf(z)));
    const float sig = 1.0f / (1.0f + expf(-z));
    const float dz = valid ? (sig - y) : 0.0f;
    float g2[LEARN_H], g1[LEARN_H];
#pragma unroll
    for (int i = 0; i < LEARN_H; ++i) g2[i] = h2[i] > 0.0f ? dz * S.P[LP_W3 + i] : 0.0f;
    for (int i = 0; i < LEARN_H; ++i) {
        float acc = 0.0f;
#pragma unroll
        for (int o = 0; o < LEARN_H; ++o) acc += S.P[LP_W2 + o * LEARN_H + i] * g2[o];
        g1[i] = h1[i] > 0.0f ? acc : 0.0f;
    }
#pragma unroll
    for (int i = 0; i < LEARN_NF; ++i) S.x[tid][i] = x[i];
#pragma unroll
    for (int i = 0; i < LEARN_H; ++i) {
        S.h1[tid][i] = h1[i];
        S.h2[tid][i] = h2[i];
        S.g1[tid][i] = g1[i];
        S.g2[tid][i] = g2[i];
    }
    S.gz[tid] = dz;
    S.loss[tid] = valid ? loss : 0.0f;
    __syncthreads();
    // this block's gradient: each entry summed over the TB samples in order
    for (int p = tid; p < LEARN_NP; p += TB) {
        float acc = 0.0f;
        if (p < LP_B1) {
            const int o = p / LEARN_K, i = p % LEARN_K;
            if (i < LEARN_NF)
                for (int s = 0; s < TB; ++s) acc += S.g1[s][o] * S.x[s][i];
        } else if (p < LP_W2) {
            const int o = p - LP_B1;
            for (int s = 0; s < TB; ++s) acc += S.g1[s][o];
        } else if (p < LP_B2) {
            const int o = (p - LP_W2) / LEARN_H, i = (p - LP_W2) % LEARN_H;
            for (int s = 0; s < TB; ++s) acc += S.g2[s][o] * S.h1[s][i];
        } else if (p < LP_W3) {
            const int o = p - LP_B2;
            for (int s = 0; s < TB; ++s) acc += S.g2[s][o];
        } else if (p < LP_B3) {
            const int i = p - LP_W3;
            for (int s = 0; s < TB; ++s) acc += S.gz[s] * S.h2[s][i];
        } else {
            for (int s = 0; s < TB; ++s) acc += S.gz[s];
        }
        partial[(size_t)blockIdx.x * LEARN_NP + p] = acc;
    }
    if (tid == 0) {
        float ls = 0.0f;
        for (int s = 0; s < TB; ++s) ls += S.loss[s];
        lpart[blockIdx.x] = ls;
    }
}

// mean over the batch: gradient entries and the loss, blocks summed in order
__global__ void k_mlp_reduce(const float *__restrict__ partial, const float *__restrict__ lpart, int nblk,
                             long long count, float *__restrict__ grad, float *__restrict__ loss_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const float inv = 1.0f / (float)count;
    if (p < LEARN_NP) {
        float acc = 0.0f;
        for (int b = 0; b < nblk; ++b) acc += partial[(size_t)b * LEARN_NP + p];
        grad[p] = acc * inv;
    }
    if (p == 0 && loss_out) {
        float acc = 0.0f;
        for (int b = 0; b < nblk; ++b) acc += lpart[b];
        *loss_out = acc * inv;
    }
}

__global__ void k_adam(float *__restrict__ P, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= LEARN_NP) return;
    const float gi = g[p];
    const float mi = b1 * m[p] + (1.0f - b1) * gi;
    const float vi = b2 * v[p] + (1.0f - b2) * gi * gi;
    m[p] = mi;
    v[p] = vi;
    P[p] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ---------------------------------------------------------------------------
// stand-alone inference on given features (one tile of 128 rows per CTA)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_mlp_infer(const MlpPacked *__restrict__ mp, const float *__restrict__ X,
                                                   int ld, long long n, float *__restrict__ logits, int *err) {
    __shared__ MlpTile tile;
    mlp_tile_setup(tile, mp);
    const long long r = (long long)blockIdx.x * 128 + threadIdx.x;
    float x[LEARN_K];
#pragma unroll
    for (int i = 0; i < LEARN_K; ++i) x[i] = (r < n && i < LEARN_NF) ? X[r * ld + i] : 0.0f;
    uint32_t phase = 0;
    float z;
    const bool ok = mlp_tile_logit(tile, x, phase, z);
    if (!ok) atomicExch(err, 1);
    if (r < n) logits[r] = z;
    mlp_tile_teardown(tile);
}

void learn_pack(const float *P, MlpPacked *out) {
    memset(out, 0, sizeof(MlpPacked));
    auto bf = [](float f) -> uint16_t {
        // round to nearest even, as __float2bfloat16_rn (finite inputs)
        uint32_t u;
        memcpy(&u, &f, 4);
        const uint32_t lsb = (u >> 16) & 1u;
        u += 0x7FFFu + lsb;
        return (uint16_t)(u >> 16);
    };
    for (int o = 0; o < LEARN_H; ++o)
        for (int i = 0; i < LEARN_K; ++i) out->W1[kmaj_off(o, i, LEARN_K)] = bf(P[LP_W1 + o * LEARN_K + i]);
    for (int o = 0; o < LEARN_H; ++o)
        for (int i = 0; i < LEARN_H; ++i) out->W2[kmaj_off(o, i, LEARN_H)] = bf(P[LP_W2 + o * LEARN_H + i]);
    for (int i = 0; i < LEARN_H; ++i) {
        out->b1[i] = P[LP_B1 + i];
        out->b2[i] = P[LP_B2 + i];
        out->w3[i] = P[LP_W3 + i];
    }
    out->b3 = P[LP_B3];
}

long long harvest_rows(const Dev &d, long long stride) {
    const long long cells = (long long)d.nx * d.ny * d.nz;
    return (cells + stride - 1) / stride;
}

void launch_harvest(const Dev &d, int dir, long long stride, float *out, cudaStream_t s) {
    const long long rows = harvest_rows(d, stride);
    const unsigned g = (unsigned)((rows + 127) / 128);
    if (dir == 0) k_learn_harvest<0><<<g, 128, 0, s>>>(d, stride, rows, out);
    else if (dir == 1) k_learn_harvest<1><<<g, 128, 0, s>>>(d, stride, rows, out);
    else k_learn_harvest<2><<<g, 128, 0, s>>>(d, stride, rows, out);
}

}  // namespace cumc

using namespace cumc;

namespace {
std::string g_learn_err;
int lfail(int code, const std::string &m) {
    g_learn_err = m;
    return code;
}
struct DevBuf {
    std::vector<void *> p;
    ~DevBuf() {
        for (void *q : p) cudaFree(q);
    }
    template <class T> T *get(size_t n) {
        void *q = nullptr;
        if (cudaMalloc(&q, n * sizeof(T) + 16) != cudaSuccess) return nullptr;
        p.push_back(q);
        return (T *)q;
    }
};
int grad_smem() { return (int)sizeof(GradSmem); }
}  // namespace

extern "C" {

const char *cumc_mlp_last_error(void) { return g_learn_err.c_str(); }

int cumc_mlp_grad(const float *params, const float *samples, long long n, float delta, float *grad_out,
                  float *loss_out) {
    if (!params || !samples || n <= 0 || !grad_out) return lfail(CUMC_EINVAL, "bad argument");
    DevBuf B;
    float *dP = B.get<float>(LEARN_NP), *dX = B.get<float>((size_t)n * LEARN_ROW);
    const int nblk = (int)((n + TB - 1) / TB);
    float *part = B.get<float>((size_t)nblk * LEARN_NP), *lp = B.get<float>(nblk);
    float *dg = B.get<float>(LEARN_NP), *dl = B.get<float>(1);
    if (!dP || !dX || !part || !lp || !dg || !dl) return lfail(CUMC_ENOMEM, "device allocation failed");
    cudaMemcpy(dP, params, LEARN_NP * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dX, samples, (size_t)n * LEARN_ROW * sizeof(float), cudaMemcpyHostToDevice);
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, grad_smem());
    k_mlp_grad<<<nblk, TB, grad_smem()>>>(dP, dX, nullptr, 0, n, delta, part, lp);
    k_mlp_reduce<<<(LEARN_NP + 255) / 256, 256>>>(part, lp, nblk, n, dg, dl);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
        return lfail(CUMC_ECUDA, "gradient kernels failed");
    cudaMemcpy(grad_out, dg, LEARN_NP * sizeof(float), cudaMemcpyDeviceToHost);
    if (loss_out) cudaMemcpy(loss_out, dl, sizeof(float), cudaMemcpyDeviceToHost);
    return CUMC_OK;
}

int cumc_mlp_train(const float *samples, long long n, const cumc_train_config *tc, float *params_inout,
                   float *loss_curve) {
    if (!samples || n <= 0 || !tc || !params_inout || tc->steps <= 0 || tc->batch <= 0)
        return lfail(CUMC_EINVAL, "bad argument");
    DevBuf B;
    float *dP = B.get<float>(LEARN_NP), *dX = B.get<float>((size_t)n * LEARN_ROW);
    const int nblk = (tc->batch + TB - 1) / TB;
    float *part = B.get<float>((size_t)nblk * LEARN_NP), *lp = B.get<float>(nblk);
    float *dg = B.get<float>(LEARN_NP), *dm = B.get<float>(LEARN_NP), *dv = B.get<float>(LEARN_NP);
    float *dl = B.get<float>(tc->steps);
    long long *idx = B.get<long long>(tc->batch);
    if (!dP || !dX || !part || !lp || !dg || !dm || !dv || !dl || !idx)
        return lfail(CUMC_ENOMEM, "device allocation failed");
    cudaMemcpy(dP, params_inout, LEARN_NP * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dX, samples, (size_t)n * LEARN_ROW * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(dm, 0, LEARN_NP * sizeof(float));
    cudaMemset(dv, 0, LEARN_NP * sizeof(float));
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, grad_smem());
    const float b1 = tc->beta1 > 0 ? tc->beta1 : 0.9f, b2 = tc->beta2 > 0 ? tc->beta2 : 0.999f;
    const float eps = tc->eps > 0 ? tc->eps : 1e-8f;
    double c1 = 1.0, c2 = 1.0;
    for (int s = 1; s <= tc->steps; ++s) {
        k_sample_idx<<<(tc->batch + 255) / 256, 256>>>(tc->seed, (unsigned long long)s, n, tc->batch, idx);
        k_mlp_grad<<<nblk, TB, grad_smem()>>>(dP, dX, idx, 0, tc->batch, tc->delta, part, lp);
        k_mlp_reduce<<<(LEARN_NP + 255) / 256, 256>>>(part, lp, nblk, tc->batch, dg, dl + (s - 1));
        c1 *= b1;
        c2 *= b2;
        k_adam<<<(LEARN_NP + 255) / 256, 256>>>(dP, dg, dm, dv, tc->lr, b1, b2, eps, (float)(1.0 - c1),
                                                (float)(1.0 - c2));
    }
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
        return lfail(CUMC_ECUDA, "training kernels failed");
    cudaMemcpy(params_inout, dP, LEARN_NP * sizeof(float), cudaMemcpyDeviceToHost);
    if (loss_curve) cudaMemcpy(loss_curve, dl, (size_t)tc->steps * sizeof(float), cudaMemcpyDeviceToHost);
    return CUMC_OK;
}

int cumc_mlp_infer(const float *params, const float *features, int ld, long long n, float *logits) {
    if (!params || !features || n <= 0 || ld < LEARN_NF || !logits) return lfail(CUMC_EINVAL, "bad argument");
    DevBuf B;
    MlpPacked hp;
    learn_pack(params, &hp);
    MlpPacked *dp = B.get<MlpPacked>(1);
    float *dX = B.get<float>((size_t)n * ld), *dz = B.get<float>(n);
    int *derr = B.get<int>(1);
    if (!dp || !dX || !dz || !derr) return lfail(CUMC_ENOMEM, "device allocation failed");
    cudaMemcpy(dp, &hp, sizeof hp, cudaMemcpyHostToDevice);
    cudaMemcpy(dX, features, (size_t)n * ld * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(derr, 0, sizeof(int));
    k_mlp_infer<<<(unsigned)((n + 127) / 128), 128>>>(dp, dX, ld, n, dz, derr);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
        return lfail(CUMC_ECUDA, "inference kernel failed");
    int herr = 0;
    cudaMemcpy(&herr, derr, sizeof herr, cudaMemcpyDeviceToHost);
    if (herr) return lfail(CUMC_ECUDA, "a tensor-core MMA did not complete");
    cudaMemcpy(logits, dz, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    return CUMC_OK;
}

}  // extern "C"
