// learned.cuh -- the learned smooth-face flag of the FP32 WENO form.
//
// A small MLP reads scale-free features of a cell's 5-point stencils (all 7
// reconstructed variables) and flags cells whose WENO-Z face values are
// within a tolerance of the linear optimal-weight (0.1, 0.6, 0.3) fifth-order
// values; a warp whose 32 cells are all flagged reconstructs with the linear
// weights and skips the smoothness indicators and nonlinear weights.
//
// Inference runs on the 5th-generation tensor cores: one CTA = 128 cells =
// the M = 128 rows of tcgen05.mma (kind::f16, BF16 operands from shared
// memory, FP32 accumulator in tensor memory), two layers of N = 32, the
// 32 -> 1 output layer on the CUDA cores from the accumulator registers.
//
// No reference counterpart (the reference always uses the nonlinear weights,
// solver/mhd/weno_module.f90:363-404).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cumc {

constexpr int LEARN_NV = 7;   // reconstructed variables per cell
constexpr int LEARN_NF = 35;  // features: 4 normalised differences + 1 relative variation per variable
constexpr int LEARN_K = 48;   // features padded to 3 MMA k-steps of 16
constexpr int LEARN_H = 32;   // hidden width of both layers
// parameter vector (FP32): W1[H][K] (out, in), b1[H], W2[H][H], b2[H], w3[H], b3
constexpr int LP_W1 = 0;
constexpr int LP_B1 = LP_W1 + LEARN_H * LEARN_K;
constexpr int LP_W2 = LP_B1 + LEARN_H;
constexpr int LP_B2 = LP_W2 + LEARN_H * LEARN_H;
constexpr int LP_W3 = LP_B2 + LEARN_H;
constexpr int LP_B3 = LP_W3 + LEARN_H;
constexpr int LEARN_NP = LP_B3 + 1;  // 2657
// one harvested sample: the features, the relative face-value change that
// the linear weights would make, the largest nonlinear-weight deviation
constexpr int LEARN_ROW = LEARN_NF + 2;
// device counters of the audits: per slot {cells audited, cells flagged,
// tiles set to fall back, audits}; 64 slots spread the atomics
constexpr int LEARN_STAT_SLOTS = 64;
constexpr int LEARN_STAT_FIELDS = 4;
// device error word: an MMA of the learned inference did not complete
constexpr int LEARN_ERR_MMA = 2;  // CUMC_ECUDA

// features of one variable's stencil a0..a4 (cells c-2..c+2): differences
// over their absolute sum (shape, scale-free) and the relative variation
__host__ __device__ inline void learn_var_features(float a0, float a1, float a2, float a3, float a4, float *f4,
                                                   float *r) {
    const float d0 = a1 - a0, d1 = a2 - a1, d2 = a3 - a2, d3 = a4 - a3;
    const float s = ((fabsf(d0) + fabsf(d1)) + fabsf(d2)) + fabsf(d3);
    const float inv = 1.0f / (s + 1.0e-30f);
    f4[0] = d0 * inv;
    f4[1] = d1 * inv;
    f4[2] = d2 * inv;
    f4[3] = d3 * inv;
    *r = s * (1.0f / ((fabsf(a2) + s) + 1.0e-30f));
}

// element offset of (row r, column k) in a K-major BF16 tile of K columns in
// the no-swizzle canonical layout of tcgen05: 8 x 8 core matrices (8 rows of
// 16 bytes, contiguous), adjacent in K 128 bytes apart (leading offset),
// 8-row groups K * 16 bytes apart (stride offset)
__host__ __device__ constexpr int kmaj_off(int r, int k, int K) {
    return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

// packed parameters for inference (prepared on the host): BF16 W1, W2 in the
// canonical layout, FP32 biases and output layer
struct MlpPacked {
    uint16_t W1[LEARN_H * LEARN_K];
    uint16_t W2[LEARN_H * LEARN_H];
    float b1[LEARN_H], b2[LEARN_H], w3[LEARN_H];
    float b3, pad[3];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "packed parameters are copied in 16-byte units");

struct __align__(128) MlpTile {
    uint16_t A[128 * LEARN_K];  // features of the CTA's 128 cells (layer-1 A operand)
    uint16_t Hd[128 * LEARN_H]; // hidden layer (layer-2 A operand)
    MlpPacked p;                // weights (B operands) and biases
    unsigned long long mbar;    // MMA completion
    unsigned int tmem;          // tensor-memory base address
    int err;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start >> 4, leading byte offset >> 4,
// stride byte offset >> 4, version 1 (bit 46), no swizzle
__device__ __forceinline__ uint64_t umma_desc(const void *p, uint32_t lbo, uint32_t sbo) {
    const uint64_t a = (smem_u32(p) >> 4) & 0x3FFFu;
    return a | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at 24
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned long long *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(unsigned long long *mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
// bounded wait on one phase of the barrier; false if it never completed
__device__ __forceinline__ bool mbar_wait(unsigned long long *mbar, uint32_t parity) {
    const uint32_t a = smem_u32(mbar);
    for (int i = 0; i < (1 << 22); ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 32 consecutive FP32 columns of this warp's 32 tensor-memory lanes; the load
// and its completion wait are one statement so no use can move between them
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
    const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
    return a | (b << 16);
}
// one row of 8 values (16 bytes) of a core matrix
__device__ __forceinline__ void store_row8(uint16_t *dst, const float *v) {
    uint4 q;
    q.x = pack_bf16x2(v[0], v[1]);
    q.y = pack_bf16x2(v[2], v[3]);
    q.z = pack_bf16x2(v[4], v[5]);
    q.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4 *>(dst) = q;
}

// Set-up of the tile (all 128 threads): tensor memory (32 columns, warp 0),
// the completion barrier and the weights.
__device__ __forceinline__ void mlp_tile_setup(MlpTile &t, const MlpPacked *gp) {
    const int tid = threadIdx.x;
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(&t.tmem))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&t.mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        t.err = 0;
    }
    const uint4 *src = reinterpret_cast<const uint4 *>(gp);
    uint4 *dst = reinterpret_cast<uint4 *>(&t.p);
    for (int i = tid; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) dst[i] = __ldg(src + i);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

__device__ __forceinline__ void mlp_tile_teardown(MlpTile &t) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(t.tmem) : "memory");
    }
}

// Logit of this thread's row (128 threads = 128 rows).  x: LEARN_K features
// (zero beyond LEARN_NF).  phase: the barrier phase to wait for next (two
// phases are used per call).  Returns false if an MMA never completed.
__device__ __forceinline__ bool mlp_tile_logit(MlpTile &t, const float *x, uint32_t &phase, float &logit) {
    const int tid = threadIdx.x;
    const uint32_t lane_base = (uint32_t)((tid >> 5) * 32) << 16;
    constexpr uint32_t idesc = umma_idesc_bf16(128, LEARN_H);
#pragma unroll
    for (int kc = 0; kc < LEARN_K / 8; ++kc) store_row8(&t.A[kmaj_off(tid, kc * 8, LEARN_K)], x + kc * 8);
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int ks = 0; ks < LEARN_K / 16; ++ks)
            umma_bf16(t.tmem, umma_desc(&t.A[ks * 128], 128, LEARN_K * 16),
                      umma_desc(&t.p.W1[ks * 128], 128, LEARN_K * 16), idesc, ks > 0 ? 1u : 0u);
        umma_commit(&t.mbar);
    }
    bool ok = mbar_wait(&t.mbar, phase);
    phase ^= 1u;
    tc_fence_after();
    float h[32];
    tmem_ld32(t.tmem + lane_base, h);
#pragma unroll
    for (int i = 0; i < 32; ++i) h[i] = fmaxf(h[i] + t.p.b1[i], 0.0f);
#pragma unroll
    for (int kc = 0; kc < LEARN_H / 8; ++kc) store_row8(&t.Hd[kmaj_off(tid, kc * 8, LEARN_H)], h + kc * 8);
    tc_fence_before();
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int ks = 0; ks < LEARN_H / 16; ++ks)
            umma_bf16(t.tmem, umma_desc(&t.Hd[ks * 128], 128, LEARN_H * 16),
                      umma_desc(&t.p.W2[ks * 128], 128, LEARN_H * 16), idesc, ks > 0 ? 1u : 0u);
        umma_commit(&t.mbar);
    }
    ok = mbar_wait(&t.mbar, phase) && ok;
    phase ^= 1u;
    tc_fence_after();
    tmem_ld32(t.tmem + lane_base, h);
    float z = t.p.b3;
#pragma unroll
    for (int i = 0; i < 32; ++i) z += t.p.w3[i] * fmaxf(h[i] + t.p.b2[i], 0.0f);
    logit = z;
    tc_fence_before();  // the next tile's MMA (after a barrier) may overwrite these columns
    return ok;
}

// host: FP32 parameter vector -> packed BF16 inference layout
void learn_pack(const float *params, MlpPacked *out);
struct Dev;
// harvest: rows of LEARN_ROW floats for every stride-th interior cell
long long harvest_rows(const Dev &d, long long stride);
void launch_harvest(const Dev &d, int dir, long long stride, float *out, cudaStream_t s);

}  // namespace cumc
