// noalloc.cu -- cumc_batch_run1_noalloc: one 1D problem through the batched
// kernel (k_batch, batch_kernel.cuh) with every device buffer taken from a
// file-scope static device array instead of cudaMalloc.
//
// Who needs it: a host program that owns all device memory itself and lets no
// library allocate, e.g. a Fortran/OpenACC code that maps its arrays once at
// start-up and sizes its pool to what is left, or an embedding whose time loop
// must not call cudaMalloc/cudaFree because both can synchronise the whole
// device and stall the host's other streams.
//
// Limits and rules:
//  * at most NOALLOC_MAX_CELLS (4096) zones; larger problems are rejected with
//    CUMC_EINVAL before any device work;
//  * the scratch is one static array per device (NOALLOC_SCRATCH_BYTES, about
//    3.5 MB), held by every device that loads the library until exit; each
//    call, with the device current, looks up its address in the current
//    context (cudaGetSymbolAddress).  The first call on a device (and the
//    first after a cudaDeviceReset) loads the module: make it before any
//    stream capture;
//  * a CUDA error left pending by the caller's earlier work is reported as
//    such (CUMC_ECUDA) before any device work, so the launch checks below
//    only ever see this call's own launches;
//  * every call clears the whole scratch array (one cudaMemsetAsync of about
//    3.5 MB) before filling it, so no state survives between calls;
//  * calls that overlap in time on the same device (other threads, other
//    streams) share the one scratch array and race: serialise them.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/cumc3d_gpu.h"
#include "batch_kernel.cuh"
#include "weights1d.cuh"

using namespace cumc;

namespace {

constexpr int NOALLOC_MAX_CELLS = 4096;
constexpr int NOALLOC_ROW = NOALLOC_MAX_CELLS + 8;  // padded cells -2..n+3, or faces -3..n+3
// per padded cell, in doubles: P 5, EPS, CS, BC 3, prim faces 5, cons 5+5
// plus the second x-face buffer, u_old 5+5, QL 7, QR 7, F 5, EY, EZ, dx,
// w 14, wf 7 (14 floats), staging 3 x 8 + 1, faces 1
constexpr int NOALLOC_PER_CELL = 10 + 5 + 11 + 10 + 14 + 5 + 2 + 1 + 14 + 7 + 25 + 1;
constexpr size_t NOALLOC_HEAD = 256;  // work counter, order, problem record
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_HEAD + (size_t)NOALLOC_PER_CELL * NOALLOC_ROW * sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// the message goes to the caller's buffer (no library-held string)
struct ErrBuf {
    char *p;
    size_t len;
    int fail(int code, const char *msg) const {
        if (p && len) {
            strncpy(p, msg, len - 1);
            p[len - 1] = '\0';
        }
        return code;
    }
};

// the static array's device address in the current device's context.  Looked
// up on every call rather than cached: a cudaDeviceReset (or another context
// made current) reloads the module and may move the array, and an address
// kept from before would then point at freed or foreign memory.  Once the
// module is loaded the lookup is a host-side table read and allocates nothing.
int scratch_base(void **out, const ErrBuf &eb) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return eb.fail(CUMC_ECUDA, "no current CUDA device");
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return eb.fail(CUMC_ECUDA, "cudaGetSymbolAddress of the static scratch failed");
    *out = p;
    return CUMC_OK;
}

struct Staging {
    const double *xF;                      // n + 7 faces
    const double *row11, *row01, *row10;  // prim(8, -2:n+3) rows (k,l) = (1,1), (0,1), (1,0)
    const double *eps11;                   // epsilon row (1,1)
    double *out;                           // prim(8, -2:n+3) of the result (reuses row11's slot)
};

// grid metrics, weights and the de-interleaved initial rows
__global__ void k_noalloc_setup(const BatchDev b, const Staging st, int n, int rec, double t_end) {
    const int NX = n + 6;
    double *dx = const_cast<double *>(b.dx);
    double *w = const_cast<double *>(b.w);
    float *wf = const_cast<float *>(b.wf);
    for (int i = threadIdx.x; i < NX; i += blockDim.x) dx[i] = st.xF[i + 1] - st.xF[i];
    __syncthreads();
    const int jlo = (rec == 3 || rec == 4) ? 0 : -1, jhi = (rec == 3 || rec == 4) ? n + 1 : n + 2;
    for (int i = threadIdx.x; i < NX; i += blockDim.x) {
        const int j = i - 2;
        double wl[14];
        if (j >= jlo && j <= jhi) batch_cell_weights(rec, dx, j, wl);
        else for (int m = 0; m < 14; ++m) wl[m] = 0.0;
        for (int m = 0; m < 14; ++m) {
            w[(size_t)i * 14 + m] = wl[m];
            wf[(size_t)i * 14 + m] = (float)wl[m];
        }
        for (int v = 0; v < 5; ++v) b.P[v][i] = st.row11[(size_t)i * 8 + v];
        b.BX[i] = st.row11[(size_t)i * 8 + 5];
        b.BY1[i] = st.row11[(size_t)i * 8 + 6];
        b.BZ1[i] = st.row11[(size_t)i * 8 + 7];
        b.BY0[i] = st.row01[(size_t)i * 8 + 6];
        b.BZ0[i] = st.row10[(size_t)i * 8 + 7];
        b.EPS[i] = st.eps11[i];
    }
    if (threadIdx.x == 0) {
        *const_cast<int *>(b.order) = 0;
        b.prob[0].off = 0;
        b.prob[0].n = n;
        b.prob[0].t_end = t_end;
    }
}

// the result row, interleaved as prim(8, -2:n+3)
__global__ void k_noalloc_pack(const BatchDev b, double *out, int n) {
    for (int i = threadIdx.x; i < n + 6; i += blockDim.x) {
        for (int v = 0; v < 5; ++v) out[(size_t)i * 8 + v] = b.P[v][i];
        out[(size_t)i * 8 + 5] = b.BX[i];
        out[(size_t)i * 8 + 6] = b.BY1[i];
        out[(size_t)i * 8 + 7] = b.BZ1[i];
    }
}

}  // namespace

extern "C" {

int cumc_batch_run1_noalloc(const cumc_batch_config *cfg, const double *prim, const double *eps, int max_steps,
                            void *stream, double *prim_row, double *eps_row, double *t_out, int *steps_out,
                            int *status_out, char *err, size_t err_len) {
    const ErrBuf eb{err, err_len};
    if (err && err_len) err[0] = '\0';
    auto nfail = [&](int code, const char *msg) { return eb.fail(code, msg); };
    if (!cfg || !prim || !eps || !prim_row || !eps_row || !cfg->nx || !cfg->xF || !cfg->t_end || !cfg->xF[0])
        return nfail(CUMC_EINVAL, "null argument");
    if (cfg->n_problems != 1) return nfail(CUMC_EINVAL, "cumc_batch_run1_noalloc runs exactly one problem");
    const int n = cfg->nx[0];
    if (n < 1) return nfail(CUMC_EINVAL, "problem with no zones");
    if (n > NOALLOC_MAX_CELLS)
        return nfail(CUMC_EINVAL, "problem larger than the static scratch: at most 4096 zones without allocation");
    if (cfg->recon < 0 || cfg->recon > 4 || cfg->riemann < 0 || cfg->riemann > 3 || cfg->precision < 0 ||
        cfg->precision > 1)
        return nfail(CUMC_EINVAL, "bad recon/riemann/precision option");
    if (cfg->gamma <= 1.0 || !(cfg->cfl > 0.0)) return nfail(CUMC_EINVAL, "bad gamma or cfl");
    if (cfg->floor_kind != CUMC_FLOOR_NONE && cfg->floor_kind != CUMC_FLOOR_EPS)
        return nfail(CUMC_EINVAL, "batched problems support the none/eps floors");
    if (cudaPeekAtLastError() != cudaSuccess)
        return nfail(CUMC_ECUDA, "a CUDA error is pending from earlier work on this thread (not from this call)");
    void *base = nullptr;
    int rc = scratch_base(&base, eb);
    if (rc != CUMC_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int NX = n + 6;

    // carve the scratch: a head block, then NOALLOC_PER_CELL rows of NOALLOC_ROW doubles
    unsigned char *head = (unsigned char *)base;
    double *cells = (double *)(head + NOALLOC_HEAD);
    int slot = 0;
    auto row = [&]() { return cells + (size_t)(slot++) * NOALLOC_ROW; };
    BatchDev d;
    memset(&d, 0, sizeof d);
    d.nprob = 1;
    d.max_steps = max_steps > 0 ? max_steps : 0x7fffffff;
    d.gamma = cfg->gamma;
    d.cfl = cfg->cfl;
    d.floor_kind = cfg->floor_kind;
    d.pos_fallback = cfg->positivity_fallback ? 1 : 0;
    d.coop_min_n = BATCH_COOP_MIN_N;
    d.next = (int *)head;
    d.order = (const int *)(head + 16);
    d.prob = (BatchProblem *)(head + 64);
    for (int i = 0; i < 5; ++i) d.P[i] = row();
    d.EPS = row(); d.CS = row();
    for (int i = 0; i < 3; ++i) d.BC[i] = row();
    d.BX = row(); d.BY1 = row(); d.BZ1 = row(); d.BY0 = row(); d.BZ0 = row();
    for (int i = 0; i < 5; ++i) d.U[i] = row();
    d.UBX = row(); d.UBXb = row(); d.UBY1 = row(); d.UBZ1 = row(); d.UBY0 = row(); d.UBZ0 = row();
    for (int i = 0; i < 5; ++i) d.O[i] = row();
    d.OBX = row(); d.OBY1 = row(); d.OBZ1 = row(); d.OBY0 = row(); d.OBZ0 = row();
    for (int i = 0; i < 7; ++i) d.QL[i] = row();
    for (int i = 0; i < 7; ++i) d.QR[i] = row();
    for (int i = 0; i < 5; ++i) d.F[i] = row();
    d.EY = row(); d.EZ = row();
    d.dx = row();
    double *w = row();
    slot += 13;  // 14 weights per cell
    d.w = w;
    float *wf = (float *)row();
    slot += 6;   // 14 floats per cell
    d.wf = wf;
    double *stage = row();
    slot += 24;  // 3 prim rows of 8 values per cell + the eps row
    double *xf = row();
    if (slot != NOALLOC_PER_CELL) return nfail(CUMC_EINVAL, "internal scratch layout mismatch");
    Staging st;
    st.row11 = stage;
    st.row01 = stage + (size_t)8 * NOALLOC_ROW;
    st.row10 = stage + (size_t)16 * NOALLOC_ROW;
    st.eps11 = stage + (size_t)24 * NOALLOC_ROW;
    st.xF = xf;
    st.out = stage;

    // clear the whole array: the head (work counter, problem record) and every
    // per-cell row, whatever the problem size (about 3.5 MB, well under a
    // microsecond of HBM time)
    bool ok = cudaMemsetAsync(head, 0, NOALLOC_HEAD, s) == cudaSuccess;
    ok = ok && cudaMemsetAsync(cells, 0, (size_t)NOALLOC_PER_CELL * NOALLOC_ROW * sizeof(double), s) == cudaSuccess;
    // inputs: the three prim rows the 1D kernel reads, the eps row and the faces
    const size_t rowb = (size_t)8 * NX * sizeof(double);
    auto prow = [&](int k, int l) { return prim + (size_t)8 * NX * ((size_t)(k + 2) + 7 * (size_t)(l + 2)); };
    ok = ok && cudaMemcpyAsync((void *)st.row11, prow(1, 1), rowb, cudaMemcpyHostToDevice, s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync((void *)st.row01, prow(0, 1), rowb, cudaMemcpyHostToDevice, s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync((void *)st.row10, prow(1, 0), rowb, cudaMemcpyHostToDevice, s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync((void *)st.eps11, eps + (size_t)NX * (3 + 7 * 3), NX * sizeof(double),
                               cudaMemcpyHostToDevice, s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync((void *)st.xF, cfg->xF[0], (size_t)(n + 7) * sizeof(double), cudaMemcpyHostToDevice,
                               s) == cudaSuccess;
    if (!ok) return nfail(CUMC_ECUDA, "input copy failed");
    k_noalloc_setup<<<1, 256, 0, s>>>(d, st, n, cfg->recon, cfg->t_end[0]);
    if (cudaGetLastError() != cudaSuccess) return nfail(CUMC_ECUDA, "set-up kernel failed to launch");
    // one cluster of BATCH_CLUSTER CTAs; one CTA if a cluster does not fit
    cudaError_t e = cfg->precision == CUMC_FP32
                        ? launch_batch_fp32(d, cfg->recon, cfg->riemann, 1, BATCH_CLUSTER, s)
                        : launch_batch_fp64(d, cfg->recon, cfg->riemann, 1, BATCH_CLUSTER, s);
    if (e == cudaErrorInvalidConfiguration || e == cudaErrorInvalidValue) {
        cudaGetLastError();
        e = cfg->precision == CUMC_FP32 ? launch_batch_fp32(d, cfg->recon, cfg->riemann, 1, 1, s)
                                        : launch_batch_fp64(d, cfg->recon, cfg->riemann, 1, 1, s);
    }
    if (e != cudaSuccess) return nfail(CUMC_ECUDA, "batch kernel failed to launch");
    k_noalloc_pack<<<1, 256, 0, s>>>(d, st.out, n);
    if (cudaGetLastError() != cudaSuccess) return nfail(CUMC_ECUDA, "pack kernel failed to launch");
    BatchProblem pr;
    ok = cudaMemcpyAsync(prim_row, st.out, rowb, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(eps_row, d.EPS, NX * sizeof(double), cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(&pr, d.prob, sizeof pr, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) return nfail(CUMC_ECUDA, "run or result copy failed");
    if (t_out) *t_out = pr.t;
    if (steps_out) *steps_out = pr.steps;
    if (status_out) *status_out = pr.status;
    if (pr.status) return nfail(CUMC_ESTATE, "the problem reached a non-finite or non-positive state");
    return CUMC_OK;
}

}  // extern "C"
