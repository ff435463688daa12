// batch_host.cu -- C-ABI of the batched 1D engine (cumc_batch_* in
// include/cumc3d_gpu.h).  Packs many 1D problems of uneven size into one set
// of device arrays and runs them in one persistent launch (batch_kernel.cuh).
#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/cumc3d_gpu.h"
#include "batch_kernel.cuh"
#include "weights1d.cuh"

using namespace cumc;

struct cumc_batch {
    BatchDev d;
    int nprob = 0, precision = 0, recon = 0, riemann = 0;
    std::vector<int> n;
    std::vector<long long> off;
    std::vector<double> t_end;
    long long total = 0;
    cudaStream_t stream = nullptr;
    std::vector<void *> allocs;
    std::string err;
    int sm_count = 148;
    int cluster_size = BATCH_CLUSTER;  // CTAs that share one large problem
    int coop_min_n = -1;               // set by cumc_batch_set_cluster; -1: chosen per run
    int64_t launches = 0;
};

static std::string g_batch_err;

static int bfail(cumc_batch *b, int code, const std::string &m) {
    if (b) b->err = m; else g_batch_err = m;
    return code;
}

// PPM/WENO/TVD weights of one axis (same formulas as the 3D handle; the
// per-cell routine is shared with the allocation-free entry point)
static void axis_weights(int rec, int n, const double *xF, double *dx_out, double *w_out) {
    for (int j = -2; j <= n + 3; ++j) dx_out[j + 2] = xF[j + 3] - xF[j + 2];
    for (int j = 0; j < (n + 6) * 14; ++j) w_out[j] = 0.0;
    const int jlo = (rec == 3 || rec == 4) ? 0 : -1, jhi = (rec == 3 || rec == 4) ? n + 1 : n + 2;
    for (int j = jlo; j <= jhi; ++j) batch_cell_weights(rec, dx_out, j, w_out + (size_t)(j + 2) * 14);
}

extern "C" {

int cumc_batch_create(const cumc_batch_config *cfg, cumc_batch **out) {
    if (!cfg || !out || cfg->n_problems <= 0 || !cfg->nx || !cfg->xF || !cfg->t_end)
        return bfail(nullptr, CUMC_EINVAL, "bad batch configuration");
    if (cfg->recon < 0 || cfg->recon > 4 || cfg->riemann < 0 || cfg->riemann > 3 || cfg->precision < 0 || cfg->precision > 1)
        return bfail(nullptr, CUMC_EINVAL, "bad recon/riemann/precision option");
    if (cfg->gamma <= 1.0 || !(cfg->cfl > 0.0)) return bfail(nullptr, CUMC_EINVAL, "bad gamma or cfl");
    if (cfg->floor_kind != CUMC_FLOOR_NONE && cfg->floor_kind != CUMC_FLOOR_EPS)
        return bfail(nullptr, CUMC_EINVAL, "batched problems support the none/eps floors");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return bfail(nullptr, CUMC_ECUDA, "no CUDA device");
    cumc_batch *b = new cumc_batch();
    b->nprob = cfg->n_problems;
    b->precision = cfg->precision;
    b->recon = cfg->recon;
    b->riemann = cfg->riemann;
    b->n.assign(cfg->nx, cfg->nx + cfg->n_problems);
    b->t_end.assign(cfg->t_end, cfg->t_end + cfg->n_problems);
    b->off.resize(b->nprob);
    long long tot = 0;
    for (int p = 0; p < b->nprob; ++p) {
        if (b->n[p] < 1) { delete b; return bfail(nullptr, CUMC_EINVAL, "problem with no zones"); }
        b->off[p] = tot;
        tot += b->n[p] + 6;
    }
    b->total = tot;
    std::vector<double> dx(tot), w((size_t)tot * 14);
    for (int p = 0; p < b->nprob; ++p)
        axis_weights(cfg->recon, b->n[p], cfg->xF[p], &dx[b->off[p]], &w[(size_t)b->off[p] * 14]);
    std::vector<float> wf(w.begin(), w.end());
    // largest problems first: the persistent CTAs then finish close together
    std::vector<int> order(b->nprob);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->n[a] > b->n[c]; });
    std::vector<BatchProblem> prob(b->nprob);
    for (int p = 0; p < b->nprob; ++p) {
        memset(&prob[p], 0, sizeof(BatchProblem));
        prob[p].off = b->off[p];
        prob[p].n = b->n[p];
        prob[p].t_end = b->t_end[p];
    }
    BatchDev &d = b->d;
    memset(&d, 0, sizeof d);
    d.nprob = b->nprob;
    d.max_steps = 0x7fffffff;
    d.gamma = cfg->gamma;
    d.cfl = cfg->cfl;
    d.floor_kind = cfg->floor_kind;
    d.pos_fallback = cfg->positivity_fallback ? 1 : 0;
    d.coop_min_n = BATCH_COOP_MIN_N;
    bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
    auto A = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) { ok = false; return nullptr; }
        cudaMemset(p, 0, bytes);
        b->allocs.push_back(p);
        return p;
    };
    const size_t nb = (size_t)tot * sizeof(double);
    for (int i = 0; i < 5; ++i) { d.P[i] = (double *)A(nb); d.U[i] = (double *)A(nb); d.O[i] = (double *)A(nb); d.F[i] = (double *)A(nb); }
    d.EPS = (double *)A(nb); d.CS = (double *)A(nb);
    for (int i = 0; i < 3; ++i) d.BC[i] = (double *)A(nb);
    d.BX = (double *)A(nb); d.BY1 = (double *)A(nb); d.BZ1 = (double *)A(nb); d.BY0 = (double *)A(nb); d.BZ0 = (double *)A(nb);
    d.UBX = (double *)A(nb); d.UBXb = (double *)A(nb); d.UBY1 = (double *)A(nb); d.UBZ1 = (double *)A(nb); d.UBY0 = (double *)A(nb); d.UBZ0 = (double *)A(nb);
    d.OBX = (double *)A(nb); d.OBY1 = (double *)A(nb); d.OBZ1 = (double *)A(nb); d.OBY0 = (double *)A(nb); d.OBZ0 = (double *)A(nb);
    for (int i = 0; i < 7; ++i) { d.QL[i] = A(nb); d.QR[i] = A(nb); }
    d.EY = (double *)A(nb); d.EZ = (double *)A(nb);
    d.next = (int *)A(sizeof(int));
    int *ord = (int *)A(sizeof(int) * b->nprob);
    d.order = ord;
    d.prob = (BatchProblem *)A(sizeof(BatchProblem) * b->nprob);
    double *ddx = (double *)A(nb), *dw = (double *)A(nb * 14);
    float *dwf = (float *)A((size_t)tot * 14 * sizeof(float));
    d.dx = ddx; d.w = dw; d.wf = dwf;
    if (!ok) { cumc_batch_destroy(b); return bfail(nullptr, CUMC_ENOMEM, "device allocation failed"); }
    cudaMemcpy(ord, order.data(), sizeof(int) * b->nprob, cudaMemcpyHostToDevice);
    cudaMemcpy(d.prob, prob.data(), sizeof(BatchProblem) * b->nprob, cudaMemcpyHostToDevice);
    cudaMemcpy(ddx, dx.data(), nb, cudaMemcpyHostToDevice);
    cudaMemcpy(dw, w.data(), nb * 14, cudaMemcpyHostToDevice);
    cudaMemcpy(dwf, wf.data(), (size_t)tot * 14 * sizeof(float), cudaMemcpyHostToDevice);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (cudaDeviceSynchronize() != cudaSuccess) { cumc_batch_destroy(b); return bfail(nullptr, CUMC_ECUDA, "device setup failed"); }
    *out = b;
    return CUMC_OK;
}

int cumc_batch_destroy(cumc_batch *b) {
    if (!b) return CUMC_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (void *p : b->allocs) cudaFree(p);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return CUMC_OK;
}

const char *cumc_batch_last_error(cumc_batch *b) { return b ? b->err.c_str() : g_batch_err.c_str(); }

// prim/eps of one 1D problem in the reference's layout (8, nx+6, 7, 7) and
// (nx+6, 7, 7): the row (k,l) = (1,1) plus the initial lower y/z faces
int cumc_batch_set_state(cumc_batch *b, int p, const double *prim, const double *eps) {
    if (!b || !prim || !eps || p < 0 || p >= b->nprob) return bfail(b, CUMC_EINVAL, "bad argument");
    const int n = b->n[p], NX = n + 6;
    auto ip = [&](int v, int j, int k, int l) { return (size_t)v + 8 * ((size_t)(j + 2) + NX * ((size_t)(k + 2) + 7 * (size_t)(l + 2))); };
    auto ie = [&](int j, int k, int l) { return (size_t)(j + 2) + NX * ((size_t)(k + 2) + 7 * (size_t)(l + 2)); };
    std::vector<double> row((size_t)NX);
    const long long o = b->off[p];
    auto up = [&](double *dst, int v, int k, int l) {
        for (int j = -2; j <= n + 3; ++j) row[j + 2] = prim[ip(v, j, k, l)];
        return cudaMemcpyAsync(dst + o, row.data(), NX * sizeof(double), cudaMemcpyHostToDevice, b->stream) == cudaSuccess;
    };
    bool ok = true;
    for (int v = 0; v < 5; ++v) ok = ok && up(b->d.P[v], v, 1, 1);
    ok = ok && up(b->d.BX, 5, 1, 1) && up(b->d.BY1, 6, 1, 1) && up(b->d.BZ1, 7, 1, 1);
    ok = ok && up(b->d.BY0, 6, 0, 1) && up(b->d.BZ0, 7, 1, 0);
    for (int j = -2; j <= n + 3; ++j) row[j + 2] = eps[ie(j, 1, 1)];
    ok = ok && cudaMemcpyAsync(b->d.EPS + o, row.data(), NX * sizeof(double), cudaMemcpyHostToDevice, b->stream) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(b->stream) == cudaSuccess;
    return ok ? CUMC_OK : bfail(b, CUMC_ECUDA, "state upload failed");
}

int cumc_batch_get_state(cumc_batch *b, int p, double *prim_row, double *eps_row) {
    if (!b || !prim_row || !eps_row || p < 0 || p >= b->nprob) return bfail(b, CUMC_EINVAL, "bad argument");
    const int n = b->n[p], NX = n + 6;
    const long long o = b->off[p];
    std::vector<double> row(NX);
    double *src[8] = {b->d.P[0], b->d.P[1], b->d.P[2], b->d.P[3], b->d.P[4], b->d.BX, b->d.BY1, b->d.BZ1};
    for (int v = 0; v < 8; ++v) {
        if (cudaMemcpy(row.data(), src[v] + o, NX * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return bfail(b, CUMC_ECUDA, "download failed");
        for (int j = 0; j < NX; ++j) prim_row[(size_t)j * 8 + v] = row[j];
    }
    if (cudaMemcpy(eps_row, b->d.EPS + o, NX * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return bfail(b, CUMC_ECUDA, "download failed");
    return CUMC_OK;
}

int cumc_batch_run(cumc_batch *b, int max_steps, double *t_out, int *steps_out, int *status_out) {
    if (!b) return bfail(b, CUMC_EINVAL, "null batch");
    b->d.max_steps = max_steps > 0 ? max_steps : 0x7fffffff;
    if (cudaMemsetAsync(b->d.next, 0, sizeof(int), b->stream) != cudaSuccess) return bfail(b, CUMC_ECUDA, "memset failed");
    // sharing threshold: a batch no larger than the clusters that can be
    // resident at once (two 256-thread CTAs per SM) leaves SMs idle, so its
    // problems are shared from 256 cells up (one cell per thread and fewer
    // steps' worth of latency); a larger one shares only its largest problems
    if (b->coop_min_n < 0) {
        const int resident = b->cluster_size > 1 ? 2 * b->sm_count / b->cluster_size : 2 * b->sm_count;
        b->d.coop_min_n = b->nprob <= resident ? BATCH_COOP_MIN_N_FEW : BATCH_COOP_MIN_N;
    } else {
        b->d.coop_min_n = b->coop_min_n;
    }
    cudaError_t e = b->precision == CUMC_FP32
                        ? launch_batch_fp32(b->d, b->recon, b->riemann, 0, b->cluster_size, b->stream)
                        : launch_batch_fp64(b->d, b->recon, b->riemann, 0, b->cluster_size, b->stream);
    if (e == cudaErrorInvalidConfiguration || e == cudaErrorInvalidValue) {
        cudaGetLastError();  // no room for a cluster: one CTA per problem
        e = b->precision == CUMC_FP32 ? launch_batch_fp32(b->d, b->recon, b->riemann, 0, 1, b->stream)
                                      : launch_batch_fp64(b->d, b->recon, b->riemann, 0, 1, b->stream);
    }
    if (e != cudaSuccess) return bfail(b, CUMC_ECUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    b->launches++;
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(b->stream) != cudaSuccess)
        return bfail(b, CUMC_ECUDA, "batch kernel failed");
    std::vector<BatchProblem> prob(b->nprob);
    cudaMemcpy(prob.data(), b->d.prob, sizeof(BatchProblem) * b->nprob, cudaMemcpyDeviceToHost);
    int bad = 0;
    for (int p = 0; p < b->nprob; ++p) {
        if (t_out) t_out[p] = prob[p].t;
        if (steps_out) steps_out[p] = prob[p].steps;
        if (status_out) status_out[p] = prob[p].status;
        if (prob[p].status) bad++;
    }
    if (bad) return bfail(b, CUMC_ESTATE, std::to_string(bad) + " problem(s) reached a non-finite or non-positive state");
    return CUMC_OK;
}

int cumc_batch_set_cluster(cumc_batch *b, int cluster_size, int coop_min_n) {
    if (!b) return bfail(b, CUMC_EINVAL, "null batch");
    if ((cluster_size != 1 && cluster_size != 2 && cluster_size != 4 && cluster_size != 8 && cluster_size != 16) ||
        coop_min_n < 1)
        return bfail(b, CUMC_EINVAL, "cluster size must be 1, 2, 4, 8 or 16 and coop_min_n >= 1");
    b->cluster_size = cluster_size;
    b->coop_min_n = coop_min_n;
    return CUMC_OK;
}

int cumc_batch_sync(cumc_batch *b) {
    if (!b) return CUMC_EINVAL;
    return cudaStreamSynchronize(b->stream) == cudaSuccess ? CUMC_OK : CUMC_ECUDA;
}

void *cumc_batch_stream(cumc_batch *b) { return b ? (void *)b->stream : nullptr; }
int64_t cumc_batch_launch_count(cumc_batch *b) { return b ? b->launches : 0; }

}  // extern "C"
