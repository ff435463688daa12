// recon_tile.cuh -- face reconstruction with the stencils staged in shared
// memory.  Same cells, same arithmetic (recon_cell) and the same outputs as
// k_recon; each state value of the tile is loaded from HBM once, coalesced
// along x, and converted to T once, instead of once per stencil that uses it.
//
// CTA = 32 x 8 threads.  Tile:
//   x sweep (DIR 0): 32 cells along x  x  8*CPT rows along y, halo H in x;
//   y/z sweep:       32 cells along x  x  8*CPT cells along the sweep,
//                    halo H rows along the sweep;
// H = 2 for the 5-point stencils (PPM, WENO), 1 for TVD.  CPT (cells per
// thread, 1 or 2) trades halo overhead for registers; the autotuner picks.
#pragma once
#include "../../include/cumc3d_gpu.h"
#include "engine.cuh"
#include "mhd_device.cuh"

namespace cumc {

// LRN = 1 (FP32 WENO with the learned flag, stages the network does not
// run) or 2 (FP64 WENO with the learned flag, every stage; the network only
// sets the flags): a warp whose 32 cells carry the stored flag, dilated by
// two cells along the sweep, in 128-cell tiles not marked to fall back,
// reconstructs with the linear optimal weights (recon_learned.cuh); the
// decision is made once per refresh, per warp (k_learned_warps).  With no
// cell flagged the arithmetic is that of LRN = 0.
__device__ __forceinline__ bool learned_refresh_stage(const Dev &d, int stage) {
    return stage == 1 && (d.flag_interval <= 1 || (d.S->steps % d.flag_interval) == 0);
}

// grid of the tiled reconstruction for one sweep
__host__ __device__ inline dim3 recon_tile_grid(const Dev &d, int dir, int cpt) {
    const int nr = 8 * cpt;
    if (dir == 0) return dim3((d.nx + 2 + 31) / 32, (d.ny + nr - 1) / nr, d.nz);
    if (dir == 1) return dim3((d.nx + 31) / 32, (d.ny + 2 + nr - 1) / nr, d.nz);
    return dim3((d.nx + 31) / 32, (d.nz + 2 + nr - 1) / nr, d.ny);
}

// The index of the warp of the staged reconstruction (learned_warps in
// engine.cuh) with x-chunk bx, sweep cell c (DIR 1, 2) or row k (DIR 0) and
// the remaining coordinate o (l for DIR 0 and 1, k for DIR 2).
template <int DIR>
__device__ __forceinline__ long long learned_warp(const Dev &d, int bx, int c, int o) {
    const long long nxc = learned_warp_nx(d, DIR);
    if (DIR == 0) return bx + nxc * ((c - 1) + (long long)d.ny * (o - 1));
    if (DIR == 1) return bx + nxc * (c + (long long)(d.ny + 2) * (o - 1));
    return bx + nxc * ((o - 1) + (long long)d.ny * c);
}

// After the flag network (refresh stages only): the linear decision of every
// warp of the staged reconstruction, from the flags of its 32 cells and of
// their neighbours within two cells along the sweep and from the per-tile
// fallback marks -- the test the staged kernel would otherwise make per cell
// with five flag loads.  A small persistent grid of 32 x 8 blocks walks the
// blocks of recon_tile_grid(d, DIR, 1), so that on the other stages (the
// kernel sits in every captured step) it costs only its early exit.
template <int DIR>
__global__ void __launch_bounds__(256) k_learned_warps(const Dev d, int stage) {
    if (d.S->done || !learned_refresh_stage(d, stage)) return;
    const dim3 tg = recon_tile_grid(d, DIR, 1);
    const long long nblk = (long long)tg.x * tg.y * tg.z;
    const int tx = threadIdx.x, r = threadIdx.y;
    for (long long bid = blockIdx.x; bid < nblk; bid += gridDim.x) {
        const int bx = (int)(bid % tg.x);
        const long long rest = bid / tg.x;
        const int by = (int)(rest % tg.y), bz = (int)(rest / tg.y);
        const int c0 = (DIR == 0) ? bx * 32 : by * 8;
        int c, j, k, l, ns, o;
        bool valid, row;
        if (DIR == 0) {
            c = c0 + tx; j = c; k = by * 8 + r + 1; l = bz + 1; ns = d.nx; o = l;
            valid = c <= d.nx + 1 && k <= d.ny;
            row = k <= d.ny;
        } else if (DIR == 1) {
            c = c0 + r; k = c; j = bx * 32 + tx + 1; l = bz + 1; ns = d.ny; o = l;
            valid = j <= d.nx && c <= d.ny + 1;
            row = c <= d.ny + 1;
        } else {
            c = c0 + r; l = c; j = bx * 32 + tx + 1; k = bz + 1; ns = d.nz; o = k;
            valid = j <= d.nx && c <= d.nz + 1;
            row = c <= d.nz + 1;
        }
        bool ok = false;
        if (valid && c >= 2 && c <= ns - 1) {
            long long t, sweep;
            if (DIR == 0) { t = c + (long long)(d.nx + 2) * ((k - 1) + (long long)d.ny * (l - 1)); sweep = 1; }
            else if (DIR == 1) { t = (j - 1) + (long long)d.nx * (c + (long long)(d.ny + 2) * (l - 1)); sweep = d.nx; }
            else { t = (j - 1) + (long long)d.nx * ((k - 1) + (long long)d.ny * c); sweep = (long long)d.nx * d.ny; }
            const unsigned char *f = d.lflag[DIR];
            // c-2 .. c+2 lie within 0 .. n+1, the cells of the enumeration
            ok = f[t] && f[t - sweep] && f[t + sweep] && f[t - 2 * sweep] && f[t + 2 * sweep] &&
                 d.lfb[DIR][t >> 7] == 0;
        }
        const bool all = __all_sync(0xffffffffu, ok);
        if (tx == 0 && row) d.lwarp[DIR][learned_warp<DIR>(d, bx, (DIR == 0) ? k : c, o)] = all ? 1 : 0;
    }
}

// The reconstruction of the cells of one staged tile (block coordinates bx,
// by, bz of recon_tile_grid).  The tile lies in shared memory as 7 slots of
// SLOT elements, each SR rows of SX values; the stencil of the cell in row r,
// lane tx sits at column tx + HO + m (x sweep) or row r + HO + m, column
// tx + XO (y, z sweeps), m = -H..H.
template <class T, int DIR, int REC, int UNI, int CPT, int LRN, int SX, int SLOT, int HO, int XO>
__device__ __forceinline__ void recon_tile_cells(const Dev &d, const T *__restrict__ s, int bx, int by, int bz, int tx,
                                                 int ty) {
    constexpr int TX = 32, TY = 8;
    constexpr int H = (REC == REC_PPM || REC == REC_WENO) ? 2 : 1;
    constexpr int NR = TY * CPT;
    const int c0 = (DIR == 0) ? bx * TX : by * NR;  // first reconstructed cell
    T *const *QL = reinterpret_cast<T *const *>(d.QL);
    T *const *QR = reinterpret_cast<T *const *>(d.QR);
    const int st = (DIR == 0) ? 1 : (DIR == 1) ? d.NX : d.NX * d.NY;
#pragma unroll
    for (int i = 0; i < CPT; ++i) {
        const int r = ty + TY * i;  // row within the tile
        int c, j, k, l, ns;
        bool valid;
        if (DIR == 0) {
            c = c0 + tx; j = c; k = by * NR + r + 1; l = bz + 1; ns = d.nx;
            valid = c <= d.nx + 1 && k <= d.ny;
        } else if (DIR == 1) {
            c = c0 + r; k = c; j = bx * TX + tx + 1; l = bz + 1; ns = d.ny;
            valid = j <= d.nx && c <= d.ny + 1;
        } else {
            c = c0 + r; l = c; j = bx * TX + tx + 1; k = bz + 1; ns = d.nz;
            valid = j <= d.nx && c <= d.nz + 1;
        }
        bool linear = false;
        if (LRN) {
            // the warp's decision, made once per refresh by k_learned_warps;
            // audit steps reconstruct with WENO-Z everywhere
            const bool row = (DIR == 0) ? k <= d.ny : (DIR == 1) ? c <= d.ny + 1 : c <= d.nz + 1;
            const bool audit = d.audit_interval > 0 && (d.S->steps % d.audit_interval) == 0;
            if (row && !audit) linear = d.lwarp[DIR][learned_warp<DIR>(d, bx, DIR == 0 ? k : c, DIR == 2 ? k : l)] != 0;
        }
        if (!valid) continue;
        const int ci = cidx(d, j, k, l);
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
        T vm_rho = T(0), vp_rho = T(0);
        bool fallback = false;
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            // the stencil c-H .. c+H of variable v
            auto at = [&](int m) -> T {
                return (DIR == 0) ? s[v * SLOT + r * SX + tx + HO + m] : s[v * SLOT + (r + HO + m) * SX + tx + XO];
            };
            T a0 = T(0), a4 = T(0);
            if (H == 2) { a0 = at(-2); a4 = at(2); }
            const T a1 = at(-1), a2 = at(0), a3 = at(1);
            T vm, vp;
            if (LRN && linear) weno_linear<T>(w, a0, a1, a2, a3, a4, vm, vp);
            else recon_cell<T, REC>(w, a0, a1, a2, a3, a4, vm, vp);
            if (v == 0) { vm_rho = vm; vp_rho = vp; }
            if (v == 4 && d.pos_fallback) {
                fallback = !(vm_rho > T(0) && vp_rho > T(0) && vm > T(0) && vp > T(0));
                if (fallback && d.fb_count) atomicAdd(d.fb_count, 1ull);
                if (fallback) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const T cv = (DIR == 0) ? s[u * SLOT + r * SX + tx + HO] : s[u * SLOT + (r + HO) * SX + tx + XO];
                        if (c <= ns) QL[u][ci] = cv;
                        if (c >= 1) QR[u][ci - st] = cv;
                    }
                }
            }
            if (fallback) vm = vp = a2;
            if (c <= ns) QL[v][ci] = vp;      // left state of face c
            if (c >= 1) QR[v][ci - st] = vm;  // right state of face c-1
        }
    }
}

// MINB: blocks per SM the register budget is sized for (1: the compiler's
// choice, about 76 registers for FP64 WENO-Z; 4: 64 registers, a third more
// resident warps)
template <class T, int DIR, int REC, int UNI, int CPT, int LRN = 0, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) k_recon_tile(const Dev d, int stage = 0) {
    if (d.S->done) return;
    if (LRN == 1 && learned_refresh_stage(d, stage)) return;  // the network kernel reconstructs this stage
    constexpr int TX = 32, TY = 8;
    constexpr int H = (REC == REC_PPM || REC == REC_WENO) ? 2 : 1;
    constexpr int NR = TY * CPT;                    // rows of reconstructed cells
    constexpr int SX = (DIR == 0) ? TX + 2 * H : TX;  // staged row length
    constexpr int SR = (DIR == 0) ? NR : NR + 2 * H;  // staged rows
    __shared__ T s[7 * SR * SX];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * TX + tx;
    constexpr int tb1 = (DIR == 0) ? 1 : 0;
    constexpr int tb2 = (DIR == 2) ? 1 : 2;

    // ---- stage the tile ----
    const int c0 = (DIR == 0) ? blockIdx.x * TX : blockIdx.y * NR;  // first reconstructed cell
    for (int idx = tid; idx < SR * SX; idx += TX * TY) {
        const int sr = idx / SX, sx = idx - sr * SX;
        int x, y, z;
        bool ok;
        if (DIR == 0) {
            x = c0 - H + sx; y = blockIdx.y * NR + sr + 1; z = blockIdx.z + 1;
            ok = x <= d.nx + 3 && y <= d.ny;
        } else if (DIR == 1) {
            x = blockIdx.x * TX + sx + 1; y = c0 - H + sr; z = blockIdx.z + 1;
            ok = x <= d.nx && y <= d.ny + 3;
        } else {
            x = blockIdx.x * TX + sx + 1; y = blockIdx.z + 1; z = c0 - H + sr;
            ok = x <= d.nx && z <= d.nz + 3;
        }
        if (ok) {
            const int ci = cidx(d, x, y, z);
#pragma unroll
            for (int v = 0; v < 7; ++v) {
                const double *src = (v < 5) ? d.P[v] : d.BC[v == 5 ? tb1 : tb2];
                s[v * SR * SX + sr * SX + sx] = (T)__ldg(src + ci);
            }
        }
    }
    __syncthreads();
    recon_tile_cells<T, DIR, REC, UNI, CPT, LRN, SX, SR * SX, H, 0>(d, s, blockIdx.x, blockIdx.y, blockIdx.z, tx, ty);
}

// ---------------------------------------------------------------------------
// The same reconstruction with the tiles staged by the tensor memory
// accelerator (FP64 form, one cell per thread): persistent CTAs walk the
// tiles of recon_tile_grid; while a CTA reconstructs one tile from shared
// memory, TMA loads the next into the other buffer (cp.async.bulk.tensor,
// one 3D box per staged array, completion on an mbarrier).  The tensor maps
// (TmaMaps, one per staged array: the five hydro primitives and the two
// transverse cell fields of the sweep) cover this GPU's own state arrays;
// no multicast.  Boxes start on even x (16-byte aligned): the x sweep loads
// cells c0-2 .. c0+33 whatever the stencil's halo, the y and z sweeps cells
// 32 bx .. 32 bx + 33 (one column before the tile's first).  Cells outside
// the padded grid come back as zeros and are never used.  A wait that does
// not complete within a bound sets the device error word and the CTA skips
// the tile, then waits (bounded) for its copies still in flight before
// exiting.
// ---------------------------------------------------------------------------
template <int DIR>
struct TmaBox {
    static constexpr int SX = (DIR == 0) ? 36 : 34;          // box x extent
    static constexpr int SR = (DIR == 0) ? 8 : 12;           // box rows (y for DIR 0, 1; z for DIR 2)
    static constexpr int BYTES = SX * SR * 8;                // one array's box
    static constexpr int SLOT = ((BYTES + 127) / 128) * 128 / 8;  // doubles per 128-byte aligned slot
    static constexpr int SMEM = 2 * 7 * SLOT * 8 + 128;      // two buffers of seven slots, 128-byte aligned
};

__device__ __forceinline__ unsigned tma_smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned phase) {
    for (int it = 0; it < (1 << 22); ++it) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(bar), "r"(phase)
                     : "memory");
        if (done) return true;
    }
    return false;
}

template <int DIR>
__device__ __forceinline__ void tma_issue(const TmaMaps &maps, double *buf, unsigned bar, int bx, int by, int bz) {
    using B = TmaBox<DIR>;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(7 * B::BYTES) : "memory");
    int x, y, z;  // padded indices of the box's first element
    if (DIR == 0) { x = bx * 32; y = by * 8 + 3; z = bz + 3; }
    else if (DIR == 1) { x = bx * 32 + 2; y = by * 8; z = bz + 3; }
    else { x = bx * 32 + 2; y = bz + 3; z = by * 8; }
#pragma unroll
    for (int v = 0; v < 7; ++v) {
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
                tma_smem_addr(buf + v * B::SLOT)),
            "l"(reinterpret_cast<unsigned long long>(&maps.m[v])), "r"(x), "r"(y), "r"(z), "r"(bar)
            : "memory");
    }
}

template <int DIR, int REC, int UNI>
__global__ void __launch_bounds__(256) k_recon_tma(const Dev d, const __grid_constant__ TmaMaps maps) {
    if (d.S->done) return;
    using B = TmaBox<DIR>;
    extern __shared__ __align__(16) unsigned char tma_raw[];
    // TMA destinations must start on 128-byte boundaries
    double *const tma_smem = reinterpret_cast<double *>((reinterpret_cast<uintptr_t>(tma_raw) + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) unsigned long long bar[2];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const dim3 tg = recon_tile_grid(d, DIR, 1);
    const long long ntiles = (long long)tg.x * tg.y * tg.z;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tma_smem_addr(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tma_smem_addr(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    auto coords = [&](long long t, int &bx, int &by, int &bz) {
        bx = (int)(t % tg.x);
        const long long rest = t / tg.x;
        by = (int)(rest % tg.y);
        bz = (int)(rest / tg.y);
    };
    unsigned phase[2] = {0u, 0u};
    int issued[2] = {0, 0};  // copies issued into each buffer and not yet waited for (thread 0)
    long long t = blockIdx.x;
    if (t < ntiles && tid == 0) {
        int bx, by, bz;
        coords(t, bx, by, bz);
        tma_issue<DIR>(maps, tma_smem, tma_smem_addr(&bar[0]), bx, by, bz);
        issued[0] = 1;
    }
    bool failed = false;
    for (int i = 0; t < ntiles; ++i, t += gridDim.x) {
        const int b = i & 1;
        const long long tn = t + gridDim.x;
        if (tn < ntiles && tid == 0 && !failed) {  // the next tile into the other buffer
            int bx, by, bz;
            coords(tn, bx, by, bz);
            tma_issue<DIR>(maps, tma_smem + (b ^ 1) * 7 * B::SLOT, tma_smem_addr(&bar[b ^ 1]), bx, by, bz);
            issued[b ^ 1] = 1;
        }
        const bool ok = !failed && mbar_wait_bounded(tma_smem_addr(&bar[b]), phase[b]);
        if (ok) {
            phase[b] ^= 1u;
            if (tid == 0) issued[b] = 0;
        } else if (!failed) {
            failed = true;
            if (atomicCAS(&d.S->err_code, 0, CUMC_ECUDA) == 0) d.S->err_stage = 100 + DIR;
        }
        if (ok) {
            int bx, by, bz;
            coords(t, bx, by, bz);
            recon_tile_cells<double, DIR, REC, UNI, 1, 0, B::SX, B::SLOT, 2, (DIR == 0) ? 0 : 1>(
                d, tma_smem + b * 7 * B::SLOT, bx, by, bz, tx, ty);
        }
        __syncthreads();  // every thread is done with buffer b before it is refilled
    }
    // copies still in flight after a failed wait: wait for them (bounded)
    if (tid == 0) {
        for (int b = 0; b < 2; ++b)
            if (issued[b]) mbar_wait_bounded(tma_smem_addr(&bar[b]), phase[b]);
    }
}

}  // namespace cumc
