// engine.cuh -- device-side layout of one solver instance.
//
// State lives in HBM as structure-of-arrays: every variable is its own
// padded (nx+6)*(ny+6)*(nz+6) double array with x fastest, so a warp reading
// 32 consecutive cells of one variable issues fully coalesced 256-byte
// transactions.  Index (j,k,l), j in -2..nx+3, maps to
// (j+2) + NX*((k+2) + NY*(l+2)), the padded extents of the reference's
// arrays (solver/mhd/setup.f90:348-375).
#pragma once
#include <cuda.h>  // CUtensorMap (the type only; the encoder is fetched at run time)
#include <cuda_runtime.h>
#include <stdint.h>

namespace cumc {

// tensor maps of the seven arrays the reconstruction of one sweep stages (the
// five hydro primitives, the two transverse cell fields), for the TMA-staged
// reconstruction (recon_tile.cuh, k_recon_tma)
struct TmaMaps {
    CUtensorMap m[7];
};

// device-resident scalars of the time loop (solver/mhd/main.f90:98-116)
struct Scalars {
    double dt;                   // step size used by the RK stages
    double t;                    // global_time
    double t_end;                // total_time
    unsigned long long dt_bits;  // FINDDT min-reduction target (bits of a positive double)
    int steps;                   // steps taken in the current evolve call
    int max_steps;
    int done;                    // set when t >= t_end or steps >= max_steps
    int err_code;                // first guard failure (0 = none)
    int err_cell;                // padded linear index of that cell
    int err_stage;
    int pad[2];
    // the collapsar model's black hole: mass, its value at the step's start,
    // the pseudo-Newtonian radius 2 m_bh / c^2
    double m_bh, mbh_old, r_sh;
};

struct Dev {
    int nx, ny, nz, n_dim, coord;
    int NX, NY, NZ;
    int N3;
    int bf[6];              // boundary_flag
    int eps_y_out_mode;     // BOUNDARY1D_NM y-outer rule for epsilon (boundary.f90:243)
    int fixn;               // carry periodic normal faces
    int pos_fallback;       // first-order fallback for non-positive edge rho/p
    int tpb_recon, tpb_riemann;  // threads per block of the split flux kernels (autotuned)
    int riemann_minb;            // blocks/SM the Riemann kernel is compiled for (1, 4, 5, 6; 14, 15, 16:
                                 // the prefetching kernel at 4, 5, 6; autotuned)
    int recon_tile;              // 0: per-cell stencil loads; 1, 2: staged tiles, cells per thread (autotuned)
    int wuni[3];                 // 1: the axis's reconstruction weights are identical in every cell
    double wu[3][14];            // those weights (FP64 form)
    float wuf[3][14];            // and in FP32
    signed char bfac[6][12];  // parity per side (xin,xout,yin,yout,zin,zout) and variable 1..11
    double gamma, cfl;
    int floor_kind, source_kind, bc_kind;
    int zcut[2];            // z side (lower, upper) shared with a neighbouring slab: 1 a cut
                            // interior to the whole grid, 2 the seam of a periodic ring
    double rho_floor, eps_floor, p_floor, g_const, r_sh;

    double *P[8];   // prim
    double *U[8];   // cons
    double *U0[8];  // u_old
    double *EPS, *CS;
    double *BC[3];  // bcell
    double *FX[5], *FY[5], *FZ[5];  // hydro face fluxes per direction
    double *EF[6];  // face EMFs (yx, zx, xy, zy, xz, yz)
    double *EC[3];  // cell EMFs
    double *EX, *EY, *EZ;  // edge EMFs
    void *QL[7], *QR[7];   // face states of the split flux path (double or float)

    // grid metrics (getgrid.f90), offsets: cells +2, faces +3
    const double *x, *dx, *xF, *xbar, *dx_cb;
    const double *y, *dy, *yF, *sine, *sinf, *dcose, *dsine;
    const double *z, *dz, *zF;
    const double *wx, *wy, *wz;  // reconstruction weights, 14 per cell
    const float *wxf, *wyf, *wzf;
    Scalars *S;

    // learned smooth-face flag of the FP32 WENO form (learned.cuh)
    int learned;                 // 1: the learned reconstruction kernel replaces k_recon
    float learn_thr;             // logit above which a cell is flagged smooth
    int flag_interval;           // the network runs every this many steps (stage 1)
    int num_sms;                 // persistent grids
    int audit_interval;          // full-WENO audit every this many steps (0: never)
    float audit_tol;             // relative face-value error a tile may show
    const void *mlp;             // MlpPacked parameters
    unsigned char *lfb[3];       // per direction, per 128-cell tile: 1 = fall back to WENO-Z
    unsigned char *lflag[3];     // per direction, per reconstructed cell: the stage-1 flag
    unsigned char *lwarp[3];     // per direction, per warp of the staged reconstruction: 1 = linear
    // the collapsar model: the self-gravity potential (colour-split, see
    // poisson.cuh; null until cumc_poisson_setup) and c in code units
    const double *phi[2];
    int phx;
    double c_code;
    unsigned long long *lstats;  // audit counters (LEARN_STAT_SLOTS x LEARN_STAT_FIELDS)
    // cells whose reconstruction took the positivity fallback, summed over
    // sweeps and stages (null: not counted; cumc_fallback_count)
    unsigned long long *fb_count;
};

__device__ __forceinline__ int cidx(const Dev &d, int j, int k, int l) {
    return (j + 2) + d.NX * ((k + 2) + d.NY * (l + 2));
}

// (a, b, e) of a flat index t = a + ex (b + ey e).  Every flat count of a
// grid the engine accepts fits 32 bits (its padded cells times 8 stay below
// 2^31), so the divisions are 32-bit ones, several times cheaper than the
// 64-bit division routine.
__device__ __forceinline__ void unflat3(unsigned t, unsigned ex, unsigned ey, int &a, int &b, int &e) {
    const unsigned r = t / ex;
    a = (int)(t - r * ex);
    const unsigned q = r / ey;
    b = (int)(r - q * ey);
    e = (int)q;
}

// host-side launchers of the face-flux kernels (one per precision unit)
void launch_flux_fp64(const Dev &d, int dir, int rec, int rs, dim3 grid, dim3 block, size_t smem, cudaStream_t s);
void launch_flux_fp32(const Dev &d, int dir, int rec, int rs, dim3 grid, dim3 block, size_t smem, cudaStream_t s);
void launch_split_fp64(const Dev &d, int dir, int rec, int rs, cudaStream_t s, const TmaMaps *tma = nullptr);
void launch_split_fp32(const Dev &d, int dir, int rec, int rs, cudaStream_t s);
void launch_split_learned_fp32(const Dev &d, int dir, int rs, int stage, cudaStream_t s);
void launch_split_learned_fp64(const Dev &d, int dir, int rs, int stage, cudaStream_t s);
void launch_learned_flags(const Dev &d, int dir, int stage, cudaStream_t s);
long long learned_tiles(const Dev &d, int dir);
// The warps of the staged reconstruction (a warp = 32 consecutive x-cells of
// one row of the tile, for every cells-per-thread): their number along x and
// in all, per sweep direction.
__device__ __host__ __forceinline__ int learned_warp_nx(const Dev &d, int dir) {
    return dir == 0 ? (d.nx + 2 + 31) / 32 : (d.nx + 31) / 32;
}
__device__ __host__ __forceinline__ long long learned_warps(const Dev &d, int dir) {
    const long long nxc = learned_warp_nx(d, dir);
    if (dir == 0) return nxc * d.ny * d.nz;
    if (dir == 1) return nxc * (d.ny + 2) * d.nz;
    return nxc * d.ny * (d.nz + 2);
}

}  // namespace cumc
