// flux_fp32.cu -- FP32 form: reconstruction, face EOS and Riemann flux in
// single precision (fused multiply-add allowed); fluxes are widened to FP64
// before the FP64 CT / RK accumulation in the stage kernels.
#include "flux_kernel.cuh"
#include "recon_learned.cuh"

namespace cumc {
void launch_flux_fp32(const Dev &d, int dir, int rec, int rs, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
    launch_flux_t<float>(d, dir, rec, rs, grid, block, smem, s);
}
void launch_split_fp32(const Dev &d, int dir, int rec, int rs, cudaStream_t s) {
    launch_split_t<float>(d, dir, rec, rs, s);
}

// tiles of 128 reconstructed cells of one sweep (the learned kernel's CTAs)
long long learned_tiles(const Dev &d, int dir) {
    const long long ex = d.nx + (dir == 0 ? 2 : 0), ey = d.ny + (dir == 1 ? 2 : 0), ez = d.nz + (dir == 2 ? 2 : 0);
    return (ex * ey * ez + 127) / 128;
}

template <int DIR>
static void launch_learned_dir(const Dev &d, int rs, int stage, cudaStream_t s) {
    const unsigned tiles = (unsigned)learned_tiles(d, DIR);
    if (stage == 1) {
        // the network kernel (persistent, 4 CTAs per SM) runs on refresh
        // stages, the staged flag kernel on the others; whichever does not
        // apply exits at once
        const unsigned pg = tiles < (unsigned)(4 * d.num_sms) ? tiles : (unsigned)(4 * d.num_sms);
        if (d.wuni[DIR]) k_recon_learned<DIR, 1, 1><<<pg, 128, 0, s>>>(d, stage);
        else k_recon_learned<DIR, 0, 1><<<pg, 128, 0, s>>>(d, stage);
        k_learned_warps<DIR><<<2 * d.num_sms, dim3(32, 8, 1), 0, s>>>(d, stage);
    }
    const dim3 tb(32, 8, 1);
    if (d.recon_tile == 1) {
        const dim3 g = recon_tile_grid(d, DIR, 1);
        if (d.wuni[DIR]) k_recon_tile<float, DIR, REC_WENO, 1, 1, 1><<<g, tb, 0, s>>>(d, stage);
        else k_recon_tile<float, DIR, REC_WENO, 0, 1, 1><<<g, tb, 0, s>>>(d, stage);
    } else {
        const dim3 g = recon_tile_grid(d, DIR, 2);
        if (d.wuni[DIR]) k_recon_tile<float, DIR, REC_WENO, 1, 2, 1><<<g, tb, 0, s>>>(d, stage);
        else k_recon_tile<float, DIR, REC_WENO, 0, 2, 1><<<g, tb, 0, s>>>(d, stage);
    }
    dim3 g, b;
    split_dims(d, DIR, false, g, b);
    switch (d.riemann_minb) {
        case 4: launch_riemann_m<float, DIR, 4>(d, rs, g, b, s); break;
        case 5: launch_riemann_m<float, DIR, 5>(d, rs, g, b, s); break;
        case 6: launch_riemann_m<float, DIR, 6>(d, rs, g, b, s); break;
        case 14: launch_riemann_pf<float, DIR, 4>(d, rs, s); break;
        case 15: launch_riemann_pf<float, DIR, 5>(d, rs, s); break;
        case 16: launch_riemann_pf<float, DIR, 6>(d, rs, s); break;
        default: launch_riemann_m<float, DIR, 1>(d, rs, g, b, s); break;
    }
}

// the flags-only network kernel of the FP64 form (refresh stages)
template <int DIR>
static void launch_flags_dir(const Dev &d, int stage, cudaStream_t s) {
    const unsigned tiles = (unsigned)learned_tiles(d, DIR);
    const unsigned pg = tiles < (unsigned)(4 * d.num_sms) ? tiles : (unsigned)(4 * d.num_sms);
    if (d.wuni[DIR]) k_recon_learned<DIR, 1, 0><<<pg, 128, 0, s>>>(d, stage);
    else k_recon_learned<DIR, 0, 0><<<pg, 128, 0, s>>>(d, stage);
    k_learned_warps<DIR><<<2 * d.num_sms, dim3(32, 8, 1), 0, s>>>(d, stage);
}
void launch_learned_flags(const Dev &d, int dir, int stage, cudaStream_t s) {
    if (stage != 1) return;
    if (dir == 0) launch_flags_dir<0>(d, stage, s);
    else if (dir == 1) launch_flags_dir<1>(d, stage, s);
    else launch_flags_dir<2>(d, stage, s);
}

void launch_split_learned_fp32(const Dev &d, int dir, int rs, int stage, cudaStream_t s) {
    if (dir == 0) launch_learned_dir<0>(d, rs, stage, s);
    else if (dir == 1) launch_learned_dir<1>(d, rs, stage, s);
    else launch_learned_dir<2>(d, rs, stage, s);
}
}  // namespace cumc
