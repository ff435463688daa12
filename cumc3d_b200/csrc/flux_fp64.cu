// flux_fp64.cu -- FP64 instantiations of the face-flux kernels (plain form,
// and the FP64 form with the learned flag).  Built with --fmad=false: each expression keeps the reference's
// rounding sequence, so results match the Fortran semantics bit for bit.
#include "flux_kernel.cuh"

namespace cumc {
void launch_flux_fp64(const Dev &d, int dir, int rec, int rs, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
    launch_flux_t<double>(d, dir, rec, rs, grid, block, smem, s);
}
void launch_split_fp64(const Dev &d, int dir, int rec, int rs, cudaStream_t s, const TmaMaps *tma) {
    launch_split_t<double>(d, dir, rec, rs, s, tma);
}

// FP64 WENO with the learned flag: the network (FP32 unit) sets the flags on
// refresh stages, the staged FP64 reconstruction uses them on every stage
template <int DIR>
static void launch_learned64_dir(const Dev &d, int rs, int stage, cudaStream_t s) {
    launch_learned_flags(d, DIR, stage, s);
    const dim3 tb(32, 8, 1);
    if (d.recon_tile == 2) {
        const dim3 g = recon_tile_grid(d, DIR, 2);
        if (d.wuni[DIR]) k_recon_tile<double, DIR, REC_WENO, 1, 2, 2><<<g, tb, 0, s>>>(d, stage);
        else k_recon_tile<double, DIR, REC_WENO, 0, 2, 2><<<g, tb, 0, s>>>(d, stage);
    } else {
        const dim3 g = recon_tile_grid(d, DIR, 1);
        if (d.wuni[DIR]) k_recon_tile<double, DIR, REC_WENO, 1, 1, 2><<<g, tb, 0, s>>>(d, stage);
        else k_recon_tile<double, DIR, REC_WENO, 0, 1, 2><<<g, tb, 0, s>>>(d, stage);
    }
    dim3 g, b;
    split_dims(d, DIR, false, g, b);
    switch (d.riemann_minb) {
        case 4: launch_riemann_m<double, DIR, 4>(d, rs, g, b, s); break;
        case 5: launch_riemann_m<double, DIR, 5>(d, rs, g, b, s); break;
        case 6: launch_riemann_m<double, DIR, 6>(d, rs, g, b, s); break;
        case 14: launch_riemann_pf<double, DIR, 4>(d, rs, s); break;
        case 15: launch_riemann_pf<double, DIR, 5>(d, rs, s); break;
        case 16: launch_riemann_pf<double, DIR, 6>(d, rs, s); break;
        default: launch_riemann_m<double, DIR, 1>(d, rs, g, b, s); break;
    }
}
void launch_split_learned_fp64(const Dev &d, int dir, int rs, int stage, cudaStream_t s) {
    if (dir == 0) launch_learned64_dir<0>(d, rs, stage, s);
    else if (dir == 1) launch_learned64_dir<1>(d, rs, stage, s);
    else launch_learned64_dir<2>(d, rs, stage, s);
}
}  // namespace cumc
