// flux_fp64.cu -- FP64 (plain form) instantiations of the fused face-flux
// kernel.  Built with --fmad=false: each expression keeps the reference's
// rounding sequence, so results match the Fortran semantics bit for bit.
#include "flux_kernel.cuh"

namespace cumc {
void launch_flux_fp64(const Dev &d, int dir, int rec, int rs, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
    launch_flux_t<double>(d, dir, rec, rs, grid, block, smem, s);
}
void launch_split_fp64(const Dev &d, int dir, int rec, int rs, cudaStream_t s) {
    launch_split_t<double>(d, dir, rec, rs, s);
}
}  // namespace cumc
