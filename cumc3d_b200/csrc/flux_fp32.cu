// flux_fp32.cu -- FP32 form: reconstruction, face EOS and Riemann flux in
// single precision (fused multiply-add allowed); fluxes are widened to FP64
// before the FP64 CT / RK accumulation in the stage kernels.
#include "flux_kernel.cuh"

namespace cumc {
void launch_flux_fp32(const Dev &d, int dir, int rec, int rs, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
    launch_flux_t<float>(d, dir, rec, rs, grid, block, smem, s);
}
void launch_split_fp32(const Dev &d, int dir, int rec, int rs, cudaStream_t s) {
    launch_split_t<float>(d, dir, rec, rs, s);
}
}  // namespace cumc
