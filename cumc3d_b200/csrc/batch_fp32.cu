// batch_fp32.cu -- FP32-form instantiations of the batched 1D kernel: FP32
// reconstruction and Riemann flux, FP64 accumulation / CT / recovery / dt.
#include "batch_kernel.cuh"

namespace cumc {
cudaError_t launch_batch_fp32(const BatchDev &b, int rec, int rs, int clusters, int cluster_size, cudaStream_t s) {
    return launch_batch_t<float>(b, rec, rs, clusters, cluster_size, s);
}
}  // namespace cumc
