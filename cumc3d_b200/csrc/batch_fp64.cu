// batch_fp64.cu -- FP64 (plain form) instantiations of the batched 1D kernel
// (built with --fmad=false, like the rest of the FP64 path).
#include "batch_kernel.cuh"

namespace cumc {
cudaError_t launch_batch_fp64(const BatchDev &b, int rec, int rs, int clusters, int cluster_size, cudaStream_t s) {
    return launch_batch_t<double>(b, rec, rs, clusters, cluster_size, s);
}
}  // namespace cumc
