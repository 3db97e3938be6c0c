// batch_inst_256.cu -- the batched kernels with 256-thread CTAs.
#include "batch_kernels_impl.cuh"

namespace loits_dev {

template __global__ void batch_forward_kernel<256, 2, false>(BatchArgs);
template __global__ void batch_backward_kernel<256, 2, false, false>(BatchArgs, double*);
template __global__ void batch_forward_kernel<256, 2, true>(BatchArgs);
template __global__ void batch_backward_kernel<256, 2, true, false>(BatchArgs, double*);
template __global__ void batch_forward_kernel<256, 4, false>(BatchArgs);
template __global__ void batch_backward_kernel<256, 4, false, false>(BatchArgs, double*);
template __global__ void batch_forward_kernel<256, 4, true>(BatchArgs);
template __global__ void batch_backward_kernel<256, 4, true, false>(BatchArgs, double*);
template __global__ void batch_forward_kernel<256, 8, false>(BatchArgs);
template __global__ void batch_backward_kernel<256, 8, false, false>(BatchArgs, double*);
template __global__ void batch_forward_kernel<256, 8, true>(BatchArgs);
template __global__ void batch_backward_kernel<256, 8, true, false>(BatchArgs, double*);
template __global__ void batch_forward_kernel<256, 16, false>(BatchArgs);
template __global__ void batch_backward_kernel<256, 16, false, false>(BatchArgs, double*);
template __global__ void batch_forward_kernel<256, 16, true>(BatchArgs);
template __global__ void batch_backward_kernel<256, 16, true, false>(BatchArgs, double*);

}  // namespace loits_dev
