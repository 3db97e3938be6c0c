// batch_inst_1024.cu -- the batched kernels with 1024-thread CTAs.
#include "batch_kernels_impl.cuh"

namespace loits_dev {

template __global__ void batch_forward_kernel<1024, 2, false>(BatchArgs);
template __global__ void batch_backward_kernel<1024, 2, false, false>(BatchArgs, double*);
template __global__ void batch_backward_kernel<1024, 2, false, true>(BatchArgs, double*);
template __global__ void batch_forward_kernel<1024, 2, true>(BatchArgs);
template __global__ void batch_backward_kernel<1024, 2, true, false>(BatchArgs, double*);
template __global__ void batch_backward_kernel<1024, 2, true, true>(BatchArgs, double*);
template __global__ void batch_forward_kernel<1024, 4, false>(BatchArgs);
template __global__ void batch_backward_kernel<1024, 4, false, false>(BatchArgs, double*);
template __global__ void batch_backward_kernel<1024, 4, false, true>(BatchArgs, double*);
template __global__ void batch_forward_kernel<1024, 4, true>(BatchArgs);
template __global__ void batch_backward_kernel<1024, 4, true, false>(BatchArgs, double*);
template __global__ void batch_backward_kernel<1024, 4, true, true>(BatchArgs, double*);
template __global__ void batch_forward_kernel<1024, 8, false>(BatchArgs);
template __global__ void batch_backward_kernel<1024, 8, false, false>(BatchArgs, double*);
template __global__ void batch_backward_kernel<1024, 8, false, true>(BatchArgs, double*);
template __global__ void batch_forward_kernel<1024, 8, true>(BatchArgs);
template __global__ void batch_backward_kernel<1024, 8, true, false>(BatchArgs, double*);
template __global__ void batch_backward_kernel<1024, 8, true, true>(BatchArgs, double*);

template __global__ void batch_forward_kernel<1024, 16, false>(BatchArgs);
template __global__ void batch_backward_kernel<1024, 16, false, false>(BatchArgs, double*);
template __global__ void batch_backward_kernel<1024, 16, false, true>(BatchArgs, double*);
template __global__ void batch_forward_kernel<1024, 16, true>(BatchArgs);
template __global__ void batch_backward_kernel<1024, 16, true, false>(BatchArgs, double*);
template __global__ void batch_backward_kernel<1024, 16, true, true>(BatchArgs, double*);

}  // namespace loits_dev
