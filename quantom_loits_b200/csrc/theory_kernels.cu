// theory_kernels.cu -- the parametric theory of the batched GAN workload.
//
// A generator emits 6 raw parameters per density; the theory maps them to a
// two-component power-law density tabulated on a shared grid:
//   a_i = -1/2 + 3/2 sigmoid(p[2i]),  b_i = 1 + 4 sigmoid(p[2i+1])  (i = 0, 1)
//   w_i = softplus(p[4+i])
//   f(x) = w_0 x^a_0 (1-x)^b_0 + w_1 x^a_1 (1-x)^b_1
// (the x^a (1-x)^b family of the sampler's synthetic densities, with a and b
// kept in the same ranges).  The VJP reduces grad_values * df/dp over the
// grid per density in a fixed order (deterministic).  fp32 throughout.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "loits_b200.h"
#include "theory.cuh"

namespace {

using loits_theory::Comp;
using loits_theory::component;

__global__ void theory_eval_kernel(int64_t nd, int64_t G, const float* __restrict__ params,
                                   const float* __restrict__ grid, float* __restrict__ values) {
  const int64_t n = nd * G;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t d = i / G;
    const float x = __ldg(&grid[i - d * G]);
    const float* p = params + d * 6;
    const Comp c0 = component(p, 0), c1 = component(p, 1);
    values[i] = loits_theory::value(c0, c1, x);
  }
}

constexpr int kVjpThreads = 256;

__global__ void __launch_bounds__(kVjpThreads) theory_vjp_kernel(
    int64_t G, const float* __restrict__ params, const float* __restrict__ grid,
    const float* __restrict__ grad_values, float* __restrict__ grad_params) {
  const int64_t d = blockIdx.x;
  const float* p = params + d * 6;
  const Comp c[2] = {component(p, 0), component(p, 1)};
  const float* gv = grad_values + d * G;
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int64_t t = threadIdx.x; t < G; t += kVjpThreads)
    loits_theory::add_grad(c, __ldg(&grid[t]), __ldg(&gv[t]), acc);
  // fixed-order reduction: warp tree, then warp 0 over the warps
  __shared__ float red[kVjpThreads / 32][6];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    float v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    float v = 0.0f;
    for (int w = 0; w < kVjpThreads / 32; ++w) v += red[w][threadIdx.x];
    grad_params[d * 6 + threadIdx.x] = v;
  }
}

}  // namespace

extern "C" int loits_theory_powerlaw(int64_t n_densities, int64_t knots, const float* params,
                                     const float* grid, float* values, void* stream) {
  if (n_densities < 0 || knots < 2 || (n_densities > 0 && (!params || !grid || !values)))
    return LOITS_ERR_INVALID;
  if (n_densities == 0) return LOITS_OK;
  const int64_t n = n_densities * knots;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>((n + threads - 1) / threads, 148 * 16);
  theory_eval_kernel<<<static_cast<int>(blocks), threads, 0, static_cast<cudaStream_t>(stream)>>>(
      n_densities, knots, params, grid, values);
  return cudaGetLastError() == cudaSuccess ? LOITS_OK : LOITS_ERR_CUDA;
}

extern "C" int loits_theory_powerlaw_vjp(int64_t n_densities, int64_t knots, const float* params,
                                         const float* grid, const float* grad_values,
                                         float* grad_params, void* stream) {
  if (n_densities < 0 || knots < 2 ||
      (n_densities > 0 && (!params || !grid || !grad_values || !grad_params)))
    return LOITS_ERR_INVALID;
  if (n_densities == 0) return LOITS_OK;
  if (n_densities > 0x7fffffff) return LOITS_ERR_UNSUPPORTED;
  theory_vjp_kernel<<<static_cast<int>(n_densities), kVjpThreads, 0,
                      static_cast<cudaStream_t>(stream)>>>(knots, params, grid, grad_values,
                                                           grad_params);
  return cudaGetLastError() == cudaSuccess ? LOITS_OK : LOITS_ERR_CUDA;
}
