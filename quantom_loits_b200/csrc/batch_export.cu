// batch_export.cu -- CDF export and quantile kernels of the batched sampler.
#include <cstdint>

#include "batch_kernels_impl.cuh"

namespace loits_dev {

// CDF export (hi + lo as fp64) and quantiles -----------------------------

__global__ void batch_cdf_export_kernel(const float4* __restrict__ rec, int64_t n,
                                        double* __restrict__ cdf) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float4 r = rec[i];
    cdf[i] = static_cast<double>(r.x) - static_cast<double>(r.y);  // key - (key - c)
  }
}

__global__ void batch_quantile_kernel(const float4* __restrict__ rec,
                                      const uint32_t* __restrict__ guide, int m, int G,
                                      bool count_all, const float* __restrict__ u, int64_t n,
                                      float* __restrict__ x, int32_t* __restrict__ intervals) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    // the guide bucket of u needs its 24-bit word: u = k * 2^-24 exactly
    const float uc = fminf(fmaxf(u[i], 0.0f), 0x1.fffffep-1f);
    const uint32_t bits = static_cast<uint32_t>(uc * 16777216.0f) << 8;
    const uint32_t k = bits >> (32 - m);
    const int j = count_all ? interval_count_all(rec, u[i], G)
                            : interval_in_range(rec, static_cast<int>(guide[k]),
                                                static_cast<int>(guide[k + 1]), u[i], G);
    float tv;
    x[i] = interval_value(rec[j], u[i], tv);
    if (intervals) intervals[i] = j;
  }
}

}  // namespace loits_dev
