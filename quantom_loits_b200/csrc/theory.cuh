// theory.cuh -- the two-component power-law theory of the batched GAN step,
// as device functions shared by the theory kernels (theory_kernels.cu) and
// the batched sampler's fused path (the CDF tiles evaluate the density from
// its parameters as they load the knots; the backward's finalize reduces the
// parameter gradient).  Every product and sum is rounded on its own
// (explicit _rn intrinsics), so both places compute bit-identical values.
//
//   a_i = -1/2 + 3/2 s(p[2i]),  b_i = 1 + 4 s(p[2i+1]),  w_i = softplus(p[4+i])
//   f(x) = w_0 x^a_0 (1-x)^b_0 + w_1 x^a_1 (1-x)^b_1,   s(z) = 1 / (1 + e^-z)
#pragma once

#include <cuda_runtime.h>

namespace loits_theory {

struct Comp {
  float a, b, w;     // exponents and weight
  float da, db, dw;  // d a / d p, d b / d p, d w / d p
};

__device__ __forceinline__ float sigmoid(float z) {
  return __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-z)));
}

__device__ __forceinline__ Comp component(const float* p, int i) {
  Comp c;
  const float sa = sigmoid(p[2 * i]), sb = sigmoid(p[2 * i + 1]), sw = sigmoid(p[4 + i]);
  c.a = __fadd_rn(-0.5f, __fmul_rn(1.5f, sa));
  c.b = __fadd_rn(1.0f, __fmul_rn(4.0f, sb));
  // softplus, written to stay finite for large arguments
  const float z = p[4 + i];
  c.w = z > 20.0f ? z : log1pf(expf(z));
  c.da = __fmul_rn(__fmul_rn(1.5f, sa), __fsub_rn(1.0f, sa));
  c.db = __fmul_rn(__fmul_rn(4.0f, sb), __fsub_rn(1.0f, sb));
  c.dw = sw;
  return c;
}

// x^a (1-x)^b from the logs of x and 1-x (0 at x = 1: b >= 1).
__device__ __forceinline__ float term(float lx, float l1x, float a, float b) {
  return expf(__fadd_rn(__fmul_rn(a, lx), __fmul_rn(b, l1x)));
}

// f(x) for the two components c0, c1.
__device__ __forceinline__ float value(const Comp& c0, const Comp& c1, float x) {
  const float lx = logf(x), l1x = logf(__fsub_rn(1.0f, x));  // -inf at x = 1: the term is 0
  return __fadd_rn(__fmul_rn(c0.w, term(lx, l1x, c0.a, c0.b)),
                   __fmul_rn(c1.w, term(lx, l1x, c1.a, c1.b)));
}

// Adds g * d f(x) / d p[j] to acc[j], j = 0..5.
__device__ __forceinline__ void add_grad(const Comp* c, float x, float g, float* acc) {
  const float lx = logf(x);
  const float one_m = __fsub_rn(1.0f, x);
  const float l1x = logf(one_m);
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float tv = term(lx, l1x, c[i].a, c[i].b);
    const float gwt = __fmul_rn(__fmul_rn(g, c[i].w), tv);
    acc[2 * i] = __fadd_rn(acc[2 * i], __fmul_rn(__fmul_rn(gwt, lx), c[i].da));
    // (1-x)^b ln(1-x) -> 0 as x -> 1 (b >= 1)
    if (one_m > 0.0f)
      acc[2 * i + 1] = __fadd_rn(acc[2 * i + 1], __fmul_rn(__fmul_rn(gwt, l1x), c[i].db));
    acc[4 + i] = __fadd_rn(acc[4 + i], __fmul_rn(__fmul_rn(g, tv), c[i].dw));
  }
}

}  // namespace loits_theory
