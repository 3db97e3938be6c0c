// common.cuh -- device building blocks shared by the LOITS kernels (sm_100a).
//
//  * Philox4x32-10 with the counter/key mapping of rng/philox.hpp:17-61
//    (counter = (block, stream), key = seed; word i of block b is slot 4b+i);
//  * error-free transforms (two-sum, two-product) for the compensated fp32
//    scans;
//  * acquire/release flag access with bounded spins (every wait has an
//    iteration limit and reports LOITS_ERR_TIMEOUT instead of hanging);
//  * warp / block scans.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "loits_b200.h"

namespace loits_dev {

// ------------------------------------------------------------------ Philox

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

// Round keys of Philox4x32-10 for one 64-bit seed: the Weyl key schedule
// (k0 + r * 0x9E3779B9, k1 + r * 0xBB67AE85) of rounds 0..9.  Built once per
// launch on the host and read from kernel parameters (constant bank), so the
// per-round key is an instruction operand instead of a per-thread add.
struct PhiloxKey {
  uint32_t k0[10];
  uint32_t k1[10];
};

__host__ __device__ inline PhiloxKey philox_key(uint64_t seed) {
  PhiloxKey k;
  uint32_t a = static_cast<uint32_t>(seed), b = static_cast<uint32_t>(seed >> 32);
  for (int r = 0; r < 10; ++r) {
    k.k0[r] = a;
    k.k1[r] = b;
    a += 0x9E3779B9u;
    b += 0xBB67AE85u;
  }
  return k;
}

// Random123 Philox4x32-10 (Salmon et al., SC'11).  rng/philox.hpp:17-56 binds
// c0,c1 = block lo/hi, c2,c3 = stream lo/hi, k0,k1 = seed lo/hi; each round
// multiplies (c0, c2) by (M0, M1) into 64-bit products.
__device__ __forceinline__ uint4 philox4x32_10(uint64_t block, uint64_t stream, const PhiloxKey& key) {
  uint32_t c0 = static_cast<uint32_t>(block), c1 = static_cast<uint32_t>(block >> 32);
  uint32_t c2 = static_cast<uint32_t>(stream), c3 = static_cast<uint32_t>(stream >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = static_cast<uint64_t>(kPhiloxM0) * c0;
    const uint64_t p1 = static_cast<uint64_t>(kPhiloxM1) * c2;
    const uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c1 ^ key.k0[r];
    const uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c3 ^ key.k1[r];
    c1 = static_cast<uint32_t>(p1);
    c3 = static_cast<uint32_t>(p0);
    c0 = n0;
    c2 = n2;
  }
  return make_uint4(c0, c1, c2, c3);
}

__device__ __forceinline__ uint4 philox4x32_10(uint64_t block, uint64_t stream, uint64_t seed) {
  const PhiloxKey key = philox_key(seed);
  return philox4x32_10(block, stream, key);
}

// rng/philox.hpp:59-61: top 24 bits, exact in fp32, in [0, 1).
__device__ __forceinline__ float uniform_from_bits(uint32_t bits) {
  return __uint2float_rn(bits >> 8) * 0x1.0p-24f;
}

__device__ __forceinline__ uint32_t word_of(const uint4& w, int i) {
  return i == 0 ? w.x : (i == 1 ? w.y : (i == 2 ? w.z : w.w));
}

// ------------------------------------------------- error-free transforms

// Knuth two-sum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// p + e == a * b exactly (FMA-based two-product).
__device__ __forceinline__ void two_prod(float a, float b, float& p, float& e) {
  p = __fmul_rn(a, b);
  e = __fmaf_rn(a, b, -p);
}

// Double-float accumulate: (hi, lo) += (a_hi, a_lo), ~48-bit result.
__device__ __forceinline__ void df_add(float& hi, float& lo, float a_hi, float a_lo) {
  float s, e;
  two_sum(hi, a_hi, s, e);
  e = __fadd_rn(e, __fadd_rn(lo, a_lo));
  hi = __fadd_rn(s, e);
  lo = __fsub_rn(e, __fsub_rn(hi, s));
}

// Trapezoid area 0.5 * (g1 - g0) * (f0 + f1) of fp32 inputs as a double-float
// pair accurate to ~2^-46 relative (the reference evaluates the same product
// exactly in fp64, cpp/loits_core.cpp:73).
__device__ __forceinline__ void trapezoid_df(float g0, float g1, float f0, float f1, float& hi,
                                             float& lo) {
  float d, de, s, se;
  two_sum(g1, -g0, d, de);
  two_sum(f0, f1, s, se);
  float p, pe;
  two_prod(d, s, p, pe);
  // cross terms d*se + de*s (+ de*se, below fp32 resolution of the result)
  const float corr = __fmaf_rn(d, se, __fmaf_rn(de, s, pe));
  float h, l;
  two_sum(p, corr, h, l);
  hi = 0.5f * h;  // exact scaling by a power of two
  lo = 0.5f * l;
}

// ------------------------------------------------------- flags and spins

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Upper bound on polls of one flag before the wait is declared failed.  Each
// poll after the first 64 sleeps ~256 ns, so a wait gives up after ~1 s.
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ void spin_pause(uint32_t iter) {
  if (iter > 64) __nanosleep(256);
}

// Record the first error of a launch (later errors keep the first code).
__device__ __forceinline__ void raise_status(int32_t* status, int32_t code) {
  if (status) atomicCAS(reinterpret_cast<int*>(status), 0, code);
}

// True once a wait of this launch has run out (its status word says so):
// every other wait then gives up at once instead of running out in turn, so
// a launch whose dependencies cannot be met ends after about one wait limit.
__device__ __forceinline__ bool launch_timed_out(const int32_t* status) {
  return status && *reinterpret_cast<const volatile int32_t*>(status) == LOITS_ERR_TIMEOUT;
}

// Wait until *counter >= target (acquire), at most `limit` polls.  Returns
// false on timeout (or when another wait of the launch has timed out).
__device__ __forceinline__ bool wait_counter(const uint32_t* counter, uint32_t target,
                                             const int32_t* status, uint32_t limit = kSpinLimit) {
  for (uint32_t it = 0; it < limit; ++it) {
    if (ld_acquire_u32(counter) >= target) return true;
    if ((it & 63u) == 63u && launch_timed_out(status)) return false;
    spin_pause(it);
  }
  return false;
}

// -------------------------------------------- bulk copies into shared memory
//
// A CTA stages a density's records and guide with the copy engine
// (cp.async.bulk, global -> shared, this GPU's own memory, no multicast):
// one thread arms an mbarrier with the byte count and issues the copies,
// every thread waits for the barrier's phase.  Both addresses and the size
// of each copy are multiples of 16 bytes.

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Once per CTA (one thread), before any bulk copy; a barrier must follow.
__device__ __forceinline__ void bulk_barrier_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One thread: earlier accesses to shared memory (ordered by a barrier)
// before the copy engine's writes; arm the barrier for `bytes`.
__device__ __forceinline__ void bulk_arm(uint64_t* bar, uint32_t bytes) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("{\n\t.reg .b64 st;\n\t"
               "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
               ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// One thread: bytes (a multiple of 16) from global src to shared dst, both
// 16-byte aligned, completing on bar.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// Every thread: wait for phase `parity` of bar to complete, at most `limit`
// polls; false when the wait ran out.
__device__ __forceinline__ bool bulk_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

// ---------------------------------------------------------------- scans

template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_inclusive_max(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = v > n ? v : n;
  }
  return v;
}

// Block-wide exclusive sum; `total` receives the block total.  `scratch`
// holds one T per warp.  Every thread of the block must call it.
template <typename T, int TPB>
__device__ __forceinline__ T block_exclusive_sum(T v, T& total, T* scratch) {
  constexpr int W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // exclusive values are formed by shifting inclusive ones (never inc - v,
  // which is inexact for floating-point T)
  const T inc = warp_inclusive_sum(v);
  T exc = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) exc = T(0);
  if (lane == 31) scratch[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const T s = lane < W ? scratch[lane] : T(0);
    const T si = warp_inclusive_sum(s);
    T se = __shfl_up_sync(0xffffffffu, si, 1);
    if (lane == 0) se = T(0);
    if (lane < W) scratch[lane] = se;
    if (lane == W - 1) scratch[W] = si;
  }
  __syncthreads();
  const T r = scratch[warp] + exc;
  total = scratch[W];
  __syncthreads();
  return r;
}

struct OpMax {
  template <typename T>
  __device__ __forceinline__ T operator()(T a, T b) const { return a > b ? a : b; }
};

// Block-wide exclusive max with identity `lowest` (thread i receives the max
// over threads < i); `total` receives the block max.  scratch: W+1 T.
template <typename T, int TPB>
__device__ __forceinline__ T block_exclusive_max(T v, T lowest, T& total, T* scratch) {
  constexpr int W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const OpMax op;
  T inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T n = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc = op(inc, n);
  }
  T exc = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) exc = lowest;
  if (lane == 31) scratch[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const T s = lane < W ? scratch[lane] : lowest;
    T si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T n = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si = op(si, n);
    }
    T se = __shfl_up_sync(0xffffffffu, si, 1);
    if (lane == 0) se = lowest;
    if (lane < W) scratch[lane] = se;
    if (lane == W - 1) scratch[W] = si;
  }
  __syncthreads();
  const T r = op(scratch[warp], exc);
  total = scratch[W];
  __syncthreads();
  return r;
}

// Block-wide exclusive SUFFIX sum: thread i receives the sum over threads > i.
template <typename T, int TPB>
__device__ __forceinline__ T block_exclusive_suffix_sum(T v, T& total, T* scratch) {
  constexpr int W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = v;  // inclusive suffix within the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T n = __shfl_down_sync(0xffffffffu, inc, o);
    if (lane + o < 32) inc += n;
  }
  T exc = __shfl_down_sync(0xffffffffu, inc, 1);
  if (lane == 31) exc = T(0);
  if (lane == 0) scratch[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const T s = lane < W ? scratch[lane] : T(0);
    T si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T n = __shfl_down_sync(0xffffffffu, si, o);
      if (lane + o < 32) si += n;
    }
    T se = __shfl_down_sync(0xffffffffu, si, 1);
    if (lane == 31) se = T(0);
    if (lane < W) scratch[lane] = se;
    if (lane == 0) scratch[W] = si;
  }
  __syncthreads();
  const T r = scratch[warp] + exc;
  total = scratch[W];
  __syncthreads();
  return r;
}

}  // namespace loits_dev
