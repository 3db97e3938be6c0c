// batch_kernels_impl.cuh -- batched ragged 1-D LOITS on sm_100a (fp32 storage).
//
// Template definitions of the persistent kernels; batch_inst_*.cu instantiate
// them (one translation unit per CTA size, compiled in parallel).
//
// One persistent forward kernel and one persistent backward kernel serve a
// whole batch of densities.  CTAs take work items from an atomic ticket in a
// fixed order, so every item an item waits on was handed out earlier to a
// CTA that is already running (no deadlock), and every wait is bounded.
//
// Forward items, in ticket order:
//   1. CDF scan tiles (density, knot range): trapezoid areas of fp32 knots as
//      double-float pairs (error-free transforms), a compensated fp32 prefix
//      per thread, fp64 block scan of thread totals, fp64 carries between
//      tiles of one density (chained look-back).  A density that fits one
//      tile is finalised in the same item.
//   2. CDF finalize items for densities spanning several tiles.
//      Finalising = clamp the prefix to be non-decreasing (unless an area is
//      negative: then the exact count semantics of cpp/loits_core.cpp:12-18
//      are used at sampling time), divide by the fp64 normaliser, store per
//      knot the smallest fp32 >= c_k (the search key) with its offset from
//      c_k and the slope of every interval.
//   3. Sampling tiles (density, run of Philox blocks): in-register Philox
//      (rng/philox.hpp), exact search of fp32 u against the fp64 CDF through
//      the per-knot keys, linear interpolation (cpp/loits_core.cpp:193-196),
//      acceptance (finite, non-zero, x > x_cut), warp scans + decoupled
//      look-back for a stable (density, slot) compaction, coalesced 16-byte
//      stores from a per-CTA staging run that stays in L2.
// Backward items:
//   1. Chunks (density, run of sampling tiles): recompute uniforms, intervals
//      and the compaction ranks of the forward, read the cotangents of the
//      kept rows, scatter the interpolation VJP (cpp/loits_core.cpp:293-300)
//      into shared-memory grad-CDF sums (fixed point or replicated fp32),
//      write them as the chunk's partial.
//   2. Density finalize: sum the partials in chunk order (fp64,
//      deterministic), reverse suffix scan (cdf_vjp, :340-368) and the
//      normaliser VJP (density_vjp, :400-435), fp32 output.
#pragma once

#include <cmath>
#include <cstdint>

#include "batch_kernels.cuh"
#include "lookback.cuh"
#include "theory.cuh"

namespace loits_dev {

constexpr double kEps = 1e-5;
constexpr double kNegInf = -__builtin_huge_val();

// Largest b in [lo, hi) with table[b] <= idx (table non-decreasing).
__device__ __forceinline__ int find_owner(const int32_t* __restrict__ table, int lo, int hi,
                                          int32_t idx) {
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&table[mid]) <= idx) lo = mid; else hi = mid;
  }
  return lo;
}

// Philox stream of the launch: 2 * sequence, the sequence read from device
// memory when the launch was given one (graph replays that advance it).
__device__ __forceinline__ uint64_t stream_of(const BatchArgs& a) {
  return a.seq_dev ? 2 * __ldg(a.seq_dev) : a.stream_id;
}

// ------------------------------------------------------------------ search

// (u >= c_k) exactly, for fp32 u: a record's key is the smallest fp32 >= c_k.
__device__ __forceinline__ bool ge_key(float u, const float4* rec, int i) { return u >= rec[i].x; }

// Interval of u: (#knots t with u >= c_t) - 1, clamped to [0, G-2].
// Non-decreasing CDF: the guide bucket k of u (top m bits of its Philox word)
// bounds the count to [L[k], L[k+1]]; with M >= G buckets the range is
// usually empty or one knot wide, decided by at most one compare, else
// finished by binary search.  Otherwise the full count over every knot
// (cpp/loits_core.cpp:12-18).
__device__ __forceinline__ int interval_in_range(const float4* __restrict__ rec, int lo, int hi,
                                                 float u, int G) {
  if (lo < hi && ge_key(u, rec, lo)) {
    ++lo;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (ge_key(u, rec, mid)) lo = mid + 1; else hi = mid;
    }
  }
  int j = lo - 1;
  j = j < 0 ? 0 : j;
  return j > G - 2 ? G - 2 : j;
}

__device__ __forceinline__ int interval_count_all(const float4* __restrict__ rec, float u, int G) {
  int cnt = 0;
  for (int t = 0; t < G; ++t) cnt += ge_key(u, rec, t) ? 1 : 0;
  int j = cnt - 1;
  j = j < 0 ? 0 : j;
  return j > G - 2 ? G - 2 : j;
}

// Inverse CDF on interval j: g_j + m_j * (u - c_j), with u - c_j formed as
// (u - key_j) + (key_j - c_j), fp32.
__device__ __forceinline__ float interval_value(float4 r, float u, float& t) {
  t = __fadd_rn(__fsub_rn(u, r.x), r.y);
  return __fmaf_rn(r.w, t, r.z);
}

__device__ __forceinline__ bool accept_event(float x, float cut) {
  // reference predicate (finite, x * q != 0 with q finite non-zero) + cut
  return isfinite(x) && x != 0.0f && x > cut;
}

// ------------------------------------------------------------- CDF phase

template <int TPB>
struct CdfShared {
  double dscan[33];
  double dmax[33];
  double cfirst[TPB];
  double tile_excl, norm, mprev, cnext;
  int nonmono, has_next;
  int tmax[32];      // kept threshold: per-warp last interval at or below the cut
  uint32_t flags;    // the density's flags, shared by publish_density
};

// Double-float prefix step for knot t of density (g, f): adds the area of
// interval [t-1, t] (t >= 1).  Returns false if that area is negative/NaN.
// A density's knots as the CDF passes read them: knot t's position and value
// at g[t - off], f[t - off] -- the density in global memory (off = 0), or a
// CDF tile's knots staged in shared memory (kS: plain loads; __ldg is for
// global memory only).
struct Knots {
  const float* g;
  const float* f;
  int64_t off;
};

template <bool kS>
__device__ __forceinline__ float knot_g(const Knots& kn, int64_t t) {
  if constexpr (kS) return kn.g[t - kn.off];
  else return __ldg(&kn.g[t - kn.off]);
}

template <bool kS>
__device__ __forceinline__ float knot_f(const Knots& kn, int64_t t) {
  if constexpr (kS) return kn.f[t - kn.off];
  else return __ldg(&kn.f[t - kn.off]);
}

template <bool kS>
__device__ __forceinline__ bool add_area(const Knots& kn, int64_t t, float& ph, float& pl) {
  if (t < 1) return true;
  float ah, al;
  trapezoid_df(knot_g<kS>(kn, t - 1), knot_g<kS>(kn, t), knot_f<kS>(kn, t - 1), knot_f<kS>(kn, t),
               ah, al);
  df_add(ph, pl, ah, al);
  return ah >= 0.0f;
}

// Pass 1 over this thread's knots [my_lo, my_hi): local total and max prefix.
// bad_grid: a knot position is not finite or below its predecessor.
template <bool kS>
__device__ __forceinline__ void cdf_pass1(const Knots& kn, int64_t my_lo, int64_t my_hi,
                                          double& total, double& maxp, bool& neg,
                                          bool& bad_grid) {
  float ph = 0.0f, pl = 0.0f;
  maxp = kNegInf;
  neg = false;
  bad_grid = false;
  for (int64_t t = my_lo; t < my_hi; ++t) {
    const float gt = knot_g<kS>(kn, t);
    bad_grid |= !isfinite(gt) || (t >= 1 && !(gt >= knot_g<kS>(kn, t - 1)));
    neg |= !add_area<kS>(kn, t, ph, pl);
    const double p = static_cast<double>(ph) + static_cast<double>(pl);
    maxp = p > maxp ? p : maxp;
  }
  total = static_cast<double>(ph) + static_cast<double>(pl);
}

// First guide bucket k with k / M >= key (0 .. M + 1).
__device__ __forceinline__ int32_t bucket_start(float key, int m) {
  const float scaled = ldexpf(key, m);  // exact: M is a power of two
  if (!(scaled > 0.0f)) return 0;
  const int32_t M = 1 << m;
  if (scaled > static_cast<float>(M)) return M + 1;
  return static_cast<int32_t>(ceilf(scaled));
}

// Write the per-knot record of knot t given c_t and (if has_next) c_{t+1}
// (fp64), and the guide buckets whose knot count becomes t + 1 at this knot.
// Record: {key, key - c, g_t, m_t}; key = the smallest fp32 >= c_t, so that
// for every fp32 u, (u >= c_t) == (u >= key) exactly.
// gd: guide of the density (nullptr when the CDF is not non-decreasing).
template <bool kS>
__device__ __forceinline__ void emit_record(const BatchArgs& a, int64_t k0, const Knots& kn,
                                            int64_t t, double c, bool has_next, double c_next,
                                            uint32_t* gd, int m) {
  const float key = __double2float_ru(c);
  const float dk = __double2float_rn(static_cast<double>(key) - c);
  const float gt = knot_g<kS>(kn, t);
  float m_slope = 0.0f, inv = 0.0f, key_next = 0.0f;
  if (has_next) {
    key_next = __double2float_ru(c_next);
    const double inv_d = 1.0 / (c_next - c + kEps);
    const double md = (static_cast<double>(knot_g<kS>(kn, t + 1)) - static_cast<double>(gt)) * inv_d;
    m_slope = __double2float_rn(md);
    inv = __double2float_rn(inv_d);
  }
  a.rec[k0 + t] = make_float4(key, dk, gt, m_slope);
  a.invd[k0 + t] = inv;
  if (gd) {
    const int32_t M = 1 << m;
    const int32_t k_lo = bucket_start(key, m);
    const int32_t k_hi = has_next ? bucket_start(key_next, m) : M + 1;
    for (int32_t k = k_lo; k < k_hi; ++k) gd[k] = static_cast<uint32_t>(t + 1);
    if (t == 0)
      for (int32_t k = 0; k < k_lo; ++k) gd[k] = 0;
  }
}

// kAcceptAll when every event of density b is provably kept: with a
// non-decreasing CDF the search gives u >= c_j, so t = u - c_j >= 0 (exactly
// evaluated), and with an ascending finite grid the slope is finite and >= 0,
// hence x = g_j + m t >= g_0.  If g_0 > 0 and the cut (if any) is below g_0,
// x is finite, non-zero and above the cut for every uniform: the stable
// compaction is the identity.
__device__ __forceinline__ uint32_t accept_all_flag(const BatchArgs& a, int b, int64_t k0,
                                                    int64_t G, double norm, uint32_t flags) {
  if (flags & (kNonMonotone | kBadGrid)) return 0u;
  if (!(norm > 0.0) || !isfinite(norm)) return 0u;
  const float g0 = __ldg(&a.grid[k0]);
  // g_last bounds every slope (g_last - g_0) / 1e-5 well inside fp32 range
  if (!(g0 > 0.0f) || !(__ldg(&a.grid[k0 + G - 1]) < 1e30f)) return 0u;
  if (a.x_cut && !(__ldg(&a.x_cut[b]) < g0)) return 0u;
  return kAcceptAll;
}

// kThreshold when the kept events of density b are exactly those whose
// uniform lies above one threshold: with a non-decreasing CDF and an
// ascending finite grid (finite slopes m_j >= 0), the fp32 value
// x(u) = g_j + m_j ((u - key_j) + d_j) is non-decreasing in u -- each step is
// a correctly rounded monotone operation, and across a knot the next
// interval starts at or above where the previous one ends -- so for a cut
// >= 0 (x > cut >= 0 is non-zero and finite) {u : x(u) > cut} = {u > u*}.
__device__ __forceinline__ uint32_t threshold_flag(const BatchArgs& a, int b, int64_t k0,
                                                   int64_t G, double norm, uint32_t flags) {
  if (flags & (kNonMonotone | kBadGrid | kAcceptAll)) return 0u;
  if (!(norm > 0.0) || !isfinite(norm)) return 0u;
  if (!(__ldg(&a.grid[k0 + G - 1]) < 1e30f) || !(__ldg(&a.grid[k0]) > -1e30f)) return 0u;
  if (!a.x_cut || !(__ldg(&a.x_cut[b]) >= 0.0f)) return 0u;
  return kThreshold;
}

// Packed guide entry of a small density (G <= 8192 knots) for the bucket
// whose counts are [lo, hi] (lo = L[k] >= 1, hi = L[k+1]): the interval the
// bucket starts in, ja = lo - 1, and the number of knots inside the bucket
// that can still move the interval, span = min(hi, G - 1) - lo (a count past
// G - 1 only moves past the last interval, which the interval clamp undoes).
// Interval of u in the bucket: ja + #{t in [lo, lo + span) : key_t <= u}.
// Clamps make every entry safe (ja + span <= G - 2) whatever L holds.  The
// entry is 8 bytes: {ja | span << 16, key_{ja+1}} -- the key the first
// compare needs rides with the entry, so a slot's search loads the entry and
// then its record, two dependent shared-memory loads instead of three.
// rec: the density's final records (global memory).
__device__ __forceinline__ uint2 pack_entry(uint32_t lo, uint32_t hi, int G, const float4* rec) {
  const int l = static_cast<int>(lo), h = min(static_cast<int>(hi), G - 1);
  const int ja = max(min(l - 1, G - 2), 0);
  const int span = max(h - (ja + 1), 0);
  return make_uint2(static_cast<uint32_t>(ja) | (static_cast<uint32_t>(span) << 16),
                    __float_as_uint(__ldcg(reinterpret_cast<const float*>(rec + ja + 1))));
}

// Pack small density b's guide for sampling from shared memory:
// gpk[k] = pack_entry(L[k], L[k+1]).  Every L entry was written (and fenced)
// before this runs.  Large densities are sampled from L itself.
template <int TPB>
__device__ __forceinline__ void pack_guide(const BatchArgs& a, int b) {
  const int64_t po = __ldg(&a.pkoff[b]);
  if (po < 0) return;
  const int M = 1 << __ldg(&a.gbits[b]);
  const int G = static_cast<int>(__ldg(&a.knot_off[b + 1]) - __ldg(&a.knot_off[b]));
  const uint32_t* L = a.gl + __ldg(&a.goff[b]);
  uint2* P = reinterpret_cast<uint2*>(a.gpk + po);
  const float4* rec = a.rec + __ldg(&a.knot_off[b]);
  for (int k = threadIdx.x; k < M; k += TPB) P[k] = pack_entry(__ldcg(&L[k]), __ldcg(&L[k + 1]), G, rec);
  __threadfence();
}

// Pass 2: recompute the prefix, clamp, normalise, emit records for this
// thread's knots [my_lo, my_hi) of the tile ending at knot `hi`.
// base = tile_excl + thread exclusive sum; run0 = max of the prefix before
// this thread (the clamp); tile_next_c is c at knot `hi` when hi < G;
// gd / m: the density's guide table (nullptr for count semantics).
template <int TPB, bool kS>
__device__ __forceinline__ void cdf_pass2(const BatchArgs& a, int64_t k0, const Knots& kn, int64_t G, int64_t hi, int64_t my_lo,
                          int64_t my_hi, double base, double run0, double norm, bool nonmono,
                          double tile_next_c, uint32_t* gd, int m, CdfShared<TPB>& sh) {
  // first knot of each thread goes to shared memory for its left neighbour
  double c_first = 0.0;
  if (my_lo < my_hi) {
    float ph = 0.0f, pl = 0.0f;
    add_area<kS>(kn, my_lo, ph, pl);
    double s = base + (static_cast<double>(ph) + static_cast<double>(pl));
    if (!nonmono) s = s > run0 ? s : run0;
    c_first = s / norm;
  }
  sh.cfirst[threadIdx.x] = c_first;
  __syncthreads();
  if (my_lo < my_hi) {
    float ph = 0.0f, pl = 0.0f;
    double run = run0, c_prev = 0.0;
    for (int64_t t = my_lo; t < my_hi; ++t) {
      add_area<kS>(kn, t, ph, pl);
      double s = base + (static_cast<double>(ph) + static_cast<double>(pl));
      if (!nonmono) {
        run = s > run ? s : run;
        s = run;
      }
      const double c = s / norm;
      if (t > my_lo) emit_record<kS>(a, k0, kn, t - 1, c_prev, true, c, gd, m);
      c_prev = c;
    }
    // last knot of this thread: end of density, next thread, or next tile
    const int64_t t = my_hi - 1;
    if (t == G - 1) emit_record<kS>(a, k0, kn, t, c_prev, false, 0.0, gd, m);
    else if (t + 1 < hi) emit_record<kS>(a, k0, kn, t, c_prev, true, sh.cfirst[threadIdx.x + 1], gd, m);
    else emit_record<kS>(a, k0, kn, t, c_prev, true, tile_next_c, gd, m);
  }
  // every thread publishes its records before thread 0 signals readiness
  __threadfence();
  __syncthreads();
}

// Chained look-back over tiles [first, ct) of one density, by one whole
// warp: publishes tile ct's aggregate, then reads 32 predecessors per step
// until it meets an inclusive sum, and publishes tile ct's inclusive sum.
// Returns the fp64 sum of the earlier tiles on every lane.  flag: 1
// aggregate, 2 inclusive.  Every poll is bounded.
__device__ __forceinline__ double chained_lookback(uint32_t* flag, double* agg_arr, double* inc_arr,
                                                   int32_t* status, int32_t first, int32_t ct,
                                                   double agg, uint32_t limit) {
  const int lane = threadIdx.x & 31;
  double excl = 0.0;
  if (ct > first) {
    if (lane == 0) {
      __stcg(&agg_arr[ct], agg);
      __threadfence();
      atomicExch(&flag[ct], 1u);
    }
    __syncwarp();
    int32_t base = ct - 1;
    uint32_t polls = 0;
    while (base >= first) {
      const int32_t i = base - lane;
      // tiles before `first` do not exist: an inclusive zero
      const uint32_t fl = i >= first ? ld_acquire_u32(&flag[i]) : 2u;
      if (__any_sync(0xffffffffu, fl == 0)) {
        if (++polls >= limit ||
            ((polls & 63u) == 0u && __any_sync(0xffffffffu, launch_timed_out(status)))) {
          if (lane == 0) raise_status(status, LOITS_ERR_TIMEOUT);
          break;
        }
        spin_pause(polls);
        continue;
      }
      const unsigned inc = __ballot_sync(0xffffffffu, fl == 2);
      const int stop = inc ? __ffs(inc) - 1 : 32;  // nearest inclusive predecessor
      double v = 0.0;
      if (i >= first && lane < stop) v = __ldcg(&agg_arr[i]);
      else if (i >= first && lane == stop) v = __ldcg(&inc_arr[i]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      excl += v;
      if (inc) break;
      base -= 32;
    }
  }
  if (lane == 0) {
    __stcg(&inc_arr[ct], excl + agg);
    __threadfence();
    atomicExch(&flag[ct], 2u);
  }
  return excl;
}

__device__ __forceinline__ double cdf_lookback(const BatchArgs& a, int32_t first, int32_t ct, double agg) {
  return chained_lookback(a.cflag, a.cagg, a.cinc, a.status, first, ct, agg, a.spin_limit);
}

// Whether a CDF item (scan or finalize) of density b can stage its knots,
// 2 floats per knot of [lo - 1, hi + 1), in the dynamic shared memory before
// the guide.
__device__ __forceinline__ bool cdf_tile_fits(const BatchArgs& a, int b, int tpb) {
  const int64_t G = __ldg(&a.knot_off[b + 1]) - __ldg(&a.knot_off[b]);
  const int64_t KT = static_cast<int64_t>(tpb) * __ldg(&a.scan_k[b]);
  const int64_t n = (G < KT ? G : KT) + 2;
  return 8 * n <= 4ll * a.fwd_guide_off;
}

// Knots [s0, s1) of density b (first knot k0) into shared memory (sg, sf):
// coalesced loads, all in flight at once, instead of each thread's strided
// chain of dependent loads.  With theory parameters the values are evaluated
// here from the knot positions: the densities never round-trip global
// memory.  The caller synchronises.
template <int TPB>
__device__ __forceinline__ void stage_knots(const BatchArgs& a, int b, int64_t k0, int64_t s0,
                                            int64_t s1, float* sg, float* sf) {
  const int64_t n = s1 - s0;
  if (a.theory) {
    const float* p = a.theory + static_cast<int64_t>(b) * 6;
    const loits_theory::Comp c0 = loits_theory::component(p, 0);
    const loits_theory::Comp c1 = loits_theory::component(p, 1);
    for (int64_t i = threadIdx.x; i < n; i += TPB) {
      const float x = __ldg(&a.grid[k0 + s0 + i]);
      sg[i] = x;
      sf[i] = loits_theory::value(c0, c1, x);
    }
    return;
  }
#pragma unroll 4
  for (int64_t i = threadIdx.x; i < n; i += TPB) {
    sg[i] = __ldg(&a.grid[k0 + s0 + i]);
    sf[i] = __ldg(&a.values[k0 + s0 + i]);
  }
}

// The knots a CDF tile [lo, hi) reads: [lo - 1, hi + 1) within the density.
// kS: staged in shared memory (stage_s, which holds 2 (s1 - s0) floats).
template <bool kS>
__device__ __forceinline__ Knots tile_knots(const BatchArgs& a, int64_t k0, int64_t G,
                                            int64_t lo, int64_t hi, float* stage_s) {
  if constexpr (kS) {
    const int64_t s0 = lo > 0 ? lo - 1 : 0, s1 = hi + 1 < G ? hi + 1 : G;
    return Knots{stage_s, stage_s + (s1 - s0), s0};
  } else {
    return Knots{a.grid + k0, a.values + k0, 0};
  }
}

__device__ __forceinline__ int density_threshold(const BatchArgs& a, int b, int64_t k0, int64_t G);
template <int TPB>
__device__ __forceinline__ int threshold_scan(const BatchArgs& a, int b, int64_t k0, int64_t G,
                                              CdfShared<TPB>& sh);

// Densities up to this many knots per CTA thread find their kept threshold
// with every thread of the CTA (threshold_scan); larger ones by one warp's
// search over the uniforms (density_threshold).
constexpr int kThresholdScanPerThread = 32;

// The end of a density's CDF, by every thread of the CTA, thread 0 holding
// the density's flags `fl`: a kThreshold density's kept threshold is found
// and stored, then the density is published ready (its records, guide,
// flags and threshold all visible first).  Every record of the density was
// written and made visible (barrier, fence) before the call.
template <int TPB>
__device__ __forceinline__ void publish_density(const BatchArgs& a, int b, int64_t k0, int64_t G,
                                                uint32_t fl, CdfShared<TPB>& sh) {
  if (threadIdx.x == 0) sh.flags = fl;
  __syncthreads();
  fl = sh.flags;
  if (fl & kThreshold) {
    if (G <= static_cast<int64_t>(kThresholdScanPerThread) * TPB) {
      const int ks = threshold_scan<TPB>(a, b, k0, G, sh);
      if (threadIdx.x == 0) a.kstar[b] = ks;
    } else if (threadIdx.x < 32) {
      const int ks = density_threshold(a, b, k0, G);
      if (threadIdx.x == 0) a.kstar[b] = ks;
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&a.cdf_ready[b], 1u);
  }
}

template <int TPB, bool kS>
__device__ __forceinline__ void cdf_scan_item(const BatchArgs& a, int32_t ct, CdfShared<TPB>& sh,
                                              float* stage_s) {
  const int b = __ldg(&a.cdf_owner[ct]);
  const int32_t first = __ldg(&a.cdf_first[b]);
  const int32_t ci = ct - first, nci = __ldg(&a.cdf_first[b + 1]) - first;
  const int64_t k0 = __ldg(&a.knot_off[b]);
  const int64_t G = __ldg(&a.knot_off[b + 1]) - k0;
  const int sk = __ldg(&a.scan_k[b]);  // knots per thread in this density's CDF tiles
  const int64_t KT = static_cast<int64_t>(TPB) * sk;
  const int64_t lo = ci * KT, hi = lo + KT < G ? lo + KT : G;
  const Knots kn = tile_knots<kS>(a, k0, G, lo, hi, stage_s);
  if constexpr (kS) {
    stage_knots<TPB>(a, b, k0, kn.off, kn.off + (kn.f - kn.g), const_cast<float*>(kn.g),
                     const_cast<float*>(kn.f));
    __syncthreads();
  }
  const int64_t my_lo_raw = lo + static_cast<int64_t>(threadIdx.x) * sk;
  const int64_t my_lo = my_lo_raw < hi ? my_lo_raw : hi;
  const int64_t my_hi = my_lo_raw + sk < hi ? my_lo_raw + sk : hi;
  double tot, maxp;
  bool neg;
  bool bad_grid;
  cdf_pass1<kS>(kn, my_lo, my_hi, tot, maxp, neg, bad_grid);
  double tile_tot;
  const double excl = block_exclusive_sum<double, TPB>(tot, tile_tot, sh.dscan);
  const double thr_max = my_lo < my_hi ? excl + maxp : kNegInf;
  double tile_max;
  const double run0 = block_exclusive_max<double, TPB>(thr_max, kNegInf, tile_max, sh.dmax);
  const bool any_neg = __syncthreads_or(neg ? 1 : 0) != 0;
  const bool any_bad = __syncthreads_or(bad_grid ? 1 : 0) != 0;
  if (nci == 1) {
    // whole density in one tile: finalise now
    uint32_t* gd = any_neg ? nullptr : a.gl + __ldg(&a.goff[b]);
    cdf_pass2<TPB, kS>(a, k0, kn, G, hi, my_lo, my_hi, excl, run0, tile_tot, any_neg, 0.0, gd,
                       __ldg(&a.gbits[b]), sh);
    if (!any_neg) pack_guide<TPB>(a, b);
    __syncthreads();
    uint32_t fl = 0;
    if (threadIdx.x == 0) {
      a.norm[b] = tile_tot;
      fl = (any_neg ? kNonMonotone : 0u) | (any_bad ? kBadGrid : 0u);
      fl |= accept_all_flag(a, b, k0, G, tile_tot, fl);
      fl |= threshold_flag(a, b, k0, G, tile_tot, fl);
      a.dflags[b] = fl;
    }
    publish_density<TPB>(a, b, k0, G, fl, sh);
    return;
  }
  (void)tile_max;
  (void)run0;
  if (threadIdx.x == 0) {
    if (any_neg || any_bad)
      atomicOr(&a.dflags[b], (any_neg ? kNonMonotone : 0u) | (any_bad ? kBadGrid : 0u));
  }
  if (threadIdx.x < 32) {
    const double excl_t = cdf_lookback(a, first, ct, tile_tot);
    if (threadIdx.x == 0) sh.tile_excl = excl_t;
  }
  __syncthreads();
  // largest unnormalised prefix of this tile, formed exactly as pass 2 forms
  // each prefix ((tile_excl + thread_excl) + local), for the clamp of later tiles
  const double tile_excl = sh.tile_excl;
  const double my_max = my_lo < my_hi ? (tile_excl + excl) + maxp : kNegInf;
  double tmax;
  block_exclusive_max<double, TPB>(my_max, kNegInf, tmax, sh.dmax);
  if (threadIdx.x == 0) {
    __stcg(&a.cmax[ct], tmax);
    if (ci == nci - 1) __stcg(&a.norm[b], tile_excl + tile_tot);
    __threadfence();
    atomicAdd(&a.cdf_scanned[b], 1u);
  }
  __syncthreads();
}

template <int TPB, bool kS>
__device__ __forceinline__ void cdf_finalize_item(const BatchArgs& a, int32_t fi, CdfShared<TPB>& sh,
                                                  float* stage_s) {
  const int b = find_owner(a.fin_first, a.d_lo, a.d_hi, fi);
  const int32_t ci = fi - __ldg(&a.fin_first[b]);
  const int32_t first = __ldg(&a.cdf_first[b]);
  const int32_t nci = __ldg(&a.cdf_first[b + 1]) - first;
  const int32_t ct = first + ci;
  const int64_t k0 = __ldg(&a.knot_off[b]);
  const int64_t G = __ldg(&a.knot_off[b + 1]) - k0;
  const int sk = __ldg(&a.scan_k[b]);  // knots per thread in this density's CDF tiles
  const int64_t KT = static_cast<int64_t>(TPB) * sk;
  const int64_t lo = ci * KT, hi = lo + KT < G ? lo + KT : G;
  const Knots kn = tile_knots<kS>(a, k0, G, lo, hi, stage_s);
  if constexpr (kS)  // made visible by the barrier after the lane-0 work below
    stage_knots<TPB>(a, b, k0, kn.off, kn.off + (kn.f - kn.g), const_cast<float*>(kn.g),
                     const_cast<float*>(kn.f));
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    if (lane == 0 && !wait_counter(&a.cdf_scanned[b], static_cast<uint32_t>(nci), a.status, a.spin_limit))
      raise_status(a.status, LOITS_ERR_TIMEOUT);
    __syncwarp();
    // largest unnormalised prefix of all earlier tiles (warp-strided max)
    double mp = kNegInf;
    for (int32_t i = first + lane; i < ct; i += 32) {
      const double v = __ldcg(&a.cmax[i]);
      mp = v > mp ? v : mp;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double v = __shfl_xor_sync(0xffffffffu, mp, o);
      mp = v > mp ? v : mp;
    }
    if (lane == 0) {
      sh.norm = __ldcg(&a.norm[b]);
      sh.nonmono = (ld_acquire_u32(&a.dflags[b]) & kNonMonotone) ? 1 : 0;
      sh.tile_excl = ci == 0 ? 0.0 : __ldcg(&a.cinc[ct - 1]);
      sh.mprev = mp;
      sh.has_next = hi < G ? 1 : 0;
      if (hi < G) {
        // first knot of the next tile, exactly as that tile's own pass 2 forms it
        float ph = 0.0f, pl = 0.0f;
        add_area<false>(Knots{a.grid + k0, a.values + k0, 0}, hi, ph, pl);
        double s = (__ldcg(&a.cinc[ct]) + 0.0) + (static_cast<double>(ph) + static_cast<double>(pl));
        if (!sh.nonmono) {
          const double m_own = __ldcg(&a.cmax[ct]);
          const double m = mp > m_own ? mp : m_own;
          s = s > m ? s : m;
        }
        sh.cnext = s / sh.norm;
      }
    }
  }
  __syncthreads();
  const double norm = sh.norm, tile_excl = sh.tile_excl, mprev = sh.mprev, cnext = sh.cnext;
  const bool nonmono = sh.nonmono != 0, has_next = sh.has_next != 0;
  const int64_t my_lo_raw = lo + static_cast<int64_t>(threadIdx.x) * sk;
  const int64_t my_lo = my_lo_raw < hi ? my_lo_raw : hi;
  const int64_t my_hi = my_lo_raw + sk < hi ? my_lo_raw + sk : hi;
  double tot, maxp;
  bool neg, bad_grid;
  cdf_pass1<kS>(kn, my_lo, my_hi, tot, maxp, neg, bad_grid);
  double tile_tot;
  const double excl = block_exclusive_sum<double, TPB>(tot, tile_tot, sh.dscan);
  const double thr_max = my_lo < my_hi ? (tile_excl + excl) + maxp : kNegInf;
  double tile_max;
  double run0 = block_exclusive_max<double, TPB>(thr_max, kNegInf, tile_max, sh.dmax);
  run0 = run0 > mprev ? run0 : mprev;
  (void)has_next;
  uint32_t* gd = nonmono ? nullptr : a.gl + __ldg(&a.goff[b]);
  cdf_pass2<TPB, kS>(a, k0, kn, G, hi, my_lo, my_hi, tile_excl + excl, run0, norm, nonmono,
                     cnext, gd, __ldg(&a.gbits[b]), sh);
  // the last finalize item of the density packs its guide and publishes it
  if (threadIdx.x == 0) sh.has_next = atomicAdd(&a.fin_done[b], 1u) == static_cast<uint32_t>(nci - 1);
  __syncthreads();
  if (sh.has_next) {
    __threadfence();
    if (!nonmono) pack_guide<TPB>(a, b);
    __syncthreads();
    uint32_t fl = 0;
    if (threadIdx.x == 0) {
      fl = ld_acquire_u32(&a.dflags[b]) & (kNonMonotone | kBadGrid);
      fl |= accept_all_flag(a, b, k0, G, norm, fl);
      fl |= threshold_flag(a, b, k0, G, norm, fl);
      a.dflags[b] = fl;
    }
    publish_density<TPB>(a, b, k0, G, fl, sh);
  }
  __syncthreads();
}

// --------------------------------------------------------- sampling phase

// Geometry of sampling tile t of density b: Philox blocks
// [blk0, blk0 + TPB*rb) clipped to the density's slots [P0, P0 + n).
struct TileGeom {
  int b;
  int rb;  // Philox blocks per thread per tile of this density (at most the launch's R)
  int64_t k0, G, n, P0, blk0;
};

template <int TPB, int R>
__device__ __forceinline__ TileGeom tile_geom(const BatchArgs& a, int32_t t) {
  TileGeom tg;
  tg.b = __ldg(&a.tile_owner[t]);
  const int32_t si = t - __ldg(&a.tile_first[tg.b]);
  tg.rb = min(max(__ldg(&a.tile_r[tg.b]), 1), R);
  tg.k0 = __ldg(&a.knot_off[tg.b]);
  tg.G = __ldg(&a.knot_off[tg.b + 1]) - tg.k0;
  tg.n = __ldg(&a.n_events[tg.b]);
  tg.P0 = (a.dbase + tg.b) * a.nmax;
  tg.blk0 = (tg.P0 >> 2) + static_cast<int64_t>(si) * TPB * tg.rb;
  return tg;
}

// Where a density's records and guide are read from:
//   kShared  small density, copied into shared memory for the tile;
//   kL2      large density in the forward: global memory written earlier in
//            the same launch, read through L2 (coherent);
//   kRO      large density in the backward: global memory, read-only for the
//            launch (read-only data cache).
enum : int { kShared = 0, kL2 = 1, kRO = 2 };

template <int kMode>
__device__ __forceinline__ float4 rec_at(const float4* rec, int i) {
  if constexpr (kMode == kL2) return __ldcg(rec + i);
  else if constexpr (kMode == kRO) return __ldg(rec + i);
  else return rec[i];
}

template <int kMode>
__device__ __forceinline__ float key_at(const float4* rec, int i) {
  const float* p = reinterpret_cast<const float*>(rec + i);
  if constexpr (kMode == kL2) return __ldcg(p);
  else if constexpr (kMode == kRO) return __ldg(p);
  else return *p;
}

// A density's sampling state.
struct DensView {
  const float4* rec;      // records (shared or global)
  const uint32_t* guide;  // small: packed entries in shared memory; large: L, global
  const uint32_t* cguide; // large, coarse: every 2^s-th count of L in shared memory
  const float* invd;      // backward weights (shared or global)
  int shift;              // 32 - m: bucket of a Philox word = word >> shift
  int G;
  bool count_all;
  bool accept_all;
  bool threshold;         // kept = uniforms above one threshold (kThreshold)
  int kstar;              // ... namely (word >> 8) > kstar
  bool skip;              // large density whose CDF is not non-decreasing: not sampled
  bool coarse;            // large: cguide in shared memory (shift covers its bits)
  bool fresh;             // large: the coarse guide was copied for this view
  int shift_full;         // large: 32 - bits of the full guide
  const float4* wrec;     // forward, large: records [wk0, wk1) in shared memory
  int wk0, wk1;
  float cut;
};

struct SampleShared {
  int warp_cnt[32];
  float red[32];
  int64_t base;
  uint32_t flags;
  float cut;
  float fix_scale;   // backward chunk: fixed-point units per cotangent unit
  float fix_cap;     // backward chunk: largest scaled term a fixed-point sum takes
  int fix_lbits;     // backward chunk: bits of a term in its low word
  int win_b;         // density whose fixed-point window win_lo belongs to
  int win_lo;
  int run_k0;        // most_probable_run's result
  int kstar;         // the density's kept threshold (kThreshold)
};

// Wait until density b's CDF is final (thread 0) and share its flags and cut.
// A large density whose CDF is not non-decreasing would need the count over
// all of its knots, O(G) per event: it is not sampled and the launch reports
// LOITS_ERR_UNSUPPORTED.
__device__ __forceinline__ void density_flags(const BatchArgs& a, int b, bool large,
                                              bool wait_ready, SampleShared& sh) {
  if (threadIdx.x == 0) {
    if (wait_ready && !wait_counter(&a.cdf_ready[b], 1u, a.status, a.spin_limit))
      raise_status(a.status, LOITS_ERR_TIMEOUT);
    // plain loads, in flight together: the wait's acquire (or the kernel
    // boundary, without a wait) already orders them after the density's
    // flags and threshold were written
    const uint32_t fl = __ldcg(&a.dflags[b]);
    const int ks = __ldcg(&a.kstar[b]);
    sh.flags = fl;
    sh.kstar = (fl & kThreshold) ? ks : 0;
    sh.cut = a.x_cut ? __ldg(&a.x_cut[b]) : -__int_as_float(0x7f800000);
    if (large && (sh.flags & kNonMonotone)) raise_status(a.status, LOITS_ERR_UNSUPPORTED);
  }
  __syncthreads();
}

// A CTA's bulk-copy barrier (shared memory) and the parity of its next phase
// (shared, advanced by thread 0 after each use).
struct BulkStage {
  uint64_t* bar;
  uint32_t* phase;
};

// The density's sampling view: small densities copy their records, packed
// guide and (backward) weights into shared memory -- records and the full
// packed guide by the copy engine (one bulk copy each, issued by the CTA's
// last thread so that warp 0 may run a look-back meanwhile), the weights
// and a coarser guide by the threads; large densities keep records and
// weights in global memory and copy a coarse guide when lguide_bits > 0 (the
// forward adds a window of records: sample_item).  Ends with a barrier.
// guide_key (shared) names the density whose coarse guide guide_s holds, so
// a CTA's consecutive items on one large density copy it once.
__device__ __forceinline__ DensView density_view(const BatchArgs& a, int b, int64_t k0, int64_t G,
                                                 bool large, float4* rec_s, uint32_t* guide_s,
                                                 float* invd_s, const SampleShared& sh,
                                                 int& guide_key, BulkStage bulk) {
  const bool nonmono = (sh.flags & kNonMonotone) != 0;
  const int m_full = __ldg(&a.gbits[b]);
  const bool coarse = large && a.lguide_bits > 0;
  const int m = large ? (coarse ? min(m_full, a.lguide_bits) : m_full) : min(m_full, a.gbits_cap);
  DensView v;
  if (large) {
    v.rec = a.rec + k0;
    v.invd = a.invd + k0;
    const uint32_t* L = a.gl + __ldg(&a.goff[b]);
    v.fresh = coarse && !nonmono && guide_key != b;
    if (v.fresh) {
      // every 2^s-th count of the guide (the guide with 2^s-times wider
      // buckets), 2^m + 1 uint32
      const int sft = m_full - m;
      for (int k = threadIdx.x; k <= (1 << m); k += blockDim.x) guide_s[k] = __ldcg(&L[k << sft]);
    }
    v.guide = L;
    v.cguide = guide_s;
  } else {
    const bool full_guide = !nonmono && m == m_full;
    const uint4* gsrc = reinterpret_cast<const uint4*>(a.gpk + __ldg(&a.pkoff[b]));
    const uint32_t rec_bytes = static_cast<uint32_t>(G) * 16u;
    const uint32_t guide_bytes = full_guide ? (8u << m) : 0u;
    if (bulk.bar && threadIdx.x == blockDim.x - 1) {
      // records (16 G bytes) and the packed guide (8 M bytes, M >= 4) start on
      // 16-byte boundaries in the workspace and in shared memory
      bulk_arm(bulk.bar, rec_bytes + guide_bytes);
      bulk_copy(rec_s, a.rec + k0, rec_bytes, bulk.bar);
      if (full_guide) bulk_copy(guide_s, gsrc, guide_bytes, bulk.bar);
    }
    if (invd_s)
      for (int64_t i = threadIdx.x; i < G; i += blockDim.x) invd_s[i] = __ldcg(&a.invd[k0 + i]);
    if (!bulk.bar) {
      for (int64_t i = threadIdx.x; i < G; i += blockDim.x) rec_s[i] = __ldcg(&a.rec[k0 + i]);
      if (full_guide) {
        uint4* dst = reinterpret_cast<uint4*>(guide_s);
        for (int i = threadIdx.x; i < (1 << m) / 2; i += blockDim.x) dst[i] = __ldcg(&gsrc[i]);
      }
    } else if (!bulk_wait(bulk.bar, *bulk.phase, a.spin_limit)) {
      // the copy did not complete within the wait limit: the launch reports
      // it and the threads copy the same bytes themselves
      raise_status(a.status, LOITS_ERR_TIMEOUT);
      for (int64_t i = threadIdx.x; i < G; i += blockDim.x) rec_s[i] = __ldcg(&a.rec[k0 + i]);
      if (full_guide) {
        uint4* dst = reinterpret_cast<uint4*>(guide_s);
        for (int i = threadIdx.x; i < (1 << m) / 2; i += blockDim.x) dst[i] = __ldcg(&gsrc[i]);
      }
    }
    if (!full_guide && !nonmono) {
      // every 2^s-th count: the guide with 2^s-times wider buckets
      const int sft = m_full - m;
      const uint32_t* L = a.gl + __ldg(&a.goff[b]);
      const int Gi = static_cast<int>(G);
      for (int k = threadIdx.x; k < (1 << m); k += blockDim.x)
        reinterpret_cast<uint2*>(guide_s)[k] =
            pack_entry(__ldcg(&L[k << sft]), __ldcg(&L[(k + 1) << sft]), Gi, a.rec + k0);
    }
    v.rec = rec_s;
    v.guide = guide_s;
    v.cguide = guide_s;
    v.invd = invd_s;
    v.fresh = false;
  }
  __syncthreads();
  // every thread has read guide_key and the bulk phase above; the next reads
  // follow the item loop's barriers
  if (threadIdx.x == 0) {
    guide_key = large ? (nonmono || !coarse ? guide_key : b) : -1;
    if (!large && bulk.bar) *bulk.phase ^= 1u;
  }
  v.shift = 32 - m;
  v.shift_full = 32 - m_full;
  v.wrec = nullptr;
  v.wk0 = v.wk1 = 0;
  v.G = static_cast<int>(G);
  v.count_all = nonmono && !large;
  v.accept_all = (sh.flags & kAcceptAll) != 0;
  v.threshold = (sh.flags & kThreshold) != 0;
  v.kstar = sh.kstar;
  v.skip = nonmono && large;
  v.coarse = coarse;
  v.cut = sh.cut;
  return v;
}

// `large` is a constant at every call site, so that after inlining each
// view's pointers are known to be shared (LDS) or global memory.
__device__ __forceinline__ DensView load_density(const BatchArgs& a, int b, int64_t k0, int64_t G,
                                                 bool large, float4* rec_s, uint32_t* guide_s,
                                                 float* invd_s, bool wait_ready, SampleShared& sh,
                                                 int& guide_key, BulkStage bulk) {
  density_flags(a, b, large, wait_ready, sh);
  return density_view(a, b, k0, G, large, rec_s, guide_s, invd_s, sh, guide_key, bulk);
}

// One slot: uniform from its Philox word, interval, value, acceptance.
struct Slot {
  float x, t, m;
  int j;
  bool ok;
};

// Interval of u whose count #{t : u >= c_t} lies in [lo, hi] (a guide
// bucket; c_0 = 0, so lo >= 1): both candidate records are loaded at once --
// interval lo-1 (count == lo) and knot/interval lo (count > lo) -- and one
// exact compare selects, without a branch.  Only a bucket holding several
// knots needs a search.  Reads record indices lo-1 .. hi only.
template <int kMode>
__device__ __forceinline__ void pick_interval(const float4* rec, int G, float u, int lo, int hi,
                                              int& j, float4& r) {
  const int ja = max(min(lo - 1, G - 2), 0);
  const float4 ra = rec_at<kMode>(rec, ja);
  const float4 rb = rec_at<kMode>(rec, ja + 1);
  const bool step = (lo < hi) & (u >= rb.x);
  // count == lo + 1 moves to interval lo, unless lo - 1 is the last one
  const bool adv = step & (lo <= G - 2);
  j = ja + (adv ? 1 : 0);
  r = adv ? rb : ra;
  if (step & (hi - lo >= 2)) {
    // count in [lo + 1, hi]: first key above u
    int l = lo + 1, h = hi;
    while (l < h) {
      const int mid = (l + h) >> 1;
      if (u >= key_at<kMode>(rec, mid)) l = mid + 1; else h = mid;
    }
    j = min(l - 1, G - 2);
    r = rec_at<kMode>(rec, j);
  }
}

// Interval of u from a small density's packed guide entry (pack_entry), the
// records in shared memory: one compare with the entry's key moves u from
// the bucket's first interval to the next (always in bounds:
// ja + 1 <= G - 1); only a bucket with two or more movable knots finishes
// with a binary search over the records' keys.  The record itself is loaded
// once, after the interval is known.
__device__ __forceinline__ int pick_packed(const float4* rec, uint2 pk2, float u) {
  const float* keys = reinterpret_cast<const float*>(rec);
  const uint32_t pk = pk2.x;
  const int ja = static_cast<int>(pk & 0xffffu);
  const int span = static_cast<int>(pk >> 16);
  const bool step = (span > 0) & (u >= __uint_as_float(pk2.y));
  int j = ja + (step ? 1 : 0);
  if (step & (span >= 2)) {
    // first key above u among knots [ja + 2, ja + 1 + span)
    int l = ja + 2, h = ja + 1 + span;
    while (l < h) {
      const int mid = (l + h) >> 1;
      if (u >= keys[4 * mid]) l = mid + 1; else h = mid;
    }
    j = l - 1;
  }
  return j;
}

template <int kMode>
__device__ __forceinline__ Slot sample_slot(const DensView& d, uint32_t bits) {
  const float u = uniform_from_bits(bits);
  int j;
  float4 r;
  if (kMode == kShared && d.count_all) {
    j = interval_count_all(d.rec, u, d.G);
    r = d.rec[j];
  } else if constexpr (kMode == kShared) {
    j = pick_packed(d.rec, reinterpret_cast<const uint2*>(d.guide)[bits >> d.shift], u);
    r = d.rec[j];
  } else if constexpr (kMode == kL2) {
    // forward, large density: when the coarse bucket's knots all lie in the
    // shared window [wk0, wk1), search there; otherwise the full guide and
    // records through L2 (written earlier in this launch)
    bool hot = false;
    if (d.coarse) {
      const uint32_t kc = bits >> d.shift;
      const int lo = static_cast<int>(d.cguide[kc]), hi = static_cast<int>(d.cguide[kc + 1]);
      hot = lo > d.wk0 && hi < d.wk1;
      if (hot) {
        // window coordinates (knot index - wk0): the clamps to [0, G-2] do
        // not bind inside the window, so the pick is the same
        pick_interval<kShared>(d.wrec, d.G - d.wk0, u, lo - d.wk0, hi - d.wk0, j, r);
        j += d.wk0;
      }
    }
    if (!hot) {
      const uint32_t k = bits >> d.shift_full;
      pick_interval<kL2>(d.rec, d.G, u, static_cast<int>(__ldcg(d.guide + k)),
                         static_cast<int>(__ldcg(d.guide + k + 1)), j, r);
    }
  } else {
    // backward, large density: the coarse guide in shared memory, or the
    // full guide through the read-only cache
    const uint32_t k = bits >> d.shift;
    int lo, hi;
    if (d.coarse) {
      lo = static_cast<int>(d.cguide[k]);
      hi = static_cast<int>(d.cguide[k + 1]);
    } else {
      lo = static_cast<int>(__ldg(d.guide + k));
      hi = static_cast<int>(__ldg(d.guide + k + 1));
    }
    pick_interval<kRO>(d.rec, d.G, u, lo, hi, j, r);
  }
  Slot o;
  o.x = interval_value(r, u, o.t);
  o.m = r.w;
  o.j = j;
  o.ok = accept_event(o.x, d.cut);
  return o;
}

// Warp-granular work layout of a sampling tile: warp w of the CTA owns
// Philox blocks blk0 + (w*rb + r)*32 + lane for rounds r = 0..rb-1, i.e. the
// 128 consecutive slots of each round, rounds in order.  A warp therefore
// ranks its kept events with one warp scan per round, and the kept events of
// a tile are the concatenation of its warps' kept events in warp order.

// Bit mask of the 4 slots of Philox block blk inside the density's slot
// range [P0, P0 + n) (0 when the block lies past the range).
__device__ __forceinline__ uint32_t block_range_mask(const TileGeom& tg, int64_t blk) {
  const int64_t s0 = (blk << 2) - tg.P0;  // density slot of word 0
  if (s0 >= 0 && s0 + 4 <= tg.n) return 0xfu;
  const int64_t lo = s0 < 0 ? -s0 : 0;
  const int64_t hi = tg.n - s0 < 4 ? tg.n - s0 : 4;
  if (hi <= lo) return 0u;
  return ((1u << static_cast<int>(hi)) - 1u) & ~((1u << static_cast<int>(lo)) - 1u);
}

// Exclusive warp prefix of per-lane counts (ints: exact); *total = warp sum.
__device__ __forceinline__ int warp_exclusive_count(int c, int& total) {
  const int inc = warp_inclusive_sum(c);
  total = __shfl_sync(0xffffffffu, inc, 31);
  return inc - c;
}

// Copy n floats src[0..n) (the warp's staging run, L2-resident) to dst[0..n)
// (final rows), 16-byte stores where dst is aligned.  One warp.
__device__ __forceinline__ void warp_store(const float* __restrict__ src, float* __restrict__ dst,
                                           int n) {
  const int lane = threadIdx.x & 31;
  const int head = static_cast<int>((4 - ((reinterpret_cast<uintptr_t>(dst) >> 2) & 3)) & 3);
  const int h = head < n ? head : n;
  if (lane < h) dst[lane] = __ldcg(&src[lane]);
  const int nv = (n - h) >> 2;
  float4* dv = reinterpret_cast<float4*>(dst + h);
  // four 16-byte groups per lane in flight (the staging run is read from L2)
  int v = lane;
  for (; v + 96 < nv; v += 128) {
    float4 q[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int s0 = h + 4 * (v + 32 * i);
      q[i] = make_float4(__ldcg(&src[s0]), __ldcg(&src[s0 + 1]), __ldcg(&src[s0 + 2]),
                         __ldcg(&src[s0 + 3]));
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) __stcs(&dv[v + 32 * i], q[i]);
  }
  for (; v < nv; v += 32) {
    const int s0 = h + 4 * v;
    __stcs(&dv[v], make_float4(__ldcg(&src[s0]), __ldcg(&src[s0 + 1]), __ldcg(&src[s0 + 2]),
                               __ldcg(&src[s0 + 3])));
  }
  const int tail0 = h + 4 * nv;
  if (tail0 + lane < n) dst[tail0 + lane] = __ldcg(&src[tail0 + lane]);
}

// Optional per-row interval (diagnostics, saved state) and offset u - c_j
// (saved state) output of a general tile: recomputed for its kept rows.
template <int TPB, int R, int kMode>
__device__ __forceinline__ void write_intervals(const BatchArgs& a, const TileGeom& tg,
                                                const DensView& d, int64_t row0) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t row = row0;
#pragma unroll 1
  for (int r = 0; r < tg.rb; ++r) {
    const int64_t blk = tg.blk0 + static_cast<int64_t>(warp * tg.rb + r) * 32 + lane;
    const uint32_t range = d.skip ? 0u : block_range_mask(tg, blk);
    int js[4] = {0, 0, 0, 0};
    float ts[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t keep = 0;
    if (range) {
      const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), stream_of(a), a.rk);
      const Slot e0 = sample_slot<kMode>(d, w.x), e1 = sample_slot<kMode>(d, w.y);
      const Slot e2 = sample_slot<kMode>(d, w.z), e3 = sample_slot<kMode>(d, w.w);
      keep = (e0.ok | (e1.ok << 1) | (e2.ok << 2) | (e3.ok << 3)) & range;
      js[0] = e0.j; js[1] = e1.j; js[2] = e2.j; js[3] = e3.j;
      ts[0] = e0.t; ts[1] = e1.t; ts[2] = e2.t; ts[3] = e3.t;
    }
    int total;
    const int excl = warp_exclusive_count(__popc(keep), total);
    int k = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (keep & (1u << i)) {
        if (a.intervals) a.intervals[row + excl + k] = js[i];
        if (a.offsets) a.offsets[row + excl + k] = ts[i];
        ++k;
      }
    }
    row += total;
  }
}

// First and one-past-last absolute slot of tile tg inside its density.
template <int TPB, int R>
__device__ __forceinline__ void tile_slot_range(const TileGeom& tg, int64_t& s_lo, int64_t& s_hi) {
  const int64_t pb = tg.blk0 << 2, pe = (tg.blk0 + static_cast<int64_t>(TPB) * tg.rb) << 2;
  const int64_t dend = tg.P0 + tg.n;
  s_lo = pb > tg.P0 ? pb : tg.P0;
  s_hi = pe < dend ? pe : dend;
}

// True when every slot of tile tg lies inside its density (all but a
// density's first and last tiles): every block's range mask is then 0xf.
template <int TPB, int R>
__device__ __forceinline__ bool tile_full(const TileGeom& tg) {
  const int64_t pb = tg.blk0 << 2, pe = (tg.blk0 + static_cast<int64_t>(TPB) * tg.rb) << 2;
  return pb >= tg.P0 && pe <= tg.P0 + tg.n;
}

// Publish tile t's kept count, take its first row from the look-back, and
// fill the row offsets its density (and trailing empty densities) own.
// Called by warp 0; returns the base on every lane.
__device__ __forceinline__ int64_t publish_tile(const BatchArgs& a, int32_t t, const TileGeom& tg,
                                                int cnt) {
  const int64_t base = lookback_exclusive(a.tile_state, t, static_cast<uint64_t>(cnt), a.status,
                                          a.spin_limit, t != a.withhold_tile);
  if ((threadIdx.x & 31) == 0) {
    a.tile_prefix[t] = base;
    if (t == __ldg(&a.tile_first[tg.b])) {
      for (int dd = __ldg(&a.rowfill_lo[tg.b]); dd <= tg.b; ++dd) a.row_offsets[dd] = base;
    }
    if (t == a.tiles_total - 1) {
      for (int dd = a.last_nonempty + 1; dd <= a.nd; ++dd) a.row_offsets[dd] = base + cnt;
      a.tile_prefix[t + 1] = base + cnt;  // one past the last row
    }
  }
  return base;
}

// Slope of interval j in fp64 from its records r0 = rec[j], r1 = rec[j + 1]:
// m_j = (g_{j+1} - g_j) / (c_{j+1} - c_j + 1e-5), c = key - d
// (cpp/loits_core.cpp:193-196).
__device__ __forceinline__ double exact_slope(float4 r0, float4 r1) {
  const double c0 = __dsub_rn(static_cast<double>(r0.x), static_cast<double>(r0.y));
  const double c1 = __dsub_rn(static_cast<double>(r1.x), static_cast<double>(r1.y));
  return __ddiv_rn(__dsub_rn(static_cast<double>(r1.z), static_cast<double>(r0.z)),
                   __dadd_rn(__dsub_rn(c1, c0), kEps));
}

// g_j + m_j (u - c_j) in fp64 at the uniform u = k 2^-24 of interval j.
__device__ __forceinline__ double value_at(float4 r0, float4 r1, double m, int k) {
  (void)r1;
  const double c0 = __dsub_rn(static_cast<double>(r0.x), static_cast<double>(r0.y));
  const double u = static_cast<double>(uniform_from_bits(static_cast<uint32_t>(k) << 8));
  return __fma_rn(m, __dsub_rn(u, c0), static_cast<double>(r0.z));
}

// The first 24-bit uniform index k (u = k 2^-24) with u >= key, in [0, 2^24].
__device__ __forceinline__ int first_index_at(float key) {
  const float s = ceilf(key * 16777216.0f);  // exact: a power-of-two scale
  return s <= 0.0f ? 0 : (s >= 16777216.0f ? (1 << 24) : static_cast<int>(s));
}

// The reference's inverse CDF at the uniform of `bits`, in fp64
// (cpp/loits_core.cpp:193-196): the interval j by the sampler's exact search,
// then g_j + m_j (u - c_j) with c_j = key_j - d_j and
// m_j = (g_{j+1} - g_j) / (c_{j+1} - c_j + 1e-5).
template <int kMode>
__device__ __forceinline__ double exact_value(const DensView& d, uint32_t bits) {
  const int j = sample_slot<kMode>(d, bits).j;
  const float4 r0 = rec_at<kMode>(d.rec, j), r1 = rec_at<kMode>(d.rec, j + 1);
  return value_at(r0, r1, exact_slope(r0, r1), bits >> 8);
}

// The threshold of a kThreshold density: the largest k in [-1, 2^24) whose
// uniform k 2^-24 the reference would not keep (x <= cut, x in fp64), found
// by one warp with a 33-ary search; slot p is kept exactly when
// (word >> 8) > k, in the forward and in the backward alike.  (The written
// event is x rounded to fp32.)
template <int kMode>
__device__ __forceinline__ int kept_threshold(const DensView& d) {
  const int lane = threadIdx.x & 31;
  const double cut = static_cast<double>(d.cut);
  int lo = -1, hi = 1 << 24;  // x(lo) <= cut (lo = -1: none), x(hi) > cut (hi = 2^24: all)
  while (hi - lo > 1) {
    const int64_t span = hi - lo;
    const int p = lo + static_cast<int>(span * (lane + 1) / 33);
    bool le = true;
    if (p > lo && p < hi) le = !(exact_value<kMode>(d, static_cast<uint32_t>(p) << 8) > cut);
    const int lo2 = __reduce_max_sync(0xffffffffu, le ? p : lo);
    int hi2 = __reduce_min_sync(0xffffffffu, le ? hi : p);
    if (hi2 <= lo2) hi2 = lo2 + 1;  // only if x were not monotone: still ends
    lo = lo2;
    hi = hi2;
  }
  return lo;
}

// kept_threshold of density b from global memory (its records and full
// guide, final once its CDF is): by one warp, in the item that finishes the
// density's CDF, so that sampling tiles and backward chunks only read it.
__device__ __forceinline__ int density_threshold(const BatchArgs& a, int b, int64_t k0, int64_t G) {
  DensView d{};
  d.rec = a.rec + k0;
  d.guide = a.gl + __ldg(&a.goff[b]);
  d.shift_full = 32 - __ldg(&a.gbits[b]);
  d.shift = d.shift_full;
  d.G = static_cast<int>(G);
  d.coarse = false;
  d.cut = __ldg(&a.x_cut[b]);
  return kept_threshold<kL2>(d);
}

// kept_threshold of density b by every thread of the CTA, from its final
// records in global memory.  With a non-decreasing CDF, the uniforms
// k 2^-24 of interval t are those with key_t <= u < key_{t+1} (interval 0
// also below key_1, interval G-2 up to the last uniform), so x(k) there is
// value_at with interval t's records -- exact_value's arithmetic without its
// search.  x is non-decreasing in k (kThreshold), so the threshold lies in
// the last interval whose first uniform gives x <= cut, where thread 0
// finishes with a binary search.  Returns the threshold on thread 0.
template <int TPB>
__device__ __forceinline__ int threshold_scan(const BatchArgs& a, int b, int64_t k0, int64_t G,
                                              CdfShared<TPB>& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double cut = static_cast<double>(__ldg(&a.x_cut[b]));
  const float4* rec = a.rec + k0;
  const int n_int = static_cast<int>(G) - 1;
  int best = -1;  // last interval (of this thread's) whose first uniform has x <= cut
  for (int t = threadIdx.x; t < n_int; t += TPB) {
    const float4 r0 = __ldcg(rec + t), r1 = __ldcg(rec + t + 1);
    const int klo = t == 0 ? 0 : first_index_at(r0.x);
    const int khi = t == n_int - 1 ? (1 << 24) - 1 : first_index_at(r1.x) - 1;
    if (klo <= khi && !(value_at(r0, r1, exact_slope(r0, r1), klo) > cut)) best = t;
  }
  best = __reduce_max_sync(0xffffffffu, best);
  if (lane == 0) sh.tmax[warp] = best;
  __syncthreads();
  int ks = -1;
  if (threadIdx.x == 0) {
    int t = -1;
    for (int w = 0; w < TPB / 32; ++w) t = sh.tmax[w] > t ? sh.tmax[w] : t;
    if (t >= 0) {
      const float4 r0 = __ldcg(rec + t), r1 = __ldcg(rec + t + 1);
      const double m = exact_slope(r0, r1);
      int lo = t == 0 ? 0 : first_index_at(r0.x);  // x(lo) <= cut
      int hi = t == n_int - 1 ? (1 << 24) : first_index_at(r1.x);  // the next interval's first
      while (hi - lo > 1) {
        const int mid = lo + ((hi - lo) >> 1);
        if (value_at(r0, r1, m, mid) > cut) hi = mid; else lo = mid;
      }
      ks = lo;
    }
  }
  return ks;
}

__device__ __forceinline__ uint32_t threshold_keep(uint4 w, int kstar) {
  return (static_cast<int>(w.x >> 8) > kstar ? 1u : 0u) |
         (static_cast<int>(w.y >> 8) > kstar ? 2u : 0u) |
         (static_cast<int>(w.z >> 8) > kstar ? 4u : 0u) |
         (static_cast<int>(w.w >> 8) > kstar ? 8u : 0u);
}

// Rounds of a warp whose first block is wblk0 that hold slots of tile tg's
// density: all rb for a full tile, else up to the density's last block (a
// warp past it has none).
__device__ __forceinline__ int warp_rounds(const TileGeom& tg, int64_t wblk0, bool full) {
  if (full) return tg.rb;
  if (tg.n <= 0) return 0;
  const int64_t last = (tg.P0 + tg.n - 1) >> 2;  // the density's last block
  const int64_t k = last - wblk0;
  return k < 0 ? 0 : static_cast<int>(k / 32 + 1 < tg.rb ? k / 32 + 1 : tg.rb);
}

// Stores the kept slots of one Philox block at rows p, p + 1, ... in slot
// order: events, and intervals / offsets when the launch writes them.
__device__ __forceinline__ void store_kept(const BatchArgs& a, int64_t p, uint32_t keep,
                                           const Slot& e0, const Slot& e1, const Slot& e2,
                                           const Slot& e3) {
  if (!keep) return;
  const int c1 = keep & 1u, c2 = c1 + ((keep >> 1) & 1u), c3 = c2 + ((keep >> 2) & 1u);
  float* ev = a.events + p;
  if (keep & 1u) __stcs(ev, e0.x);
  if (keep & 2u) __stcs(ev + c1, e1.x);
  if (keep & 4u) __stcs(ev + c2, e2.x);
  if (keep & 8u) __stcs(ev + c3, e3.x);
  if (a.intervals) {
    int32_t* iv = a.intervals + p;
    if (keep & 1u) __stcs(iv, e0.j);
    if (keep & 2u) __stcs(iv + c1, e1.j);
    if (keep & 4u) __stcs(iv + c2, e2.j);
    if (keep & 8u) __stcs(iv + c3, e3.j);
  }
  if (a.offsets) {
    float* ov = a.offsets + p;
    if (keep & 1u) __stcs(ov, e0.t);
    if (keep & 2u) __stcs(ov + c1, e1.t);
    if (keep & 4u) __stcs(ov + c2, e2.t);
    if (keep & 8u) __stcs(ov + c3, e3.t);
  }
}

// Tile of a kThreshold density: each warp counts its kept slots from the
// Philox words alone, the tile publishes its count and takes its first row
// from the look-back, then every warp samples again and stores its kept
// events straight to their final rows (no staging).  Generating the words
// twice measured faster than keeping them in an L2-resident run between
// the passes.
template <int TPB, int R, int kMode>
__device__ __forceinline__ void sample_tile_threshold(const BatchArgs& a, int32_t t,
                                                      const TileGeom& tg, const DensView& d,
                                                      SampleShared& sh) {
  constexpr int W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int kstar = d.kstar;
  const bool full = tile_full<TPB, R>(tg);
  const uint64_t sid = stream_of(a);
  const int64_t wblk0 = tg.blk0 + static_cast<int64_t>(warp * tg.rb) * 32;
  const int rounds = warp_rounds(tg, wblk0, full);
  int cnt = 0;
#pragma unroll 1
  for (int r = 0; r < rounds; ++r) {
    const int64_t blk = wblk0 + r * 32 + lane;
    const uint32_t range = full ? 0xfu : block_range_mask(tg, blk);
    if (!range) continue;
    const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), sid, a.rk);
    cnt += __popc(threshold_keep(w, kstar) & range);
  }
  cnt = warp_sum(cnt);
  if (lane == 0) sh.warp_cnt[warp] = cnt;
  __syncthreads();
  int tile_cnt = 0, warp_excl = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const int c = sh.warp_cnt[w];
    warp_excl += w < warp ? c : 0;
    tile_cnt += c;
  }
  if (lane == 0) a.warp_off[static_cast<int64_t>(t) * W + warp] = warp_excl;
  if (warp == 0) {
    const int64_t base = publish_tile(a, t, tg, tile_cnt);
    if (lane == 0) sh.base = base;
  }
  __syncthreads();
  const int64_t row = sh.base + warp_excl;
  // rows of this warp relative to its first (a tile holds < 2^31 rows)
  float* const evb = a.events + row;
  int32_t* const ivb = a.intervals ? a.intervals + row : nullptr;
  float* const ovb = a.offsets ? a.offsets + row : nullptr;
  int rrow = 0;
  DensView dd = d;
  dd.count_all = false;  // a kThreshold density's CDF is non-decreasing
#pragma unroll 1
  for (int r = 0; r < rounds; ++r) {
    const int64_t blk = wblk0 + r * 32 + lane;
    const uint32_t range = full ? 0xfu : block_range_mask(tg, blk);
    const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), sid, a.rk);
    const uint32_t keep = threshold_keep(w, kstar) & range;
    int total;
    const int excl = warp_exclusive_count(__popc(keep), total);
    const Slot e0 = sample_slot<kMode>(dd, w.x), e1 = sample_slot<kMode>(dd, w.y);
    const Slot e2 = sample_slot<kMode>(dd, w.z), e3 = sample_slot<kMode>(dd, w.w);
    if (keep) {
      const int p = rrow + excl;
      const int c1 = keep & 1u, c2 = c1 + ((keep >> 1) & 1u), c3 = c2 + ((keep >> 2) & 1u);
      if (keep & 1u) __stcs(evb + p, e0.x);
      if (keep & 2u) __stcs(evb + p + c1, e1.x);
      if (keep & 4u) __stcs(evb + p + c2, e2.x);
      if (keep & 8u) __stcs(evb + p + c3, e3.x);
      if (ivb) {
        if (keep & 1u) __stcs(ivb + p, e0.j);
        if (keep & 2u) __stcs(ivb + p + c1, e1.j);
        if (keep & 4u) __stcs(ivb + p + c2, e2.j);
        if (keep & 8u) __stcs(ivb + p + c3, e3.j);
      }
      if (ovb) {
        if (keep & 1u) __stcs(ovb + p, e0.t);
        if (keep & 2u) __stcs(ovb + p + c1, e1.t);
        if (keep & 4u) __stcs(ovb + p + c2, e2.t);
        if (keep & 8u) __stcs(ovb + p + c3, e3.t);
      }
    }
    rrow += total;
  }
}

// Tile of a density whose every event is kept (kAcceptAll): the tile's count
// is its number of slots, published (by the caller, before any event is
// computed) with first row `base`, and slot p lands in row p + (base - s_lo)
// -- the identity compaction, no staging.
template <int TPB, int R, int kMode>
__device__ __forceinline__ void sample_tile_all(const BatchArgs& a, const TileGeom& tg,
                                                const DensView& d, int64_t base) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t s_lo, s_hi;
  tile_slot_range<TPB, R>(tg, s_lo, s_hi);
  const int64_t shiftrow = base - s_lo;
  const bool full = tile_full<TPB, R>(tg);
  const uint64_t sid = stream_of(a);
  const int64_t wblk0 = tg.blk0 + static_cast<int64_t>(warp * tg.rb) * 32;
  const int rounds = warp_rounds(tg, wblk0, full);
#pragma unroll 1
  for (int r = 0; r < rounds; ++r) {
    const int64_t blk = wblk0 + r * 32 + lane;
    const uint32_t range = full ? 0xfu : block_range_mask(tg, blk);
    if (!range) continue;
    const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), sid, a.rk);
    const Slot e0 = sample_slot<kMode>(d, w.x), e1 = sample_slot<kMode>(d, w.y);
    const Slot e2 = sample_slot<kMode>(d, w.z), e3 = sample_slot<kMode>(d, w.w);
    const int64_t row0 = (blk << 2) + shiftrow;
    if (range == 0xfu && (row0 & 3) == 0) {
      // rows row0 .. row0 + 3, 16-byte aligned (events, intervals and offsets
      // buffers start on 16-byte boundaries)
      __stcs(reinterpret_cast<float4*>(a.events + row0), make_float4(e0.x, e1.x, e2.x, e3.x));
      if (a.intervals)
        __stcs(reinterpret_cast<int4*>(a.intervals + row0), make_int4(e0.j, e1.j, e2.j, e3.j));
      if (a.offsets)
        __stcs(reinterpret_cast<float4*>(a.offsets + row0), make_float4(e0.t, e1.t, e2.t, e3.t));
    } else {
      // the kept (in-range) slots at consecutive rows from the first one's
      const int first = __ffs(range) - 1;
      store_kept(a, row0 + first, range, e0, e1, e2, e3);
    }
  }
}

// General tile: kept events are ranked per warp, staged, and stored once the
// tile's first row is known.
template <int TPB, int R, int kMode>
__device__ __forceinline__ void sample_tile_general(const BatchArgs& a, int32_t t,
                                                    const TileGeom& tg, const DensView& d,
                                                    float* stage, SampleShared& sh) {
  constexpr int W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* sw = stage + warp * (tg.rb * 128);
  int acc = 0;
  const bool full = tile_full<TPB, R>(tg);
#pragma unroll 1
  for (int r = 0; r < tg.rb; ++r) {
    const int64_t blk = tg.blk0 + static_cast<int64_t>(warp * tg.rb + r) * 32 + lane;
    const uint32_t range = d.skip ? 0u : (full ? 0xfu : block_range_mask(tg, blk));
    float x0 = 0.f, x1 = 0.f, x2 = 0.f, x3 = 0.f;
    uint32_t keep = 0;
    if (range) {
      const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), stream_of(a), a.rk);
      const Slot e0 = sample_slot<kMode>(d, w.x), e1 = sample_slot<kMode>(d, w.y);
      const Slot e2 = sample_slot<kMode>(d, w.z), e3 = sample_slot<kMode>(d, w.w);
      keep = (e0.ok | (e1.ok << 1) | (e2.ok << 2) | (e3.ok << 3)) & range;
      x0 = e0.x; x1 = e1.x; x2 = e2.x; x3 = e3.x;
    }
    int total;
    int pos = acc + warp_exclusive_count(__popc(keep), total);
    if (keep & 1u) __stcg(&sw[pos++], x0);
    if (keep & 2u) __stcg(&sw[pos++], x1);
    if (keep & 4u) __stcg(&sw[pos++], x2);
    if (keep & 8u) __stcg(&sw[pos], x3);
    acc += total;
  }
  if (lane == 0) sh.warp_cnt[warp] = acc;
  __syncthreads();
  int tile_cnt = 0, warp_excl = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const int c = sh.warp_cnt[w];
    warp_excl += w < warp ? c : 0;
    tile_cnt += c;
  }
  if (lane == 0) a.warp_off[static_cast<int64_t>(t) * W + warp] = warp_excl;
  if (warp == 0) {
    const int64_t base = publish_tile(a, t, tg, tile_cnt);
    if (lane == 0) sh.base = base;
  }
  __syncthreads();
  const int64_t row0 = sh.base + warp_excl;
  warp_store(sw, a.events + row0, acc);
  if (a.intervals || a.offsets) write_intervals<TPB, R, kMode>(a, tg, d, row0);
}

// ------------------------------------------------------- histogram mode
//
// Instead of compacting and writing the kept events, a histogram-mode launch
// bins them: event x adds (1 - f) to bin k and f to bin k + 1 of its
// density's histogram, where k + f = (x - lo) / h - 1/2 (bins of width h
// centred at lo + (k + 1/2) h; weight falling outside the bins is dropped).
// The weights are piecewise linear in x, so d hist_k / d x is defined almost
// everywhere and the backward forms each event's cotangent from the
// histogram's cotangent: (gh[k + 1] - gh[k]) / h.  Order does not matter to a
// histogram: no compaction, no look-back, no event traffic.

__device__ __forceinline__ void hist_bin(const BatchArgs& a, float x, int& k, float& f) {
  float sc = __fmaf_rn(x - a.hist_lo, a.hist_inv_h, -0.5f);
  sc = fminf(fmaxf(sc, -2.0f), static_cast<float>(a.hist_bins) + 1.0f);
  const float fk = floorf(sc);
  k = static_cast<int>(fk);
  f = sc - fk;
}

// Bins a kept event into a tile's shared copy of the histogram in fixed
// point: weights 2^S - w and w = f 2^S rounded (S = hist_shift, so that a
// copy's bins cannot overflow within a tile), one native uint32 atomic each
// (fp32 shared-memory atomicAdd is a compare-and-swap loop).
__device__ __forceinline__ void hist_add(const BatchArgs& a, uint32_t* h, float x) {
  int k;
  float f;
  hist_bin(a, x, k, f);
  const uint32_t one = 1u << a.hist_shift;
  const uint32_t w1 = __float2uint_rn(ldexpf(f, a.hist_shift));
  if (k >= 0 && k < a.hist_bins) atomicAdd(&h[k], one - w1);
  if (k + 1 >= 0 && k + 1 < a.hist_bins) atomicAdd(&h[k + 1], w1);
}

__device__ __forceinline__ float hist_cotangent(const BatchArgs& a, const float* gh, float x) {
  int k;
  float f;
  hist_bin(a, x, k, f);
  const float g0 = (k >= 0 && k < a.hist_bins) ? gh[k] : 0.0f;
  const float g1 = (k + 1 >= 0 && k + 1 < a.hist_bins) ? gh[k + 1] : 0.0f;
  return (g1 - g0) * a.hist_inv_h;
}

// One tile in histogram mode: kept events go into `hist_rep` shared copies
// of the density's histogram (lane l into copy l % rep; copies of one bin
// fall in different banks), merged into the global histogram at the end.
template <int TPB, int R, int kMode>
__device__ __forceinline__ void sample_tile_hist(const BatchArgs& a, const TileGeom& tg,
                                                 const DensView& d, float* hs) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nb = a.hist_bins, stride = nb + 1;
  const int rep = a.hist_rep;
  uint32_t* hu = reinterpret_cast<uint32_t*>(hs);
  for (int i = threadIdx.x; i < rep * stride; i += TPB) hu[i] = 0u;
  __syncthreads();
  uint32_t* mine = hu + (lane & (rep - 1)) * stride;
  const bool full = tile_full<TPB, R>(tg);
  const int kstar = d.kstar;
  int kept = 0;
#pragma unroll 1
  for (int r = 0; r < tg.rb; ++r) {
    const int64_t blk = tg.blk0 + static_cast<int64_t>(warp * tg.rb + r) * 32 + lane;
    const uint32_t range = d.skip ? 0u : (full ? 0xfu : block_range_mask(tg, blk));
    if (!range) continue;
    const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), stream_of(a), a.rk);
    const Slot e0 = sample_slot<kMode>(d, w.x), e1 = sample_slot<kMode>(d, w.y);
    const Slot e2 = sample_slot<kMode>(d, w.z), e3 = sample_slot<kMode>(d, w.w);
    const uint32_t keep = (d.threshold ? threshold_keep(w, kstar)
                                       : (e0.ok | (e1.ok << 1) | (e2.ok << 2) | (e3.ok << 3))) &
                          range;
    if (keep & 1u) hist_add(a, mine, e0.x);
    if (keep & 2u) hist_add(a, mine, e1.x);
    if (keep & 4u) hist_add(a, mine, e2.x);
    if (keep & 8u) hist_add(a, mine, e3.x);
    kept += __popc(keep);
  }
  kept = warp_sum(kept);
  if (lane == 0 && kept) atomicAdd(&a.kept[tg.b], static_cast<unsigned long long>(kept));
  __syncthreads();
  float* out = a.hist + static_cast<int64_t>(tg.b) * nb;
  for (int k = threadIdx.x; k < nb; k += TPB) {
    unsigned long long v = hu[k];
    for (int c = 1; c < rep; ++c) v += hu[c * stride + k];
    if (v != 0ull) atomicAdd(&out[k], ldexpf(static_cast<float>(v), -a.hist_shift));
  }
  __syncthreads();
}

// The first bucket k0 of the run of coarse-guide buckets [k0, k1] that holds
// the most uniforms while L[k1] - L[k0] <= room, i.e. whose knots fit a window
// of room + 1 counts: the density's most probable stretch.  Each thread tries
// every 4th bucket start (binary search for k1); ties go to the smallest k0.
// Returns the same k0 on every thread; ends with a barrier.
template <int TPB>
__device__ __forceinline__ int most_probable_run(const uint32_t* L, int M, uint32_t room,
                                                 SampleShared& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int best_span = -1, best_k0 = 0;
  for (int k0 = threadIdx.x * 4; k0 < M; k0 += TPB * 4) {
    const uint32_t lim = L[k0] + room;
    int lo = k0, hi = M;  // largest k1 in [k0, M] with L[k1] <= lim
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (L[mid] <= lim) lo = mid; else hi = mid - 1;
    }
    if (lo - k0 > best_span) { best_span = lo - k0; best_k0 = k0; }
  }
  const int wspan = __reduce_max_sync(0xffffffffu, best_span);
  const int wk0 = __reduce_min_sync(0xffffffffu, best_span == wspan ? best_k0 : 0x7fffffff);
  if (lane == 0) { sh.warp_cnt[warp] = wspan; sh.red[warp] = __int_as_float(wk0); }
  __syncthreads();
  if (threadIdx.x == 0) {
    int span = -1, k0 = 0;
    for (int w = 0; w < TPB / 32; ++w) {
      const int k = __float_as_int(sh.red[w]);
      if (sh.warp_cnt[w] > span || (sh.warp_cnt[w] == span && k < k0)) {
        span = sh.warp_cnt[w];
        k0 = k;
      }
    }
    sh.run_k0 = k0;
  }
  __syncthreads();
  return sh.run_k0;
}

// Forward, large density with a coarse guide: the window of fwin_n records
// [wk0, wk1) around its most probable stretch, copied to shared memory (rec_s)
// when the view is fresh (its coarse guide was just copied: a small density
// or another large one used the slot since).  Slots whose coarse bucket lies
// inside the window are searched there (sample_slot).  Ends with a barrier.
template <int TPB>
__device__ __forceinline__ void forward_window(const BatchArgs& a, DensView& d, int64_t k0,
                                               float4* rec_s, int2& win, SampleShared& sh) {
  if (d.skip) {  // not sampled
    d.wk0 = d.wk1 = 0;
    return;
  }
  if (d.fresh) {
    const int W = min(a.fwin_n, d.G);
    const int M = 1 << (32 - d.shift);
    // buckets [k0, k1] with L[k1] <= L[k0] + W - 2 hold counts the window
    // [L[k0] - 1, L[k0] - 1 + W) answers (see sample_slot)
    const int kb = most_probable_run<TPB>(d.cguide, M, static_cast<uint32_t>(W - 2), sh);
    const int w0 = max(min(static_cast<int>(d.cguide[kb]) - 1, d.G - W), 0);
    for (int i = threadIdx.x; i < W; i += TPB) rec_s[i] = __ldcg(&a.rec[k0 + w0 + i]);
    if (threadIdx.x == 0) win = make_int2(w0, w0 + W);
    __syncthreads();
  }
  d.wrec = rec_s;
  d.wk0 = win.x;
  d.wk1 = win.y;
}

// kLarge: the plan has densities above the shared-memory limit (compiled
// separately so that plans without them carry none of the global-memory path).
template <int TPB, int R, bool kLarge>
__device__ __forceinline__ void sample_item(const BatchArgs& a, int32_t t, float4* rec_s,
                                            uint32_t* guide_s, float* stage, SampleShared& sh,
                                            int& guide_key, int2& win, BulkStage bulk) {
  const TileGeom tg = tile_geom<TPB, R>(a, t);
  const bool large = kLarge && tg.G > a.gcap;
  density_flags(a, tg.b, large, true, sh);
  if (a.hist) {
    float* hs = reinterpret_cast<float*>(rec_s) + a.hist_smem_off;
    if (large) {
      DensView d = density_view(a, tg.b, tg.k0, tg.G, true, rec_s, guide_s, nullptr, sh,
                                guide_key, bulk);
      if (d.coarse) forward_window<TPB>(a, d, tg.k0, rec_s, win, sh);
      sample_tile_hist<TPB, R, kL2>(a, tg, d, hs);
    } else {
      const DensView d = density_view(a, tg.b, tg.k0, tg.G, false, rec_s, guide_s, nullptr, sh,
                                     guide_key, bulk);
      sample_tile_hist<TPB, R, kShared>(a, tg, d, hs);
    }
    return;
  }
  if ((sh.flags & kAcceptAll) && threadIdx.x < 32) {
    // identity compaction: the count is known now, so the row look-back runs
    // while the other warps copy the density
    int64_t s_lo, s_hi;
    tile_slot_range<TPB, R>(tg, s_lo, s_hi);
    const int64_t base = publish_tile(a, t, tg, static_cast<int>(s_hi - s_lo));
    if (threadIdx.x == 0) sh.base = base;
  }
  // one view per branch: each sees constant `large` (shared or global loads)
  if (large) {
    DensView d = density_view(a, tg.b, tg.k0, tg.G, true, rec_s, guide_s, nullptr, sh,
                              guide_key, bulk);
    if (d.coarse) forward_window<TPB>(a, d, tg.k0, rec_s, win, sh);
    if (d.accept_all) sample_tile_all<TPB, R, kL2>(a, tg, d, sh.base);
    else if (d.threshold) sample_tile_threshold<TPB, R, kL2>(a, t, tg, d, sh);
    else sample_tile_general<TPB, R, kL2>(a, t, tg, d, stage, sh);
  } else {
    const DensView d = density_view(a, tg.b, tg.k0, tg.G, false, rec_s, guide_s, nullptr, sh,
                                   guide_key, bulk);
    if (d.accept_all) sample_tile_all<TPB, R, kShared>(a, tg, d, sh.base);
    else if (d.threshold) sample_tile_threshold<TPB, R, kShared>(a, t, tg, d, sh);
    else sample_tile_general<TPB, R, kShared>(a, t, tg, d, stage, sh);
  }
}

// --------------------------------------------------------- backward phase

// Where a backward chunk accumulates its grad-CDF.
//  * small densities, fp32: gacc (shared memory), two fp32 atomics per kept
//    slot;
//  * small densities, fixed point (fix): per interval j the two sums
//    A_j = sum g and B_j = sum g w of integer terms (units of 1/scale), each
//    held as two uint32 words (alo/ahi/blo/bhi, planar so that consecutive
//    intervals use consecutive banks): a term v is split into its low s bits
//    v mod 2^s and its high part v >> s (arithmetic), and each part is added
//    to its word with one native uint32 shared-memory reduction -- no
//    returned value, no carry to propagate.  Shared-memory fp32 atomicAdd is
//    a compare-and-swap loop, slow where many lanes hit one interval; uint32
//    reductions are native even then, and integer sums do not depend on their
//    order.  The chunk's grad-CDF is formed from A and B when the chunk ends:
//    gcdf_k = m_k (B_k - A_k) - m_{k-1} B_{k-1};
//  * large densities: the same fixed-point sums for the intervals of a window
//    [win_lo, win_lo + win_n) (the most probable ones), one float2 global
//    atomic per kept slot for the others (gc).
// Neither word can wrap: with at most 2^lg kept rows in the chunk, s =
// 32 - lg keeps the low words below 2^32, and a term is added only while its
// scaled magnitude stays below cap = 2^min(30, 30 + s - lg), which keeps the
// high words inside int32.  A larger (or non-finite) cotangent's terms take
// the fp32 path instead, as global fp32 reductions: into the chunk's partial
// (`spill`, zeroed when the chunk starts and added to the fixed-point sums
// when it ends) for small densities, into gc for large ones.  Non-finite
// values therefore reach the gradient as they would through fp32 sums.
struct Acc {
  float* gacc;
  uint32_t *alo, *ahi, *blo, *bhi;
  float2* gc;
  float* spill;
  float scale, cap;
  int lbits;       // s: bits of a term in its low word
  uint32_t lmask;  // 2^s - 1
  int win_lo, win_n;
};

// Adds integer term v (|v| < 2^30) to the split sum (lo, hi) at index i: its
// low s bits to lo, its (signed) high part to hi.  Skipping the zero high
// parts measured slower: the lanes of a warp diverge on the sign.
__device__ __forceinline__ void fix_add(const Acc& acc, uint32_t* lo, uint32_t* hi, int i, int v) {
  atomicAdd(&lo[i], static_cast<uint32_t>(v) & acc.lmask);  // no return value: reductions
  atomicAdd(&hi[i], static_cast<uint32_t>(v >> acc.lbits));
}

// The split sum's value (hi 2^s + lo) in cotangent units.
__device__ __forceinline__ double fix_value(uint32_t lo, uint32_t hi, int lbits, double inv_scale) {
  return (ldexp(static_cast<double>(static_cast<int32_t>(hi)), lbits) + static_cast<double>(lo)) *
         inv_scale;
}

// One kept slot's (g, g w) into fixed-point slot i, when both scaled terms
// are below the chunk's cap (false: nothing added, the caller takes the fp32
// path).
__device__ __forceinline__ bool fix_pair(const Acc& acc, int i, float g, float w) {
  const float f0 = g * acc.scale, f1 = (g * w) * acc.scale;
  if (!(fabsf(f0) < acc.cap) || !(fabsf(f1) < acc.cap)) return false;
  fix_add(acc, acc.alo, acc.ahi, i, __float2int_rn(f0));
  fix_add(acc, acc.blo, acc.bhi, i, __float2int_rn(f1));
  return true;
}

__device__ __forceinline__ void red_add_f32x2(float2* p, float x, float y) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(x), "f"(y) : "memory");
}

// Scatter of one kept slot's cotangent into the grad-CDF:
// d x / d c_j = m (w - 1), d x / d c_{j+1} = -m w, w = (u - c_j) / d_j
// (cpp/loits_core.cpp:293-300).
// kFix (small densities): fixed-point sums instead of fp32 atomics.
template <int kMode, bool kFix>
__device__ __forceinline__ void scatter_slot(const Slot& e, float g, const DensView& d,
                                             const Acc& acc) {
  float inv;
  if constexpr (kMode == kShared) inv = d.invd[e.j];
  else inv = __ldg(&d.invd[e.j]);
  const float w = e.t * inv;
  if constexpr (kMode == kShared) {
    if constexpr (kFix) {
      if (!fix_pair(acc, e.j, g, w)) {
        const float mg = e.m * g;
        atomicAdd(&acc.spill[e.j], mg * (w - 1.0f));  // no return value: a reduction
        atomicAdd(&acc.spill[e.j + 1], -(mg * w));
      }
    } else {
      const float mg = e.m * g;
      atomicAdd(&acc.gacc[e.j], mg * (w - 1.0f));
      atomicAdd(&acc.gacc[e.j + 1], -(mg * w));
    }
  } else {
    const unsigned wj = static_cast<unsigned>(e.j - acc.win_lo);
    if (!(wj < static_cast<unsigned>(acc.win_n) && fix_pair(acc, static_cast<int>(wj), g, w))) {
      const float mg = e.m * g;
      red_add_f32x2(&acc.gc[e.j], mg * (w - 1.0f), -(mg * w));
    }
  }
}

// Backward chunk from a saved state: the chunk's kept rows [r0, r1) carry
// their interval and offset u - c_j, so no uniform is regenerated and no
// interval searched; each row scatters exactly what scatter_slot would for
// the replayed slot.  Saved intervals are clamped to [0, G - 2], so reads
// stay inside the density for any state contents.
template <int TPB, int kMode, bool kFix>
__device__ __forceinline__ void vjp_chunk_rows(const BatchArgs& a, const DensView& d, int64_t r0,
                                               int64_t r1, const Acc& acc) {
  constexpr int U = 4;  // rows per thread in flight
  const int jmax = d.G - 2;
  if (jmax < 0) return;
#pragma unroll 1
  for (int64_t base = r0; base < r1; base += static_cast<int64_t>(TPB) * U) {
    Slot e[U];
    float g[U];
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const int64_t r = base + i * TPB + threadIdx.x;
      e[i].ok = r < r1;
      e[i].j = 0;
      e[i].t = 0.0f;
      g[i] = 0.0f;
      if (e[i].ok) {
        e[i].j = min(max(__ldcs(&a.st_intervals[r]), 0), jmax);
        e[i].t = __ldcs(&a.st_offsets[r]);
        g[i] = __ldcs(&a.grad[r]);
      }
    }
#pragma unroll
    for (int i = 0; i < U; ++i) {
      if (!e[i].ok) continue;
      const float* m = reinterpret_cast<const float*>(d.rec + e[i].j) + 3;
      if constexpr (kMode == kShared) e[i].m = *m;
      else e[i].m = __ldg(m);
      scatter_slot<kMode, kFix>(e[i], g[i], d, acc);
    }
  }
}

// The tiles [t_first, t_end) of one backward chunk.  Every warp replays its
// own slots of each tile; the forward recorded where its kept rows start
// (tile_prefix + warp_off), so no scan across warps and no barrier is needed.
template <int TPB, int R, int kMode, bool kFix>
__device__ __forceinline__ void vjp_chunk_tiles(const BatchArgs& a, const DensView& d, TileGeom tg,
                                                int32_t tb, int32_t t_first, int32_t t_end,
                                                const Acc& acc, const float* gh) {
  constexpr int W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (d.skip) return;
  if (a.st_intervals) {
    // saved state: the chunk's rows run from its first tile's first row to
    // the next tile's (tile_prefix has an entry past the last tile)
    vjp_chunk_rows<TPB, kMode, kFix>(a, d, __ldcg(&a.tile_prefix[t_first]),
                               __ldcg(&a.tile_prefix[t_end]), acc);
    return;
  }
  // kThreshold densities keep exactly the slots the forward kept by threshold
  const int kstar = d.kstar;
  if (gh) {
    // histogram mode: every kept slot's cotangent comes from the histogram's
#pragma unroll 1
    for (int32_t t = t_first; t < t_end; ++t) {
      tg.blk0 = (tg.P0 >> 2) + static_cast<int64_t>(t - tb) * TPB * tg.rb;
      const bool full = tile_full<TPB, R>(tg);
#pragma unroll 1
      for (int r = 0; r < tg.rb; ++r) {
        const int64_t blk = tg.blk0 + static_cast<int64_t>(warp * tg.rb + r) * 32 + lane;
        const uint32_t range = full ? 0xfu : block_range_mask(tg, blk);
        if (!range) continue;
        const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), stream_of(a), a.rk);
        const Slot e0 = sample_slot<kMode>(d, w.x), e1 = sample_slot<kMode>(d, w.y);
        const Slot e2 = sample_slot<kMode>(d, w.z), e3 = sample_slot<kMode>(d, w.w);
        const uint32_t keep = (d.threshold ? threshold_keep(w, kstar)
                                           : (e0.ok | (e1.ok << 1) | (e2.ok << 2) | (e3.ok << 3))) &
                              range;
        if (keep & 1u) scatter_slot<kMode, kFix>(e0, hist_cotangent(a, gh, e0.x), d, acc);
        if (keep & 2u) scatter_slot<kMode, kFix>(e1, hist_cotangent(a, gh, e1.x), d, acc);
        if (keep & 4u) scatter_slot<kMode, kFix>(e2, hist_cotangent(a, gh, e2.x), d, acc);
        if (keep & 8u) scatter_slot<kMode, kFix>(e3, hist_cotangent(a, gh, e3.x), d, acc);
      }
    }
    return;
  }
  if (d.accept_all) {
    // identity compaction: slot p of tile t is row p + (tile_prefix[t] - s_lo)
#pragma unroll 1
    for (int32_t t = t_first; t < t_end; ++t) {
      tg.blk0 = (tg.P0 >> 2) + static_cast<int64_t>(t - tb) * TPB * tg.rb;
      int64_t s_lo, s_hi;
      tile_slot_range<TPB, R>(tg, s_lo, s_hi);
      const int64_t shiftrow = __ldcg(&a.tile_prefix[t]) - s_lo;
      const bool full = tile_full<TPB, R>(tg);
#pragma unroll 1
      for (int r = 0; r < tg.rb; ++r) {
        const int64_t blk = tg.blk0 + static_cast<int64_t>(warp * tg.rb + r) * 32 + lane;
        const uint32_t range = full ? 0xfu : block_range_mask(tg, blk);
        if (!range) continue;
        const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), stream_of(a), a.rk);
        const int64_t row0 = (blk << 2) + shiftrow;
        float4 g4;
        if (range == 0xfu && (row0 & 3) == 0) {
          g4 = __ldcs(reinterpret_cast<const float4*>(a.grad + row0));
        } else {
          g4.x = (range & 1u) ? __ldcs(a.grad + row0) : 0.0f;
          g4.y = (range & 2u) ? __ldcs(a.grad + row0 + 1) : 0.0f;
          g4.z = (range & 4u) ? __ldcs(a.grad + row0 + 2) : 0.0f;
          g4.w = (range & 8u) ? __ldcs(a.grad + row0 + 3) : 0.0f;
        }
        // all four slots first: their record loads must not wait behind the
        // grad-CDF atomics (which the compiler cannot prove disjoint)
        const Slot e0 = sample_slot<kMode>(d, w.x), e1 = sample_slot<kMode>(d, w.y);
        const Slot e2 = sample_slot<kMode>(d, w.z), e3 = sample_slot<kMode>(d, w.w);
        if (range & 1u) scatter_slot<kMode, kFix>(e0, g4.x, d, acc);
        if (range & 2u) scatter_slot<kMode, kFix>(e1, g4.y, d, acc);
        if (range & 4u) scatter_slot<kMode, kFix>(e2, g4.z, d, acc);
        if (range & 8u) scatter_slot<kMode, kFix>(e3, g4.w, d, acc);
      }
    }
    return;
  }
#pragma unroll 1
  for (int32_t t = t_first; t < t_end; ++t) {
    tg.blk0 = (tg.P0 >> 2) + static_cast<int64_t>(t - tb) * TPB * tg.rb;
    int64_t row = __ldcg(&a.tile_prefix[t]) + __ldcg(&a.warp_off[static_cast<int64_t>(t) * W + warp]);
    const bool full = tile_full<TPB, R>(tg);
#pragma unroll 1
    for (int r = 0; r < tg.rb; ++r) {
      const int64_t blk = tg.blk0 + static_cast<int64_t>(warp * tg.rb + r) * 32 + lane;
      const uint32_t range = full ? 0xfu : block_range_mask(tg, blk);
      Slot e0, e1, e2, e3;
      uint32_t keep = 0;
      if (range) {
        const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), stream_of(a), a.rk);
        e0 = sample_slot<kMode>(d, w.x);
        e1 = sample_slot<kMode>(d, w.y);
        e2 = sample_slot<kMode>(d, w.z);
        e3 = sample_slot<kMode>(d, w.w);
        keep = (d.threshold ? threshold_keep(w, kstar)
                            : (e0.ok | (e1.ok << 1) | (e2.ok << 2) | (e3.ok << 3))) &
               range;
      }
      int total;
      int64_t my = row + warp_exclusive_count(__popc(keep), total);
      if (keep & 1u) scatter_slot<kMode, kFix>(e0, __ldcs(&a.grad[my++]), d, acc);
      if (keep & 2u) scatter_slot<kMode, kFix>(e1, __ldcs(&a.grad[my++]), d, acc);
      if (keep & 4u) scatter_slot<kMode, kFix>(e2, __ldcs(&a.grad[my++]), d, acc);
      if (keep & 8u) scatter_slot<kMode, kFix>(e3, __ldcs(&a.grad[my]), d, acc);
      row += total;
    }
  }
}

// The fixed-point paths are compiled for CTAs of 512 and 1024 threads only
// (64 registers; the 48 of a 256-thread CTA would spill), whose shared memory
// has room for them.
template <int TPB>
constexpr bool kFixPaths = TPB >= 512;

// Fixed-point geometry of a backward chunk of at most `rows` kept rows (in
// histogram mode its slots), into sh: with rows <= 2^lg, the low-word bits
// s = 32 - lg, the term bound cap = 2^min(30, 30 + s - lg) (see Acc), and
// the scale, a power of two that puts the mean |cotangent| of up to TPB of
// the chunk's kept rows near 2^p, p = min(20, log2(cap) - 10): one unit is
// about 1e-6 of a typical contribution where the chunk allows, and terms up
// to 2^10 times the mean stay in fixed point.  Histogram mode: the mean
// histogram-cotangent step instead.  Ends with a barrier.
template <int TPB>
__device__ __forceinline__ void chunk_scale(const BatchArgs& a, const float* gh, int64_t r0,
                                            int64_t r1, int64_t rows, SampleShared& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float v = 0.0f, c = 0.0f;
  if (gh) {
    const int nb = a.hist_bins;
    for (int k = threadIdx.x; k <= nb; k += TPB) {
      const float g1 = k < nb ? gh[k] : 0.0f, g0 = k > 0 ? gh[k - 1] : 0.0f;
      const float q = fabsf(g1 - g0) * a.hist_inv_h;
      if (q < 3.0e38f) { v += q; c += 1.0f; }
    }
  } else if (r0 + threadIdx.x < r1) {
    const float q = fabsf(__ldcg(&a.grad[r0 + threadIdx.x]));
    if (q < 3.0e38f) { v = q; c = 1.0f; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if (lane == 0) { sh.red[warp] = v; sh.warp_cnt[warp] = static_cast<int>(c); }
  __syncthreads();
  if (threadIdx.x == 0) {
    float sum = 0.0f;
    int cnt = 0;
    for (int w = 0; w < TPB / 32; ++w) { sum += sh.red[w]; cnt += sh.warp_cnt[w]; }
    int e = 0;
    if (cnt > 0 && sum > 0.0f) frexpf(sum / cnt, &e);
    e = min(max(e, -100), 100);
    const int lg = rows > 1 ? 64 - __clzll(static_cast<unsigned long long>(rows - 1)) : 0;
    const int lbits = max(1, min(31, 32 - lg));
    const int cap_log = min(30, 30 + lbits - lg);
    sh.fix_scale = ldexpf(1.0f, min(20, cap_log - 10) - e);
    sh.fix_cap = ldexpf(1.0f, cap_log);
    sh.fix_lbits = lbits;
  }
  __syncthreads();
}

// The window of a large density's fixed-point sums (into sh.win_lo): the run
// of win_n intervals that holds the most probability (buckets k0 .. k1 of
// the coarse guide map to intervals L[k0] - 1 .. L[k1] - 1).  Ends with a
// barrier.
template <int TPB>
__device__ __forceinline__ void large_window(const BatchArgs& a, const DensView& d, int b,
                                             SampleShared& sh) {
  const int M = 1 << (32 - d.shift);
  const int k0 = most_probable_run<TPB>(d.cguide, M, static_cast<uint32_t>(a.win_n - 1), sh);
  if (threadIdx.x == 0) {
    const int n_int = d.G - 1;  // intervals of the density
    const int lo = min(static_cast<int>(d.cguide[k0]) - 1, n_int - a.win_n);
    sh.win_lo = max(lo, 0);
    sh.win_b = b;
  }
  __syncthreads();
}

// Saved-state chunk of a small density with a non-decreasing CDF, in fixed
// point: the weights 1/d_j in shared memory (smem[0, G)), the sums A, B
// after them, the chunk's partial `part` taking the fp32 reductions of terms
// above the cap; each kept row reads its interval, offset and cotangent
// (coalesced) and one weight; the slopes enter per interval when the chunk
// ends, read from the records in global memory.  Ends with every partial
// written (not fenced).
template <int TPB>
__device__ __forceinline__ void vjp_state_chunk_fix(const BatchArgs& a, int64_t k0, int G,
                                                    int64_t r0, int64_t r1, float* part,
                                                    float* smem, SampleShared& sh) {
  float* invd_s = smem;
  uint32_t* base = reinterpret_cast<uint32_t*>(smem + ((G + 3) & ~3));
  for (int i = threadIdx.x; i < G; i += TPB) {
    invd_s[i] = __ldg(&a.invd[k0 + i]);
    __stcg(&part[i], 0.0f);
  }
  for (int i = threadIdx.x; i < 4 * G; i += TPB) base[i] = 0u;
  chunk_scale<TPB>(a, nullptr, r0, r1, r1 - r0, sh);
  Acc acc{};
  acc.alo = base;
  acc.ahi = base + G;
  acc.blo = base + 2 * G;
  acc.bhi = base + 3 * G;
  acc.scale = sh.fix_scale;
  acc.cap = sh.fix_cap;
  acc.lbits = sh.fix_lbits;
  acc.lmask = (1u << acc.lbits) - 1u;
  const float4* rec = a.rec + k0;
  const int jmax = G - 2;
  // one row's fixed-point terms (or, above the chunk's cap, fp32 reductions)
  auto add_row = [&](int j, float t, float g) {
    j = min(max(j, 0), jmax);
    const float w = t * invd_s[j];
    if (!fix_pair(acc, j, g, w)) {
      const float mg = __ldg(&rec[j].w) * g;
      atomicAdd(&part[j], mg * (w - 1.0f));  // no return value: reductions
      atomicAdd(&part[j + 1], -(mg * w));
    }
  };
  // rows up to the first multiple of 4 and past the last one singly; the
  // rest as 16-byte vectors of 4 rows per array (the three arrays start on
  // 16-byte boundaries when their base pointers do)
  const bool vec = ((reinterpret_cast<uintptr_t>(a.st_intervals) |
                     reinterpret_cast<uintptr_t>(a.st_offsets) |
                     reinterpret_cast<uintptr_t>(a.grad)) & 15) == 0;
  const int64_t q0 = vec ? (r0 + 3) >> 2 : r1, q1 = vec ? r1 >> 2 : r1;  // quads [q0, q1)
  const int64_t body0 = q0 < q1 ? 4 * q0 : r1, body1 = q0 < q1 ? 4 * q1 : r1;
  for (int64_t r = r0 + threadIdx.x; r < body0; r += TPB)
    add_row(__ldcs(&a.st_intervals[r]), __ldcs(&a.st_offsets[r]), __ldcs(&a.grad[r]));
  for (int64_t r = body1 + threadIdx.x; r < r1; r += TPB)
    add_row(__ldcs(&a.st_intervals[r]), __ldcs(&a.st_offsets[r]), __ldcs(&a.grad[r]));
  const int4* iv4 = reinterpret_cast<const int4*>(a.st_intervals);
  const float4* of4 = reinterpret_cast<const float4*>(a.st_offsets);
  const float4* gr4 = reinterpret_cast<const float4*>(a.grad);
#pragma unroll 1
  for (int64_t q = q0 + threadIdx.x; q < q1; q += TPB) {
    const int4 j4 = __ldcs(&iv4[q]);
    const float4 t4 = __ldcs(&of4[q]);
    const float4 g4 = __ldcs(&gr4[q]);
    add_row(j4.x, t4.x, g4.x);
    add_row(j4.y, t4.y, g4.y);
    add_row(j4.z, t4.z, g4.z);
    add_row(j4.w, t4.w, g4.w);
  }
  __threadfence();
  __syncthreads();
  const double inv_scale = 1.0 / static_cast<double>(acc.scale);
  for (int i = threadIdx.x; i < G; i += TPB) {
    // gcdf_i = m_i (B_i - A_i) - m_{i-1} B_{i-1} (no interval starts at knot G-1)
    double v = 0.0;
    if (i + 1 < G)
      v = static_cast<double>(__ldg(&rec[i].w)) *
          (fix_value(acc.blo[i], acc.bhi[i], acc.lbits, inv_scale) -
           fix_value(acc.alo[i], acc.ahi[i], acc.lbits, inv_scale));
    if (i > 0)
      v -= static_cast<double>(__ldg(&rec[i - 1].w)) *
           fix_value(acc.blo[i - 1], acc.bhi[i - 1], acc.lbits, inv_scale);
    __stcg(&part[i], static_cast<float>(v + static_cast<double>(__ldcg(&part[i]))));
  }
}

// Backward chunk (density, run of sampling tiles).  kFix: the plan has small
// densities that sum in fixed point (compiled separately: the fp32 path
// alone needs fewer registers).
template <int TPB, int R, bool kLarge, bool kFix>
__device__ __forceinline__ void vjp_chunk_item(const BatchArgs& a, int32_t k, float4* rec_s,
                                               uint32_t* guide_s, float* invd_s, float* gacc_s,
                                               SampleShared& sh, int& guide_key, BulkStage bulk) {
  const int b = __ldg(&a.chunk_owner[k]);
  const int32_t ki = k - __ldg(&a.chunk_first[b]);
  const int32_t tb = __ldg(&a.tile_first[b]);
  const int32_t t_first = tb + ki * a.tiles_per_chunk;
  const int32_t t_end0 = t_first + a.tiles_per_chunk;
  const int32_t t_end = t_end0 < __ldg(&a.tile_first[b + 1]) ? t_end0 : __ldg(&a.tile_first[b + 1]);
  const TileGeom tg = tile_geom<TPB, R>(a, t_first);
  const int G = static_cast<int>(tg.G);
  // histogram mode: the density's histogram cotangent, in shared memory
  float* gh = nullptr;
  if (a.grad_hist) {
    gh = reinterpret_cast<float*>(rec_s) + a.hist_smem_off;
    const float* src = a.grad_hist + static_cast<int64_t>(b) * a.hist_bins;
    for (int k = threadIdx.x; k < a.hist_bins; k += TPB) gh[k] = __ldg(&src[k]);
  }
  // the chunk's kept rows (event modes): [tile_prefix[t_first], tile_prefix[t_end])
  const int64_t r0 = gh ? 0 : __ldcg(&a.tile_prefix[t_first]);
  const int64_t r1 = gh ? 0 : __ldcg(&a.tile_prefix[t_end]);
  // an upper bound on the chunk's kept rows (histogram mode: its slots)
  const int64_t chunk_rows =
      gh ? static_cast<int64_t>(t_end - t_first) * TPB * tg.rb * 4 : r1 - r0;
  Acc acc{};
  if (kLarge && tg.G > a.gcap) {
    const DensView d = load_density(a, b, tg.k0, tg.G, true, nullptr, guide_s, nullptr, false,
                                    sh, guide_key, bulk);
    acc.gc = a.gcdf + __ldg(&a.gc_off[b]);
    const bool win = kFixPaths<TPB> && a.win_n > 0 && d.coarse && !d.skip && G - 1 > a.win_n;
    if (win) {
      // the window's sums live where small densities keep their records
      if (sh.win_b != b) large_window<TPB>(a, d, b, sh);
      uint32_t* base = reinterpret_cast<uint32_t*>(rec_s);
      for (int i = threadIdx.x; i < 4 * a.win_n; i += TPB) base[i] = 0u;
      chunk_scale<TPB>(a, gh, r0, r1, chunk_rows, sh);
      acc.alo = base;
      acc.ahi = base + a.win_n;
      acc.blo = base + 2 * a.win_n;
      acc.bhi = base + 3 * a.win_n;
      acc.scale = sh.fix_scale;
      acc.cap = sh.fix_cap;
      acc.lbits = sh.fix_lbits;
      acc.lmask = (1u << acc.lbits) - 1u;
      acc.win_lo = sh.win_lo;
      acc.win_n = a.win_n;
    }
    vjp_chunk_tiles<TPB, R, kRO, false>(a, d, tg, tb, t_first, t_end, acc, gh);
    if (win) {
      __syncthreads();
      const double inv_scale = 1.0 / static_cast<double>(acc.scale);
      for (int i = threadIdx.x; i < a.win_n; i += TPB) {
        if ((acc.alo[i] | acc.ahi[i] | acc.blo[i] | acc.bhi[i]) == 0u) continue;
        const int j = acc.win_lo + i;
        const double A = fix_value(acc.alo[i], acc.ahi[i], acc.lbits, inv_scale);
        const double Bs = fix_value(acc.blo[i], acc.bhi[i], acc.lbits, inv_scale);
        const double m = static_cast<double>(__ldg(reinterpret_cast<const float*>(d.rec + j) + 3));
        red_add_f32x2(&acc.gc[j], static_cast<float>(m * (Bs - A)), static_cast<float>(-m * Bs));
      }
    }
    // the density's grad-CDF atomics are performed before the chunk counts
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&a.chunks_done[b], 1u);
    return;
  }
  float* part = a.partials + __ldg(&a.part_off[b]) + static_cast<int64_t>(ki) * G;
  // fp32 sums, replicated `rep` times in the shared slot sized for the
  // largest density (copy c at c * (G + 1): copies of one knot fall in
  // different banks); lane l adds into copy l % rep, so lanes whose events
  // share an interval (small, peaked densities) rarely collide
  int rep = 1;
  while (rep < 32 && 2 * rep * (G + 1) <= a.gcap) rep *= 2;
  // Saved state: each kept row carries its interval and offset, so the chunk
  // needs only the weights 1/d_j in shared memory (no records, no guide) and
  // sums every row in fixed point.
  if (kFixPaths<TPB> && a.st_intervals && 20ll * G <= 4ll * a.bwd_guide_off) {
    density_flags(a, b, false, false, sh);
    if (!(sh.flags & kNonMonotone)) {
      vjp_state_chunk_fix<TPB>(a, tg.k0, G, r0, r1, part, reinterpret_cast<float*>(rec_s), sh);
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) atomicAdd(&a.chunks_done[b], 1u);
      return;
    }
  }
  // Fixed-point sums instead (native uint32 reductions, fast however many
  // lanes share an interval) where the density's records, weights and sums
  // (36 bytes per knot) fit the slot before the guide: records at 0,
  // weights at 16 G, sums A, B at 20 G bytes.
  if (kFix && kFixPaths<TPB> && 36ll * G <= 4ll * a.bwd_guide_off) {
    float4* rec_f = rec_s;
    float* invd_f = reinterpret_cast<float*>(rec_s + G);
    uint32_t* base = reinterpret_cast<uint32_t*>(invd_f + G);
    const DensView d = load_density(a, b, tg.k0, tg.G, false, rec_f, guide_s, invd_f, false, sh,
                                    guide_key, bulk);
    if (d.count_all) {
      // count semantics: intervals and offsets are not bounded, fp32 sums
      float* gacc = reinterpret_cast<float*>(base);
      for (int i = threadIdx.x; i < G; i += TPB) gacc[i] = 0.0f;
      __syncthreads();
      acc.gacc = gacc;
      vjp_chunk_tiles<TPB, R, kShared, false>(a, d, tg, tb, t_first, t_end, acc, gh);
      __syncthreads();
      for (int i = threadIdx.x; i < G; i += TPB) __stcg(&part[i], gacc[i]);
    } else {
      // the chunk's partial takes the fp32 reductions of terms above the cap
      for (int i = threadIdx.x; i < 4 * G; i += TPB) base[i] = 0u;
      for (int i = threadIdx.x; i < G; i += TPB) __stcg(&part[i], 0.0f);
      chunk_scale<TPB>(a, gh, r0, r1, chunk_rows, sh);
      acc.alo = base;
      acc.ahi = base + G;
      acc.blo = base + 2 * G;
      acc.bhi = base + 3 * G;
      acc.scale = sh.fix_scale;
      acc.cap = sh.fix_cap;
      acc.lbits = sh.fix_lbits;
      acc.lmask = (1u << acc.lbits) - 1u;
      acc.spill = part;
      vjp_chunk_tiles<TPB, R, kShared, true>(a, d, tg, tb, t_first, t_end, acc, gh);
      __threadfence();
      __syncthreads();
      const double inv_scale = 1.0 / static_cast<double>(acc.scale);
      for (int i = threadIdx.x; i < G; i += TPB) {
        // gcdf_i = m_i (B_i - A_i) - m_{i-1} B_{i-1} (no interval starts at knot G-1)
        double v = 0.0;
        if (i + 1 < G)
          v = static_cast<double>(rec_f[i].w) *
              (fix_value(acc.blo[i], acc.bhi[i], acc.lbits, inv_scale) -
               fix_value(acc.alo[i], acc.ahi[i], acc.lbits, inv_scale));
        if (i > 0)
          v -= static_cast<double>(rec_f[i - 1].w) *
               fix_value(acc.blo[i - 1], acc.bhi[i - 1], acc.lbits, inv_scale);
        __stcg(&part[i], static_cast<float>(v + static_cast<double>(__ldcg(&part[i]))));
      }
    }
  } else {
    const DensView d = load_density(a, b, tg.k0, tg.G, false, rec_s, guide_s, invd_s, false, sh,
                                    guide_key, bulk);
    const int stride = rep > 1 ? G + 1 : G;  // rep * stride <= gcap
    for (int i = threadIdx.x; i < rep * stride; i += TPB) gacc_s[i] = 0.0f;
    __syncthreads();
    acc.gacc = gacc_s + ((threadIdx.x & 31) & (rep - 1)) * stride;
    vjp_chunk_tiles<TPB, R, kShared, false>(a, d, tg, tb, t_first, t_end, acc, gh);
    __syncthreads();
    for (int i = threadIdx.x; i < G; i += TPB) {
      float v = gacc_s[i];
      for (int c = 1; c < rep; ++c) v += gacc_s[c * stride + i];
      __stcg(&part[i], v);
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(&a.chunks_done[b], 1u);
}

template <int TPB>
struct FinShared {
  double dscan[33];
  double sfirst[TPB];
  double red[33];
  double carry;
  float tred[TPB / 32][6];  // per-warp parameter gradients (theory)
};

// Reverse-mode chain of density b: grad_cdf (sum of chunk partials) ->
// suffix scan -> grad_rho -> normaliser VJP -> grad_values (with theory
// parameters: -> their gradient, the theory's VJP, reduced here).
template <int TPB>
__device__ __forceinline__ void vjp_finalize_item(const BatchArgs& a, int b, double* grho, FinShared<TPB>& sh) {
  const int32_t nch = __ldg(&a.chunk_first[b + 1]) - __ldg(&a.chunk_first[b]);
  const int64_t k0 = __ldg(&a.knot_off[b]);
  const int64_t G = __ldg(&a.knot_off[b + 1]) - k0;
  if (G > a.gcap) return;  // large density: reverse-scan tiles instead
  if (threadIdx.x == 0) {
    if (!wait_counter(&a.chunks_done[b], static_cast<uint32_t>(nch), a.status, a.spin_limit))
      raise_status(a.status, LOITS_ERR_TIMEOUT);
    sh.carry = 0.0;
  }
  __syncthreads();
  const float* g = a.grid + k0;
  const float* f = a.values ? a.values + k0 : nullptr;
  // with theory parameters: the density's components, to evaluate its values
  // and to take its parameter gradient here
  loits_theory::Comp th[2];
  if (a.theory) {
    th[0] = loits_theory::component(a.theory + static_cast<int64_t>(b) * 6, 0);
    th[1] = loits_theory::component(a.theory + static_cast<int64_t>(b) * 6, 1);
  }
  const double norm = __ldcg(&a.norm[b]);
  const float* part = a.partials + __ldg(&a.part_off[b]);
  constexpr int E = 4;
  const int64_t SEG = static_cast<int64_t>(TPB) * E;
  double gn_local = 0.0;  // sum grho_t * f_t
  const int64_t nseg = (G + SEG - 1) / SEG;
  for (int64_t sgi = nseg - 1; sgi >= 0; --sgi) {
    const int64_t s0 = sgi * SEG;
    const int64_t s1 = s0 + SEG < G ? s0 + SEG : G;
    const int64_t my_lo = s0 + static_cast<int64_t>(threadIdx.x) * E;
    const int64_t my_hi = my_lo + E < s1 ? my_lo + E : s1;
    double gc[E];
    double tot = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int64_t t = my_lo + e;
      double v = 0.0;
      if (t < my_hi)
        for (int32_t c = 0; c < nch; ++c) v += static_cast<double>(__ldcg(&part[static_cast<int64_t>(c) * G + t]));
      gc[e] = v;
    }
    // inclusive suffix within the thread: S_t = sum_{s >= t} gc_s
#pragma unroll
    for (int e = E - 1; e >= 0; --e) {
      tot += gc[e];
      gc[e] = tot;
    }
    double seg_tot;
    const double later = block_exclusive_suffix_sum<double, TPB>(tot, seg_tot, sh.dscan);
    const double carry = sh.carry;
    // S_t for my knots, and S of the knot after my last one
#pragma unroll
    for (int e = 0; e < E; ++e) gc[e] = gc[e] + (later + carry);
    sh.sfirst[threadIdx.x] = my_lo < my_hi ? gc[0] : 0.0;
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int64_t t = my_lo + e;
      if (t >= my_hi) break;
      // S_{t+1}: next knot in this thread, the next thread, or the next segment
      double s_next;
      if (e + 1 < E && t + 1 < my_hi) s_next = gc[e + 1];
      else if (t + 1 >= G) s_next = 0.0;
      else if (t + 1 >= s1) s_next = carry;
      else s_next = sh.sfirst[threadIdx.x + 1];
      const double h_t = t >= 1 ? 0.5 * (static_cast<double>(__ldg(&g[t])) - static_cast<double>(__ldg(&g[t - 1]))) : 0.0;
      const double h_n = t + 1 < G ? 0.5 * (static_cast<double>(__ldg(&g[t + 1])) - static_cast<double>(__ldg(&g[t]))) : 0.0;
      const double gr = h_n * s_next + h_t * gc[e];
      grho[k0 + t] = gr;
      const float ft = a.theory ? loits_theory::value(th[0], th[1], __ldg(&g[t])) : __ldg(&f[t]);
      gn_local += gr * static_cast<double>(ft);
    }
    __syncthreads();
    if (threadIdx.x == 0) sh.carry = carry + seg_tot;
    __syncthreads();
  }
  double gn_total;
  block_exclusive_sum<double, TPB>(gn_local, gn_total, sh.red);
  const double inv_n = 1.0 / norm;
  const double gnorm = -gn_total * inv_n * inv_n;
  __threadfence_block();
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // with theory: d loss / d parameters
  for (int64_t t = threadIdx.x; t < G; t += TPB) {
    const double h_t = t >= 1 ? 0.5 * (static_cast<double>(__ldg(&g[t])) - static_cast<double>(__ldg(&g[t - 1]))) : 0.0;
    const double h_n = t + 1 < G ? 0.5 * (static_cast<double>(__ldg(&g[t + 1])) - static_cast<double>(__ldg(&g[t]))) : 0.0;
    const double v = grho[k0 + t] * inv_n + (h_t + h_n) * gnorm;
    if (a.theory) loits_theory::add_grad(th, __ldg(&g[t]), __double2float_rn(v), acc);
    else a.grad_values[k0 + t] = __double2float_rn(v);
  }
  if (a.theory) {
    // the density's parameter gradient: warp trees, then the warps in order
    // (deterministic)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      float v = acc[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) sh.tred[warp][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
      float v = 0.0f;
      for (int w = 0; w < TPB / 32; ++w) v += sh.tred[w][threadIdx.x];
      a.grad_theory[static_cast<int64_t>(b) * 6 + threadIdx.x] = v;
    }
  }
  __syncthreads();
}

// Reverse-scan tiles of a large density.  Tile ti (ti = 0 is the LAST
// segment of knots) covers [s1 - SEG, s1), s1 = G - ti * SEG, SEG = TPB * 4.
template <int TPB>
__device__ __forceinline__ void large_tile_range(int64_t G, int32_t ti, int64_t& s0, int64_t& s1) {
  constexpr int64_t SEG = static_cast<int64_t>(TPB) * 4;
  s1 = G - static_cast<int64_t>(ti) * SEG;
  s0 = s1 - SEG > 0 ? s1 - SEG : 0;
}

// Phase 1 of a large density's reverse-mode chain, one tile: suffix sums of
// the fp64 grad-CDF (in-thread, block, then a chained look-back over the
// later tiles), grad_rho of the tile's knots, and the tile's share of
// sum(grad_rho * value) for the normaliser VJP (cpp/loits_core.cpp:340-435).
template <int TPB>
__device__ __forceinline__ void vjp_large_scan_item(const BatchArgs& a, int32_t li, double* grho,
                                                    FinShared<TPB>& sh) {
  constexpr int E = 4;
  const int b = find_owner(a.lfin_first, a.d_lo, a.d_hi, li);
  const int32_t first = __ldg(&a.lfin_first[b]);
  const int32_t nch = __ldg(&a.chunk_first[b + 1]) - __ldg(&a.chunk_first[b]);
  const int64_t k0 = __ldg(&a.knot_off[b]);
  const int64_t G = __ldg(&a.knot_off[b + 1]) - k0;
  int64_t s0, s1;
  large_tile_range<TPB>(G, li - first, s0, s1);
  if (threadIdx.x == 0 && !wait_counter(&a.chunks_done[b], static_cast<uint32_t>(nch), a.status, a.spin_limit))
    raise_status(a.status, LOITS_ERR_TIMEOUT);
  __syncthreads();
  const float2* gc = a.gcdf + __ldg(&a.gc_off[b]);
  const float* g = a.grid + k0;
  const float* f = a.values + k0;
  const int64_t my_lo = s0 + static_cast<int64_t>(threadIdx.x) * E;
  const int64_t my_hi = my_lo + E < s1 ? my_lo + E : s1;
  double S[E];
  double tot = 0.0;
#pragma unroll
  for (int e = E - 1; e >= 0; --e) {
    const int64_t t = my_lo + e;
    // grad-CDF of knot t: interval t's share plus interval t-1's
    double v = 0.0;
    if (t < my_hi) {
      v = static_cast<double>(__ldcg(&gc[t].x));
      if (t >= 1) v += static_cast<double>(__ldcg(&gc[t - 1].y));
    }
    tot += v;
    S[e] = tot;
  }
  double seg_tot;
  const double later = block_exclusive_suffix_sum<double, TPB>(tot, seg_tot, sh.dscan);
  if (threadIdx.x < 32) {
    const double carry_t =
        chained_lookback(a.lflag, a.lagg, a.linc, a.status, first, li, seg_tot, a.spin_limit);
    if (threadIdx.x == 0) sh.carry = carry_t;
  }
  __syncthreads();
  const double carry = sh.carry;  // sum of grad-CDF over every knot >= s1
#pragma unroll
  for (int e = 0; e < E; ++e) S[e] += later + carry;
  sh.sfirst[threadIdx.x] = my_lo < my_hi ? S[0] : 0.0;
  __syncthreads();
  double gn_local = 0.0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int64_t t = my_lo + e;
    if (t >= my_hi) break;
    double s_next;
    if (e + 1 < E && t + 1 < my_hi) s_next = S[e + 1];
    else if (t + 1 >= G) s_next = 0.0;
    else if (t + 1 >= s1) s_next = carry;
    else s_next = sh.sfirst[threadIdx.x + 1];
    const double h_t = t >= 1 ? 0.5 * (static_cast<double>(__ldg(&g[t])) - static_cast<double>(__ldg(&g[t - 1]))) : 0.0;
    const double h_n = t + 1 < G ? 0.5 * (static_cast<double>(__ldg(&g[t + 1])) - static_cast<double>(__ldg(&g[t]))) : 0.0;
    const double gr = h_n * s_next + h_t * S[e];
    grho[k0 + t] = gr;
    gn_local += gr * static_cast<double>(__ldg(&f[t]));
  }
  double gn_tile;
  block_exclusive_sum<double, TPB>(gn_local, gn_tile, sh.red);
  if (threadIdx.x == 0) {
    __stcg(&a.lgn[li], gn_tile);
    __threadfence();
    atomicAdd(&a.lfin_done[b], 1u);
  }
  __syncthreads();
}

// Phase 2, one tile: once every tile of the density has its share, the
// normaliser gradient (shares summed in tile order: deterministic) and the
// value gradients of the tile's knots.
template <int TPB>
__device__ __forceinline__ void vjp_large_out_item(const BatchArgs& a, int32_t li,
                                                   const double* grho, FinShared<TPB>& sh) {
  const int b = find_owner(a.lfin_first, a.d_lo, a.d_hi, li);
  const int32_t first = __ldg(&a.lfin_first[b]);
  const int32_t nl = __ldg(&a.lfin_first[b + 1]) - first;
  const int64_t k0 = __ldg(&a.knot_off[b]);
  const int64_t G = __ldg(&a.knot_off[b + 1]) - k0;
  int64_t s0, s1;
  large_tile_range<TPB>(G, li - first, s0, s1);
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    if (lane == 0 && !wait_counter(&a.lfin_done[b], static_cast<uint32_t>(nl), a.status, a.spin_limit))
      raise_status(a.status, LOITS_ERR_TIMEOUT);
    __syncwarp();
    double v = 0.0;
    for (int32_t i = lane; i < nl; i += 32) v += __ldcg(&a.lgn[first + i]);
    v = warp_sum(v);
    if (lane == 0) sh.carry = v;
  }
  __syncthreads();
  const double norm = __ldcg(&a.norm[b]);
  const double inv_n = 1.0 / norm;
  const double gnorm = -sh.carry * inv_n * inv_n;
  const float* g = a.grid + k0;
  for (int64_t t = s0 + threadIdx.x; t < s1; t += TPB) {
    const double h_t = t >= 1 ? 0.5 * (static_cast<double>(__ldg(&g[t])) - static_cast<double>(__ldg(&g[t - 1]))) : 0.0;
    const double h_n = t + 1 < G ? 0.5 * (static_cast<double>(__ldg(&g[t + 1])) - static_cast<double>(__ldg(&g[t]))) : 0.0;
    const double v = __ldcg(&grho[k0 + t]) * inv_n + (h_t + h_n) * gnorm;
    a.grad_values[k0 + t] = __double2float_rn(v);
  }
  __syncthreads();
}

// ---------------------------------------------------------------- kernels

// Register cap: 1280 threads per SM, i.e. 48 registers for five resident
// 256-thread CTAs, 64 for two 512-thread CTAs or one 1024-thread CTA.
template <int TPB, int R, bool kLarge>
__global__ void __launch_bounds__(TPB, 1280 / TPB) batch_forward_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* rec_s = reinterpret_cast<float4*>(smem_raw);
  uint32_t* guide_s = reinterpret_cast<uint32_t*>(smem_raw) + a.fwd_guide_off;
  // CDF items stage their tile's knots where sampling items later keep
  // records (a CTA takes every CDF ticket it gets before any sampling ticket)
  float* stage_s = reinterpret_cast<float*>(smem_raw);
  // this CTA's staging run in global memory (TPB * R * 4 floats): kept
  // events wait there for their tile's row base; they stay in L2
  float* stage = a.stage_g + static_cast<int64_t>(blockIdx.x) * (TPB * R * 4);
  __shared__ union {
    CdfShared<TPB> cdf;
    SampleShared smp;
  } sh;
  __shared__ uint32_t s_item;
  __shared__ int s_guide_key;  // density whose coarse guide guide_s holds
  __shared__ int2 s_win;       // ... and its window of records in rec_s
  __shared__ __align__(8) uint64_t s_bar;  // bulk copies of density views
  __shared__ uint32_t s_phase;
  if (threadIdx.x == 0) {
    s_guide_key = -1;
    s_phase = 0;
    bulk_barrier_init(&s_bar);
  }
  const BulkStage bulk{&s_bar, &s_phase};
  const int32_t nC = a.c_hi - a.c_lo, nF = a.f_hi - a.f_lo, nT = a.t_hi - a.t_lo;
  const uint32_t n_items = static_cast<uint32_t>(nC + nF + nT);
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const uint32_t item = s_item;
    __syncthreads();
    if (item >= n_items) break;
    if (item < static_cast<uint32_t>(nC)) {
      const int32_t ct = a.c_lo + static_cast<int32_t>(item);
      if (cdf_tile_fits(a, __ldg(&a.cdf_owner[ct]), TPB)) cdf_scan_item<TPB, true>(a, ct, sh.cdf, stage_s);
      else cdf_scan_item<TPB, false>(a, ct, sh.cdf, stage_s);
    } else if (item < static_cast<uint32_t>(nC + nF)) {
      const int32_t fi = a.f_lo + static_cast<int32_t>(item) - nC;
      if (cdf_tile_fits(a, find_owner(a.fin_first, a.d_lo, a.d_hi, fi), TPB))
        cdf_finalize_item<TPB, true>(a, fi, sh.cdf, stage_s);
      else cdf_finalize_item<TPB, false>(a, fi, sh.cdf, stage_s);
    } else {
      sample_item<TPB, R, kLarge>(a, a.t_lo + static_cast<int32_t>(item) - nC - nF, rec_s,
                                  guide_s, stage, sh.smp, s_guide_key, s_win, bulk);
    }
  }
}

template <int TPB, int R, bool kLarge, bool kFix>
__global__ void __launch_bounds__(TPB, 1280 / TPB) batch_backward_kernel(BatchArgs a, double* grho) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* rec_s = reinterpret_cast<float4*>(smem_raw);
  float* invd_s = reinterpret_cast<float*>(rec_s + a.gcap);
  float* gacc_s = invd_s + a.gcap;
  uint32_t* guide_s = reinterpret_cast<uint32_t*>(smem_raw) + a.bwd_guide_off;
  __shared__ union {
    FinShared<TPB> fin;
    SampleShared smp;
  } sh;
  __shared__ uint32_t s_item[2];
  __shared__ int s_guide_key;  // density whose coarse guide guide_s holds
  __shared__ __align__(8) uint64_t s_bar;  // bulk copies of density views
  __shared__ uint32_t s_phase;
  if (threadIdx.x == 0) {
    s_guide_key = -1;
    sh.smp.win_b = -1;  // no fixed-point window chosen yet
    s_phase = 0;
    bulk_barrier_init(&s_bar);
  }
  const BulkStage bulk{&s_bar, &s_phase};
  const int32_t nK = a.k_hi - a.k_lo, nD = a.d_hi - a.d_lo, nL = a.l_hi - a.l_lo;
  const uint32_t n_items = static_cast<uint32_t>(nK + nD + 2 * nL);
  // two ticket slots used in turn: a slot is written again only after the
  // next item's barrier, which every thread reaches after reading it
  for (int par = 0;; par ^= 1) {
    if (threadIdx.x == 0) s_item[par] = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const uint32_t item = s_item[par];
    if (item >= n_items) break;
    if (item < static_cast<uint32_t>(nK)) {
      vjp_chunk_item<TPB, R, kLarge, kFix>(a, a.k_lo + static_cast<int32_t>(item), rec_s, guide_s,
                                     invd_s, gacc_s, sh.smp, s_guide_key, bulk);
    } else if (item < static_cast<uint32_t>(nK + nD)) {
      vjp_finalize_item<TPB>(a, a.d_lo + static_cast<int32_t>(item) - nK, grho, sh.fin);
    } else if constexpr (kLarge) {
      if (item < static_cast<uint32_t>(nK + nD + nL))
        vjp_large_scan_item<TPB>(a, a.l_lo + static_cast<int32_t>(item) - nK - nD, grho, sh.fin);
      else
        vjp_large_out_item<TPB>(a, a.l_lo + static_cast<int32_t>(item) - nK - nD - nL, grho,
                                sh.fin);
    }
  }
}

}  // namespace loits_dev
