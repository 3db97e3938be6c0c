// tuple_kernels.cu -- the reference's 2-D theory tuple on sm_100a (fp64).
//
// Drop-in for the reference's native module (cpp/bindings.cpp:24-208): same
// Philox counters (padded slot p = (b*cells + cell)*nmax + slot, x stream
// 2*sequence, q stream 2*sequence+1, cpp/bindings.cpp:79-92), same int16
// count-semantics intervals, same epsilon, same compaction predicate and
// (b, cell, slot) order.  This file is compiled with -fmad=false so that every
// fp64 product and sum is rounded on its own, in the order the reference
// writes it (cpp/loits_core.cpp), which makes the forward bit-identical to
// the reference built without contraction.
//
// Kernels:
//   fill_uniform_kernel    cpp/loits_core.cpp:39-53
//   tuple_prepare_kernel   allocate_counts :22-37 + density :55-109 + cdf :111-165,
//                          one thread per cell (each cell owns one x and one q curve)
//   cell_scan_kernel       exclusive prefix of counts, nmax, active (one CTA)
//   tuple_sample_kernel    fill_uniform + interpolate :167-237 + compact :239-266
//                          fused; uniforms live in registers only; stable
//                          compaction by decoupled look-back over ordered tiles
//   tuple_rows_kernel,     interpolation_vjp :268-338 + cdf_vjp :340-398 +
//   tuple_chunk_kernel,    density_vjp :400-472: rows cut into chunks of at
//   tuple_cell_kernel      most 256 rows per cell, one warp per chunk with
//                          lane-private accumulators, per-cell ordered sum of
//                          the chunk partials, then the reverse chain;
//                          deterministic (every sum has a fixed order)
#include <cmath>
#include <cstdint>
#include <mutex>

#include "common.cuh"
#include "lookback.cuh"

namespace loits_dev {

constexpr double kEpsilon = 1e-5;

// ------------------------------------------------------------ fill_uniform

__global__ void fill_uniform_kernel(float* __restrict__ out, int64_t count, uint64_t seed,
                                    uint64_t stream_id) {
  const int64_t nblocks = (count + 3) >> 2;
  for (int64_t blk = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; blk < nblocks;
       blk += (int64_t)gridDim.x * blockDim.x) {
    const uint4 w = philox4x32_10(static_cast<uint64_t>(blk), stream_id, seed);
    const int64_t p = blk << 2;
    if (p + 3 < count && (reinterpret_cast<uintptr_t>(out + p) & 15) == 0) {
      *reinterpret_cast<float4*>(out + p) =
          make_float4(uniform_from_bits(w.x), uniform_from_bits(w.y), uniform_from_bits(w.z),
                      uniform_from_bits(w.w));
    } else {
      for (int i = 0; i < 4 && p + i < count; ++i) out[p + i] = uniform_from_bits(word_of(w, i));
    }
  }
}

// --------------------------------------------------------------- prepare

struct TupleGeom {
  int64_t batch, nx, ny, kx, kq, cells;
};

// Trapezoid norm + CDF of one curve, in the reference's operation order.
__device__ double curve_cdf(const double* __restrict__ bins, const double* __restrict__ xs,
                            int64_t k, double acc, double* __restrict__ cdf) {
  double n = 0.0;
  for (int64_t t = 1; t < k; ++t) {
    const double hw = 0.5 * (bins[t] - bins[t - 1]);
    n += hw * (xs[t - 1] + xs[t]);
  }
  const double inv_n = 1.0 / n;
  double cum = 0.0;
  double r_prev = xs[0] * inv_n;
  cdf[0] = 0.0;
  for (int64_t t = 1; t < k; ++t) {
    const double r_t = xs[t] * inv_n;
    const double hw = 0.5 * (bins[t] - bins[t - 1]);
    cum += hw * (r_prev + r_t);
    cdf[t] = cum * acc;
    r_prev = r_t;
  }
  return n;
}

__global__ void tuple_prepare_kernel(TupleGeom g, const double* __restrict__ x_bins,
                                     const double* __restrict__ xsec_x,
                                     const double* __restrict__ q_bins,
                                     const double* __restrict__ xsec_q,
                                     const double* __restrict__ weights,
                                     const uint8_t* __restrict__ acceptance, int64_t n_events,
                                     int64_t* __restrict__ counts, double* __restrict__ norm_x,
                                     double* __restrict__ norm_q, double* __restrict__ cdf_x,
                                     double* __restrict__ cdf_q) {
  const int64_t ncell = g.batch * g.cells;
  const double scale = static_cast<double>(n_events);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ncell;
       i += (int64_t)gridDim.x * blockDim.x) {
    counts[i] = static_cast<int64_t>(fabs(weights[i] * scale));
    const int64_t b = i / g.cells, cell = i - b * g.cells;
    const int64_t ix = cell / g.ny, iy = cell - ix * g.ny;
    const double acc = acceptance[i] ? 1.0 : 0.0;
    const int64_t xi = (b * g.ny + iy) * g.nx + ix;  // x curve, y-major storage
    norm_x[xi] = curve_cdf(x_bins + (b * g.nx + ix) * g.kx, xsec_x + xi * g.kx, g.kx, acc,
                           cdf_x + xi * g.kx);
    norm_q[i] = curve_cdf(q_bins + (b * g.ny + iy) * g.kq, xsec_q + i * g.kq, g.kq, acc,
                          cdf_q + i * g.kq);
  }
}

// One CTA: cell_offsets = exclusive prefix of counts; alloc = {nmax, active}.
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads)
    cell_scan_kernel(const int64_t* __restrict__ counts, int64_t ncell,
                     int64_t* __restrict__ cell_offsets, int64_t* __restrict__ alloc) {
  __shared__ long long s_sum[kScanThreads / 32 + 1];
  __shared__ long long s_max[kScanThreads / 32 + 1];
  const int64_t per = (ncell + kScanThreads - 1) / kScanThreads;
  const int64_t lo = threadIdx.x * per;
  const int64_t hi = lo + per < ncell ? lo + per : ncell;
  long long local = 0, mx = 0;
  for (int64_t i = lo; i < hi; ++i) {
    local += counts[i];
    mx = counts[i] > mx ? counts[i] : mx;
  }
  long long total;
  long long run = block_exclusive_sum<long long, kScanThreads>(local, total, s_sum);
  long long gmax;
  block_exclusive_max<long long, kScanThreads>(mx, 0ll, gmax, s_max);
  for (int64_t i = lo; i < hi; ++i) {
    cell_offsets[i] = run;
    run += counts[i];
  }
  if (threadIdx.x == 0) {
    cell_offsets[ncell] = total;
    alloc[0] = gmax;
    alloc[1] = total;
  }
}

// ----------------------------------------------------------------- sample

// Count-semantics interval of cpp/loits_core.cpp:12-18 (all k knots, then
// clamp to [0, k-2], int16).
__device__ __forceinline__ int interval_count(const double* __restrict__ c, int64_t k, double u) {
  int64_t sel = -1;
  for (int64_t t = 0; t < k; ++t) sel += (u >= c[t]) ? 1 : 0;
  if (sel < 0) sel = 0;
  if (sel > k - 2) sel = k - 2;
  return static_cast<int16_t>(sel);
}

__device__ __forceinline__ double curve_value(const double* __restrict__ bins,
                                              const double* __restrict__ c, int j, double u) {
  const double c0 = c[j];
  const double inv_d = 1.0 / (c[j + 1] - c0 + kEpsilon);
  const double m = (bins[j + 1] - bins[j]) * inv_d;
  return bins[j] + m * (u - c0);
}

constexpr int kSampleThreads = 256;
constexpr int kSampleEPT = 4;  // consecutive active events per thread
constexpr int kSampleTile = kSampleThreads * kSampleEPT;

struct TupleSampleArgs {
  TupleGeom g;
  const double* x_bins;
  const double* q_bins;
  const double* cdf_x;
  const double* cdf_q;
  const int64_t* cell_offsets;
  int64_t nmax, active;
  uint64_t seed, stream_x, stream_q;
  double* events;
  int64_t* packed;
  int16_t* interval_x;
  int16_t* interval_q;
  int64_t* valid;
  int32_t* status;
  uint32_t* ticket;
  unsigned long long* tile_state;
  int64_t n_tiles;
  const int64_t* alloc;  // when set: {nmax, active} read here (the launch has n_tiles for
                         // `capacity` active slots, an upper bound)
  int64_t capacity;
};

// Three CTAs per SM (80 registers, no spills) instead of two at 118.
// Last cell c in [lo, hi) with off[c] <= e, given off[lo] <= e, for a
// non-decreasing per-cell table off (cell offsets, chunk starts): a 33-ary
// search by one whole warp (three rounds of loads for ten thousand cells
// instead of a thread's chain of fourteen).  The probes grow with the lane,
// so the lanes whose entry is <= e are a prefix of the warp.
__device__ __forceinline__ int64_t warp_find_cell(const int64_t* __restrict__ off, int64_t lo,
                                                  int64_t hi, int64_t e) {
  const int lane = threadIdx.x & 31;
  while (hi - lo > 1) {
    const int64_t span = hi - lo;
    int64_t p = lo + span * (lane + 1) / 33;
    p = p <= lo ? lo + 1 : (p >= hi ? hi - 1 : p);
    const unsigned le = __ballot_sync(0xffffffffu, off[p] <= e);
    const int n = __popc(le);
    const int64_t new_lo = n > 0 ? __shfl_sync(0xffffffffu, p, n - 1) : lo;
    const int64_t new_hi = n < 32 ? __shfl_sync(0xffffffffu, p, n < 32 ? n : 31) : hi;
    lo = new_lo;
    hi = new_hi;
  }
  return lo;
}

__global__ void __launch_bounds__(kSampleThreads, 3) tuple_sample_kernel(TupleSampleArgs a) {
  __shared__ long long s_scan[kSampleThreads / 32 + 1];
  __shared__ long long s_base;
  __shared__ uint32_t s_tile;
  __shared__ int64_t s_cells[2];  // cells of the tile's first and last active events
  if (threadIdx.x == 0) s_tile = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  if (a.alloc) {
    // counts on the device: the launch covers `capacity` slots; a larger
    // count is an error (nothing sampled), tiles past the count do nothing
    a.nmax = a.alloc[0];
    a.active = a.alloc[1];
    if (a.active > a.capacity) {
      if (tile == 0 && threadIdx.x == 0) raise_status(a.status, LOITS_ERR_CAPACITY);
      return;
    }
    a.n_tiles = (a.active + kSampleTile - 1) / kSampleTile;
    if (tile >= a.n_tiles) return;  // the whole CTA: no later tile waits on it
  }
  const int64_t ncell = a.g.batch * a.g.cells;
  const int64_t e0 = tile * kSampleTile + threadIdx.x * kSampleEPT;
  if (threadIdx.x < 32) {
    // the tile's active events [e_first, e_last] span cells [c_first, c_last]
    const int64_t e_first = tile * kSampleTile;
    const int64_t e_last = (e_first + kSampleTile < a.active ? e_first + kSampleTile : a.active) - 1;
    const int64_t c_first = warp_find_cell(a.cell_offsets, 0, ncell, e_first);
    const int64_t c_last = warp_find_cell(a.cell_offsets, c_first, ncell, e_last);
    if (threadIdx.x == 0) {
      s_cells[0] = c_first;
      s_cells[1] = c_last;
    }
  }
  __syncthreads();

  double xs[kSampleEPT], qs[kSampleEPT];
  int64_t ps[kSampleEPT];
  int16_t jxs[kSampleEPT], jqs[kSampleEPT];
  int keep = 0;
  if (e0 < a.active) {
    // cell holding active event e0: last c with cell_offsets[c] <= e0, among
    // the tile's cells
    int64_t lo = s_cells[0], hi = s_cells[1] + 1;  // answer in [lo, hi)
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (a.cell_offsets[mid] <= e0) lo = mid; else hi = mid;
    }
    int64_t c = lo;
    uint64_t cached_blk = ~0ull;
    uint4 wx = make_uint4(0, 0, 0, 0), wq = wx;
#pragma unroll
    for (int i = 0; i < kSampleEPT; ++i) {
      const int64_t e = e0 + i;
      if (e >= a.active) break;
      while (a.cell_offsets[c + 1] <= e) ++c;
      const int64_t p = c * a.nmax + (e - a.cell_offsets[c]);
      const uint64_t blk = static_cast<uint64_t>(p) >> 2;
      if (blk != cached_blk) {
        wx = philox4x32_10(blk, a.stream_x, a.seed);
        wq = philox4x32_10(blk, a.stream_q, a.seed);
        cached_blk = blk;
      }
      const double ux = static_cast<double>(uniform_from_bits(word_of(wx, p & 3)));
      const double uq = static_cast<double>(uniform_from_bits(word_of(wq, p & 3)));
      const int64_t b = c / a.g.cells, cell = c - b * a.g.cells;
      const int64_t ix = cell / a.g.ny, iy = cell - ix * a.g.ny;
      const double* xc = a.cdf_x + ((b * a.g.ny + iy) * a.g.nx + ix) * a.g.kx;
      const double* xb = a.x_bins + (b * a.g.nx + ix) * a.g.kx;
      const double* qc = a.cdf_q + c * a.g.kq;
      const double* qb = a.q_bins + (b * a.g.ny + iy) * a.g.kq;
      const int jx = interval_count(xc, a.g.kx, ux);
      const int jq = interval_count(qc, a.g.kq, uq);
      const double x = curve_value(xb, xc, jx, ux);
      const double q = curve_value(qb, qc, jq, uq);
      const bool ok = isfinite(x) && isfinite(q) && x * q != 0.0;
      xs[i] = x;
      qs[i] = q;
      ps[i] = p;
      jxs[i] = static_cast<int16_t>(jx);
      jqs[i] = static_cast<int16_t>(jq);
      keep |= ok ? (1 << i) : 0;
    }
  }
  long long tile_count;
  const long long rank0 =
      block_exclusive_sum<long long, kSampleThreads>(__popc(keep), tile_count, s_scan);
  if (threadIdx.x < 32) {
    const int64_t base = lookback_exclusive(a.tile_state, tile, tile_count, a.status);
    if (threadIdx.x == 0) s_base = base;
  }
  __syncthreads();
  int64_t row = s_base + rank0;
#pragma unroll
  for (int i = 0; i < kSampleEPT; ++i) {
    if (!(keep & (1 << i))) continue;
    a.events[2 * row] = xs[i];
    a.events[2 * row + 1] = qs[i];
    a.packed[row] = ps[i];
    if (a.interval_x) a.interval_x[row] = jxs[i];
    if (a.interval_q) a.interval_q[row] = jqs[i];
    ++row;
  }
  if (tile == a.n_tiles - 1 && threadIdx.x == 0) *a.valid = s_base + tile_count;
}

// --------------------------------------------------------------- backward

struct TupleBackwardArgs {
  TupleGeom g;
  const double* grad;
  const int64_t* packed;
  int64_t nvalid, nmax;
  uint64_t seed, stream_x, stream_q;
  const double* x_bins;
  const double* xsec_x;
  const double* q_bins;
  const double* xsec_q;
  const uint8_t* acceptance;
  const double* norm_x;
  const double* norm_q;
  const double* cdf_x;
  const double* cdf_q;
  double* grad_x;
  double* grad_q;
  const int64_t* valid_dev;  // when set: the kept-row count (nvalid is then an upper bound)
  const int64_t* nmax_dev;   // when set: nmax
};

// First row whose packed index is >= key (packed is strictly increasing).
__device__ __forceinline__ int64_t lower_bound_i64(const int64_t* __restrict__ v, int64_t n,
                                                   int64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (v[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Contribution of one row to grad_cdf[j] and grad_cdf[j+1]
// (cpp/loits_core.cpp:293-300).
__device__ __forceinline__ void value_vjp(const double* __restrict__ bins,
                                          const double* __restrict__ c, int j, double u, double g,
                                          double& to_j, double& to_j1) {
  const double c0 = c[j];
  const double d = c[j + 1] - c0 + kEpsilon;
  const double inv_d = 1.0 / d;
  const double t = u - c0;
  const double db = bins[j + 1] - bins[j];
  const double up = g * db;
  to_j = up * (-inv_d + t * inv_d * inv_d);
  to_j1 = -(up * t * inv_d * inv_d);
}

// Reverse suffix scan + normaliser VJP of one curve (cpp/loits_core.cpp:
// 340-472), sequential; gx doubles as grad_rho scratch.
__device__ void curve_chain(const double* __restrict__ bins, const double* __restrict__ xs,
                            double n, double acc, const double* __restrict__ gcdf, int64_t k,
                            double* __restrict__ gx) {
  for (int64_t t = 0; t < k; ++t) gx[t] = 0.0;
  double suffix = 0.0;
  for (int64_t t = k - 1; t > 0; --t) {
    suffix += gcdf[t];
    const double g = 0.5 * (bins[t] - bins[t - 1]) * acc * suffix;
    gx[t - 1] += g;
    gx[t] += g;
  }
  const double inv_n = 1.0 / n;
  const double inv_n2 = inv_n * inv_n;
  double gnorm = 0.0;
  for (int64_t t = 0; t < k; ++t) {
    const double gr = gx[t];
    gx[t] = gr * inv_n;
    gnorm -= gr * xs[t] * inv_n2;
  }
  for (int64_t t = 1; t < k; ++t) {
    const double g = 0.5 * (bins[t] - bins[t - 1]) * gnorm;
    gx[t - 1] += g;
    gx[t] += g;
  }
}

// The backward is balanced over rows, not cells (cell sizes follow the
// weights and differ by an order of magnitude): a cell's kept rows are cut
// into chunks of at most kChunkRows rows, each chunk's grad-CDF partial is
// formed by one warp, and each cell sums its chunks' partials in chunk order
// before the reverse chain -- every sum has a fixed order (deterministic).
constexpr int kChunkRows = 256;

// Per cell: first kept row (lower bound of its first padded slot in the
// strictly increasing packed rows) and its number of chunks.
__global__ void tuple_rows_kernel(TupleBackwardArgs a, int64_t* __restrict__ cell_rows,
                                  int64_t* __restrict__ chunks) {
  const int64_t ncell = a.g.batch * a.g.cells;
  int64_t nvalid = a.nvalid, nmax = a.nmax;
  if (a.valid_dev) nvalid = min(*a.valid_dev, nvalid);
  if (a.nmax_dev) nmax = *a.nmax_dev;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c <= ncell;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r0 = lower_bound_i64(a.packed, nvalid, c * nmax);
    cell_rows[c] = r0;
    if (c < ncell) {
      const int64_t r1 = lower_bound_i64(a.packed, nvalid, (c + 1) * nmax);
      chunks[c] = (r1 - r0 + kChunkRows - 1) / kChunkRows;
    }
  }
}

// Grad-CDF contributions of one row, in the order of its four targets
// (x knot jx, jx+1, q knot jq, jq+1).
struct RowVjp {
  int jx, jq;
  double ax, bx, aq, bq;
};

__device__ __forceinline__ RowVjp row_vjp(const TupleBackwardArgs& a, int64_t r, const double* xb,
                                          const double* xc, const double* qb, const double* qc) {
  RowVjp o;
  const int64_t p = a.packed[r];
  const uint64_t blk = static_cast<uint64_t>(p) >> 2;
  const double ux =
      static_cast<double>(uniform_from_bits(word_of(philox4x32_10(blk, a.stream_x, a.seed), p & 3)));
  const double uq =
      static_cast<double>(uniform_from_bits(word_of(philox4x32_10(blk, a.stream_q, a.seed), p & 3)));
  o.jx = interval_count(xc, a.g.kx, ux);
  o.jq = interval_count(qc, a.g.kq, uq);
  value_vjp(xb, xc, o.jx, ux, a.grad[2 * r], o.ax, o.bx);
  value_vjp(qb, qc, o.jq, uq, a.grad[2 * r + 1], o.aq, o.bq);
  return o;
}

struct CellCurves {
  int64_t xi;
  const double *xc, *xb, *qc, *qb;
};

__device__ __forceinline__ CellCurves cell_curves(const TupleBackwardArgs& a, int64_t gc) {
  CellCurves cc;
  const int64_t b = gc / a.g.cells, cell = gc - b * a.g.cells;
  const int64_t ix = cell / a.g.ny, iy = cell - ix * a.g.ny;
  cc.xi = (b * a.g.ny + iy) * a.g.nx + ix;
  cc.xc = a.cdf_x + cc.xi * a.g.kx;
  cc.xb = a.x_bins + (b * a.g.nx + ix) * a.g.kx;
  cc.qc = a.cdf_q + gc * a.g.kq;
  cc.qb = a.q_bins + (b * a.g.ny + iy) * a.g.kq;
  return cc;
}

// One warp per chunk.  Lane-private accumulators (kx + kq doubles per lane,
// stride kx + kq + 1) in shared memory take each lane's rows in order; the
// chunk partial is their fixed-order sum over lanes.  Large K (lane copies
// would not fit) uses per-knot warp reductions instead.
__global__ void tuple_chunk_kernel(TupleBackwardArgs a, const int64_t* __restrict__ cell_rows,
                                   const int64_t* __restrict__ chunk_first,
                                   const int64_t* __restrict__ n_chunks,
                                   double* __restrict__ partials, int lane_private) {
  extern __shared__ double s_acc[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int64_t k = static_cast<int64_t>(blockIdx.x) * wpb + warp;
  if (k >= *n_chunks) return;  // whole warp leaves together
  const int64_t ncell = a.g.batch * a.g.cells;
  // owner cell: last c with chunk_first[c] <= k (chunk_first[0] = 0)
  const int64_t gc = warp_find_cell(chunk_first, 0, ncell, k);
  const int64_t r_begin = cell_rows[gc] + (k - chunk_first[gc]) * kChunkRows;
  const int64_t r_end0 = r_begin + kChunkRows;
  const int64_t r_end = r_end0 < cell_rows[gc + 1] ? r_end0 : cell_rows[gc + 1];
  const CellCurves cc = cell_curves(a, gc);
  const int64_t kx = a.g.kx, kq = a.g.kq, kt = kx + kq;
  double* out = partials + k * kt;
  if (lane_private) {
    const int64_t stride = kt + 1;
    double* base = s_acc + static_cast<int64_t>(warp) * 32 * stride;
    double* mine = base + lane * stride;
    for (int64_t t = 0; t < kt; ++t) mine[t] = 0.0;
    for (int64_t r = r_begin + lane; r < r_end; r += 32) {
      const RowVjp v = row_vjp(a, r, cc.xb, cc.xc, cc.qb, cc.qc);
      mine[v.jx] += v.ax;
      mine[v.jx + 1] += v.bx;
      mine[kx + v.jq] += v.aq;
      mine[kx + v.jq + 1] += v.bq;
    }
    __syncwarp();
    for (int64_t t = lane; t < kt; t += 32) {
      double sum = 0.0;
      for (int l = 0; l < 32; ++l) sum += base[l * stride + t];
      out[t] = sum;
    }
  } else {
    double* acc = s_acc + static_cast<int64_t>(warp) * kt;
    for (int64_t t = lane; t < kt; t += 32) acc[t] = 0.0;
    __syncwarp();
    for (int64_t r0 = r_begin; r0 < r_end; r0 += 32) {
      const int64_t r = r0 + lane;
      RowVjp v{-2, -2, 0.0, 0.0, 0.0, 0.0};
      if (r < r_end) v = row_vjp(a, r, cc.xb, cc.xc, cc.qb, cc.qc);
      for (int64_t t = 0; t < kx; ++t) {
        double x = (v.jx == t ? v.ax : 0.0) + (v.jx + 1 == t ? v.bx : 0.0);
        x = warp_sum(x);
        if (lane == 0) acc[t] += x;
      }
      for (int64_t t = 0; t < kq; ++t) {
        double x = (v.jq == t ? v.aq : 0.0) + (v.jq + 1 == t ? v.bq : 0.0);
        x = warp_sum(x);
        if (lane == 0) acc[kx + t] += x;
      }
    }
    __syncwarp();
    for (int64_t t = lane; t < kt; t += 32) out[t] = acc[t];
  }
}

// One warp per cell: its chunks' partials summed in chunk order (lane t owns
// knot t), then the reverse chain of each curve (cpp/loits_core.cpp:340-472).
__global__ void tuple_cell_kernel(TupleBackwardArgs a, const int64_t* __restrict__ chunk_first,
                                  const double* __restrict__ partials) {
  extern __shared__ double s_gc[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int64_t gc = static_cast<int64_t>(blockIdx.x) * wpb + warp;
  const int64_t ncell = a.g.batch * a.g.cells;
  if (gc >= ncell) return;
  const int64_t kx = a.g.kx, kq = a.g.kq, kt = kx + kq;
  double* acc = s_gc + static_cast<int64_t>(warp) * kt;
  const int64_t k0 = chunk_first[gc], k1 = chunk_first[gc + 1];
  for (int64_t t = lane; t < kt; t += 32) {
    double sum = 0.0;
    for (int64_t k = k0; k < k1; ++k) sum += partials[k * kt + t];
    acc[t] = sum;
  }
  __syncwarp();
  const CellCurves cc = cell_curves(a, gc);
  const double acc_cell = a.acceptance[gc] ? 1.0 : 0.0;
  if (lane == 0) {
    curve_chain(cc.xb, a.xsec_x + cc.xi * kx, a.norm_x[cc.xi], acc_cell, acc, kx,
                a.grad_x + cc.xi * kx);
  } else if (lane == 1) {
    curve_chain(cc.qb, a.xsec_q + gc * kq, a.norm_q[gc], acc_cell, acc + kx, kq,
                a.grad_q + gc * kq);
  }
}

}  // namespace loits_dev

// ===================================================================== C ABI

using namespace loits_dev;

namespace {

int launch_status(cudaError_t e) { return e == cudaSuccess ? LOITS_OK : LOITS_ERR_CUDA; }

bool valid_shape(const loits_shape* s) {
  return s && s->batch >= 0 && s->nx >= 1 && s->ny >= 1 && s->kx >= 2 && s->kq >= 2;
}

TupleGeom geom_of(const loits_shape* s) {
  return TupleGeom{s->batch, s->nx, s->ny, s->kx, s->kq, s->nx * s->ny};
}

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return static_cast<int>(g);
}

}  // namespace

extern "C" int loits_fill_uniform(float* values, int64_t count, uint64_t seed, uint64_t stream_id,
                                  void* stream) {
  if (count < 0 || (count > 0 && !values)) return LOITS_ERR_INVALID;
  if (count == 0) return LOITS_OK;
  const int threads = 256;
  fill_uniform_kernel<<<grid_for((count + 3) / 4, threads), threads, 0,
                        static_cast<cudaStream_t>(stream)>>>(values, count, seed, stream_id);
  return launch_status(cudaGetLastError());
}

extern "C" int loits_tuple_prepare(const loits_shape* shape, const double* x_bins,
                                   const double* xsec_x, const double* q_bins,
                                   const double* xsec_q, const double* weights,
                                   const uint8_t* acceptance, int64_t n_events, int64_t* counts,
                                   int64_t* cell_offsets, double* norm_x, double* norm_q,
                                   double* cdf_x, double* cdf_q, int64_t* alloc, void* stream) {
  if (!valid_shape(shape) || n_events < 0) return LOITS_ERR_INVALID;
  if (shape->kx > 32767 || shape->kq > 32767) return LOITS_ERR_UNSUPPORTED;  // int16 intervals
  const TupleGeom g = geom_of(shape);
  const int64_t ncell = g.batch * g.cells;
  if (!alloc || !cell_offsets) return LOITS_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (ncell > 0) {
    if (!x_bins || !xsec_x || !q_bins || !xsec_q || !weights || !acceptance || !counts ||
        !norm_x || !norm_q || !cdf_x || !cdf_q)
      return LOITS_ERR_INVALID;
    tuple_prepare_kernel<<<grid_for(ncell, 128), 128, 0, st>>>(
        g, x_bins, xsec_x, q_bins, xsec_q, weights, acceptance, n_events, counts, norm_x, norm_q,
        cdf_x, cdf_q);
    if (cudaGetLastError() != cudaSuccess) return LOITS_ERR_CUDA;
  }
  cell_scan_kernel<<<1, kScanThreads, 0, st>>>(counts, ncell, cell_offsets, alloc);
  return launch_status(cudaGetLastError());
}

extern "C" size_t loits_tuple_sample_workspace(int64_t active) {
  if (active <= 0) return 16;
  // whole tiles, formed without overflow for any positive active
  const int64_t tiles = active / kSampleTile + (active % kSampleTile != 0 ? 1 : 0);
  return 16 + static_cast<size_t>(tiles) * sizeof(unsigned long long);
}

namespace {

// The sampling launch; alloc (device {nmax, active}) set: active is the
// capacity the launch covers and the counts are read on the device.
int tuple_sample_launch(const loits_shape* shape, const double* x_bins, const double* q_bins,
                        const double* cdf_x, const double* cdf_q, const int64_t* cell_offsets,
                        int64_t nmax, int64_t active, const int64_t* alloc, uint64_t seed,
                        uint64_t sequence, double* events, int64_t* packed, int16_t* interval_x,
                        int16_t* interval_q, int64_t* valid, int32_t* status, void* workspace,
                        size_t workspace_bytes, void* stream) {
  if (!valid_shape(shape) || nmax < 0 || active < 0 || !valid || !status) return LOITS_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(status, 0, sizeof(int32_t), st) != cudaSuccess) return LOITS_ERR_CUDA;
  if (alloc && cudaMemsetAsync(valid, 0, sizeof(int64_t), st) != cudaSuccess) return LOITS_ERR_CUDA;
  if (active == 0) return launch_status(cudaMemsetAsync(valid, 0, sizeof(int64_t), st));
  if (!x_bins || !q_bins || !cdf_x || !cdf_q || !cell_offsets || !events || !packed || !workspace)
    return LOITS_ERR_INVALID;
  if (sequence > (UINT64_MAX - 1) / 2) return LOITS_ERR_INVALID;
  const size_t need = loits_tuple_sample_workspace(active);
  if (workspace_bytes < need) return LOITS_ERR_CAPACITY;
  if (cudaMemsetAsync(workspace, 0, need, st) != cudaSuccess) return LOITS_ERR_CUDA;
  TupleSampleArgs a;
  a.g = geom_of(shape);
  a.x_bins = x_bins;
  a.q_bins = q_bins;
  a.cdf_x = cdf_x;
  a.cdf_q = cdf_q;
  a.cell_offsets = cell_offsets;
  a.nmax = nmax;
  a.active = active;
  a.seed = seed;
  a.stream_x = 2 * sequence;
  a.stream_q = 2 * sequence + 1;
  a.events = events;
  a.packed = packed;
  a.interval_x = interval_x;
  a.interval_q = interval_q;
  a.valid = valid;
  a.status = status;
  a.ticket = static_cast<uint32_t*>(workspace);
  a.tile_state = reinterpret_cast<unsigned long long*>(static_cast<char*>(workspace) + 16);
  a.n_tiles = (active + kSampleTile - 1) / kSampleTile;
  a.alloc = alloc;
  a.capacity = active;
  if (a.n_tiles > 0x7fffffff) return LOITS_ERR_UNSUPPORTED;
  tuple_sample_kernel<<<static_cast<unsigned>(a.n_tiles), kSampleThreads, 0, st>>>(a);
  return launch_status(cudaGetLastError());
}

}  // namespace

extern "C" int loits_tuple_sample(const loits_shape* shape, const double* x_bins,
                                  const double* q_bins, const double* cdf_x, const double* cdf_q,
                                  const int64_t* cell_offsets, int64_t nmax, int64_t active,
                                  uint64_t seed, uint64_t sequence, double* events,
                                  int64_t* packed, int16_t* interval_x, int16_t* interval_q,
                                  int64_t* valid, int32_t* status, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  return tuple_sample_launch(shape, x_bins, q_bins, cdf_x, cdf_q, cell_offsets, nmax, active,
                             nullptr, seed, sequence, events, packed, interval_x, interval_q,
                             valid, status, workspace, workspace_bytes, stream);
}

extern "C" int loits_tuple_sample_bounded(const loits_shape* shape, const double* x_bins,
                                          const double* q_bins, const double* cdf_x,
                                          const double* cdf_q, const int64_t* cell_offsets,
                                          const int64_t* alloc, int64_t capacity, uint64_t seed,
                                          uint64_t sequence, double* events, int64_t* packed,
                                          int16_t* interval_x, int16_t* interval_q,
                                          int64_t* valid, int32_t* status, void* workspace,
                                          size_t workspace_bytes, void* stream) {
  if (!alloc) return LOITS_ERR_INVALID;
  return tuple_sample_launch(shape, x_bins, q_bins, cdf_x, cdf_q, cell_offsets, 0, capacity,
                             alloc, seed, sequence, events, packed, interval_x, interval_q,
                             valid, status, workspace, workspace_bytes, stream);
}

namespace {

// Workspace of the tuple backward: cell row starts, chunk counts and offsets,
// the scan's {max, total}, and one grad-CDF partial per chunk.
struct BackwardLayout {
  size_t cell_rows, chunks, chunk_first, alloc, partials, total;
  int64_t max_chunks;
};

BackwardLayout backward_layout(const TupleGeom& g, int64_t nvalid) {
  BackwardLayout L{};
  const int64_t ncell = g.batch * g.cells;
  L.max_chunks = nvalid / kChunkRows + ncell;
  size_t o = 0;
  auto take = [&o](size_t bytes) {
    const size_t at = o;
    o = (o + bytes + 255) / 256 * 256;
    return at;
  };
  L.cell_rows = take(static_cast<size_t>(ncell + 1) * 8);
  L.chunks = take(static_cast<size_t>(ncell) * 8);
  L.chunk_first = take(static_cast<size_t>(ncell + 1) * 8);
  L.alloc = take(16);
  L.partials = take(static_cast<size_t>(L.max_chunks) * (g.kx + g.kq) * 8);
  L.total = o;
  return L;
}

}  // namespace

extern "C" size_t loits_tuple_backward_workspace(const loits_shape* shape, int64_t nvalid) {
  if (!valid_shape(shape) || nvalid < 0) return 0;
  return backward_layout(geom_of(shape), nvalid).total;
}

namespace {

int tuple_backward_launch(const loits_shape* shape, const double* grad_events,
                          const int64_t* packed, int64_t nvalid, int64_t nmax,
                          const int64_t* valid_dev, const int64_t* nmax_dev, uint64_t seed,
                          uint64_t sequence, const double* x_bins, const double* xsec_x,
                          const double* q_bins, const double* xsec_q, const uint8_t* acceptance,
                          const double* norm_x, const double* norm_q, const double* cdf_x,
                          const double* cdf_q, double* grad_xsec_x, double* grad_xsec_q,
                          void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_shape(shape) || nvalid < 0 || nmax < 0) return LOITS_ERR_INVALID;
  const TupleGeom g = geom_of(shape);
  const int64_t ncell = g.batch * g.cells;
  if (ncell == 0) return LOITS_OK;
  if (!x_bins || !xsec_x || !q_bins || !xsec_q || !acceptance || !norm_x || !norm_q || !cdf_x ||
      !cdf_q || !grad_xsec_x || !grad_xsec_q || !workspace ||
      (nvalid > 0 && (!grad_events || !packed)))
    return LOITS_ERR_INVALID;
  if (sequence > (UINT64_MAX - 1) / 2) return LOITS_ERR_INVALID;
  const BackwardLayout L = backward_layout(g, nvalid);
  if (workspace_bytes < L.total) return LOITS_ERR_CAPACITY;
  TupleBackwardArgs a;
  a.g = g;
  a.grad = grad_events;
  a.packed = packed;
  a.nvalid = nvalid;
  a.nmax = nmax;
  a.seed = seed;
  a.stream_x = 2 * sequence;
  a.stream_q = 2 * sequence + 1;
  a.x_bins = x_bins;
  a.xsec_x = xsec_x;
  a.q_bins = q_bins;
  a.xsec_q = xsec_q;
  a.acceptance = acceptance;
  a.norm_x = norm_x;
  a.norm_q = norm_q;
  a.cdf_x = cdf_x;
  a.cdf_q = cdf_q;
  a.grad_x = grad_xsec_x;
  a.grad_q = grad_xsec_q;
  a.valid_dev = valid_dev;
  a.nmax_dev = nmax_dev;
  char* ws = static_cast<char*>(workspace);
  int64_t* cell_rows = reinterpret_cast<int64_t*>(ws + L.cell_rows);
  int64_t* chunks = reinterpret_cast<int64_t*>(ws + L.chunks);
  int64_t* chunk_first = reinterpret_cast<int64_t*>(ws + L.chunk_first);
  int64_t* alloc = reinterpret_cast<int64_t*>(ws + L.alloc);
  double* partials = reinterpret_cast<double*>(ws + L.partials);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t kt = g.kx + g.kq;
  tuple_rows_kernel<<<grid_for(ncell + 1, 256), 256, 0, st>>>(a, cell_rows, chunks);
  cell_scan_kernel<<<1, kScanThreads, 0, st>>>(chunks, ncell, chunk_first, alloc);
  // chunk partials: lane-private accumulators when 32 copies fit
  const size_t lane_bytes = static_cast<size_t>(32) * (kt + 1) * sizeof(double);
  const bool lane_private = lane_bytes <= 24 * 1024;
  const size_t per_warp = lane_private ? lane_bytes : static_cast<size_t>(kt) * sizeof(double);
  int wpb = 8;
  while (wpb > 1 && per_warp * wpb > 48 * 1024) wpb >>= 1;
  size_t smem = per_warp * wpb;
  if (smem > 200 * 1024) return LOITS_ERR_UNSUPPORTED;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(tuple_chunk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return LOITS_ERR_CUDA;
  const int64_t cblocks = (L.max_chunks + wpb - 1) / wpb;
  if (cblocks > 0x7fffffff) return LOITS_ERR_UNSUPPORTED;
  if (cblocks > 0)
    tuple_chunk_kernel<<<static_cast<unsigned>(cblocks), wpb * 32, smem, st>>>(
        a, cell_rows, chunk_first, alloc + 1, partials, lane_private ? 1 : 0);
  // per cell: ordered sum of its chunks, reverse chain
  const size_t cell_warp = static_cast<size_t>(kt) * sizeof(double);
  int wpc = 8;
  while (wpc > 1 && cell_warp * wpc > 48 * 1024) wpc >>= 1;
  smem = cell_warp * wpc;
  if (smem > 200 * 1024) return LOITS_ERR_UNSUPPORTED;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(tuple_cell_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return LOITS_ERR_CUDA;
  const int64_t blocks = (ncell + wpc - 1) / wpc;
  if (blocks > 0x7fffffff) return LOITS_ERR_UNSUPPORTED;
  tuple_cell_kernel<<<static_cast<unsigned>(blocks), wpc * 32, smem, st>>>(a, chunk_first,
                                                                          partials);
  return launch_status(cudaGetLastError());
}

}  // namespace

extern "C" int loits_tuple_backward(const loits_shape* shape, const double* grad_events,
                                    const int64_t* packed, int64_t nvalid, int64_t nmax,
                                    uint64_t seed, uint64_t sequence, const double* x_bins,
                                    const double* xsec_x, const double* q_bins,
                                    const double* xsec_q, const uint8_t* acceptance,
                                    const double* norm_x, const double* norm_q,
                                    const double* cdf_x, const double* cdf_q,
                                    double* grad_xsec_x, double* grad_xsec_q, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  return tuple_backward_launch(shape, grad_events, packed, nvalid, nmax, nullptr, nullptr, seed,
                               sequence, x_bins, xsec_x, q_bins, xsec_q, acceptance, norm_x,
                               norm_q, cdf_x, cdf_q, grad_xsec_x, grad_xsec_q, workspace,
                               workspace_bytes, stream);
}

extern "C" int loits_tuple_backward_bounded(const loits_shape* shape, const double* grad_events,
                                            const int64_t* packed, const int64_t* valid,
                                            const int64_t* alloc, int64_t capacity,
                                            uint64_t seed, uint64_t sequence,
                                            const double* x_bins, const double* xsec_x,
                                            const double* q_bins, const double* xsec_q,
                                            const uint8_t* acceptance, const double* norm_x,
                                            const double* norm_q, const double* cdf_x,
                                            const double* cdf_q, double* grad_xsec_x,
                                            double* grad_xsec_q, void* workspace,
                                            size_t workspace_bytes, void* stream) {
  if (!valid || !alloc) return LOITS_ERR_INVALID;
  return tuple_backward_launch(shape, grad_events, packed, capacity, 0, valid, alloc, seed,
                               sequence, x_bins, xsec_x, q_bins, xsec_q, acceptance, norm_x,
                               norm_q, cdf_x, cdf_q, grad_xsec_x, grad_xsec_q, workspace,
                               workspace_bytes, stream);
}

// ============================================== allocation-free sampling call
//
// Some callers cannot allocate device memory at the point where they sample:
// code running inside a framework that owns every byte of the GPU through
// its own pool (the pool would have to hand out a buffer, and cudaMalloc
// beside it can fail or fragment it), or real-time loops that forbid any
// allocation after start-up.  loits_tuple_sample_noalloc serves them: the
// only scratch loits_tuple_sample needs (a ticket counter and the look-back
// words of its tiles) lives in the fixed array below, which is part of the
// library image and exists on every GPU that loads the library until the
// process exits.  The caller still passes all inputs and outputs.

namespace {

// 16 bytes of ticket + 8 bytes of look-back state per 1024-slot tile.
constexpr int64_t kNoAllocMaxTiles = LOITS_TUPLE_NOALLOC_MAX_ACTIVE / kSampleTile;
static_assert(kNoAllocMaxTiles * kSampleTile == LOITS_TUPLE_NOALLOC_MAX_ACTIVE,
              "the limit is a whole number of tiles");
constexpr size_t kNoAllocScratchBytes = 16 + static_cast<size_t>(kNoAllocMaxTiles) * 8;

}  // namespace

static __device__ __align__(256) unsigned char g_tuple_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device.  In host code
// the array's name is a host-side stand-in, not a device address, so the
// address is looked up once per device (with that device current) and kept
// for the life of the process's context on that device: a process that
// destroys that context (cudaDeviceReset) must not call this entry point on
// the device again, since the kept address would be stale.
int noalloc_scratch(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return LOITS_ERR_CUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return LOITS_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tuple_noalloc_scratch) != cudaSuccess || !p)
      return LOITS_ERR_CUDA;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return LOITS_OK;
}

}  // namespace

extern "C" int loits_tuple_sample_noalloc(const loits_shape* shape, const double* x_bins,
                                          const double* q_bins, const double* cdf_x,
                                          const double* cdf_q, const int64_t* cell_offsets,
                                          int64_t nmax, int64_t active, uint64_t seed,
                                          uint64_t sequence, double* events, int64_t* packed,
                                          int16_t* interval_x, int16_t* interval_q,
                                          int64_t* valid, int32_t* status, void* stream) {
  if (active < 0) return LOITS_ERR_INVALID;
  if (active > LOITS_TUPLE_NOALLOC_MAX_ACTIVE ||
      loits_tuple_sample_workspace(active) > kNoAllocScratchBytes)
    return LOITS_ERR_CAPACITY;
  void* scratch = nullptr;
  const int rc = noalloc_scratch(&scratch);
  if (rc != LOITS_OK) return rc;
  // the sampling call clears the part of the scratch that must start at zero
  return loits_tuple_sample(shape, x_bins, q_bins, cdf_x, cdf_q, cell_offsets, nmax, active, seed,
                            sequence, events, packed, interval_x, interval_q, valid, status,
                            scratch, kNoAllocScratchBytes, stream);
}
