// batch_kernels.cuh -- shared definitions of the batched (ragged 1-D) sampler.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace loits_dev {

// Per-knot state written by the forward's CDF phase and read by sampling,
// the backward and the quantile entry:
//   rec[k]  = {key_k, d_k, grid_k, m_k}: key_k is the smallest fp32 >= c_k
//             (the normalised fp64 CDF at knot k), so (u >= c_k) == (u >=
//             key_k) exactly for every fp32 u; d_k = fl32(key_k - c_k) >= 0,
//             so c_k = key_k - d_k to ~2^-48; the knot position; the
//             inverse-CDF slope of interval k, m_k = (g_{k+1} - g_k) /
//             (c_{k+1} - c_k + 1e-5) (0 on the last knot);
//   invd[k] = 1 / (c_{k+1} - c_k + 1e-5), the backward's weight of interval k;
//   guide   = per density with a non-decreasing CDF, M = 2^m buckets of
//             u: L[k] = number of knots with c_t <= k / M (M >= 16 G where
//             shared memory allows; fewer when it or the large-density cap
//             limits it), so the interval of u in [k/M, (k+1)/M) is found
//             among knots [L[k], L[k+1]]; small densities also keep it
//             packed (pack_entry) for sampling from shared memory.
//
// Densities of at most `gcap` knots are sampled from shared memory (records
// and packed guide copied per tile); larger ones ("large densities", more
// than 8192 knots) keep records and the uint32 guide in global memory: the
// forward searches a window of records around the most probable stretch in
// shared memory (coarse guide beside it) and the rest through L2; the
// backward sums the window's intervals in fixed point in shared memory,
// sends every other event's pair of grad-CDF sums to its two knots with one
// float2 global reduction, and finalizes with a multi-tile reverse scan.
struct BatchArgs {
  // plan tables (device)
  const int64_t* knot_off;     // [B+1]
  const int64_t* n_events;     // [B]
  const int32_t* tile_first;   // [B+1] sampling tiles
  const int32_t* tile_owner;   // [tiles] density of each sampling tile
  const int32_t* cdf_owner;    // [CDF scan tiles] density of each
  const int32_t* chunk_owner;  // [backward chunks] density of each
  const int32_t* cdf_first;    // [B+1] CDF scan tiles
  const int32_t* fin_first;    // [B+1] CDF finalize items (multi-tile densities only)
  const int32_t* chunk_first;  // [B+1] backward chunks
  const int64_t* part_off;     // [B] offset of a density's chunk partials
  const int32_t* rowfill_lo;   // [B] first density whose row offset tile 0 of b writes
  const int64_t* goff;         // [B] offset of a density's guide table (entries)
  const int64_t* pkoff;        // [B] offset of a small density's packed guide (-1: large)
  const int32_t* gbits;        // [B] log2 of a density's guide buckets M
  const int64_t* gc_off;       // [B] offset of a large density's interval pairs (-1: small)
  const int32_t* lfin_first;   // [B+1] reverse-scan tiles of large densities
  int32_t nd;
  int32_t last_nonempty;       // last density with events (-1 if none)
  // item ranges of this launch (global indices)
  int32_t c_lo, c_hi;          // CDF scan tiles
  int32_t f_lo, f_hi;          // CDF finalize items
  int32_t t_lo, t_hi;          // sampling tiles
  int32_t k_lo, k_hi;          // backward chunks
  int32_t d_lo, d_hi;          // densities (backward finalize items)
  int32_t l_lo, l_hi;          // reverse-scan tiles of large densities (each run twice)
  int32_t tiles_total;         // sampling tiles of the whole plan
  const int32_t* tile_r;       // [B] Philox blocks per thread per sampling tile (<= R)
  const int32_t* scan_k;       // [B] knots per thread per CDF tile
  int32_t gcap;                // knots a sampling CTA holds in shared memory
  int32_t mcap;                // guide entries (M + 1) a sampling CTA holds
  int32_t gbits_cap;           // most guide bits this launch copies to shared memory
  int32_t lguide_bits;         // large densities: bits of the coarse guide in shared memory
  int32_t win_n;               // backward: large densities' fixed-point window (intervals, 0: none)
  int32_t fwin_n;              // forward: large densities' window of records in shared memory
  int32_t fwd_guide_off;       // forward: uint32 words from the start of dynamic shared
                               // memory to the guide
  int32_t bwd_guide_off;       // backward: uint32 words from the start of dynamic shared
                               // memory to the guide
                               // (a larger guide is read every 2^s-th count)
  int32_t tiles_per_chunk;
  uint32_t spin_limit;         // polls of one wait before it gives up (LOITS_ERR_TIMEOUT)
  int32_t withhold_tile;       // a sampling tile whose look-back state is never published
                               // (tests of the bounded waits); -1: none
  int64_t nmax;                // Philox slots per density (slot stride)
  int64_t dbase;               // global index of plan density 0
  uint64_t seed, stream_id;
  const uint64_t* seq_dev;     // when set: the sequence, read on the device
  PhiloxKey rk;                // round keys of `seed`
  // inputs
  const float* grid;
  const float* values;
  const float* theory;         // B x 6 power-law parameters: knot values are evaluated from
                               // them (theory.cuh) instead of read from `values`, or null
  const float* x_cut;
  // state (workspace)
  float4* rec;
  float* invd;
  uint32_t* gl;                // per density: L[k] = #{t : c_t <= k / M}, k = 0..M
  uint32_t* gpk;               // per small density: packed entries (first interval of
                               // bucket k | movable knots << 16), k = 0..M-1
  double* norm;
  uint32_t* dflags;            // bit 0: CDF not non-decreasing (count semantics)
  int32_t* kstar;              // kThreshold densities: slot kept iff (word >> 8) > kstar
  uint32_t* cdf_ready;         // 1 once a density's records and packed guide are final
  uint32_t* cdf_scanned;       // scanned CDF tiles per density
  uint32_t* fin_done;          // finalized CDF tiles per density (multi-tile densities)
  uint32_t* cflag;             // per CDF tile: 1 aggregate, 2 inclusive
  double* cagg;
  double* cinc;
  double* cmax;                // per CDF tile: max unnormalised prefix seen
  unsigned long long* tile_state;
  int64_t* tile_prefix;        // first kept row of each sampling tile
  int32_t* warp_off;           // kept rows of earlier warps in the tile, per (tile, warp)
  float* stage_g;              // per forward CTA: TPB * R * 4 floats of staged kept events
  uint32_t* ticket;            // this launch's ticket counter
  int32_t* status;
  uint32_t* chunks_done;       // per density
  float* partials;
  float2* gcdf;                // large densities, per interval j: (to knot j, to knot j+1)
                               // grad-CDF sums (zeroed per backward)
  uint32_t* lflag;             // per reverse-scan tile: 1 aggregate, 2 inclusive
  double* lagg;
  double* linc;
  double* lgn;                 // per reverse-scan tile: sum of grad_rho * value
  uint32_t* lfin_done;         // per density: reverse-scan tiles done
  // forward outputs
  float* events;
  int64_t* row_offsets;
  int32_t* intervals;
  float* offsets;              // saved state: u - c_j of each kept row (with intervals)
  // backward
  const float* grad;
  float* grad_values;
  float* grad_theory;          // with `theory`: B x 6 parameter gradient instead of grad_values
  const int32_t* st_intervals; // saved state read instead of replaying the uniforms
  const float* st_offsets;
  // histogram mode (events are binned instead of written; see hist_bin)
  float* hist;                 // forward: [B * hist_bins], accumulated
  unsigned long long* kept;    // forward: [B] kept events per density
  const float* grad_hist;      // backward: [B * hist_bins]
  int32_t hist_bins;
  int32_t hist_rep;            // shared copies of a tile's histogram (lane % rep), power of 2
  int32_t hist_smem_off;       // floats from the start of dynamic shared memory
  int32_t hist_shift;          // forward: fixed-point bits of a unit weight
  float hist_lo, hist_inv_h;
};

// Histogram mode: the most bins, and the shared memory a tile's copies of
// its histogram may take (one copy per lane when they fit).
constexpr int kMaxHistBins = 1024;
constexpr int kHistSmemBytes = 16 * 1024;

// Per-density flags (dflags):
constexpr uint32_t kNonMonotone = 1u;  // an area is negative/NaN: count semantics
constexpr uint32_t kBadGrid = 2u;      // grid not ascending or not finite
constexpr uint32_t kAcceptAll = 4u;    // every event provably kept (see accept_all_flag)
constexpr uint32_t kThreshold = 8u;    // kept events = uniforms above one threshold (threshold_flag)

}  // namespace loits_dev
