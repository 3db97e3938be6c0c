/*
 * loits_b200.h -- C ABI of the B200 LOITS sampler (libloits_b200.so).
 *
 * Plain pointers and sizes only.  Every buffer is caller-owned DEVICE memory
 * unless a comment says "host"; nothing in the library allocates or frees a
 * caller buffer.  Every launching entry point takes the CUDA stream to launch
 * on as `void* stream` (a cudaStream_t; NULL = legacy default stream), returns
 * immediately (asynchronous), and returns a loits_status code for errors it
 * can see on the host.  Errors seen on the device (a bounded wait that ran
 * out, an output that would not fit) are written to a device int32 status
 * word that the caller reads after synchronising.
 *
 * Two input modes share the kernels' building blocks:
 *
 *  - "tuple": the reference's own 2-D theory tuple (x_bins, xsec_x, q_bins,
 *    xsec_q, weights, acceptance), fp64, one x curve and one q curve per cell.
 *    This is the drop-in for the reference's native pybind module
 *    (cpp/bindings.cpp:24-208, openmp/bindings.cpp); results are those of the
 *    reference cpp core: same Philox counters, same compaction order, same
 *    int16 intervals, same epsilon.
 *  - "batch": B independent 1-D densities of ragged size described by offset
 *    tables, fp32 storage, per-density event counts and an optional
 *    per-density cut x > x_cut.  A batch is exactly the reference's x curve
 *    of a one-cell theory per density (nx = ny = 1), so slot s of density b
 *    uses Philox counter b * nmax + s on stream 2 * sequence, nmax = max n_b.
 */
#ifndef LOITS_B200_H
#define LOITS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------- status */

enum loits_status {
  LOITS_OK = 0,
  LOITS_ERR_INVALID = 1,     /* bad pointer, shape, size or argument */
  LOITS_ERR_UNSUPPORTED = 2, /* outside the supported range (e.g. K > 32767) */
  LOITS_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  LOITS_ERR_TIMEOUT = 4,     /* a bounded device-side wait ran out */
  LOITS_ERR_CAPACITY = 5,    /* an output buffer or workspace is too small */
  LOITS_ERR_EPSILON = 6      /* epsilon other than the reference's 1e-5 */
};

/* Human-readable name of a status code (static string). */
const char* loits_status_string(int status);

/* Library ABI version (major * 10000 + minor * 100 + patch). */
int loits_version(void);

/* ------------------------------------------------------------ uniforms */

/* values[p] = uniform of word (p & 3) of Philox4x32-10 block p >> 2 on
 * (stream, seed), p in [0, count): top 24 bits * 2^-24, in [0, 1).
 * Replaces cpp/loits_core.cpp:39-53 fill_uniform (rng/philox.hpp:17-61). */
int loits_fill_uniform(float* values, int64_t count, uint64_t seed, uint64_t stream_id,
                       void* stream);

/* ------------------------------------------------------ tuple (fp64, 2-D) */

/* {batch, nx, ny, kx, kq}; cells = nx * ny (cpp/bindings.cpp:36-37). */
typedef struct loits_shape {
  int64_t batch, nx, ny, kx, kq;
} loits_shape;

/* Stages allocation + density + cdf of cpp/bindings.cpp:39-77
 * (allocate_counts cpp/loits_core.cpp:22-37, density_x/q :55-109,
 * cdf_x/q :111-165).
 *   weights, acceptance (uint8 0/1): batch * cells, index (b*nx+ix)*ny+iy
 *   counts:       batch * cells int64, trunc(|w * n_events|)
 *   cell_offsets: batch * cells + 1 int64, exclusive prefix of counts
 *   norm_x: (batch, ny, nx), cdf_x like xsec_x; norm_q: (batch, nx, ny),
 *   cdf_q like xsec_q
 *   alloc: 2 int64 {nmax, active}; the caller reads it back to size the
 *   sampling outputs. */
int loits_tuple_prepare(const loits_shape* shape, const double* x_bins, const double* xsec_x,
                        const double* q_bins, const double* xsec_q, const double* weights,
                        const uint8_t* acceptance, int64_t n_events, int64_t* counts,
                        int64_t* cell_offsets, double* norm_x, double* norm_q, double* cdf_x,
                        double* cdf_q, int64_t* alloc, void* stream);

/* Bytes of scratch loits_tuple_sample needs for `active` slots. */
size_t loits_tuple_sample_workspace(int64_t active);

/* Stages random_x/q + interpolation_x/q + stream_compaction of
 * cpp/bindings.cpp:79-124 fused in one kernel (fill_uniform
 * cpp/loits_core.cpp:39-53, interpolate_x/q :167-237, compact :239-266):
 * Philox uniforms are generated in registers for active slots only.
 *   events: capacity `active` rows of (x, q); packed: padded slot index of
 *   each kept row; interval_x / interval_q (may be NULL): int16 interval of
 *   each kept row; valid: 1 int64, the number of kept rows;
 *   status: 1 int32 device status word (LOITS_OK or a device error). */
int loits_tuple_sample(const loits_shape* shape, const double* x_bins, const double* q_bins,
                       const double* cdf_x, const double* cdf_q, const int64_t* cell_offsets,
                       int64_t nmax, int64_t active, uint64_t seed, uint64_t sequence,
                       double* events, int64_t* packed, int16_t* interval_x, int16_t* interval_q,
                       int64_t* valid, int32_t* status, void* workspace, size_t workspace_bytes,
                       void* stream);

/* Allocation-free form of loits_tuple_sample.  No counterpart in the
 * reference.  For callers that cannot allocate device memory where they
 * sample (a framework that owns the whole GPU through its own memory pool,
 * or a loop that must not allocate after start-up): the look-back scratch is
 * a fixed array of 524,304 bytes inside the library (16 B of ticket + 8 B per
 * 1024-slot tile, 65,536 tiles), so `active` may be at most
 * LOITS_TUPLE_NOALLOC_MAX_ACTIVE (67,108,864); more returns
 * LOITS_ERR_CAPACITY without launching.  The first call on a device looks up
 * that array's device address (cudaGetSymbolAddress) and keeps it for the
 * life of the process's context on that device, so make that call before any
 * stream capture, and do not call this entry point again on a device whose
 * context was destroyed (cudaDeviceReset).  Every call on a device shares the
 * one array and leaves its contents behind: calls that may overlap on the GPU
 * (different streams without ordering between them) race. */
#define LOITS_TUPLE_NOALLOC_MAX_ACTIVE 67108864
int loits_tuple_sample_noalloc(const loits_shape* shape, const double* x_bins,
                               const double* q_bins, const double* cdf_x, const double* cdf_q,
                               const int64_t* cell_offsets, int64_t nmax, int64_t active,
                               uint64_t seed, uint64_t sequence, double* events,
                               int64_t* packed, int16_t* interval_x, int16_t* interval_q,
                               int64_t* valid, int32_t* status, void* stream);

/* loits_tuple_sample with the counts left on the device, for a caller that
 * must not wait for them (a CUDA graph replaying prepare + sample + backward
 * of a fixed tuple): alloc is loits_tuple_prepare's {nmax, active} in device
 * memory; capacity, a host-known upper bound on active (at most
 * trunc(|w| * n_events) slots per cell: n_events * sum |w| bounds it), sizes
 * the launch, the outputs (capacity rows) and the workspace
 * (loits_tuple_sample_workspace(capacity)).  valid receives the kept rows;
 * an active count above capacity samples nothing and sets status to
 * LOITS_ERR_CAPACITY.  Results equal loits_tuple_sample's. */
int loits_tuple_sample_bounded(const loits_shape* shape, const double* x_bins,
                               const double* q_bins, const double* cdf_x, const double* cdf_q,
                               const int64_t* cell_offsets, const int64_t* alloc,
                               int64_t capacity, uint64_t seed, uint64_t sequence,
                               double* events, int64_t* packed, int16_t* interval_x,
                               int16_t* interval_q, int64_t* valid, int32_t* status,
                               void* workspace, size_t workspace_bytes, void* stream);

/* Bytes of device workspace loits_tuple_backward needs for nvalid rows. */
size_t loits_tuple_backward_workspace(const loits_shape* shape, int64_t nvalid);

/* Replaces the pybind backward of cpp/bindings.cpp:132-208
 * (interpolation_vjp_x/q cpp/loits_core.cpp:268-338, cdf_vjp_x/q :340-398,
 * density_vjp_x/q :400-472).  grad_events: nvalid rows of 2; packed: the
 * forward's packed rows (ascending); uniforms and intervals are recomputed
 * from (seed, sequence) instead of being stored.  Writes every entry of
 * grad_xsec_x / grad_xsec_q (same shapes as xsec_x / xsec_q).  workspace:
 * loits_tuple_backward_workspace() bytes of caller device memory (no
 * initial contents needed); deterministic. */
int loits_tuple_backward(const loits_shape* shape, const double* grad_events,
                         const int64_t* packed, int64_t nvalid, int64_t nmax, uint64_t seed,
                         uint64_t sequence, const double* x_bins, const double* xsec_x,
                         const double* q_bins, const double* xsec_q, const uint8_t* acceptance,
                         const double* norm_x, const double* norm_q, const double* cdf_x,
                         const double* cdf_q, double* grad_xsec_x, double* grad_xsec_q,
                         void* workspace, size_t workspace_bytes, void* stream);

/* loits_tuple_backward of a loits_tuple_sample_bounded forward: the kept-row
 * count (valid) and nmax (alloc[0]) are read on the device; capacity (the
 * forward's) bounds the rows and sizes the workspace
 * (loits_tuple_backward_workspace(shape, capacity)); grad_events and packed
 * hold capacity rows, of which the first *valid are used. */
int loits_tuple_backward_bounded(const loits_shape* shape, const double* grad_events,
                                 const int64_t* packed, const int64_t* valid,
                                 const int64_t* alloc, int64_t capacity, uint64_t seed,
                                 uint64_t sequence, const double* x_bins, const double* xsec_x,
                                 const double* q_bins, const double* xsec_q,
                                 const uint8_t* acceptance, const double* norm_x,
                                 const double* norm_q, const double* cdf_x, const double* cdf_q,
                                 double* grad_xsec_x, double* grad_xsec_q, void* workspace,
                                 size_t workspace_bytes, void* stream);

/* ------------------------------------------------ batch (fp32, ragged 1-D) */

typedef struct loits_batch_plan loits_batch_plan; /* opaque, host object */

/* Launch geometry of the batched kernels.  Zero fields take defaults. */
typedef struct loits_batch_config {
  int32_t threads;         /* threads per CTA of the sampling kernels: 256, 512 or 1024;
                              0 = the size with the most resident threads per SM */
  int32_t blocks_per_item; /* Philox blocks (4 slots each) per thread per tile, at
                              most: 2,4,8,16; default 16 (8 with 1024 threads); a
                              density's tiles are evened out below this length */
  int32_t scan_knots;      /* knots per thread in the CDF scan: 1..64, default 8 */
  int32_t ctas_per_sm;     /* persistent CTAs per SM (0 = as many as fit) */
  int32_t plain;           /* 1 = one launch per density (no persistent queue) */
  int32_t guide_ratio;     /* log2 of guide buckets per knot of a small density, 1..6;
                              0 = 2 (4 buckets per knot), lowered where the guide
                              would cost resident CTAs */
  int32_t wait_limit;      /* polls of one device-side wait before it gives up and
                              reports LOITS_ERR_TIMEOUT; 0 = the default (about 1 s) */
  int32_t withhold_tile;   /* testing the bounded waits only: 1 + the index of a
                              sampling tile that never publishes its compaction
                              state, so that the next tile's wait runs out (the
                              launch then reports LOITS_ERR_TIMEOUT); 0 = none */
  int64_t density_base;    /* global index of density 0 of this plan (sharding) */
  int64_t slot_stride;     /* Philox slots per density, >= max n_b (0 = max n_b) */
} loits_batch_config;

/* Slot s of (plan-local) density b uses Philox counter
 * (density_base + b) * slot_stride + s.  A batch split into shards, each
 * planned with its first density's global index as density_base and the
 * whole batch's max n_b as slot_stride, samples bit-identically to the
 * unsplit batch. */

/* Build a plan for B densities.  Host arrays: knot_offsets (B+1, knots of
 * density b are [knot_offsets[b], knot_offsets[b+1]), at least 2 each) and
 * event_counts (B, >= 0).  cfg may be NULL (defaults).  The plan owns a
 * small device table (cudaMalloc at creation, cudaFree at destroy). */
int loits_batch_plan_create(int64_t n_densities, const int64_t* knot_offsets,
                            const int64_t* event_counts, const loits_batch_config* cfg,
                            loits_batch_plan** plan);
void loits_batch_plan_destroy(loits_batch_plan* plan);

/* loits_batch_plan_create with geometry per density (host arrays of B, or
 * NULL for the config's value): blocks_per_density[b] in
 * [1, cfg->blocks_per_item] caps density b's sampling tile at threads *
 * blocks_per_density[b] Philox blocks (every plan then evens out a density's
 * tiles: the same tile count, the fewest blocks per thread that cover the
 * density), scan_knots_per_density[b] in [1, 64]
 * its knots per thread in the CDF scan -- so that one launch serves small and
 * large densities each at its own tuned tile length and scan width (the
 * autotuner's per-bucket tables).  No counterpart in the reference (its
 * launch geometry is fixed). */
int loits_batch_plan_create_ex(int64_t n_densities, const int64_t* knot_offsets,
                               const int64_t* event_counts, const loits_batch_config* cfg,
                               const int32_t* blocks_per_density,
                               const int32_t* scan_knots_per_density, loits_batch_plan** plan);

/* Sizes of the caller buffers of a plan. */
int64_t loits_batch_capacity(const loits_batch_plan* plan);      /* sum n_b: events rows */
int64_t loits_batch_total_knots(const loits_batch_plan* plan);   /* knot_offsets[B] */
size_t loits_batch_workspace_bytes(const loits_batch_plan* plan); /* state + scratch */
/* Offset (bytes) of the int32 device status word inside the workspace. */
size_t loits_batch_status_offset(const loits_batch_plan* plan);
/* The config the plan resolved (defaults filled in). */
int loits_batch_plan_config(const loits_batch_plan* plan, loits_batch_config* cfg);

/* Forward: per-density normalisation, trapezoid CDF (compensated fp32 scan,
 * fp64 carries and normaliser), in-kernel Philox, inverse-CDF search and
 * interpolation, acceptance and stable compaction in (density, slot) order.
 *   grid, values: total_knots fp32; x_cut: B fp32 or NULL (no cut);
 *   events: capacity fp32 rows; row_offsets: B+1 int64, kept rows of
 *   density b are [row_offsets[b], row_offsets[b+1]);
 *   intervals: capacity int32 (may be NULL), interval of each kept row.
 * events and intervals start on 16-byte boundaries (rows are written as
 * vectors of four where they can be). 
 * The workspace keeps the CDF state the backward needs.  Replaces, for a
 * batch, cpp/bindings.cpp:24-130 on the embedded tuple. */
int loits_batch_forward(const loits_batch_plan* plan, const float* grid, const float* values,
                        const float* x_cut, uint64_t seed, uint64_t sequence, float* events,
                        int64_t* row_offsets, int32_t* intervals, void* workspace, void* stream);

/* Backward: d(sum_r g_r * x_r)/d(values), with the uniforms, intervals and
 * compaction recomputed from (seed, sequence) and the forward's workspace.
 *   grad_events: capacity fp32 (first row_offsets[B] used);
 *   grad_values: total_knots fp32, every entry written. */
int loits_batch_backward(const loits_batch_plan* plan, const float* grid, const float* values,
                         const float* x_cut, uint64_t seed, uint64_t sequence,
                         const float* grad_events, float* grad_values, void* workspace,
                         void* stream);

/* Saved-state forward: loits_batch_forward plus, for every kept row, the
 * two per-event quantities its VJP needs besides the cotangent -- the
 * interval j (int32) and the offset t = u - c_j inside it (fp32, the value
 * the sampler interpolated with).  This is the compact form of the state the
 * reference saves for its backward (u_x / interval_x / packed / row_offsets,
 * openmp/bindings.cpp:85-131, read by interpolation_vjp_x,
 * cpp/loits_core.cpp:268-338): 8 bytes per kept row in row order instead of
 * padded per-slot arrays.  intervals, offsets: capacity entries each, each
 * starting on a 16-byte boundary. */
int loits_batch_forward_state(const loits_batch_plan* plan, const float* grid,
                              const float* values, const float* x_cut, uint64_t seed,
                              uint64_t sequence, float* events, int64_t* row_offsets,
                              int32_t* intervals, float* offsets, void* workspace, void* stream);

/* VJP from a saved state: the same gradient as loits_batch_backward (up to
 * fp32 accumulation order), reading each kept row's interval, offset and
 * cotangent instead of regenerating its uniform and searching its interval.
 * intervals / offsets: as written by loits_batch_forward_state with this
 * workspace (intervals are clamped to the density's range).  The rows are
 * read four at a time when grad_events, like the state, starts on a 16-byte
 * boundary; otherwise one at a time (same result). */
int loits_batch_backward_state(const loits_batch_plan* plan, const float* grid,
                               const float* values, const float* x_cut, const int32_t* intervals,
                               const float* offsets, const float* grad_events, float* grad_values,
                               void* workspace, void* stream);

/* The forward's CDF of every knot as fp64 (hi + lo), total_knots entries;
 * norm: B fp64 normalisers (may be NULL). */
int loits_batch_cdf(const loits_batch_plan* plan, const void* workspace, double* cdf,
                    double* norm, void* stream);

/* Inverse CDF of density b at n caller uniforms (fp32 in [0,1)), using the
 * forward's CDF state: x and (optional) interval per uniform, no acceptance. */
int loits_batch_quantile(const loits_batch_plan* plan, const void* workspace, int64_t density,
                         const float* u, int64_t n, float* x, int32_t* intervals, void* stream);

/* ------------------------------------------- histogram mode and theory
 *
 * For consumers that only need per-density histograms of the events (the
 * discriminator of the batched GAN step), the sampler bins the kept events
 * instead of compacting and writing them: no reference counterpart (the
 * reference's GAN feeds raw events to its discriminator, pytorch/gan.py:11-24,
 * :84-94).  Event x adds (1 - f) to bin k and f to bin k + 1, where
 * k + f = (x - lo) / h - 1/2 and h = (hi - lo) / bins (triangular weights of
 * bins centred at lo + (k + 1/2) h; weight outside the bins is dropped).  hist
 * is B x bins fp32 and kept B int64 (kept events per density), both written
 * (zeroed first) by the call; the sampled events are those of
 * loits_batch_forward with the same seed and sequence.  1 <= bins <= 1024.
 * sequence_dev (may be NULL): device address of the sequence, read by the
 * kernels instead of `sequence` -- a CUDA graph replaying the call can then
 * advance it between replays. */
int loits_batch_forward_hist(const loits_batch_plan* plan, const float* grid, const float* values,
                             const float* x_cut, uint64_t seed, uint64_t sequence, int32_t bins,
                             float lo, float hi, float* hist, int64_t* kept, void* workspace,
                             const uint64_t* sequence_dev, void* stream);

/* VJP of loits_batch_forward_hist: grad_hist (B x bins) -> grad_values; each
 * kept event's cotangent is (grad_hist[k + 1] - grad_hist[k]) / h.  Needs the
 * workspace of a forward (either form) of the same plan, seed and sequence. */
int loits_batch_backward_hist(const loits_batch_plan* plan, const float* grid, const float* values,
                              const float* x_cut, uint64_t seed, uint64_t sequence, int32_t bins,
                              float lo, float hi, const float* grad_hist, float* grad_values,
                              void* workspace, const uint64_t* sequence_dev, void* stream);

/* loits_batch_forward_hist / loits_batch_backward_hist with the densities
 * given by the power-law theory's parameters (loits_theory_powerlaw below)
 * instead of tabulated values: the CDF tiles evaluate each knot's value from
 * params (B x 6 fp32) and the knot position as they load the knots, so the
 * densities are never written to or read from global memory, and the
 * backward reduces the theory's VJP into grad_params (B x 6, every entry
 * written) where it would write grad_values.  Results equal those of
 * loits_theory_powerlaw followed by the tabulated-value calls (the same
 * values, bit for bit; grad_params to fp32 summation order).  Every density
 * must be one CDF tile staged in shared memory (at most the plan's
 * shared-memory knot count, and threads * scan_knots); otherwise
 * LOITS_ERR_UNSUPPORTED.  The grid is the plan's concatenated knots (each
 * density's own).  Fuses the theory map of pytorch/theory.py:37-126 into the
 * sampler for batched theories. */
int loits_batch_forward_hist_powerlaw(const loits_batch_plan* plan, const float* grid,
                                      const float* params, const float* x_cut, uint64_t seed,
                                      uint64_t sequence, int32_t bins, float lo, float hi,
                                      float* hist, int64_t* kept, void* workspace,
                                      const uint64_t* sequence_dev, void* stream);
int loits_batch_backward_hist_powerlaw(const loits_batch_plan* plan, const float* grid,
                                       const float* params, const float* x_cut, uint64_t seed,
                                       uint64_t sequence, int32_t bins, float lo, float hi,
                                       const float* grad_hist, float* grad_params,
                                       void* workspace, const uint64_t* sequence_dev,
                                       void* stream);

/* Two-component power-law theory of the batched GAN step (replaces, for
 * batched densities, the theory map of pytorch/theory.py:37-126): params is
 * B x 6 fp32 raw generator outputs p; with s(z) = 1 / (1 + e^-z),
 *   a_i = -1/2 + 3/2 s(p[2i]), b_i = 1 + 4 s(p[2i+1]), w_i = log(1 + e^p[4+i]),
 *   values[b][t] = sum_i w_i grid[t]^a_i (1 - grid[t])^b_i   (i = 0, 1),
 * on a grid of `knots` points inside (0, 1] shared by all densities. */
int loits_theory_powerlaw(int64_t n_densities, int64_t knots, const float* params,
                          const float* grid, float* values, void* stream);

/* VJP of loits_theory_powerlaw: grad_params[b][j] = sum_t grad_values[b][t]
 * d values[b][t] / d params[b][j], summed in a fixed order. */
int loits_theory_powerlaw_vjp(int64_t n_densities, int64_t knots, const float* params,
                              const float* grid, const float* grad_values, float* grad_params,
                              void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LOITS_B200_H */
