/*
 * loits_oracle.c -- CPU oracle for the LOITS sampler.  TEST INFRASTRUCTURE.
 *
 * This library is the checker, never the product: only the test-suite, the
 * smoke check and the CPU-baseline leg of bench.py load it.  The CUDA product
 * path does not link, import or call anything in this directory.
 *
 * It restates in plain C (IEEE-754 binary64, built with -ffp-contract=off so
 * every product and sum is rounded on its own, exactly as written) the
 * algorithm of niteya-shah/quantom_loits:
 *
 *   rng/philox.hpp:17-56        Philox4x32-10, counter (block, stream), key seed
 *   rng/philox.hpp:59-61        uniform_float: (bits >> 8) * 2^-24
 *   cpp/loits_core.cpp:12-18    interval: count of knots <= u, minus one, clamp
 *   cpp/loits_core.cpp:22-37    allocate_counts: trunc(|w * n_events|)
 *   cpp/loits_core.cpp:39-53    fill_uniform: slot p = word (p & 3) of block p >> 2
 *   cpp/loits_core.cpp:55-109   density_x/q: trapezoid norm, rho = xsec * (1/n)
 *   cpp/loits_core.cpp:111-165  cdf_x/q: running trapezoid sum times acceptance
 *   cpp/loits_core.cpp:167-237  interpolate_x/q: b_j + (db * 1/(dc + 1e-5)) * (u - c_j)
 *   cpp/loits_core.cpp:239-266  compact: keep finite x, q with x * q != 0
 *   cpp/loits_core.cpp:268-338  interpolation_vjp_x/q
 *   cpp/loits_core.cpp:340-398  cdf_vjp_x/q (reverse suffix sum)
 *   cpp/loits_core.cpp:400-472  density_vjp_x/q
 *
 * Two front ends share the per-curve helpers:
 *   oracle_r_*  the reference's own 2-D input tuple (cells with an x curve and
 *               a q curve each), bit-for-bit the reference arithmetic;
 *   oracle_d_*  B independent 1-D densities described by offset tables.  A
 *               1-D density is the reference's x curve of a one-cell theory
 *               (nx = ny = 1, weight (n_b + 0.5) / nmax, n_events = nmax), so
 *               counter p = b * nmax + slot and stream 2 * sequence; the extra
 *               per-density acceptance x > x_cut is applied after the
 *               reference predicate, which keeps the order of the survivors.
 *               Intervals are int32 (no int16 wrap) and found by binary
 *               search when the CDF is non-decreasing (equal to the count),
 *               by the count otherwise.
 *
 * Parity of this restatement is pinned by tests/test_oracle_golden.py against
 * the Random123 known answer used by the reference (tests/test_native_rng.py:
 * 43-55) and against vectors produced by the reference's own compiled cores
 * (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_EPSILON 1e-5

/* ------------------------------------------------------------------ Philox */

void oracle_philox4x32_10(uint64_t block, uint64_t stream, uint64_t seed, uint32_t out[4]) {
  /* Random123 Philox4x32-10 (Salmon et al., SC'11): two 32x32->64 multiplies
     per round, Weyl key schedule, 10 rounds. */
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  uint32_t x0 = (uint32_t)block, x1 = (uint32_t)(block >> 32);
  uint32_t x2 = (uint32_t)stream, x3 = (uint32_t)(stream >> 32);
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int r = 0; r < 10; ++r) {
    uint64_t pa = (uint64_t)M0 * x0;
    uint64_t pb = (uint64_t)M1 * x2;
    uint32_t y0 = (uint32_t)(pb >> 32) ^ x1 ^ k0;
    uint32_t y1 = (uint32_t)pb;
    uint32_t y2 = (uint32_t)(pa >> 32) ^ x3 ^ k1;
    uint32_t y3 = (uint32_t)pa;
    x0 = y0; x1 = y1; x2 = y2; x3 = y3;
    k0 += W0; k1 += W1;  /* the bump after the last round is never used */
  }
  out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

float oracle_uniform_float(uint32_t bits) { return (float)(bits >> 8) * 0x1.0p-24f; }

/* Uniform of padded slot p on one stream. */
static float slot_uniform(int64_t p, uint64_t seed, uint64_t stream) {
  uint32_t w[4];
  oracle_philox4x32_10((uint64_t)p >> 2, stream, seed, w);
  return oracle_uniform_float(w[p & 3]);
}

void oracle_fill_uniform(float* values, int64_t count, uint64_t seed, uint64_t stream) {
  for (int64_t p = 0; p < count; p += 4) {
    uint32_t w[4];
    oracle_philox4x32_10((uint64_t)p >> 2, stream, seed, w);
    for (int i = 0; i < 4 && p + i < count; ++i) values[p + i] = oracle_uniform_float(w[i]);
  }
}

/* ------------------------------------------------------- per-curve helpers */

/* Trapezoid normaliser and CDF of one curve with k knots (cpp/loits_core.cpp:
   55-165).  acc is 0 or 1.  Returns the norm. */
static double curve_cdf(const double* bins, const double* xs, int64_t k, double acc, double* cdf) {
  double n = 0.0;
  for (int64_t t = 1; t < k; ++t) {
    double half_width = 0.5 * (bins[t] - bins[t - 1]);
    n += half_width * (xs[t - 1] + xs[t]);
  }
  const double inv_n = 1.0 / n;
  double cum = 0.0;
  double r_prev = xs[0] * inv_n;
  cdf[0] = 0.0;
  for (int64_t t = 1; t < k; ++t) {
    double r_t = xs[t] * inv_n;
    double half_width = 0.5 * (bins[t] - bins[t - 1]);
    cum += half_width * (r_prev + r_t);
    cdf[t] = cum * acc;
    r_prev = r_t;
  }
  return n;
}

/* Count semantics of cpp/loits_core.cpp:12-18, without the int16 narrowing. */
static int64_t interval_count(const double* cdf, int64_t k, double u) {
  int64_t sel = -1;
  for (int64_t t = 0; t < k; ++t) sel += (u >= cdf[t]) ? 1 : 0;
  if (sel < 0) sel = 0;
  if (sel > k - 2) sel = k - 2;
  return sel;
}

/* Same value as interval_count on a non-decreasing cdf: upper bound - 1. */
static int64_t interval_search(const double* cdf, int64_t k, double u) {
  int64_t lo = 0, hi = k; /* first t with cdf[t] > u lies in [lo, hi] */
  while (lo < hi) {
    int64_t mid = lo + (hi - lo) / 2;
    if (u >= cdf[mid]) lo = mid + 1; else hi = mid;
  }
  int64_t sel = lo - 1;
  if (sel < 0) sel = 0;
  if (sel > k - 2) sel = k - 2;
  return sel;
}

static int is_nondecreasing(const double* cdf, int64_t k) {
  for (int64_t t = 1; t < k; ++t) if (!(cdf[t] >= cdf[t - 1])) return 0;
  return 1;
}

/* Inverse-CDF value on interval j (cpp/loits_core.cpp:193-196). */
static double curve_value(const double* bins, const double* cdf, int64_t j, double u) {
  const double c0 = cdf[j];
  const double inv_d = 1.0 / (cdf[j + 1] - c0 + ORACLE_EPSILON);
  const double m = (bins[j + 1] - bins[j]) * inv_d;
  return bins[j] + m * (u - c0);
}

/* Scatter of one event's cotangent g into grad_cdf (cpp/loits_core.cpp:293-300). */
static void curve_value_vjp(const double* bins, const double* cdf, int64_t j, double u, double g,
                            double* gcdf) {
  const double c0 = cdf[j];
  const double d = cdf[j + 1] - c0 + ORACLE_EPSILON;
  const double inv_d = 1.0 / d;
  const double t = u - c0;
  const double db = bins[j + 1] - bins[j];
  const double up = g * db;
  gcdf[j] += up * (-inv_d + t * inv_d * inv_d);
  gcdf[j + 1] -= up * t * inv_d * inv_d;
}

/* Reverse suffix scan then normaliser VJP of one curve (cpp/loits_core.cpp:
   340-472).  gxs receives d(loss)/d(xsec); grho is k doubles of scratch. */
static void curve_cdf_vjp(const double* bins, const double* xs, double n, double acc,
                          const double* gcdf, double* grho, double* gxs, int64_t k) {
  for (int64_t t = 0; t < k; ++t) grho[t] = 0.0;
  double suffix = 0.0;
  for (int64_t t = k - 1; t > 0; --t) {
    suffix += gcdf[t];
    const double g = 0.5 * (bins[t] - bins[t - 1]) * acc * suffix;
    grho[t - 1] += g;
    grho[t] += g;
  }
  const double inv_n = 1.0 / n;
  const double inv_n2 = inv_n * inv_n;
  double gnorm = 0.0;
  for (int64_t t = 0; t < k; ++t) {
    gxs[t] = grho[t] * inv_n;
    gnorm -= grho[t] * xs[t] * inv_n2;
  }
  for (int64_t t = 1; t < k; ++t) {
    const double g = 0.5 * (bins[t] - bins[t - 1]) * gnorm;
    gxs[t - 1] += g;
    gxs[t] += g;
  }
}

static int event_kept(double x, double q) { return isfinite(x) && isfinite(q) && x * q != 0.0; }

/* ------------------------------------------------------ reference 2-D tuple */

typedef struct {
  int64_t batch, nx, ny, kx, kq;
} oracle_shape_t;

/* Offsets of the two curves of cell (b, ix, iy); the x curve is stored
   y-major, the q curve x-major (pytorch/theory.py:94-126). */
static int64_t xcurve_index(const oracle_shape_t* s, int64_t b, int64_t ix, int64_t iy) {
  return (b * s->ny + iy) * s->nx + ix;
}
static int64_t qcurve_index(const oracle_shape_t* s, int64_t b, int64_t ix, int64_t iy) {
  return (b * s->nx + ix) * s->ny + iy;
}

void oracle_r_allocate(const oracle_shape_t* s, const double* weights, int64_t n_events,
                       int64_t* counts, int64_t* nmax, int64_t* active) {
  const int64_t n = s->batch * s->nx * s->ny;
  const double scale = (double)n_events;
  int64_t mx = 0, tot = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t c = (int64_t)fabs(weights[i] * scale);
    counts[i] = c;
    tot += c;
    if (c > mx) mx = c;
  }
  *nmax = mx;
  *active = tot;
}

/* norm and CDF of every x curve (axis 0) or q curve (axis 1). */
void oracle_r_cdf(const oracle_shape_t* s, int axis, const double* bins, const double* xsec,
                  const uint8_t* acceptance, double* norm, double* cdf) {
  const int64_t k = axis == 0 ? s->kx : s->kq;
  for (int64_t b = 0; b < s->batch; ++b)
    for (int64_t ix = 0; ix < s->nx; ++ix)
      for (int64_t iy = 0; iy < s->ny; ++iy) {
        const int64_t ci = axis == 0 ? xcurve_index(s, b, ix, iy) : qcurve_index(s, b, ix, iy);
        const int64_t bi = axis == 0 ? b * s->nx + ix : b * s->ny + iy;
        const double acc = acceptance[(b * s->nx + ix) * s->ny + iy] ? 1.0 : 0.0;
        norm[ci] = curve_cdf(bins + bi * k, xsec + ci * k, k, acc, cdf + ci * k);
      }
}

/* Fused interpolation and stable compaction over the active slots.  Writes
   rows in (b, cell, slot) order; interval_x/q (may be NULL) receive the
   int16 interval of each kept row.  Returns the number of kept rows. */
int64_t oracle_r_sample(const oracle_shape_t* s, const double* x_bins, const double* q_bins,
                        const double* cdf_x, const double* cdf_q, const int64_t* counts,
                        int64_t nmax, uint64_t seed, uint64_t sequence, double* events,
                        int64_t* packed, int16_t* interval_x, int16_t* interval_q) {
  const int64_t cells = s->nx * s->ny;
  int64_t row = 0;
  for (int64_t b = 0; b < s->batch; ++b)
    for (int64_t cell = 0; cell < cells; ++cell) {
      const int64_t ix = cell / s->ny, iy = cell % s->ny;
      const double* xc = cdf_x + xcurve_index(s, b, ix, iy) * s->kx;
      const double* xb = x_bins + (b * s->nx + ix) * s->kx;
      const double* qc = cdf_q + qcurve_index(s, b, ix, iy) * s->kq;
      const double* qb = q_bins + (b * s->ny + iy) * s->kq;
      const int64_t count = counts[b * cells + cell];
      const int64_t base = (b * cells + cell) * nmax;
      for (int64_t slot = 0; slot < count; ++slot) {
        const int64_t p = base + slot;
        const double ux = (double)slot_uniform(p, seed, 2 * sequence);
        const double uq = (double)slot_uniform(p, seed, 2 * sequence + 1);
        const int64_t jx = interval_count(xc, s->kx, ux);
        const int64_t jq = interval_count(qc, s->kq, uq);
        const double x = curve_value(xb, xc, (int16_t)jx, ux);
        const double q = curve_value(qb, qc, (int16_t)jq, uq);
        if (!event_kept(x, q)) continue;
        events[2 * row] = x;
        events[2 * row + 1] = q;
        packed[row] = p;
        if (interval_x) interval_x[row] = (int16_t)jx;
        if (interval_q) interval_q[row] = (int16_t)jq;
        ++row;
      }
    }
  return row;
}

/* Reverse VJP of the 2-D sampler w.r.t. xsec_x and xsec_q. */
void oracle_r_backward(const oracle_shape_t* s, const double* grad_events, const int64_t* packed,
                       int64_t nvalid, int64_t nmax, uint64_t seed, uint64_t sequence,
                       const double* x_bins, const double* xsec_x, const double* q_bins,
                       const double* xsec_q, const uint8_t* acceptance, const double* norm_x,
                       const double* norm_q, const double* cdf_x, const double* cdf_q,
                       double* grad_xsec_x, double* grad_xsec_q) {
  const int64_t cells = s->nx * s->ny;
  const int64_t nx_tot = s->batch * cells * s->kx, nq_tot = s->batch * cells * s->kq;
  double* gcx = (double*)calloc((size_t)nx_tot, sizeof(double));
  double* gcq = (double*)calloc((size_t)nq_tot, sizeof(double));
  const int64_t kmax = s->kx > s->kq ? s->kx : s->kq;
  double* grho = (double*)malloc((size_t)kmax * sizeof(double));
  for (int64_t r = 0; r < nvalid; ++r) {
    const int64_t p = packed[r];
    const int64_t gc = p / nmax; /* b * cells + cell */
    const int64_t b = gc / cells, cell = gc % cells;
    const int64_t ix = cell / s->ny, iy = cell % s->ny;
    const int64_t xi = xcurve_index(s, b, ix, iy), qi = qcurve_index(s, b, ix, iy);
    const double ux = (double)slot_uniform(p, seed, 2 * sequence);
    const double uq = (double)slot_uniform(p, seed, 2 * sequence + 1);
    const double* xc = cdf_x + xi * s->kx;
    const double* qc = cdf_q + qi * s->kq;
    const int64_t jx = interval_count(xc, s->kx, ux);
    const int64_t jq = interval_count(qc, s->kq, uq);
    curve_value_vjp(x_bins + (b * s->nx + ix) * s->kx, xc, jx, ux, grad_events[2 * r], gcx + xi * s->kx);
    curve_value_vjp(q_bins + (b * s->ny + iy) * s->kq, qc, jq, uq, grad_events[2 * r + 1], gcq + qi * s->kq);
  }
  for (int64_t b = 0; b < s->batch; ++b)
    for (int64_t ix = 0; ix < s->nx; ++ix)
      for (int64_t iy = 0; iy < s->ny; ++iy) {
        const double acc = acceptance[(b * s->nx + ix) * s->ny + iy] ? 1.0 : 0.0;
        const int64_t xi = xcurve_index(s, b, ix, iy), qi = qcurve_index(s, b, ix, iy);
        curve_cdf_vjp(x_bins + (b * s->nx + ix) * s->kx, xsec_x + xi * s->kx, norm_x[xi], acc,
                      gcx + xi * s->kx, grho, grad_xsec_x + xi * s->kx, s->kx);
        curve_cdf_vjp(q_bins + (b * s->ny + iy) * s->kq, xsec_q + qi * s->kq, norm_q[qi], acc,
                      gcq + qi * s->kq, grho, grad_xsec_q + qi * s->kq, s->kq);
      }
  free(gcx);
  free(gcq);
  free(grho);
}

/* ---------------------------------------------------- batched 1-D densities */

int64_t oracle_d_nmax(int64_t nd, const int64_t* eoff) {
  int64_t m = 0;
  for (int64_t b = 0; b < nd; ++b) {
    const int64_t n = eoff[b + 1] - eoff[b];
    if (n > m) m = n;
  }
  return m;
}

/* Norm, CDF and monotone flag of every density. */
void oracle_d_cdf(int64_t nd, const int64_t* koff, const double* grid, const double* values,
                  double* norm, double* cdf, uint8_t* monotone) {
  for (int64_t b = 0; b < nd; ++b) {
    const int64_t o = koff[b], k = koff[b + 1] - koff[b];
    norm[b] = curve_cdf(grid + o, values + o, k, 1.0, cdf + o);
    if (monotone) monotone[b] = (uint8_t)is_nondecreasing(cdf + o, k);
  }
}

static int64_t d_interval(const double* c, int64_t k, double u, int mono) {
  return mono ? interval_search(c, k, u) : interval_count(c, k, u);
}

static int d_accept(double x, const double* x_cut, int64_t b) {
  /* q of the embedding is finite and non-zero, so x * q != 0 iff x != 0 */
  if (!(isfinite(x) && x != 0.0)) return 0;
  return x_cut == NULL || x > x_cut[b];
}

/* Philox slots per density: slot_stride if given (> 0), else max n_b. */
static int64_t d_stride(int64_t nd, const int64_t* eoff, int64_t slot_stride) {
  return slot_stride > 0 ? slot_stride : oracle_d_nmax(nd, eoff);
}

/* Sample every density; rows in (density, slot) order.  row_offsets has nd+1
   entries.  intervals / u_rows / slots (each may be NULL) receive the
   interval, the uniform and the slot of each kept row.  Slot s of density b
   draws counter (density_base + b) * stride + s.  Returns kept rows. */
int64_t oracle_d_sample(int64_t nd, const int64_t* koff, const int64_t* eoff, const double* grid,
                        const double* cdf, const uint8_t* monotone, const double* x_cut,
                        uint64_t seed, uint64_t sequence, int64_t density_base,
                        int64_t slot_stride, double* events, int64_t* row_offsets,
                        int32_t* intervals, float* u_rows, int64_t* slots) {
  const int64_t nmax = d_stride(nd, eoff, slot_stride);
  int64_t row = 0;
  for (int64_t b = 0; b < nd; ++b) {
    row_offsets[b] = row;
    const int64_t o = koff[b], k = koff[b + 1] - koff[b];
    const int64_t n = eoff[b + 1] - eoff[b];
    const int mono = monotone ? monotone[b] : is_nondecreasing(cdf + o, k);
    for (int64_t slot = 0; slot < n; ++slot) {
      const float u32 = slot_uniform((density_base + b) * nmax + slot, seed, 2 * sequence);
      const double u = (double)u32;
      const int64_t j = d_interval(cdf + o, k, u, mono);
      const double x = curve_value(grid + o, cdf + o, j, u);
      if (!d_accept(x, x_cut, b)) continue;
      events[row] = x;
      if (intervals) intervals[row] = (int32_t)j;
      if (u_rows) u_rows[row] = u32;
      if (slots) slots[row] = slot;
      ++row;
    }
  }
  row_offsets[nd] = row;
  return row;
}

/* Inverse CDF of density b at the given uniforms (no acceptance). */
void oracle_d_quantile(int64_t b, const int64_t* koff, const double* grid, const double* cdf,
                       const double* u, int64_t n, double* x, int32_t* intervals) {
  const int64_t o = koff[b], k = koff[b + 1] - koff[b];
  const int mono = is_nondecreasing(cdf + o, k);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t j = d_interval(cdf + o, k, u[i], mono);
    x[i] = curve_value(grid + o, cdf + o, j, u[i]);
    if (intervals) intervals[i] = (int32_t)j;
  }
}

/* Reverse VJP of the batched sampler w.r.t. the density values. */
void oracle_d_backward(int64_t nd, const int64_t* koff, const int64_t* eoff, const double* grid,
                       const double* values, const double* norm, const double* cdf,
                       const uint8_t* monotone, const double* x_cut, uint64_t seed,
                       uint64_t sequence, int64_t density_base, int64_t slot_stride,
                       const double* grad_events, double* grad_values) {
  const int64_t nmax = d_stride(nd, eoff, slot_stride);
  int64_t kmax = 2;
  for (int64_t b = 0; b < nd; ++b) if (koff[b + 1] - koff[b] > kmax) kmax = koff[b + 1] - koff[b];
  double* gcdf = (double*)malloc((size_t)kmax * sizeof(double));
  double* grho = (double*)malloc((size_t)kmax * sizeof(double));
  int64_t row = 0;
  for (int64_t b = 0; b < nd; ++b) {
    const int64_t o = koff[b], k = koff[b + 1] - koff[b];
    const int64_t n = eoff[b + 1] - eoff[b];
    const int mono = monotone ? monotone[b] : is_nondecreasing(cdf + o, k);
    memset(gcdf, 0, (size_t)k * sizeof(double));
    for (int64_t slot = 0; slot < n; ++slot) {
      const double u = (double)slot_uniform((density_base + b) * nmax + slot, seed, 2 * sequence);
      const int64_t j = d_interval(cdf + o, k, u, mono);
      const double x = curve_value(grid + o, cdf + o, j, u);
      if (!d_accept(x, x_cut, b)) continue;
      curve_value_vjp(grid + o, cdf + o, j, u, grad_events[row], gcdf);
      ++row;
    }
    curve_cdf_vjp(grid + o, values + o, norm[b], 1.0, gcdf, grho, grad_values + o, k);
  }
  free(gcdf);
  free(grho);
}

/* Central finite difference of L = sum_rows g_row * x_row w.r.t. values[knot]
   of density b, with every event's interval and acceptance frozen at the
   unperturbed state (the derivative along the branch the analytic VJP
   differentiates).  *flips counts events whose interval or acceptance would
   change under +-h.  g_rows are the cotangents of density b's kept rows; nd is the
   number of densities (nmax is taken over the whole table). */
double oracle_d_fd(int64_t nd, int64_t b, int64_t knot, double h, const int64_t* koff,
                      const int64_t* eoff, const double* grid, const double* values,
                      const double* x_cut, uint64_t seed, uint64_t sequence,
                      const double* g_rows, int64_t* flips) {
  const int64_t nmax = oracle_d_nmax(nd, eoff);
  const int64_t o = koff[b], k = koff[b + 1] - koff[b];
  const int64_t n = eoff[b + 1] - eoff[b];
  double* f = (double*)malloc((size_t)k * sizeof(double));
  double* c0 = (double*)malloc((size_t)k * sizeof(double));
  double* cp = (double*)malloc((size_t)k * sizeof(double));
  double* cm = (double*)malloc((size_t)k * sizeof(double));
  memcpy(f, values + o, (size_t)k * sizeof(double));
  curve_cdf(grid + o, f, k, 1.0, c0);
  const double fk = f[knot];
  f[knot] = fk + h;
  curve_cdf(grid + o, f, k, 1.0, cp);
  f[knot] = fk - h;
  curve_cdf(grid + o, f, k, 1.0, cm);
  const int m0 = is_nondecreasing(c0, k), mp = is_nondecreasing(cp, k), mm = is_nondecreasing(cm, k);
  double lp = 0.0, lm = 0.0;
  int64_t row = 0, nflip = 0;
  for (int64_t slot = 0; slot < n; ++slot) {
    const double u = (double)slot_uniform(b * nmax + slot, seed, 2 * sequence);
    const int64_t j = d_interval(c0, k, u, m0);
    const double x = curve_value(grid + o, c0, j, u);
    if (!d_accept(x, x_cut, b)) {
      const int64_t jp = d_interval(cp, k, u, mp), jm = d_interval(cm, k, u, mm);
      if (d_accept(curve_value(grid + o, cp, jp, u), x_cut, b) ||
          d_accept(curve_value(grid + o, cm, jm, u), x_cut, b))
        ++nflip;
      continue;
    }
    const double xp = curve_value(grid + o, cp, j, u);
    const double xm = curve_value(grid + o, cm, j, u);
    const int64_t jp = d_interval(cp, k, u, mp), jm = d_interval(cm, k, u, mm);
    if (jp != j || jm != j || !d_accept(xp, x_cut, b) || !d_accept(xm, x_cut, b)) ++nflip;
    lp += g_rows[row] * xp;
    lm += g_rows[row] * xm;
    ++row;
  }
  free(f);
  free(c0);
  free(cp);
  free(cm);
  if (flips) *flips = nflip;
  return (lp - lm) / (2.0 * h);
}
