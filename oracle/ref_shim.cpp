// ref_shim.cpp -- C entry points around the reference's OWN compiled core.
// TEST INFRASTRUCTURE: built by oracle/Makefile into oracle/_ref/ together
// with the reference's unmodified cpp/loits_core.cpp or openmp/loits_core.cpp
// (compiled where they lie in the reference tree; no reference source is
// copied here).  Only the test-suite, the smoke check and bench.py's CPU
// baseline / reference arm load the result; the CUDA product never does.
//
// The call sequence is the one of the reference's pybind layer:
//   forward  = cpp/bindings.cpp:24-130  (openmp/bindings.cpp adds row_offsets)
//   backward = cpp/bindings.cpp:132-208
// with PyTorch's tensor allocation replaced by caller-provided host buffers
// (the reference sizes them by allocation.nmax / allocation.active, which
// ref_allocate returns first).
#include <cstdint>
#include <vector>

#include "loits_core.hpp"  // resolved with -I<reference>/cpp or -I<reference>/openmp

#ifdef REF_OPENMP
#include <omp.h>
namespace ref = openmp_loits;
#else
namespace ref = loits;
#endif

namespace {

ref::Shape make_shape(const int64_t dims[5]) {
  // dims = {batch, nx, ny, kx, kq}; cells = nx * ny (cpp/bindings.cpp:36-37)
  return ref::Shape{dims[0], dims[1], dims[2], dims[3], dims[4], dims[1] * dims[2]};
}

}  // namespace

extern "C" {

int ref_is_openmp() {
#ifdef REF_OPENMP
  return 1;
#else
  return 0;
#endif
}

void ref_set_threads(int n) {
#ifdef REF_OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int ref_max_threads() {
#ifdef REF_OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// counts: batch * cells int64.  Returns nmax / active through the pointers.
void ref_allocate(const int64_t dims[5], const double* weights, int64_t n_events, int64_t* counts,
                  int64_t* nmax, int64_t* active) {
  const ref::Shape s = make_shape(dims);
  const ref::Allocation a = ref::allocate_counts(weights, counts, n_events, s);
  *nmax = a.nmax;
  *active = a.active;
}

// Full forward.  Padded outputs (u_x, u_q, interval_x, interval_q) hold
// batch * cells * nmax entries; events (2 per row) and packed hold `active`
// rows; row_offsets (batch * cells + 1) is written by the openmp core only and
// may be null for the cpp core.  Returns the number of kept rows.
int64_t ref_forward(const int64_t dims[5], const double* x_bins, const double* xsec_x,
                    const double* q_bins, const double* xsec_q, const uint8_t* acceptance,
                    const int64_t* counts, int64_t nmax, uint64_t seed, uint64_t sequence,
                    double* norm_x, double* norm_q, double* cdf_x, double* cdf_q, float* u_x,
                    float* u_q, int16_t* interval_x, int16_t* interval_q, double* events,
                    int64_t* packed, int64_t* row_offsets) {
  const ref::Shape s = make_shape(dims);
  const bool* acc = reinterpret_cast<const bool*>(acceptance);
  const int64_t nxs = s.batch * s.cells * s.kx, nqs = s.batch * s.cells * s.kq;
  std::vector<double> rho_x(nxs), rho_q(nqs);
  ref::density_x(x_bins, xsec_x, norm_x, rho_x.data(), s);
  ref::density_q(q_bins, xsec_q, norm_q, rho_q.data(), s);
  ref::cdf_x(x_bins, rho_x.data(), acc, cdf_x, s);
  ref::cdf_q(q_bins, rho_q.data(), acc, cdf_q, s);
  const int64_t total = s.batch * s.cells * nmax;
  ref::fill_uniform(u_x, total, seed, sequence * 2);
  ref::fill_uniform(u_q, total, seed, sequence * 2 + 1);
  std::vector<double> dense_x(total), dense_q(total);
  ref::interpolate_x(x_bins, cdf_x, u_x, counts, nmax, dense_x.data(), interval_x, s);
  ref::interpolate_q(q_bins, cdf_q, u_q, counts, nmax, dense_q.data(), interval_q, s);
#ifdef REF_OPENMP
  return ref::compact(dense_x.data(), dense_q.data(), counts, nmax, events, packed, row_offsets, s);
#else
  (void)row_offsets;
  return ref::compact(dense_x.data(), dense_q.data(), counts, nmax, events, packed, s);
#endif
}

// Full backward; grad_events has 2 * nvalid entries.
void ref_backward(const int64_t dims[5], const double* grad_events, const double* x_bins,
                  const double* xsec_x, const double* q_bins, const double* xsec_q,
                  const uint8_t* acceptance, const double* norm_x, const double* norm_q,
                  const double* cdf_x, const double* cdf_q, const float* u_x, const float* u_q,
                  const int16_t* interval_x, const int16_t* interval_q, const int64_t* packed,
                  int64_t nvalid, const int64_t* row_offsets, int64_t nmax, double* grad_xsec_x,
                  double* grad_xsec_q) {
  const ref::Shape s = make_shape(dims);
  const bool* acc = reinterpret_cast<const bool*>(acceptance);
  const int64_t nxs = s.batch * s.cells * s.kx, nqs = s.batch * s.cells * s.kq;
  std::vector<double> gcx(nxs), gcq(nqs), grx(nxs), grq(nqs);
#ifdef REF_OPENMP
  (void)nvalid;
  ref::interpolation_vjp_x(grad_events, packed, row_offsets, x_bins, cdf_x, u_x, interval_x, nmax,
                           gcx.data(), s);
  ref::interpolation_vjp_q(grad_events, packed, row_offsets, q_bins, cdf_q, u_q, interval_q, nmax,
                           gcq.data(), s);
#else
  (void)row_offsets;
  ref::interpolation_vjp_x(grad_events, packed, nvalid, x_bins, cdf_x, u_x, interval_x, nmax,
                           gcx.data(), s);
  ref::interpolation_vjp_q(grad_events, packed, nvalid, q_bins, cdf_q, u_q, interval_q, nmax,
                           gcq.data(), s);
#endif
  ref::cdf_vjp_x(x_bins, acc, gcx.data(), grx.data(), s);
  ref::cdf_vjp_q(q_bins, acc, gcq.data(), grq.data(), s);
  ref::density_vjp_x(x_bins, xsec_x, norm_x, grx.data(), grad_xsec_x, s);
  ref::density_vjp_q(q_bins, xsec_q, norm_q, grq.data(), grad_xsec_q, s);
}

}  // extern "C"
