// Test infrastructure only: a C-ABI shim around the reference's vendored ducc0
// w-gridder, compiled in place from the reference sources by oracle/Makefile into
// oracle/_ref/.  It is the parity checker and the timed CPU baseline; nothing in
// the product links it.
//
// The call pattern follows WSClean's WGriddingGridder_Simple
// (wgridder/wgriddinggridder_simple.cpp:56-63 and :106-113): ducc0::ms2dirty /
// dirty2ms (external/wgridder/ducc0/wgridder/wgridder.h:1696-1729) and the
// "tuned" variants (wgridder.h:1781-1877), with the full ducc0 argument set
// exposed so tests can pin negate_v / divide_by_n / sigma / center shifts.
//
// Type instances: prec 0 = <float,float> (Tcalc=Tacc=float), prec 1 =
// <double,double>.  vis_double selects complex<double> visibilities (Tms=double,
// only with prec 1) versus complex<float> (WSClean's boundary type).  The dirty
// image has the calc type (WSClean's NumT).
#include <complex>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <stdexcept>

#include "ducc0/wgridder/wgridder.h"

using namespace ducc0;

namespace {

thread_local std::string g_err;

template <typename Tcalc, typename Tms>
void run_ms2dirty(int tuning, size_t nrows, size_t nchan, const double *uvw,
                  const double *freq, const void *vis, const void *wgt,
                  const uint8_t *mask, size_t nx, size_t ny, double px,
                  double py, double eps, int do_w, size_t nthreads,
                  void *dirty, size_t verbosity, int negate_v, int divide_by_n,
                  double smin, double smax, double cx, double cy) {
  cmav<double, 2> uvw2(uvw, {nrows, 3});
  cmav<double, 1> freq2(freq, {nchan});
  cmav<std::complex<Tms>, 2> ms(
      reinterpret_cast<const std::complex<Tms> *>(vis), {nrows, nchan});
  cmav<Tms, 2> w2(reinterpret_cast<const Tms *>(wgt),
                  wgt ? std::array<size_t, 2>{nrows, nchan}
                      : std::array<size_t, 2>{0, 0});
  cmav<uint8_t, 2> m2(mask, mask ? std::array<size_t, 2>{nrows, nchan}
                                 : std::array<size_t, 2>{0, 0});
  vmav<Tcalc, 2> d(reinterpret_cast<Tcalc *>(dirty), {nx, ny});
  if (tuning)
    ms2dirty_tuning<Tcalc, Tcalc>(uvw2, freq2, ms, w2, m2, px, py, eps,
                                  do_w != 0, nthreads, d, verbosity,
                                  negate_v != 0, divide_by_n != 0, smin, smax,
                                  cx, cy);
  else
    ms2dirty<Tcalc, Tcalc>(uvw2, freq2, ms, w2, m2, px, py, eps, do_w != 0,
                           nthreads, d, verbosity, negate_v != 0,
                           divide_by_n != 0, smin, smax, cx, cy);
}

template <typename Tcalc, typename Tms>
void run_dirty2ms(int tuning, size_t nrows, size_t nchan, const double *uvw,
                  const double *freq, const void *dirty, const void *wgt,
                  const uint8_t *mask, size_t nx, size_t ny, double px,
                  double py, double eps, int do_w, size_t nthreads, void *vis,
                  size_t verbosity, int negate_v, int divide_by_n, double smin,
                  double smax, double cx, double cy) {
  cmav<double, 2> uvw2(uvw, {nrows, 3});
  cmav<double, 1> freq2(freq, {nchan});
  vmav<std::complex<Tms>, 2> ms(reinterpret_cast<std::complex<Tms> *>(vis),
                                {nrows, nchan});
  cmav<Tms, 2> w2(reinterpret_cast<const Tms *>(wgt),
                  wgt ? std::array<size_t, 2>{nrows, nchan}
                      : std::array<size_t, 2>{0, 0});
  cmav<uint8_t, 2> m2(mask, mask ? std::array<size_t, 2>{nrows, nchan}
                                 : std::array<size_t, 2>{0, 0});
  cmav<Tcalc, 2> d(reinterpret_cast<const Tcalc *>(dirty), {nx, ny});
  if (tuning)
    dirty2ms_tuning<Tcalc, Tcalc>(uvw2, freq2, d, w2, m2, px, py, eps,
                                  do_w != 0, nthreads, ms, verbosity,
                                  negate_v != 0, divide_by_n != 0, smin, smax,
                                  cx, cy);
  else
    dirty2ms<Tcalc, Tcalc>(uvw2, freq2, d, w2, m2, px, py, eps, do_w != 0,
                           nthreads, ms, verbosity, negate_v != 0,
                           divide_by_n != 0, smin, smax, cx, cy);
}

// Captures std::cout while f runs (ducc0 prints its verbosity report there).
template <typename F>
int captured(char *report, size_t report_len, F &&f) {
  std::ostringstream ss;
  std::streambuf *old = nullptr;
  if (report && report_len) old = std::cout.rdbuf(ss.rdbuf());
  int rc = 0;
  try {
    f();
  } catch (const std::exception &e) {
    g_err = e.what();
    rc = 1;
  }
  if (old) {
    std::cout.rdbuf(old);
    std::string s = ss.str();
    size_t n = std::min(s.size(), report_len - 1);
    std::memcpy(report, s.data(), n);
    report[n] = 0;
  }
  return rc;
}

}  // namespace

extern "C" {

const char *ducc_ref_last_error(void) { return g_err.c_str(); }

// prec: 0 float, 1 double.  vis_double: 1 -> complex<double> vis and double
// weights.  Returns 0 on success, 1 on a ducc0 exception (message via
// ducc_ref_last_error), 2 on an unsupported type combination.
int ducc_ref_ms2dirty(int prec, int vis_double, int tuning, size_t nrows,
                      size_t nchan, const double *uvw, const double *freq,
                      const void *vis, const void *wgt, const uint8_t *mask,
                      size_t nx, size_t ny, double px, double py, double eps,
                      int do_w, size_t nthreads, void *dirty, size_t verbosity,
                      int negate_v, int divide_by_n, double smin, double smax,
                      double cx, double cy, char *report, size_t report_len) {
  return captured(report, report_len, [&] {
    if (prec == 0 && !vis_double)
      run_ms2dirty<float, float>(tuning, nrows, nchan, uvw, freq, vis, wgt,
                                 mask, nx, ny, px, py, eps, do_w, nthreads,
                                 dirty, verbosity, negate_v, divide_by_n, smin,
                                 smax, cx, cy);
    else if (prec == 1 && !vis_double)
      run_ms2dirty<double, float>(tuning, nrows, nchan, uvw, freq, vis, wgt,
                                  mask, nx, ny, px, py, eps, do_w, nthreads,
                                  dirty, verbosity, negate_v, divide_by_n,
                                  smin, smax, cx, cy);
    else if (prec == 1 && vis_double)
      run_ms2dirty<double, double>(tuning, nrows, nchan, uvw, freq, vis, wgt,
                                   mask, nx, ny, px, py, eps, do_w, nthreads,
                                   dirty, verbosity, negate_v, divide_by_n,
                                   smin, smax, cx, cy);
    else
      throw std::runtime_error("unsupported type combination");
  });
}

int ducc_ref_dirty2ms(int prec, int vis_double, int tuning, size_t nrows,
                      size_t nchan, const double *uvw, const double *freq,
                      const void *dirty, const void *wgt, const uint8_t *mask,
                      size_t nx, size_t ny, double px, double py, double eps,
                      int do_w, size_t nthreads, void *vis, size_t verbosity,
                      int negate_v, int divide_by_n, double smin, double smax,
                      double cx, double cy, char *report, size_t report_len) {
  return captured(report, report_len, [&] {
    if (prec == 0 && !vis_double)
      run_dirty2ms<float, float>(tuning, nrows, nchan, uvw, freq, dirty, wgt,
                                 mask, nx, ny, px, py, eps, do_w, nthreads, vis,
                                 verbosity, negate_v, divide_by_n, smin, smax,
                                 cx, cy);
    else if (prec == 1 && !vis_double)
      run_dirty2ms<double, float>(tuning, nrows, nchan, uvw, freq, dirty, wgt,
                                  mask, nx, ny, px, py, eps, do_w, nthreads,
                                  vis, verbosity, negate_v, divide_by_n, smin,
                                  smax, cx, cy);
    else if (prec == 1 && vis_double)
      run_dirty2ms<double, double>(tuning, nrows, nchan, uvw, freq, dirty, wgt,
                                   mask, nx, ny, px, py, eps, do_w, nthreads,
                                   vis, verbosity, negate_v, divide_by_n, smin,
                                   smax, cx, cy);
    else
      throw std::runtime_error("unsupported type combination");
  });
}

}  // extern "C"
