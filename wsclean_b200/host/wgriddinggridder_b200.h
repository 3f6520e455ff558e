// WGriddingGridder_B200: the drop-in replacement for WSClean's
// WGriddingGridder_Simple<NumT> (wgridder/wgriddinggridder_simple.h:34-144),
// implemented over libwsg's C ABI (include/wsg.h).  WSClean's
// WGriddingMSGridder::MakeGridder (wgridder/wgriddingmsgridder.cpp:39-52)
// returns one of these instead; the imager, the threaded scheduler and Radler
// are unchanged.  Errors from the library are rethrown as std::runtime_error,
// the exception type of the reference's MR_assert, so the scheduler's
// capture-and-rethrow path (scheduling/threadedscheduler.cpp:63-67) works as
// before.
#ifndef WSG_WGRIDDINGGRIDDER_B200_H
#define WSG_WGRIDDINGGRIDDER_B200_H

#include <complex>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "wgridding_gridder_base.h"
#include "wsg.h"

class WGriddingGridder_B200 final : public WGriddingGridderBase {
 public:
  // Same arguments as the reference constructor
  // (wgriddinggridder_simple.h:64-68).  precision: WSG_PREC_MIXED (the
  // reference's NumT=float), WSG_PREC_FP64 (NumT=double) or -1 to choose as
  // WSClean does: FP64 when epsilon <= 1.01e-5 (wgriddingmsgridder.cpp:41).
  WGriddingGridder_B200(size_t width, size_t height, size_t width_t, size_t height_t,
                        double pixelSizeX, double pixelSizeY, double l_shift, double m_shift,
                        size_t nthreads, double epsilon = 1e-4, size_t verbosity = 0,
                        bool tuning = false, int precision = -1, int device = -1);
  ~WGriddingGridder_B200() override;
  WGriddingGridder_B200(const WGriddingGridder_B200 &) = delete;
  WGriddingGridder_B200 &operator=(const WGriddingGridder_B200 &) = delete;

  void MemoryUsage(size_t &constant, size_t &per_vis) const override;
  void InitializeInversion() override;
  void AddInversionData(size_t nrows, size_t nchan, const double *uvw, const double *freq,
                        const std::complex<float> *vis) override;
  void FinalizeImage(double multiplicationFactor) override;
  std::vector<float> RealImage() override;
  void InitializePrediction(const float *image_data) override;
  void PredictVisibilities(size_t nrows, size_t nchan, const double *uvw, const double *freq,
                           std::complex<float> *vis) const override;

  // Parameters and phase timings of the last call (ducc0's verbosity report).
  wsg_stats Stats() const;

 private:
  static void Check(int rc);
  wsg_gridder *handle_ = nullptr;
  size_t width_, height_;
};

#endif
