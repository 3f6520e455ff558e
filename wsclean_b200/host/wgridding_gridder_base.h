// The gridder interface WSClean's WGriddingMSGridder drives
// (wgridder/wgriddinggridder_simple.h:8-22 in WSClean).  Inside a WSClean
// build define WSG_USE_WSCLEAN_HEADERS so the real declaration is used; this
// file restates the same pure-virtual interface, with identical signatures,
// so the adapter also builds and is tested outside WSClean.
#ifndef WSG_WGRIDDING_GRIDDER_BASE_H
#define WSG_WGRIDDING_GRIDDER_BASE_H

#ifdef WSG_USE_WSCLEAN_HEADERS
#include "wgridder/wgriddinggridder_simple.h"
#else
#include <complex>
#include <cstddef>
#include <vector>

class WGriddingGridderBase {
 public:
  virtual ~WGriddingGridderBase() = default;
  virtual void MemoryUsage(size_t &constant, size_t &per_vis) const = 0;
  virtual void InitializeInversion() = 0;
  virtual void AddInversionData(size_t nrows, size_t nchan, const double *uvw,
                                const double *freq, const std::complex<float> *vis) = 0;
  virtual void FinalizeImage(double multiplicationFactor) = 0;
  virtual std::vector<float> RealImage() = 0;
  virtual void InitializePrediction(const float *image_data) = 0;
  virtual void PredictVisibilities(size_t nrows, size_t nchan, const double *uvw,
                                   const double *freq, std::complex<float> *vis) const = 0;
};
#endif

#endif
