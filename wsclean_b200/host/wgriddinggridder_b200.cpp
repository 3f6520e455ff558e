#include "wgriddinggridder_b200.h"

void WGriddingGridder_B200::Check(int rc) {
  if (rc != WSG_OK) throw std::runtime_error(std::string("wsg: ") + wsg_last_error());
}

WGriddingGridder_B200::WGriddingGridder_B200(size_t width, size_t height, size_t width_t,
                                             size_t height_t, double pixelSizeX,
                                             double pixelSizeY, double l_shift, double m_shift,
                                             size_t nthreads, double epsilon, size_t verbosity,
                                             bool tuning, int precision, int device)
    : width_(width), height_(height) {
  wsg_gridder_params p;
  p.width = width;
  p.height = height;
  p.width_t = width_t;
  p.height_t = height_t;
  p.pixel_size_x = pixelSizeX;
  p.pixel_size_y = pixelSizeY;
  p.l_shift = l_shift;
  p.m_shift = m_shift;
  p.nthreads = nthreads;
  p.epsilon = epsilon;
  p.verbosity = verbosity;
  p.tuning = tuning ? 1 : 0;
  p.precision = precision >= 0 ? precision : (epsilon <= 1.01e-5 ? WSG_PREC_FP64 : WSG_PREC_MIXED);
  p.device = device;
  Check(wsg_gridder_create(&p, &handle_));
}

WGriddingGridder_B200::~WGriddingGridder_B200() {
  if (handle_) wsg_gridder_destroy(handle_);
}

void WGriddingGridder_B200::MemoryUsage(size_t &constant, size_t &per_vis) const {
  Check(wsg_gridder_memory_usage(handle_, &constant, &per_vis));
}

void WGriddingGridder_B200::InitializeInversion() {
  Check(wsg_gridder_initialize_inversion(handle_));
}

void WGriddingGridder_B200::AddInversionData(size_t nrows, size_t nchan, const double *uvw,
                                             const double *freq,
                                             const std::complex<float> *vis) {
  Check(wsg_gridder_add_inversion_data(handle_, nrows, nchan, uvw, freq, vis));
}

void WGriddingGridder_B200::FinalizeImage(double multiplicationFactor) {
  Check(wsg_gridder_finalize_image(handle_, multiplicationFactor));
}

std::vector<float> WGriddingGridder_B200::RealImage() {
  std::vector<float> image(width_ * height_);
  Check(wsg_gridder_real_image(handle_, image.data()));
  return image;
}

void WGriddingGridder_B200::InitializePrediction(const float *image_data) {
  Check(wsg_gridder_initialize_prediction(handle_, image_data));
}

void WGriddingGridder_B200::PredictVisibilities(size_t nrows, size_t nchan, const double *uvw,
                                                const double *freq,
                                                std::complex<float> *vis) const {
  Check(wsg_gridder_predict_visibilities(handle_, nrows, nchan, uvw, freq, vis));
}

wsg_stats WGriddingGridder_B200::Stats() const {
  wsg_stats s;
  Check(wsg_get_stats(wsg_gridder_ctx(handle_), &s));
  return s;
}
