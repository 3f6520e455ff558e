// Imaging weights on the GPU (wsg_weights_*).
#include "wsg_host.cuh"

namespace wsg {

// ------------------------------------------------------- image weights

ImageWeightsGpu::ImageWeightsGpu(Context &cx, int mode, double robust, size_t width,
                                 size_t height, double psx, double psy, bool as_taper,
                                 double super_weight)
    : cx_(cx), mode_(mode), robust_(robust), psx_(psx), psy_(psy), as_taper_(as_taper) {
  require(mode >= 0 && mode <= 2, "weight mode must be natural (0), uniform (1) or Briggs (2)");
  require(super_weight > 0 && psx > 0 && psy > 0, "bad image-weight geometry");
  // the grid size (structures/imageweights.cpp:36-47)
  W_ = size_t(std::round(double(width) / super_weight));
  H_ = size_t(std::round(double(height) / super_weight));
  if (W_ % 2) ++W_;
  if (H_ % 2) ++H_;
  require(W_ >= 2 && H_ >= 2, "image-weight grid too small");
  CK(cudaSetDevice(cx_.device));
  grid_.ensure(W_ * (H_ / 2) * sizeof(double));
  sums_.ensure(2 * sizeof(double));
  CK(cudaMemsetAsync(grid_.p, 0, W_ * (H_ / 2) * sizeof(double), cx_.stream));
  CK(cudaMemsetAsync(sums_.p, 0, 2 * sizeof(double), cx_.stream));
  CK(cudaStreamSynchronize(cx_.stream));
}

ImageWeightsGpu::~ImageWeightsGpu() {
  cudaSetDevice(cx_.device);
  cudaStreamSynchronize(cx_.stream);
  for (DevBuf *b : {&grid_, &sums_, &lambda_, &in_, &out_}) b->release();
}

// wavelength per channel, c / f (aocommon BandData::ChannelWavelength)
const double *ImageWeightsGpu::lambdas(size_t nchan, const double *freq) {
  std::vector<double> f(nchan), l(nchan);
  if (is_device_pointer(freq))
    CK(cudaMemcpy(f.data(), freq, nchan * sizeof(double), cudaMemcpyDeviceToHost));
  else
    std::memcpy(f.data(), freq, nchan * sizeof(double));
  for (size_t c = 0; c < nchan; ++c) {
    require(f[c] > 0, "channel frequencies must be positive");
    l[c] = kSpeedOfLight / f[c];
  }
  double *d = reinterpret_cast<double *>(lambda_.ensure(nchan * sizeof(double)));
  CK(cudaMemcpyAsync(d, l.data(), nchan * sizeof(double), cudaMemcpyHostToDevice, cx_.stream));
  CK(cudaStreamSynchronize(cx_.stream));
  return d;
}

void ImageWeightsGpu::grid(size_t nrows, size_t nchan, size_t npol, const double *uvw,
                           const double *freq, const float *w) {
  require(!finished_, "grid() after finish()");
  require(uvw && freq && nchan > 0 && npol > 0, "uvw and freq are required");
  if (nrows == 0) return;
  CK(cudaSetDevice(cx_.device));
  const double *lam = lambdas(nchan, freq);
  const double *du = reinterpret_cast<const double *>(cx_.stage_in(uvw, nrows * 3 * sizeof(double), cx_.b_uvw));
  const float *dw = reinterpret_cast<const float *>(cx_.stage_in(w, nrows * nchan * npol * sizeof(float), in_));
  WeightGrid g{int(W_), int(H_), psx_, psy_};
  const int nb = std::min(launch_blocks(nrows, 256), cx_.num_sms * 8);
  k_weights_grid<<<nb, 256, 0, cx_.stream>>>(nrows, int(nchan), int(npol), du, lam, dw,
                                             as_taper_ ? 1 : 0, g, reinterpret_cast<double *>(grid_.p),
                                             reinterpret_cast<double *>(sums_.p));
  cuda_check(cudaGetLastError(), "k_weights_grid launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  CK(cudaStreamSynchronize(cx_.stream));
}

void ImageWeightsGpu::finish() {
  require(!finished_, "finish() called twice");
  CK(cudaSetDevice(cx_.device));
  const size_t n = W_ * (H_ / 2);
  double *sums = reinterpret_cast<double *>(sums_.p);
  const int nb = std::min(launch_blocks(n, 256), cx_.num_sms * 8);
  if (mode_ == 2) {
    k_weights_sumsq<<<nb, 256, 0, cx_.stream>>>(n, reinterpret_cast<const double *>(grid_.p), sums + 1);
    cuda_check(cudaGetLastError(), "k_weights_sumsq launch");
  }
  const double num = 5.0 * std::exp(-M_LN10 * robust_);
  k_weights_finish<<<nb, 256, 0, cx_.stream>>>(n, reinterpret_cast<double *>(grid_.p), mode_, sums,
                                               num * num);
  cuda_check(cudaGetLastError(), "k_weights_finish launch");
  g_kernel_launches.fetch_add(mode_ == 2 ? 2 : 1, std::memory_order_relaxed);
  CK(cudaStreamSynchronize(cx_.stream));
  finished_ = true;
}

void ImageWeightsGpu::apply(size_t nrows, size_t nchan, size_t npol, const double *uvw,
                            const double *freq, const float *in, float *out) {
  require(finished_, "apply() before finish()");
  require(uvw && freq && out && nchan > 0 && npol > 0, "uvw, freq and out are required");
  if (nrows == 0) return;
  CK(cudaSetDevice(cx_.device));
  const size_t nv = nrows * nchan * npol;
  const double *lam = lambdas(nchan, freq);
  const double *du = reinterpret_cast<const double *>(cx_.stage_in(uvw, nrows * 3 * sizeof(double), cx_.b_uvw));
  const float *din = reinterpret_cast<const float *>(cx_.stage_in(in, nv * sizeof(float), in_));
  const bool odev = is_device_pointer(out);
  float *dout = odev ? out : reinterpret_cast<float *>(out_.ensure(nv * sizeof(float)));
  WeightGrid g{int(W_), int(H_), psx_, psy_};
  const int nb = std::min(launch_blocks(nrows, 256), cx_.num_sms * 8);
  k_weights_apply<<<nb, 256, 0, cx_.stream>>>(nrows, int(nchan), int(npol), du, lam, g,
                                              reinterpret_cast<const double *>(grid_.p), din, dout);
  cuda_check(cudaGetLastError(), "k_weights_apply launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  if (!odev) CK(cudaMemcpyAsync(out, dout, nv * sizeof(float), cudaMemcpyDeviceToHost, cx_.stream));
  CK(cudaStreamSynchronize(cx_.stream));
}

void ImageWeightsGpu::get(double *grid, size_t *width, size_t *height, double *total) {
  CK(cudaSetDevice(cx_.device));
  if (width) *width = W_;
  if (height) *height = H_;
  if (total)
    CK(cudaMemcpy(total, sums_.p, sizeof(double), cudaMemcpyDeviceToHost));
  if (grid)
    CK(cudaMemcpy(grid, grid_.p, W_ * (H_ / 2) * sizeof(double),
                  is_device_pointer(grid) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
}

}  // namespace wsg
