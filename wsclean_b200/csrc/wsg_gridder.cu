// The stateful gridder (WGriddingGridder_Simple through wsg_gridder_*).
#include "wsg_host.cuh"

namespace wsg {

// ----------------------------------------------------- stateful gridder

Gridder::Gridder(const wsg_gridder_params &p) : prm(p), ctx(p.device) {
  require(p.verbosity <= 2, "verbosity must be 0, 1, or 2");
  require(p.width_t <= p.width && p.height_t <= p.height, "trimmed size exceeds image size");
  require(p.width_t % 2 == 0 && p.height_t % 2 == 0, "trimmed image size must be even");
  ctx.verbosity = int(p.verbosity);
}

wsg_args Gridder::args(size_t nrows, size_t nchan, const double *uvw, const double *freq) const {
  wsg_args a;
  wsg_args_init(&a);
  a.nrows = nrows;
  a.nchan = nchan;
  a.uvw = uvw;
  a.freq = freq;
  a.npix_x = prm.width_t;
  a.npix_y = prm.height_t;
  a.pixsize_x = prm.pixel_size_x;
  a.pixsize_y = prm.pixel_size_y;
  a.epsilon = prm.epsilon;
  a.do_wgridding = 1;
  // WSClean's call pattern (wgriddinggridder_simple.cpp:56-58)
  a.negate_v = 1;
  a.divide_by_n = 0;
  a.sigma_min = 1.1;
  a.sigma_max = 2.0;
  a.center_x = -prm.l_shift;
  a.center_y = -prm.m_shift;
  a.precision = prm.precision;
  a.vis_type = WSG_C64;
  a.dirty_type = WSG_F64;
  return a;
}

void Gridder::memory_usage(size_t &constant, size_t &per_vis) const {
  // host-side figures for WSClean's row chunking: the trimmed image plus the
  // staging of one chunk; per visibility the device sort keys, indices and
  // record (the host holds nothing extra per visibility)
  constant = prm.width_t * prm.height_t * sizeof(double);
  per_vis = 8;
}

void Gridder::initialize_inversion() {
  CK(cudaSetDevice(ctx.device));
  void *p = ctx.b_img2.ensure(prm.width_t * prm.height_t * sizeof(double));
  CK(cudaMemsetAsync(p, 0, prm.width_t * prm.height_t * sizeof(double), ctx.stream));
  CK(cudaStreamSynchronize(ctx.stream));
  have_img = true;
}

void Gridder::add_inversion_data(size_t nrows, size_t nchan, const double *uvw, const double *freq,
                                 const void *vis) {
  require(have_img, "InitializeInversion must be called first");
  wsg_args a = args(nrows, nchan, uvw, freq);
  ctx.validate(a);
  CK(cudaSetDevice(ctx.device));
  const size_t nvis = nrows * nchan;
  Staged s;
  s.uvw = reinterpret_cast<const double *>(ctx.stage_in(uvw, nrows * 3 * sizeof(double), ctx.b_uvw));
  s.vis = ctx.stage_in(vis, nvis * 8, ctx.b_vis);
  double *img = reinterpret_cast<double *>(ctx.b_img2.p);
  // -gridder tuned-wgridder: ms2dirty_tuning (wgriddinggridder_simple.cpp:59-63)
  if (prm.tuning) {
    if (a.precision == WSG_PREC_FP64)
      ctx.grid_tuned<double>(a, s, img, true, nullptr);
    else
      ctx.grid_tuned<float>(a, s, img, true, nullptr);
  } else if (a.precision == WSG_PREC_FP64) {
    ctx.grid_core<double>(a, s, img, true);
  } else {
    ctx.grid_core<float>(a, s, img, true);
  }
  CK(cudaStreamSynchronize(ctx.stream));
}

void Gridder::finalize_image(double f) {
  require(have_img, "no image to finalize");
  size_t n = prm.width_t * prm.height_t;
  k_scale<<<launch_blocks(n, 256), 256, 0, ctx.stream>>>(n, reinterpret_cast<double *>(ctx.b_img2.p), f);
  cuda_check(cudaGetLastError(), "k_scale launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  CK(cudaStreamSynchronize(ctx.stream));
}

void Gridder::real_image(float *out) {
  require(have_img, "no image available");
  size_t n = prm.width * prm.height;
  const bool odev = is_device_pointer(out);
  float *d = odev ? out : reinterpret_cast<float *>(ctx.b_out.ensure(n * sizeof(float)));
  int dx = int((prm.width - prm.width_t) / 2), dy = int((prm.height - prm.height_t) / 2);
  k_retrim<<<launch_blocks(n, 256), 256, 0, ctx.stream>>>(
      int(prm.width_t), int(prm.height_t), int(prm.width), int(prm.height), dx, dy,
      reinterpret_cast<const double *>(ctx.b_img2.p), d);
  cuda_check(cudaGetLastError(), "k_retrim launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  if (!odev) CK(cudaMemcpyAsync(out, d, n * sizeof(float), cudaMemcpyDeviceToHost, ctx.stream));
  CK(cudaStreamSynchronize(ctx.stream));
}

void Gridder::initialize_prediction(const float *image) {
  require(image != nullptr, "image is required");
  CK(cudaSetDevice(ctx.device));
  size_t n = prm.width * prm.height;
  const float *d = reinterpret_cast<const float *>(ctx.stage_in(image, n * sizeof(float), ctx.b_out));
  double *img = reinterpret_cast<double *>(ctx.b_img2.ensure(prm.width_t * prm.height_t * sizeof(double)));
  int dx = int((prm.width - prm.width_t) / 2), dy = int((prm.height - prm.height_t) / 2);
  k_untrim<<<launch_blocks(prm.width_t * prm.height_t, 256), 256, 0, ctx.stream>>>(
      int(prm.width_t), int(prm.height_t), int(prm.width), dx, dy, d, img);
  cuda_check(cudaGetLastError(), "k_untrim launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  CK(cudaStreamSynchronize(ctx.stream));
  have_img = true;
}

void Gridder::predict_visibilities(size_t nrows, size_t nchan, const double *uvw, const double *freq,
                                   void *vis) {
  require(have_img, "InitializePrediction must be called first");
  wsg_args a = args(nrows, nchan, uvw, freq);
  ctx.validate(a);
  CK(cudaSetDevice(ctx.device));
  Staged s;
  s.uvw = reinterpret_cast<const double *>(ctx.stage_in(uvw, nrows * 3 * sizeof(double), ctx.b_uvw));
  // dirty2ms_tuning when tuned (wgriddinggridder_simple.cpp:109-113)
  ctx.degrid_from_image(a, s, reinterpret_cast<const double *>(ctx.b_img2.p), vis, nrows * nchan * 8,
                        prm.tuning != 0);
}

}  // namespace wsg
