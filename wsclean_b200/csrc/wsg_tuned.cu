// The tuned schedule (ms2dirty_tuning / dirty2ms_tuning).
#include "wsg_host.cuh"

namespace wsg {

// ------------------------------------------------------ tuned schedule
//
// ducc0's ms2dirty_tuning / dirty2ms_tuning (wgridder.h:1781-1877), which
// WSClean calls for -gridder tuned-wgridder: the |w| histogram of the
// masked-in visibilities decides (tuning_choice) whether to subdivide; if
// so, the visibilities at or above the cut bin are gridded facet by facet,
// each facet an image of its own with its own phase centre (and so its own,
// smaller n-1 range and fewer w planes), written into its block of the
// image, and those below the cut are gridded on the whole image and added.
// Each part is one grid_core / degrid_core call on the device-resident
// inputs with a mask selecting its visibilities.

TuningChoice Context::tuning_for(const wsg_args &a, const Staged &s) {
  const size_t nrows = a.nrows, nchan = a.nchan;
  std::vector<double> freq(nchan), fovc(nchan);
  if (is_device_pointer(a.freq))
    CK(cudaMemcpy(freq.data(), a.freq, nchan * sizeof(double), cudaMemcpyDeviceToHost));
  else
    std::memcpy(freq.data(), a.freq, nchan * sizeof(double));
  for (size_t c = 0; c < nchan; ++c) fovc[c] = freq[c] / kSpeedOfLight;
  double *d_fovc = reinterpret_cast<double *>(b_tfovc.ensure(nchan * sizeof(double)));
  CK(cudaMemcpyAsync(d_fovc, fovc.data(), nchan * sizeof(double), cudaMemcpyHostToDevice, stream));
  auto *d = reinterpret_cast<unsigned long long *>(b_tune.ensure((3 + kTuningBins) * 8));
  unsigned long long h[3 + kTuningBins] = {0x7ff0000000000000ull, 0, 0};
  CK(cudaMemcpyAsync(d, h, sizeof h, cudaMemcpyHostToDevice, stream));
  const int nb = std::min(launch_blocks(nrows, 256), num_sms * 8);
  k_wrange<<<nb, 256, 0, stream>>>(nrows, int(nchan), s.uvw, d_fovc, s.mask, d);
  cuda_check(cudaGetLastError(), "k_wrange launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  CK(cudaMemcpyAsync(h, d, 3 * 8, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  TuningChoice none;
  if (h[2] == 0) return none;
  double wmin, wmax;
  std::memcpy(&wmin, &h[0], 8);
  std::memcpy(&wmax, &h[1], 8);
  none.wmin = wmin;
  none.wmax = wmax;
  if (!(wmax > wmin)) return none;
  const double xdw = kTuningBins / (wmax - wmin);
  k_whist<<<nb, 256, 0, stream>>>(nrows, int(nchan), s.uvw, d_fovc, s.mask, wmin, xdw, d + 3);
  cuda_check(cudaGetLastError(), "k_whist launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  CK(cudaMemcpyAsync(h + 3, d + 3, kTuningBins * 8, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  std::vector<uint64_t> hist(h + 3, h + 3 + kTuningBins);
  TuningChoice tc = tuning_choice(a.npix_x, a.npix_y, a.pixsize_x, a.pixsize_y, a.epsilon,
                                  a.do_wgridding != 0, tune_center_set ? tune_center_x : a.center_x,
                                  tune_center_set ? tune_center_y : a.center_y, nrows * nchan, wmin,
                                  wmax, hist.data());
  if (tc.split() && tc.icut > 0) {
    uint8_t *hi = reinterpret_cast<uint8_t *>(b_mhi.ensure(nrows * nchan));
    uint8_t *lo = reinterpret_cast<uint8_t *>(b_mlo.ensure(nrows * nchan));
    k_wsplit<<<launch_blocks(nrows, 256), 256, 0, stream>>>(nrows, int(nchan), s.uvw, d_fovc,
                                                            s.mask, wmin, xdw, tc.icut, hi, lo);
    cuda_check(cudaGetLastError(), "k_wsplit launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  }
  if (verbosity > 0) {
    if (!tc.split())
      std::printf("Tuning decision:\n  no subdivision\n");
    else if (tc.icut == 0)
      std::printf("Tuning decision:\n  subdividing into %dx%d facets.\n", tc.nfx, tc.nfy);
    else
      std::printf("Tuning decision:\n  subdividing w range at w=%g, subdividing high w part into "
                  "%dx%d facets.\n", wmin + tc.icut * (wmax - wmin) / kTuningBins, tc.nfx, tc.nfy);
    std::fflush(stdout);
  }
  return tc;
}

// The arguments of facet (i, j): its size and phase centre.  The facet's
// pixels must land where they lie in the whole image.  Along y that depends
// on negate_v: the gridder places pixel j at m = -center_y + (j - ny/2) py
// when v is negated, so a facet above the middle needs its centre moved the
// other way.  (The reference's faceting moves it the same way in both cases,
// so with negate_v -- WSClean's call -- its tuned images have their facets
// mirrored along y; the results here equal the plain operator's.)
static wsg_args facet_args(const wsg_args &a, const TuningChoice &tc, int i, int j) {
  const Facet f = tuning_facet(a.npix_x, a.npix_y, tc.nfx, tc.nfy, i, j, a.pixsize_x,
                               a.pixsize_y, a.center_x, a.center_y);
  wsg_args af = a;
  af.npix_x = f.x1 - f.x0;
  af.npix_y = f.y1 - f.y0;
  af.center_x = f.cx;
  af.center_y = a.negate_v ? 2.0 * a.center_y - f.cy : f.cy;
  return af;
}

template <typename R>
bool Context::grid_tuned(const wsg_args &a, const Staged &s, double *img, bool accumulate,
                         void *direct_out) {
  const TuningChoice tc = tuning_for(a, s);
  last_tuning = tc;
  if (!tc.split()) return grid_core<R>(a, s, img, accumulate, direct_out);
  const size_t nx = a.npix_x, ny = a.npix_y;
  if (!accumulate) CK(cudaMemsetAsync(img, 0, nx * ny * sizeof(double), stream));
  const uint8_t *hi = tc.icut > 0 ? reinterpret_cast<const uint8_t *>(b_mhi.p) : s.mask;
  for (int i = 0; i < tc.nfx; ++i)
    for (int j = 0; j < tc.nfy; ++j) {
      const Facet f = tuning_facet(nx, ny, tc.nfx, tc.nfy, i, j, a.pixsize_x, a.pixsize_y,
                                   a.center_x, a.center_y);
      wsg_args af = facet_args(a, tc, i, j);
      af.mask = hi;
      Staged sf = s;
      sf.mask = hi;
      grid_core<R>(af, sf, img + f.x0 * ny + f.y0, true, nullptr, ny);
    }
  if (tc.icut > 0) {
    wsg_args al = a;
    Staged sl = s;
    al.mask = sl.mask = reinterpret_cast<const uint8_t *>(b_mlo.p);
    grid_core<R>(al, sl, img, true, nullptr);
  }
  return false;
}

template <typename R>
void Context::degrid_tuned(const wsg_args &a, const Staged &s, const double *img, void *vis_out,
                           const void *direct_in) {
  const TuningChoice tc = tuning_for(a, s);
  last_tuning = tc;
  if (!tc.split()) {
    degrid_core<R>(a, s, img, vis_out, direct_in);
    return;
  }
  // every part adds its visibilities (the caller zeroed vis_out)
  const size_t nx = a.npix_x, ny = a.npix_y;
  const size_t dsz = a.dirty_type == WSG_F64 ? 8 : 4;
  const uint8_t *hi = tc.icut > 0 ? reinterpret_cast<const uint8_t *>(b_mhi.p) : s.mask;
  for (int i = 0; i < tc.nfx; ++i)
    for (int j = 0; j < tc.nfy; ++j) {
      const Facet f = tuning_facet(nx, ny, tc.nfx, tc.nfy, i, j, a.pixsize_x, a.pixsize_y,
                                   a.center_x, a.center_y);
      wsg_args af = facet_args(a, tc, i, j);
      af.mask = hi;
      Staged sf = s;
      sf.mask = hi;
      const size_t off = f.x0 * ny + f.y0;
      degrid_core<R>(af, sf, img ? img + off : nullptr, vis_out,
                     direct_in ? static_cast<const char *>(direct_in) + off * dsz : nullptr, ny,
                     true);
    }
  if (tc.icut > 0) {
    wsg_args al = a;
    Staged sl = s;
    al.mask = sl.mask = reinterpret_cast<const uint8_t *>(b_mlo.p);
    degrid_core<R>(al, sl, img, vis_out, direct_in, 0, true);
  }
}

// Marks a raw operator call as tuned while alive; for a padded odd-size
// image, also the centre the subdivision rule is given.
struct TunedCall {
  Context &cx;
  explicit TunedCall(Context &c) : cx(c) { cx.tuned_call = true; }
  TunedCall(Context &c, double cx_rule, double cy_rule) : cx(c) {
    cx.tuned_call = true;
    cx.tune_center_set = true;
    cx.tune_center_x = cx_rule;
    cx.tune_center_y = cy_rule;
  }
  ~TunedCall() {
    cx.tuned_call = false;
    cx.tune_center_set = false;
  }
};

// The even image one pixel larger along each odd axis of a, centred so that
// its pixel (i, j) lies where pixel (i, j) of a does: half a pixel further
// along x, and along y in the direction pixels run (opposite with negate_v).
static wsg_args padded_odd(const wsg_args &a) {
  const size_t xodd = a.npix_x & 1, yodd = a.npix_y & 1;
  wsg_args ap = a;
  ap.npix_x += xodd;
  ap.npix_y += yodd;
  ap.center_x += 0.5 * a.pixsize_x * double(xodd);
  ap.center_y += (a.negate_v ? -0.5 : 0.5) * a.pixsize_y * double(yodd);
  return ap;
}

void Context::ms2dirty_tuning(const wsg_args &a, const void *vis, void *dirty, int accumulate) {
  require(vis && dirty, "vis and dirty are required");
  const size_t xodd = a.npix_x & 1, yodd = a.npix_y & 1;
  if (!xodd && !yodd) {
    TunedCall tc(*this);
    ms2dirty(a, vis, dirty, accumulate);
    return;
  }
  // odd sizes (the reference's tuned calls take them, wgridder.h:1789-1801):
  // an image one pixel larger along each odd axis whose first npix_x x
  // npix_y pixels lie where pixel (i, j) of the odd image lies,
  // l = center_x + (i - npix_x/2) px (and likewise m), and are kept
  require(a.npix_x > 0 && a.npix_y > 0, "empty image");
  CK(cudaSetDevice(device));
  const wsg_args ap = padded_odd(a);
  const size_t dsz = a.dirty_type == WSG_F64 ? 8 : 4;
  void *tmp = b_pad.ensure(ap.npix_x * ap.npix_y * dsz);
  if (accumulate) {
    CK(cudaMemsetAsync(tmp, 0, ap.npix_x * ap.npix_y * dsz, stream));
    CK(cudaMemcpy2DAsync(tmp, ap.npix_y * dsz, dirty, a.npix_y * dsz, a.npix_y * dsz, a.npix_x,
                         cudaMemcpyDefault, stream));
  }
  CK(cudaStreamSynchronize(stream));
  {
    // the reference's rule sees the padded image centred half a pixel
    // further along both odd axes
    TunedCall tc(*this, a.center_x + 0.5 * a.pixsize_x * double(xodd),
                 a.center_y + 0.5 * a.pixsize_y * double(yodd));
    ms2dirty(ap, vis, tmp, accumulate);
  }
  CK(cudaMemcpy2DAsync(dirty, a.npix_y * dsz, tmp, ap.npix_y * dsz, a.npix_y * dsz, a.npix_x,
                       cudaMemcpyDefault, stream));
  CK(cudaStreamSynchronize(stream));
}

void Context::dirty2ms_tuning(const wsg_args &a, const void *dirty, void *vis) {
  require(vis && dirty, "vis and dirty are required");
  const size_t xodd = a.npix_x & 1, yodd = a.npix_y & 1;
  if (!xodd && !yodd) {
    TunedCall tc(*this);
    dirty2ms(a, dirty, vis);
    return;
  }
  // odd sizes: the image zero-padded to the even image of ms2dirty_tuning,
  // whose pixels lie at the same places, so that the pair stays adjoint (the
  // reference pads here without moving the centre, wgridder.h:1829-1838,
  // which puts the image half a pixel away from its gridding direction)
  require(a.npix_x > 0 && a.npix_y > 0, "empty image");
  CK(cudaSetDevice(device));
  const wsg_args ap = padded_odd(a);
  const size_t dsz = a.dirty_type == WSG_F64 ? 8 : 4;
  void *tmp = b_pad.ensure(ap.npix_x * ap.npix_y * dsz);
  CK(cudaMemsetAsync(tmp, 0, ap.npix_x * ap.npix_y * dsz, stream));
  CK(cudaMemcpy2DAsync(tmp, ap.npix_y * dsz, dirty, a.npix_y * dsz, a.npix_y * dsz, a.npix_x,
                       cudaMemcpyDefault, stream));
  CK(cudaStreamSynchronize(stream));
  TunedCall tc(*this, a.center_x, a.center_y);  // the centre the reference's rule sees
  dirty2ms(ap, tmp, vis);
}


template bool Context::grid_tuned<float>(const wsg_args &, const Staged &, double *, bool, void *);
template bool Context::grid_tuned<double>(const wsg_args &, const Staged &, double *, bool, void *);
template void Context::degrid_tuned<float>(const wsg_args &, const Staged &, const double *, void *,
                                           const void *);
template void Context::degrid_tuned<double>(const wsg_args &, const Staged &, const double *,
                                            void *, const void *);

}  // namespace wsg
