// The autotuner: timed kernel and tile choices, kept per process.
#include "wsg_host.cuh"

namespace wsg {

// ------------------------------------------------------------ autotuner
//
// Process-wide table of timed choices: (image size, precision, accuracy,
// w-gridding, log2 of the visibility count) -> (W, sigma, tile).

namespace {
struct TuneKey {
  size_t nx, ny;
  int prec, do_w, nlog;
  double eps;
  bool operator<(const TuneKey &o) const {
    return std::tie(nx, ny, prec, do_w, nlog, eps) < std::tie(o.nx, o.ny, o.prec, o.do_w, o.nlog, o.eps);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tuned;

TuneKey tune_key(const wsg_args &a, size_t nvis) {
  int nl = 0;
  while ((size_t(1) << (nl + 1)) <= nvis) ++nl;
  return TuneKey{a.npix_x, a.npix_y, a.precision, a.do_wgridding != 0, nl, a.epsilon};
}
}  // namespace

bool tuned_choice(const wsg_args &a, size_t nvis, TuneChoice &out) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(tune_key(a, nvis));
  if (it == g_tuned.end()) return false;
  out = it->second;
  return true;
}

void store_tuned(const wsg_args &a, size_t nvis, const TuneChoice &c) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[tune_key(a, nvis)] = c;
}

// ------------------------------------------------------- the autotuner

void Context::autotune(const wsg_args &a, const void *vis, int candidates, wsg_stats &best) {
  validate(a);
  require(vis != nullptr, "vis is required");
  require(candidates >= 1, "at least one candidate");
  CK(cudaSetDevice(device));
  const size_t nvis = a.nrows * a.nchan;
  const size_t vsz = a.vis_type == WSG_C128 ? 16 : 8, dsz = a.dirty_type == WSG_F64 ? 8 : 4;
  // inputs on the device once, so that the timings are the kernels'
  DevBuf t_uvw, t_vis, t_wgt, t_mask, t_dirty, t_out;
  auto dev = [&](const void *p, size_t bytes, DevBuf &b) -> const void * {
    if (!p || is_device_pointer(p)) return p;
    void *d = b.ensure(bytes);
    CK(cudaMemcpy(d, p, bytes, cudaMemcpyHostToDevice));
    return d;
  };
  wsg_args ad = a;
  ad.uvw = reinterpret_cast<const double *>(dev(a.uvw, a.nrows * 3 * sizeof(double), t_uvw));
  ad.wgt = dev(a.wgt, nvis * (a.wgt_type == WSG_F64 ? 8 : 4), t_wgt);
  ad.mask = reinterpret_cast<const uint8_t *>(dev(a.mask, nvis, t_mask));
  const void *vd = dev(vis, nvis * vsz, t_vis);
  void *dirty = t_dirty.ensure(a.npix_x * a.npix_y * dsz);
  void *vout = t_out.ensure(nvis * vsz);

  // the data extent and the model's choice
  tune_W = 0;
  ms2dirty(ad, vd, dirty, 0);
  const wsg_stats s0 = stats;
  if (s0.nvis == 0) {
    best = s0;
    return;
  }
  GridPlan gp;
  gp.nx = a.npix_x;
  gp.ny = a.npix_y;
  gp.px = a.pixsize_x;
  gp.py = a.pixsize_y;
  gp.eps = a.epsilon;
  gp.do_w = a.do_wgridding != 0;
  gp.fp32 = a.precision != WSG_PREC_FP64;
  gp.negate_v = a.negate_v != 0;
  gp.divide_by_n = a.divide_by_n != 0;
  gp.lshift = a.center_x;
  gp.mshift = a.negate_v ? -a.center_y : a.center_y;
  gp.nvis = s0.nvis;
  gp.wmin_d = s0.wmin;
  gp.wmax_d = s0.wmax;
  // max |u|, |v| from the band the model chose: rows [0, L] hold |u| <= L
  // cells; recompute from the data instead, on the host copy of uvw
  {
    std::vector<double> h(a.nrows * 3), f(a.nchan);
    CK(cudaMemcpy(h.data(), ad.uvw, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    if (is_device_pointer(a.freq))
      CK(cudaMemcpy(f.data(), a.freq, f.size() * sizeof(double), cudaMemcpyDeviceToHost));
    else
      std::memcpy(f.data(), a.freq, f.size() * sizeof(double));
    double um = 0, vm = 0, fm = 0;
    for (size_t r = 0; r < a.nrows; ++r) {
      um = std::max(um, std::fabs(h[3 * r]));
      vm = std::max(vm, std::fabs(h[3 * r + 1]));
    }
    for (double x : f) fm = std::max(fm, x / kSpeedOfLight);
    gp.umax = um * fm;
    gp.vmax = vm * fm;
  }
  const int tile0 = default_tile(gp.fp32);
  auto cands = rank_kernels(gp, a.sigma_min, a.sigma_max, tile0, size_t(candidates));
  std::vector<int> tiles{12, 16, 20, 24};
  TuneChoice win;
  win.ms = 1e300;
  auto time_pair = [&]() {
    double t = 1e300;
    for (int rep = 0; rep < 3; ++rep) {  // the first one also builds FFT plans
      auto t0 = std::chrono::steady_clock::now();
      ms2dirty(ad, vd, dirty, 0);
      dirty2ms(ad, dirty, vout);
      const double ms =
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (rep > 0) t = std::min(t, ms);
    }
    return t;
  };
  try {
    for (const auto &c : cands)
      for (int T : tiles) {
        if (T > 33 - c.first) continue;
        tune_W = c.first;
        tune_sigma = c.second;
        tune_tile = T;
        double ms;
        try {
          ms = time_pair();
        } catch (const std::exception &e) {  // a candidate that cannot run is skipped
          cudaGetLastError();
          if (verbosity > 0)
            std::printf("autotune: W=%d sigma=%.3f tile=%d skipped: %s\n", c.first, c.second, T,
                        e.what());
          continue;
        }
        if (verbosity > 0)
          std::printf("autotune: W=%d sigma=%.3f tile=%d nu=%zu planes=%zu  %.3f ms per pair\n",
                      c.first, c.second, T, stats.nu, stats.nplanes, ms);
        if (ms < win.ms) win = TuneChoice{c.first, c.second, T, ms};
      }
  } catch (...) {
    tune_W = tune_tile = 0;
    throw;
  }
  tune_W = tune_tile = 0;
  require(win.W > 0, "the autotuner found no candidate that runs");
  store_tuned(a, s0.nvis, win);
  ms2dirty(ad, vd, dirty, 0);
  best = stats;
  best.ms_total = win.ms;
}

}  // namespace wsg
