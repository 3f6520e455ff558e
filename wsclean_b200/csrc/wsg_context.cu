// Host orchestration of libwsg: execution contexts, buffer cache, cuFFT plans,
// and the ms2dirty / dirty2ms drivers (the analogues of ducc0's
// Params::x2dirty and Params::dirty2x, wgridder.h:1430-1501).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "wsg_host.cuh"

namespace wsg {

// libwsg kernels launched by this process (cuFFT and CUB kernels excluded).
std::atomic<size_t> g_kernel_launches{0};

// ------------------------------------------------------------ utilities

void cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation)
    throw OutOfMemory(std::string(what) + ": " + cudaGetErrorString(e));
  throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

void cufft_check(cufftResult r, const char *what) {
  if (r == CUFFT_SUCCESS) return;
  if (r == CUFFT_ALLOC_FAILED) throw OutOfMemory(std::string(what) + ": cuFFT allocation failed");
  throw CufftError(std::string(what) + ": cuFFT error " + std::to_string(int(r)));
}

bool is_device_pointer(const void *p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

void *DevBuf::ensure(size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (n < bytes) {
    release();
    cuda_check(cudaMalloc(&p, bytes), "cudaMalloc");
    n = bytes;
  }
  return p;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  n = 0;
}

int env_int(const char *name, int dflt) {
  const char *s = std::getenv(name);
  return (s && *s) ? std::atoi(s) : dflt;
}

// Bin tile edge asked of the planner (which shrinks it until the W-plane
// tile fits shared memory): measured on the 8.1M-visibility 4096^2 pair,
// 20 is the fastest in mixed precision (3 -> 2 CTAs per SM, but half the
// tile flushes of 16) and 24 in FP64; WSG_TILE overrides it.
int default_tile(bool fp32) { return env_int("WSG_TILE", fp32 ? 20 : 24); }

// --------------------------------------------------------------- context

Context::Context(int dev) {
  if (dev < 0) CK(cudaGetDevice(&dev));
  device = dev;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
  stream = own_stream;
  CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
  for (auto &e : ev) CK(cudaEventCreate(&e));
  // the copy stream also runs a staged call's scan, which the host waits
  // for before it can plan and return; at the highest priority its blocks
  // are scheduled ahead of the previous call's kernels on the main stream
  int prio_lo = 0, prio_hi = 0;
  CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  CK(cudaStreamCreateWithPriority(&cpy, cudaStreamNonBlocking, prio_hi));
  CK(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
  for (cudaEvent_t *e : {&ev_start, &ev_in, &ev_done, &ev_scan, &ev_keys})
    CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  CK(cudaHostAlloc(&h_scan, sizeof(ScanOut), cudaHostAllocMapped));
  CK(cudaHostGetDevicePointer(&h_scan_dev, h_scan, 0));
  for (auto &sl : slots) CK(cudaEventCreateWithFlags(&sl.free_ev, cudaEventDisableTiming));
  std::memset(&stats, 0, sizeof(stats));
  verbosity = env_int("WSG_VERBOSITY", 0);
}

void Context::mark(const char *what) {
  if (verbosity < 2) return;
  marks.emplace_back(what, std::chrono::steady_clock::now());
}

void Context::print_marks(const char *title) {
  if (verbosity < 2 || marks.empty()) return;
  std::printf("  host timeline (%s):", title);
  for (size_t i = 1; i < marks.size(); ++i)
    std::printf(" %s %.3f ms;", marks[i].first,
                std::chrono::duration<double, std::milli>(marks[i].second - marks[i - 1].second).count());
  std::printf("\n");
  std::fflush(stdout);
  marks.clear();
}

Context::~Context() {
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  for (auto &kv : fft_plans) cufftDestroy(kv.second);
  for (auto *b : all_buffers()) b->release();
  for (auto &e : ev) cudaEventDestroy(e);
  for (cudaStream_t st : {cpy, d2h})
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  for (cudaEvent_t e : {ev_start, ev_in, ev_done, ev_scan, ev_keys})
    if (e) cudaEventDestroy(e);
  for (auto &sl : slots)
    if (sl.free_ev) cudaEventDestroy(sl.free_ev);
  for (auto &sl : slots)
    for (DevBuf *b : {&sl.uvw, &sl.vis, &sl.wgt, &sl.mask, &sl.out, &sl.fovc}) b->release();
  if (h_scan) cudaFreeHost(h_scan);
  if (h_small) cudaFreeHost(h_small);
  if (own_stream) cudaStreamDestroy(own_stream);
}

std::vector<DevBuf *> Context::all_buffers() {
  return {&b_uvw, &b_fovc, &b_vis, &b_wgt, &b_mask, &b_keys_a, &b_keys_b, &b_vals_a,
          &b_vals_b, &b_cub, &b_rec, &b_chunks, &b_small, &b_band, &b_bandf, &b_bandd, &b_H,
          &b_img, &b_img2, &b_acc, &b_fftwork, &b_out, &corr_cache[0].buf, &corr_cache[1].buf,
          &tw_cache[0].buf, &tw_cache[1].buf, &b_tune, &b_tfovc, &b_mhi, &b_mlo, &b_pad};
}

void Context::invalidate_tables() {
  for (auto &e : corr_cache) e.valid = false;
  for (auto &e : tw_cache) e.valid = false;
  cf_cur = nullptr;
}

void Context::synchronize() {
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(stream));
  CK(cudaStreamSynchronize(d2h));
  if (err_pending) {
    err_pending = false;
    check_device_error(reinterpret_cast<const int *>(reinterpret_cast<char *>(b_small.p) + 3072));
  }
  for (int *w : plan_err) {
    int h = 0;
    CK(cudaMemcpy(&h, w, sizeof(int), cudaMemcpyDeviceToHost));
    if (h == 0) continue;
    CK(cudaMemset(w, 0, sizeof(int)));
    if (h & 2) throw std::runtime_error("internal error: a staged copy into shared memory did not complete");
    throw std::runtime_error("internal error: a visibility record fell outside its tile");
  }
}

void Context::release_buffers() {
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(stream));
  CK(cudaStreamSynchronize(d2h));
  CK(cudaStreamSynchronize(cpy));
  for (auto &sl : slots)
    for (DevBuf *b : {&sl.uvw, &sl.vis, &sl.wgt, &sl.mask, &sl.out, &sl.fovc}) b->release();
  for (auto &kv : fft_plans) cufftDestroy(kv.second);
  fft_plans.clear();
  for (auto *b : all_buffers()) b->release();
  band_dirty = BandDirty{};
  bandd_zero = BandDirty{};
  invalidate_tables();
}

size_t Context::device_bytes() {
  size_t s = 0;
  for (auto *b : all_buffers()) s += b->n;
  return s;
}

cufftHandle Context::fft_plan(int n, int istride, int idist, int ostride, int odist,
                              int batch, bool dbl) {
  auto key = std::make_tuple(n, istride, idist, ostride, odist, batch, int(dbl));
  auto it = fft_plans.find(key);
  if (it != fft_plans.end()) return it->second;
  cufftHandle h;
  CF(cufftCreate(&h));
  CF(cufftSetAutoAllocation(h, 0));
  size_t work = 0;
  // the 64-bit interface only where an element index can pass 2^31 (a large
  // band grid)
  const long long last_in = (long long)(batch - 1) * idist + (long long)(n - 1) * istride;
  const long long last_out = (long long)(batch - 1) * odist + (long long)(n - 1) * ostride;
  if (std::max(last_in, last_out) < (1LL << 31) - 1) {
    int nn = n, inembed = n, onembed = n;
    CF(cufftMakePlanMany(h, 1, &nn, &inembed, istride, idist, &onembed, ostride, odist,
                         dbl ? CUFFT_Z2Z : CUFFT_C2C, batch, &work));
  } else {
    long long nn = n, inembed = n, onembed = n;
    CF(cufftMakePlanMany64(h, 1, &nn, &inembed, istride, idist, &onembed, ostride, odist,
                           dbl ? CUFFT_Z2Z : CUFFT_C2C, batch, &work));
  }
  fft_work_need = std::max(fft_work_need, work);
  fft_plans[key] = h;
  return h;
}

void Context::fft_exec(cufftHandle h, void *in, void *out, int dir, bool dbl) {
  void *work = b_fftwork.ensure(std::max<size_t>(fft_work_need, 256));
  CF(cufftSetStream(h, stream));
  CF(cufftSetWorkArea(h, work));
  if (dbl)
    CF(cufftExecZ2Z(h, reinterpret_cast<cufftDoubleComplex *>(in),
                    reinterpret_cast<cufftDoubleComplex *>(out), dir));
  else
    CF(cufftExecC2C(h, reinterpret_cast<cufftComplex *>(in),
                    reinterpret_cast<cufftComplex *>(out), dir));
}

// ------------------------------------------------------------ staging

// Returns a device pointer holding `bytes` of p: p itself if it is device
// memory, else a copy in buf (asynchronous on the context stream).
const void *Context::stage_in(const void *p, size_t bytes, DevBuf &buf, cudaStream_t st) {
  if (!p) return nullptr;
  if (is_device_pointer(p)) return p;
  void *d = buf.ensure(bytes);
  CK(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, st ? st : stream));
  return d;
}

void Context::validate(const wsg_args &a) {
  require(a.uvw && a.freq, "uvw and freq are required");
  require(a.nrows < (size_t(1) << 32), "too many rows in the MS");
  require(a.nchan < (size_t(1) << 16), "too many channels in the MS");
  require(a.nrows * a.nchan < (size_t(1) << 31), "at most 2^31-1 visibilities per call");
  require(a.npix_x % 2 == 0, "nx_dirty must be even");
  require(a.npix_y % 2 == 0, "ny_dirty must be even");
  require(a.epsilon > 0, "epsilon must be positive");
  require(a.pixsize_x > 0, "pixsize_x must be positive");
  require(a.pixsize_y > 0, "pixsize_y must be positive");
  require(a.precision == WSG_PREC_MIXED || a.precision == WSG_PREC_FP64, "bad precision");
  require(a.vis_type == WSG_C64 || a.vis_type == WSG_C128, "bad vis_type");
  require(a.dirty_type == WSG_F32 || a.dirty_type == WSG_F64, "bad dirty_type");
  require(a.sigma_min > 1.0 && a.sigma_max >= a.sigma_min, "bad sigma range");
}

// Scans the data, chooses the grid, sorts and builds records.  Returns false
// if no visibility is active.
template <typename R>
bool Context::prepare(const wsg_args &a, const Staged &s, bool gridding, void *vis_out_dev,
                      GridPlan &gp) {
  const size_t nvis_tot = a.nrows * a.nchan;
  mark("enter");
  // freq checks (Baselines ctor, wgridder.h:300-309) and f/c
  std::vector<double> freq(a.nchan), fovc(a.nchan);
  if (is_device_pointer(a.freq))
    CK(cudaMemcpy(freq.data(), a.freq, a.nchan * sizeof(double), cudaMemcpyDeviceToHost));
  else
    std::memcpy(freq.data(), a.freq, a.nchan * sizeof(double));
  for (size_t i = 0; i < a.nchan; ++i) {
    require(freq[i] > 0, "negative channel frequency encountered");
    if (i > 0) require(freq[i] >= freq[i - 1], "channel frequencies must be sorted in ascending order");
    fovc[i] = freq[i] / kSpeedOfLight;
  }
  // the scan runs on scan_st when the raw operators staged every input it
  // reads on the copy stream: its read-back then waits for this call's
  // copies only, not for earlier calls' kernels on the main stream
  cudaStream_t sst = scan_st ? scan_st : stream;
  DevBuf &fbuf = fovc_buf ? *fovc_buf : b_fovc;
  double *d_fovc = reinterpret_cast<double *>(fbuf.ensure(a.nchan * sizeof(double)));
  const size_t small_bytes = sizeof(ScanOut) + a.nchan * sizeof(double);
  if (h_small_cap < small_bytes) {
    if (h_small) CK(cudaFreeHost(h_small));
    h_small = nullptr;
    h_small_cap = 0;
    CK(cudaHostAlloc(&h_small, small_bytes, cudaHostAllocDefault));
    h_small_cap = small_bytes;
  }
  unsigned char *hsm = reinterpret_cast<unsigned char *>(h_small);
  std::memcpy(hsm + sizeof(ScanOut), fovc.data(), a.nchan * sizeof(double));
  CK(cudaMemcpyAsync(d_fovc, hsm + sizeof(ScanOut), a.nchan * sizeof(double),
                     cudaMemcpyHostToDevice, sst));
  Staged st = s;
  st.fovc = d_fovc;

  // scan
  ScanOut h0{};
  h0.wmin_bits = 0x7ff0000000000000ull;
  ScanOut *d_scan = reinterpret_cast<ScanOut *>(b_small.ensure(4096));
  std::memcpy(hsm, &h0, sizeof h0);
  CK(cudaMemcpyAsync(d_scan, hsm, sizeof(h0), cudaMemcpyHostToDevice, sst));
  // (off the main stream the caller zeroes the whole output itself)
  void *zero_out = scan_st ? nullptr : vis_out_dev;
  // the sort keys of the expected grid come out of the same pass: the fixed
  // grid of a stream, else the previous call's, checked after planning
  const bool have_spec = gp.fixed || spec_geom.size() == sizeof(DevGeom);
  DevGeom spec;
  if (gp.fixed)
    spec = make_geom(gp);
  else if (have_spec)
    std::memcpy(&spec, spec_geom.data(), sizeof spec);
  // keys are 4 or 8 bytes (the expected grid's width; sized for the wider)
  void *ka = b_keys_a.ensure(nvis_tot * 8);
  uint32_t *va = reinterpret_cast<uint32_t *>(b_vals_a.ensure(nvis_tot * 4));
  // off the main stream, the scan must not overwrite the keys and indices
  // that the previous call's sort and records may still be reading there
  if (sst != stream) CK(cudaStreamWaitEvent(sst, ev_keys, 0));
  with_types(a, [&](auto *tw, auto *tv) {
    using TW = std::remove_pointer_t<decltype(tw)>;
    using TV = std::remove_pointer_t<decltype(tv)>;
    if (have_spec) {
      const int nb = std::min(launch_blocks(a.nrows, 256), num_sms * 8);
      auto go = [&](auto *kp) {
        using K = std::remove_pointer_t<decltype(kp)>;
        k_scan_keys<TV, TW, K><<<nb, 256, 0, sst>>>(
            a.nrows, int(a.nchan), st.uvw, st.fovc, reinterpret_cast<const TV *>(st.vis),
            reinterpret_cast<const TW *>(st.wgt), st.mask, gridding ? 1 : 0,
            a.negate_v ? -1.0 : 1.0, d_scan, reinterpret_cast<TV *>(zero_out), spec, kp, va,
            st.iw);
      };
      if (spec.wide)
        go(reinterpret_cast<unsigned long long *>(ka));
      else
        go(reinterpret_cast<uint32_t *>(ka));
      cuda_check(cudaGetLastError(), "k_scan_keys launch");
      g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    } else {
      launch_scan<TW, TV>(*this, a, st, gridding, reinterpret_cast<TV *>(zero_out), d_scan, sst);
    }
  });
  k_scan_readback<<<1, 32, 0, sst>>>(d_scan, reinterpret_cast<ScanOut *>(h_scan_dev));
  cuda_check(cudaGetLastError(), "k_scan_readback launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  mark("scan-submit");
  CK(cudaStreamSynchronize(sst));
  ScanOut hs;
  std::memcpy(&hs, h_scan, sizeof hs);
  if (sst != stream) {  // keys and records read the uploaded f/c
    CK(cudaEventRecord(ev_scan, sst));
    CK(cudaStreamWaitEvent(stream, ev_scan, 0));
  }
  mark("scan-sync");
  gp.nvis = hs.nvis;
  if (gp.nvis == 0) return false;
  auto bits2d = [](unsigned long long b) {
    double d;
    std::memcpy(&d, &b, 8);
    return d;
  };
  if (gp.fixed) {
    const double wmin = bits2d(hs.wmin_bits), wmax = bits2d(hs.wmax_bits);
    const double umax = bits2d(hs.umax_bits), vmax = bits2d(hs.vmax_bits);
    auto within = [](double x, double lim) { return x <= lim * (1.0 + 1e-12) + 1e-9; };
    require(wmin >= gp.wmin_d * (1.0 - 1e-12) - 1e-9 && within(wmax, gp.wmax_d),
            "a chunk's |w| range lies outside the extent declared for the stream");
    require(within(umax, gp.umax) && within(vmax, gp.vmax),
            "a chunk's |u| or |v| exceeds the extent declared for the stream");
  } else {
    gp.wmin_d = bits2d(hs.wmin_bits);
    gp.wmax_d = bits2d(hs.wmax_bits);
    gp.umax = bits2d(hs.umax_bits);
    gp.vmax = bits2d(hs.vmax_bits);
    int tile = default_tile(sizeof(R) == 4);
    if (tune_W) {  // a candidate being timed by the autotuner
      gp.force_W = tune_W;
      gp.force_sigma = tune_sigma;
      if (tune_tile) tile = tune_tile;
    } else if (!gp.force_W) {
      TuneChoice tc;
      if (tuned_choice(a, gp.nvis, tc)) {
        gp.force_W = tc.W;
        gp.force_sigma = tc.sigma;
        tile = tc.tile;
      }
    }
    // the same data statistics and arguments give the same plan: repeated
    // calls reuse the previous one of their direction
    const std::array<double, 22> key{
        double(gp.nx), double(gp.ny), gp.px, gp.py, gp.eps, double(gp.do_w), double(gp.fp32),
        double(gp.negate_v), double(gp.divide_by_n), gp.lshift, gp.mshift, double(gp.nvis),
        gp.wmin_d, gp.wmax_d, gp.umax, gp.vmax, double(gp.force_W), gp.force_sigma,
        a.sigma_min, a.sigma_max, double(tile), double(gp.gridding)};
    GridMemo &gm = grid_memo[gridding ? 1 : 0];
    if (gm.valid && gm.key == key) {
      gp = gm.plan;
    } else {
      choose_grid(gp, a.sigma_min, a.sigma_max, tile);
      gm.key = key;
      gm.plan = gp;
      gm.valid = true;
    }
  }
  DevGeom g = make_geom(gp);
  const bool keyed = have_spec && std::memcmp(&g, &spec, sizeof g) == 0;
  spec_geom.assign(reinterpret_cast<const unsigned char *>(&g),
                   reinterpret_cast<const unsigned char *>(&g) + sizeof g);
  mark("choose_grid");

  // keys (unless the scan wrote them for this grid) + sort
  void *kb = b_keys_b.ensure(nvis_tot * 8);
  uint32_t *vb = reinterpret_cast<uint32_t *>(b_vals_b.ensure(nvis_tot * 4));
  const int end_bit = gp.key_bits + 1;
  auto keys_and_sort = [&](auto *kap, auto *kbp) {
    using K = std::remove_pointer_t<decltype(kap)>;
    if (!keyed) {
      with_types(a, [&](auto *tw, auto *tv) {
        using TW = std::remove_pointer_t<decltype(tw)>;
        using TV = std::remove_pointer_t<decltype(tv)>;
        launch_keys<TW, TV, K>(*this, a, st, gridding, g, kap, va);
      });
    }
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kap, kbp, va, vb, int(nvis_tot), 0, end_bit,
                                       stream));
    void *dtmp = b_cub.ensure(tmp);
    CK(cub::DeviceRadixSort::SortPairs(dtmp, tmp, kap, kbp, va, vb, int(nvis_tot), 0, end_bit,
                                       stream));
  };
  if (gp.wide_keys)
    keys_and_sort(reinterpret_cast<unsigned long long *>(ka),
                  reinterpret_cast<unsigned long long *>(kb));
  else
    keys_and_sort(reinterpret_cast<uint32_t *>(ka), reinterpret_cast<uint32_t *>(kb));

  // records
  void *rec = b_rec.ensure(gp.nvis * sizeof(typename RecOf<R>::type));
  with_types(a, [&](auto *tw, auto *tv) {
    using TW = std::remove_pointer_t<decltype(tw)>;
    using TV = std::remove_pointer_t<decltype(tv)>;
    // (the unsorted indices va are free after the sort: they hold the ranks)
    launch_records<R, TW, TV>(gp.nvis, a, st, gridding, g, vb, va, rec, stream);
  });

  // chunk boundaries
  int *chunks = reinterpret_cast<int *>(b_chunks.ensure((gp.nvis + 1) * sizeof(int)));
  int *d_nch = reinterpret_cast<int *>(reinterpret_cast<char *>(b_small.p) + 1024);
  auto select = [&](auto *kbp) {
    using K = std::remove_pointer_t<decltype(kbp)>;
    ChunkStartPred<K> pred{kbp, 2 * gp.lbits, chunk_size};
    thrust::counting_iterator<int> it(0);
    size_t tmp = 0;
    CK(cub::DeviceSelect::If(nullptr, tmp, it, chunks, d_nch, int(gp.nvis), pred, stream));
    void *dtmp = b_cub.ensure(std::max(tmp, b_cub.n));
    CK(cub::DeviceSelect::If(dtmp, tmp, it, chunks, d_nch, int(gp.nvis), pred, stream));
  };
  if (gp.wide_keys)
    select(reinterpret_cast<unsigned long long *>(kb));
  else
    select(reinterpret_cast<uint32_t *>(kb));
  CK(cudaEventRecord(ev_keys, stream));
  mark("sort+records-submit");
  return true;
}

// Grid-correction tables for the chosen kernel: 1/Phi as a Chebyshev series
// in v^2 (evaluated per pixel on the device for the w term) and the 1-D u/v
// correction arrays; cached per geometry (two entries), the chosen entry's
// device copy left in cf_cur.
ChebCorr Context::upload_corrections(const GridPlan &g) {
  double vmax = 0.5 * std::max(double(g.nx) / g.nu, double(g.ny) / g.nv) * 1.0000001;
  if (g.do_w) {
    vmax = std::max(vmax, 0.5 / g.ofactor * 1.0000001);
    // pixels beyond the horizon use (sqrt(r^2-1)-1)*dw (wgridder.h:1376-1377)
    double xmin = g.lshift - 0.5 * g.nx * g.px, xmax = xmin + (g.nx - 1) * g.px;
    double ymin = g.mshift - 0.5 * g.ny * g.py, ymax = ymin + (g.ny - 1) * g.py;
    for (double xc : {xmin, xmax})
      for (double yc : {ymin, ymax}) {
        double r2 = xc * xc + yc * yc;
        if (r2 > 1.0) vmax = std::max(vmax, std::fabs((std::sqrt(r2 - 1.0) - 1.0) * g.dw));
      }
    vmax = std::min(vmax, 1.0);
  }
  auto key = std::make_tuple(g.kernel.W, g.kernel.beta, g.kernel.e0, g.nx, g.ny, g.nu, g.nv, vmax);
  for (auto &e : corr_cache)
    if (e.valid && e.key == key) {
      e.used = ++cache_tick;
      cf_cur = reinterpret_cast<const double *>(e.buf.p);
      return e.cc;
    }
  CorrEntry &e = corr_cache[0].used <= corr_cache[1].used ? corr_cache[0] : corr_cache[1];
  KernelTransform tr(g.kernel);
  ChebCorr cc = fit_cheb_corr(tr, vmax);
  std::vector<double> cf(g.nx / 2 + 1 + g.ny / 2 + 1);
  for (size_t i = 0; i <= g.nx / 2; ++i) cf[i] = cc(double(i) / g.nu);
  for (size_t i = 0; i <= g.ny / 2; ++i) cf[g.nx / 2 + 1 + i] = cc(double(i) / g.nv);
  double *d = reinterpret_cast<double *>(e.buf.ensure(cf.size() * sizeof(double)));
  // stream-ordered: kernels of earlier (pipelined) calls may still read it
  CK(cudaMemcpyAsync(d, cf.data(), cf.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
  cheb_err = cc.max_rel_err;
  e.key = key;
  e.cc = cc;
  e.valid = true;
  e.used = ++cache_tick;
  cf_cur = d;
  return cc;
}

// FP64-computed twiddle tables: the per-stage tables of the length-M
// shared-memory FFT (M entries) and exp(+2 pi i t / nu) for the twist (nu
// entries), stored in the arithmetic type, cached per (M, nu, type).
// Twiddle tables of the pruned u transform (nu = K M), as interleaved
// (re, im) doubles: the per-stage FFT tables exp(+2 pi i r k / (NS R)),
// [r-1][k] in stage order (M entries); the twist bases exp(+2 pi i t k2 / nu),
// [k2][t] for t < M/16; and the per-slot factors exp(+2 pi i (M/16 q - neg M)
// k2 / nu), [k2][q][neg].  Angles are reduced exactly in integers before the
// FP64 sin/cos.
size_t col_table_entries(size_t M, size_t K) { return M + K * (M / 16) + 32 * K; }

std::vector<double> col_twiddle_table(size_t M, size_t nu, size_t K) {
  const size_t TPF = M / 16;
  std::vector<double> h(2 * col_table_entries(M, K), 0.0);
  auto put = [&](size_t idx, long long num, long long den) {
    long long r = num % den;
    if (r < 0) r += den;
    double f = double(r) / double(den);
    if (f > 0.5) f -= 1.0;
    h[2 * idx] = std::cos(2.0 * M_PI * f);
    h[2 * idx + 1] = std::sin(2.0 * M_PI * f);
  };
  size_t off = 0;
  for (size_t NS = 1; NS < M;) {
    const size_t R = (M / NS >= 16) ? 16 : M / NS;
    if (NS > 1) {
      for (size_t r = 1; r < R; ++r)
        for (size_t k = 0; k < NS; ++k) put(off + (r - 1) * NS + k, (long long)(r * k), (long long)(NS * R));
      off += (R - 1) * NS;
    }
    NS *= R;
  }
  for (size_t k2 = 0; k2 < K; ++k2)
    for (size_t t = 0; t < TPF; ++t) put(M + k2 * TPF + t, (long long)(t * k2), (long long)nu);
  for (size_t k2 = 0; k2 < K; ++k2)
    for (size_t q = 0; q < 16; ++q)
      for (int neg = 0; neg < 2; ++neg)
        put(M + K * TPF + (k2 * 16 + q) * 2 + neg,
            ((long long)(TPF * q) - (neg ? (long long)M : 0)) * (long long)k2, (long long)nu);
  return h;
}

const void *Context::upload_twiddles(const GridPlan &g, bool dbl) {
  const size_t M = size_t(1) << g.logM;
  auto key = std::make_tuple(M, g.nu, int(dbl));
  const size_t cs = dbl ? 16 : 8;
  for (auto &e : tw_cache)
    if (e.valid && e.key == key) {
      e.used = ++cache_tick;
      return e.buf.p;
    }
  TwEntry &e = tw_cache[0].used <= tw_cache[1].used ? tw_cache[0] : tw_cache[1];
  {
    const std::vector<double> h = col_twiddle_table(M, g.nu, size_t(g.K));
    void *d = e.buf.ensure(h.size() / 2 * cs);
    // stream-ordered (pageable sources are staged before the call returns)
    if (dbl) {
      CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    } else {
      std::vector<float> hf(h.begin(), h.end());
      CK(cudaMemcpyAsync(d, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
    }
    e.key = key;
    e.valid = true;
    e.used = ++cache_tick;
  }
  return e.buf.p;
}

// Planes resident per pass: as many as fit in 55% of the device memory and
// in what is free (plus what this context already holds).  cudaMemGetInfo is
// a slow driver query (milliseconds, and tens of them when other processes
// query the GPU), so a repeated plan whose buffers are still held reuses the
// previous answer -- kept per direction, for alternating ms2dirty / dirty2ms.
// Zeroes the spread's band grid before a pass: whole when its layout or
// address changed (or nothing is known), else only the v columns the last
// spread into it can have written.
void Context::clear_band(void *band, size_t rows, size_t nv, size_t cs) {
  const BandDirty d = band_dirty;
  band_dirty = BandDirty{};  // unknown until the caller records the new spread
  if (d.p == band && d.rows == rows && d.nv == nv && d.cs == cs && d.Lv >= 0) {
    const size_t L = size_t(d.Lv);
    CK(cudaMemset2DAsync(band, nv * cs, 0, (L + 1) * cs, rows, stream));
    CK(cudaMemset2DAsync(static_cast<char *>(band) + (nv - L) * cs, nv * cs, 0, L * cs, rows,
                         stream));
  } else {
    CK(cudaMemsetAsync(band, 0, rows * nv * cs, stream));
  }
}

size_t Context::choose_planes(const GridPlan &g, bool gridding) {
  const size_t per = plan_bytes(g, 1, gridding);
  const size_t held = b_band.n + b_bandf.n + b_bandd.n + b_H.n;
  const auto key = std::make_tuple(per, g.nplanes, int(gridding));
  PlanesMemo &pm = planes_memo[gridding ? 1 : 0];
  if (!(pm.valid && key == pm.key && held >= pm.P * per)) {
    size_t total = 0, freeb = 0;
    CK(cudaMemGetInfo(&freeb, &total));
    double budget = 0.55 * double(total);
    size_t avail = size_t(std::min<double>(budget, double(freeb + held) - 2e9));
    pm.P = std::max<size_t>(1, std::min<size_t>(g.nplanes, per ? avail / per : g.nplanes));
    pm.key = key;
    pm.valid = true;
  }
  size_t P = pm.P;
  const int lim = env_int("WSG_MAX_PLANES", 0);  // a test and debugging limit
  if (lim > 0) P = std::min<size_t>(P, size_t(lim));
  return std::min(P, g.nplanes);
}

// The 2-D transform of one plane in place in the grid layout [nu][P][nv]
// (row stride P nv), the whole-grid layout's transform (GridPlan::ucufft).
// 64-bit sizes: the rows of a large grid span more than 2^31 entries.
cufftHandle make_grid_fft_plan(size_t nu, size_t nv, size_t P, bool dbl, size_t &work) {
  cufftHandle h;
  CF(cufftCreate(&h));
  CF(cufftSetAutoAllocation(h, 0));
  long long n[2] = {(long long)nu, (long long)nv};
  long long emb[2] = {(long long)nu, (long long)(P * nv)};
  work = 0;
  CF(cufftMakePlanMany64(h, 2, n, emb, 1, (long long)nv, emb, 1, (long long)nv,
                         dbl ? CUFFT_Z2Z : CUFFT_C2C, 1, &work));
  return h;
}

// Runs the plane transform of make_grid_fft_plan on npl consecutive planes
// starting at grid (plane p at p nv entries).
void exec_grid_fft(cufftHandle h, void *grid, size_t nv, size_t npl, int dir, bool dbl,
                   cudaStream_t st, void *work) {
  const size_t cs = dbl ? 16 : 8;
  CF(cufftSetStream(h, st));
  CF(cufftSetWorkArea(h, work));
  for (size_t p = 0; p < npl; ++p) {
    void *g = static_cast<char *>(grid) + p * nv * cs;
    if (dbl)
      CF(cufftExecZ2Z(h, reinterpret_cast<cufftDoubleComplex *>(g),
                      reinterpret_cast<cufftDoubleComplex *>(g), dir));
    else
      CF(cufftExecC2C(h, reinterpret_cast<cufftComplex *>(g), reinterpret_cast<cufftComplex *>(g),
                      dir));
  }
}

// The context's cached plane transform for a grid layout of P planes.
void Context::grid_fft(void *grid, const GridPlan &g, size_t P, size_t npl, int dir, bool dbl) {
  auto key = std::make_tuple(-int(g.nu), int(g.nv), int(P), 0, 0, 1, int(dbl));
  auto it = fft_plans.find(key);
  cufftHandle h;
  if (it != fft_plans.end()) {
    h = it->second;
  } else {
    size_t work = 0;
    h = make_grid_fft_plan(g.nu, g.nv, P, dbl, work);
    fft_work_need = std::max(fft_work_need, work);
    fft_plans[key] = h;
  }
  void *work = b_fftwork.ensure(std::max<size_t>(fft_work_need, 256));
  exec_grid_fft(h, grid, g.nv, npl, dir, dbl, stream, work);
}

template <typename R>
bool Context::grid_core(const wsg_args &a, const Staged &s, double *img, bool accumulate,
                        void *direct_out, size_t ld) {
  const bool dbl = sizeof(R) == 8;
  GridPlan gp;
  gp.nx = a.npix_x;
  gp.ny = a.npix_y;
  gp.px = a.pixsize_x;
  gp.py = a.pixsize_y;
  gp.eps = a.epsilon;
  gp.do_w = a.do_wgridding != 0;
  gp.fp32 = !dbl;
  gp.gridding = true;
  gp.negate_v = a.negate_v != 0;
  gp.divide_by_n = a.divide_by_n != 0;
  gp.lshift = a.center_x;
  gp.mshift = a.negate_v ? -a.center_y : a.center_y;
  if (ld == 0) ld = a.npix_y;
  // zeroes the FP64 image (a strided block when it is a facet)
  auto clear_img = [&]() {
    CK(cudaMemset2DAsync(img, ld * sizeof(double), 0, a.npix_y * sizeof(double), a.npix_x, stream));
  };

  CK(cudaEventRecord(ev[0], stream));
  if (!prepare<R>(a, s, true, nullptr, gp)) {
    if (!accumulate) clear_img();
    record_stats(gp, true, 0);
    return false;
  }
  CK(cudaEventRecord(ev[1], stream));
  ChebCorr cc = upload_corrections(gp);
  DevGeom g = make_geom(gp);
  DevKernel<R> kc = make_kernel<R>(gp.poly);
  mark("corrections");
  const size_t P = choose_planes(gp, true);
  mark("choose_planes");
  // one pass over all planes and nothing to accumulate: the w-screen sum
  // goes straight to the caller's image, else through the FP64 accumulator
  const bool direct = direct_out && !accumulate && P >= gp.nplanes && ld == a.npix_y;
  const int out_mode = direct ? (a.dirty_type == WSG_F64 ? 2 : 1) : 0;
  if (!accumulate && !direct) clear_img();
  const size_t cs = 2 * sizeof(R);
  const size_t nv = gp.nv;
  // the spread writes `band`; the v transform goes out of place to `bandf`,
  // so `band` stays zero outside the columns the spread wrote
  const size_t rowsP = gp.band_rows * P;
  char *band = reinterpret_cast<char *>(b_band.ensure(rowsP * nv * cs));
  // (the whole-grid layout transforms in place and screens the grid itself)
  char *bandf = gp.ucufft ? nullptr : reinterpret_cast<char *>(b_bandf.ensure(rowsP * nv * cs));
  char *H = gp.ucufft ? nullptr : reinterpret_cast<char *>(b_H.ensure(P * gp.ny * gp.hrow() * cs));
  ColArgs ca{};
  if (!gp.ucufft) ca = make_col(gp, P, upload_twiddles(gp, dbl), bandf, H);
  const long Lv = band_v_halfwidth(gp);
  const TileLayout tl = make_layout(gp.T, gp.kernel.W);
  const size_t smem = grid_smem_bytes<R>(tl, gp.kernel.W, true);
  int *counter = reinterpret_cast<int *>(reinterpret_cast<char *>(b_small.p) + 2048);
  int *d_nch = reinterpret_cast<int *>(reinterpret_cast<char *>(b_small.p) + 1024);
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(b_small.p) + 3072);
  if (!err_pending) CK(cudaMemsetAsync(d_err, 0, sizeof(int), stream));  // sticky while pipelined
  GridArgs ga{};
  ga.err = d_err;
  ga.rec = b_rec.p;
  ga.chunk_start = reinterpret_cast<const int *>(b_chunks.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(gp.nvis);
  ga.grid = band;
  ga.P = int(P);
  ga.tl = tl;
  ga.sb = grid_sb<R>();

  const int dir = CUFFT_INVERSE;
  float t_grid = 0, t_fft = 0, t_screen = 0;
  for (size_t pb0 = 0; pb0 < gp.nplanes; pb0 += P) {
    const size_t npl = std::min(P, gp.nplanes - pb0);
    CK(cudaEventRecord(ev[2], stream));
    clear_band(band, rowsP, nv, cs);
    CK(cudaMemsetAsync(counter, 0, sizeof(int), stream));
    ga.pb0 = int(pb0);
    ga.pb1 = int(pb0 + npl);
    grid_dispatch<R>(gp.kernel.W, true, num_sms, smem, stream, ga, g, kc);
    band_dirty = BandDirty{band, rowsP, nv, cs, Lv};
    CK(cudaEventRecord(ev[3], stream));
    if (gp.ucufft) {
      // the whole grid: each plane's 2-D transform in place
      grid_fft(band, gp, P, npl, dir, dbl);
      band_dirty = BandDirty{};  // every entry of `band` written
    } else {
      // transform along v: every (band row, plane) is a contiguous row of nv
      cufftHandle h = fft_plan(int(nv), 1, int(nv), 1, int(nv), int(rowsP), dbl);
      fft_exec(h, band, bandf, dir, dbl);
      // pruned transform along u: band rows of the image columns -> image rows
      col_run<R>(gp.logM, true, ca, int(npl), stream, d_err);
    }
    CK(cudaEventRecord(ev[4], stream));
    ScreenArgs sa = make_screen(gp, cf_cur, cc, P);
    sa.pb0 = int(pb0);
    sa.npl = int(npl);
    sa.ld = ld;
    const dim3 sg = screen_grid(gp);
    if (gp.ucufft)
      launch_screen_add_grid<R>(sg, stream, sa, band, img, direct_out, out_mode);
    else
      launch_screen_add<R>(sg, stream, sa, H, img, direct_out, out_mode);
    CK(cudaEventRecord(ev[5], stream));
    float t = 0;
    if (!async_mode) CK(cudaEventSynchronize(ev[5]));
    if (!async_mode) {
      CK(cudaEventElapsedTime(&t, ev[2], ev[3]));
      t_grid += t;
      CK(cudaEventElapsedTime(&t, ev[3], ev[4]));
      t_fft += t;
      CK(cudaEventElapsedTime(&t, ev[4], ev[5]));
      t_screen += t;
    }
  }
  float t_prep = 0;
  if (async_mode) {
    err_pending = true;
  } else {
    check_device_error(d_err);
    CK(cudaEventElapsedTime(&t_prep, ev[0], ev[1]));
  }
  record_stats(gp, true, P);
  stats.ms_prep = t_prep;
  stats.ms_grid = t_grid;
  stats.ms_fft = t_fft;
  stats.ms_screen = t_screen;
  mark("passes-done");
  if (verbosity > 0) print_report(gp, true, P);
  print_marks("ms2dirty");
  return direct;
}

template <typename R>
void Context::degrid_core(const wsg_args &a, const Staged &s, const double *img, void *vis_out,
                          const void *direct_in, size_t ld, bool vis_acc) {
  const bool dbl = sizeof(R) == 8;
  GridPlan gp;
  gp.nx = a.npix_x;
  gp.ny = a.npix_y;
  gp.px = a.pixsize_x;
  gp.py = a.pixsize_y;
  gp.eps = a.epsilon;
  gp.do_w = a.do_wgridding != 0;
  gp.fp32 = !dbl;
  gp.gridding = false;
  gp.negate_v = a.negate_v != 0;
  gp.divide_by_n = a.divide_by_n != 0;
  gp.lshift = a.center_x;
  gp.mshift = a.negate_v ? -a.center_y : a.center_y;

  if (ld == 0) ld = a.npix_y;

  CK(cudaEventRecord(ev[0], stream));
  if (!prepare<R>(a, s, false, vis_acc ? nullptr : vis_out, gp)) {
    record_stats(gp, false, 0);
    return;
  }
  CK(cudaEventRecord(ev[1], stream));
  ChebCorr cc = upload_corrections(gp);
  DevGeom g = make_geom(gp);
  DevKernel<R> kc = make_kernel<R>(gp.poly);
  mark("corrections");
  const size_t P = choose_planes(gp, false);
  mark("choose_planes");
  const size_t cs = 2 * sizeof(R);
  const size_t nv = gp.nv;
  // the transposed u transform fills the image columns of `bandi`, whose
  // other columns stay zero from call to call; the v transform goes out of
  // place to `band`, which the interpolation reads
  const size_t rowsP = gp.band_rows * P;
  // (the whole-grid layout: the screen writes the grid `band` itself, which
  // is transformed in place)
  char *bandi = gp.ucufft ? nullptr : reinterpret_cast<char *>(b_bandd.ensure(rowsP * nv * cs));
  char *band = reinterpret_cast<char *>(b_bandf.ensure(rowsP * nv * cs));
  char *H = gp.ucufft ? nullptr : reinterpret_cast<char *>(b_H.ensure(P * gp.ny * gp.hrow() * cs));
  ColArgs ca{};
  if (!gp.ucufft) ca = make_col(gp, P, upload_twiddles(gp, dbl), bandi, H);
  const TileLayout tl = make_layout(gp.T, gp.kernel.W);
  const size_t smem = grid_smem_bytes<R>(tl, gp.kernel.W, false);
  int *counter = reinterpret_cast<int *>(reinterpret_cast<char *>(b_small.p) + 2048);
  int *d_nch = reinterpret_cast<int *>(reinterpret_cast<char *>(b_small.p) + 1024);
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(b_small.p) + 3072);
  if (!err_pending) CK(cudaMemsetAsync(d_err, 0, sizeof(int), stream));  // sticky while pipelined
  GridArgs ga{};
  ga.err = d_err;
  ga.rec = b_rec.p;
  ga.chunk_start = reinterpret_cast<const int *>(b_chunks.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(gp.nvis);
  ga.grid = band;
  ga.P = int(P);
  ga.tl = tl;
  ga.sb = grid_sb<R>();
  ga.vis_out = vis_out;
  ga.vis_double = a.vis_type == WSG_C128;
  ga.vis_accumulate = vis_acc ? 1 : 0;
  const bool multi = P < gp.nplanes;
  const bool need_acc = multi || grid_needs_acc<R>(gp.kernel.W);
  ga.acc = need_acc ? b_acc.ensure(gp.nvis * cs) : nullptr;
  if (need_acc) CK(cudaMemsetAsync(ga.acc, 0, gp.nvis * cs, stream));

  const int dir = CUFFT_FORWARD;
  float t_grid = 0, t_fft = 0, t_screen = 0;
  for (size_t pb0 = 0; pb0 < gp.nplanes; pb0 += P) {
    const size_t npl = std::min(P, gp.nplanes - pb0);
    CK(cudaEventRecord(ev[2], stream));
    ScreenArgs sa = make_screen(gp, cf_cur, cc, P);
    sa.pb0 = int(pb0);
    sa.npl = int(npl);
    sa.ld = ld;
    const dim3 sg = screen_grid(gp);
    // the caller's image itself (FP32 or FP64) when given, else the FP64 copy
    const void *src = direct_in ? direct_in : static_cast<const void *>(img);
    const int src_f32 = (direct_in && a.dirty_type == WSG_F32) ? 1 : 0;
    if (gp.ucufft) {
      // zero outside the image's rows and columns, which the screen leaves
      CK(cudaMemsetAsync(band, 0, rowsP * nv * cs, stream));
      launch_screen_put_grid<R>(sg, stream, sa, src, src_f32, band);
    } else {
      launch_screen_put<R>(sg, stream, sa, src, src_f32, H);
    }
    CK(cudaEventRecord(ev[3], stream));
    if (gp.ucufft) {
      grid_fft(band, gp, P, npl, dir, dbl);  // each plane's 2-D transform in place
    } else {
      // pruned transform along u (transposed): image rows -> band rows of the
      // image columns; the other columns of the band grid stay zero
      const BandDirty zl{bandi, rowsP, nv, cs, long(gp.ny)};
      if (!(bandd_zero.p == zl.p && bandd_zero.rows == zl.rows && bandd_zero.nv == zl.nv &&
            bandd_zero.cs == zl.cs && bandd_zero.Lv == zl.Lv)) {
        bandd_zero = BandDirty{};
        clear_outside_columns(bandi, rowsP, nv, gp.ny, cs, stream);
        bandd_zero = zl;
      }
      col_run<R>(gp.logM, false, ca, int(npl), stream, d_err);
      // transform along v
      cufftHandle h = fft_plan(int(nv), 1, int(nv), 1, int(nv), int(rowsP), dbl);
      fft_exec(h, bandi, band, dir, dbl);
    }
    CK(cudaEventRecord(ev[4], stream));
    CK(cudaMemsetAsync(counter, 0, sizeof(int), stream));
    ga.pb0 = int(pb0);
    ga.pb1 = int(pb0 + npl);
    ga.first_pass = pb0 == 0;
    ga.last_pass = pb0 + npl >= gp.nplanes;
    grid_dispatch<R>(gp.kernel.W, false, num_sms, smem, stream, ga, g, kc);
    CK(cudaEventRecord(ev[5], stream));
    float t = 0;
    if (!async_mode) CK(cudaEventSynchronize(ev[5]));
    if (!async_mode) {
      CK(cudaEventElapsedTime(&t, ev[2], ev[3]));
      t_screen += t;
      CK(cudaEventElapsedTime(&t, ev[3], ev[4]));
      t_fft += t;
      CK(cudaEventElapsedTime(&t, ev[4], ev[5]));
      t_grid += t;
    }
  }
  if (need_acc) {
    k_finalize<R><<<launch_blocks(gp.nvis, 256), 256, 0, stream>>>(
        int(gp.nvis), b_rec.p, ga.acc, vis_out, ga.vis_double, ga.vis_accumulate);
    cuda_check(cudaGetLastError(), "k_finalize launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  }
  float t_prep = 0;
  if (async_mode) {
    err_pending = true;
  } else {
    check_device_error(d_err);
    CK(cudaEventElapsedTime(&t_prep, ev[0], ev[1]));
  }
  record_stats(gp, false, P);
  stats.ms_prep = t_prep;
  stats.ms_grid = t_grid;
  stats.ms_fft = t_fft;
  stats.ms_screen = t_screen;
  mark("passes-done");
  if (verbosity > 0) print_report(gp, false, P);
  print_marks("dirty2ms");
}

void Context::check_device_error(const int *d_err) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (h & 2) throw std::runtime_error("internal error: a staged copy into shared memory did not complete");
  if (h) throw std::runtime_error("internal error: a visibility record fell outside its tile");
}

void Context::record_stats(const GridPlan &g, bool gridding, size_t P) {
  std::memset(&stats, 0, sizeof(stats));
  stats.nvis = g.nvis;
  stats.nu = g.nu;
  stats.nv = g.nv;
  stats.nplanes = g.nplanes;
  stats.supp = g.kernel.W;
  stats.plane_batch = P;
  stats.band_rows = g.band_rows;
  stats.degree = g.poly.D;
  stats.sigma = g.ofactor;
  stats.beta = g.kernel.beta;
  stats.e0 = g.kernel.e0;
  stats.kernel_err = g.kernel.err;
  stats.wmin = g.wmin_d;
  stats.wmax = g.wmax_d;
  stats.dw = g.dw;
  stats.nshift = g.nshift;
  stats.gridding = gridding;
  stats.precision = g.fp32 ? WSG_PREC_MIXED : WSG_PREC_FP64;
  stats.device_bytes = device_bytes();
  stats.kernel_launches = g_kernel_launches.load();
}

void Context::print_report(const GridPlan &g, bool gridding, size_t P) {
  std::printf("%s:\n  dirty=(%zux%zu), grid=(%zux%zu", gridding ? "Gridding" : "Degridding", g.nx,
              g.ny, g.nu, g.nv);
  if (g.do_w) std::printf("x%zu", g.nplanes);
  std::printf("), supp=%d, eps=%g (kernel %.3g, sigma %.2f)\n", g.kernel.W, g.eps, g.kernel.err,
              g.kernel.sigma);
  std::printf("  nvis=%zu, w=[%g; %g], dw=%g, planes per pass=%zu, u band rows=%zu%s\n", g.nvis,
              g.wmin_d, g.wmax_d, g.dw, P, g.band_rows,
              g.ucufft ? " (whole grid, 2-D library FFT a plane)" : "");
  std::fflush(stdout);
}

// ------------------------------------------------------- public drivers

// While alive, prepare() scans on the copy stream with the slot's f/c
// buffer -- when every input the scan reads was copied into the slot.
struct ScanPlacement {
  Context &cx;
  ScanPlacement(Context &c, Context::Slot &sl, bool staged) : cx(c) {
    if (staged) {
      cx.scan_st = cx.cpy;
      cx.fovc_buf = &sl.fovc;
    }
  }
  ~ScanPlacement() {
    cx.scan_st = nullptr;
    cx.fovc_buf = nullptr;
  }
};

// Ends a raw operator call: the slot is free once the main stream (and the
// device-to-host copy, when there is one) is done; synchronous mode waits.
void Context::finish_call(const wsg_args &a, Slot &sl, cudaStream_t last) {
  CK(cudaEventRecord(sl.free_ev, last));
  stats.kernel_launches = g_kernel_launches.load();
  stats.nrows = a.nrows;
  stats.nchan = a.nchan;
  if (async_mode) return;
  CK(cudaEventRecord(ev[6], last));
  CK(cudaStreamSynchronize(stream));
  CK(cudaStreamSynchronize(d2h));
  float t;
  CK(cudaEventElapsedTime(&t, ev[0], ev[6]));
  stats.ms_total = t;
}

void Context::ms2dirty(const wsg_args &a, const void *vis, void *dirty, int accumulate) {
  validate(a);
  require(vis && dirty, "vis and dirty are required");
  CK(cudaSetDevice(device));
  const size_t nvis = a.nrows * a.nchan;
  const size_t vbytes = nvis * (a.vis_type == WSG_C128 ? 16 : 8);
  const size_t npix = a.npix_x * a.npix_y;
  const size_t dsz = a.dirty_type == WSG_F64 ? 8 : 4;
  const bool ddev = is_device_pointer(dirty);
  // host inputs are copied into this call's slot on the copy stream, which
  // runs ahead of the main stream (device inputs are used in place, in the
  // order of the main stream); the slot is reused once its previous call
  // has finished with it
  Slot &sl = slots[slot_k++ % kSlots];
  CK(cudaEventSynchronize(sl.free_ev));
  Staged s;
  s.uvw = reinterpret_cast<const double *>(stage_in(a.uvw, a.nrows * 3 * sizeof(double), sl.uvw, cpy));
  s.vis = stage_in(vis, vbytes, sl.vis, cpy);
  s.wgt = stage_in(a.wgt, nvis * (a.wgt_type == WSG_F64 ? 8 : 4), sl.wgt, cpy);
  s.mask = reinterpret_cast<const uint8_t *>(stage_in(a.mask, nvis, sl.mask, cpy));
  const void *din = (accumulate && !ddev) ? stage_in(dirty, npix * dsz, sl.out, cpy) : dirty;
  CK(cudaEventRecord(ev_in, cpy));
  CK(cudaStreamWaitEvent(stream, ev_in, 0));
  // (stage_in returns device inputs unchanged: a new pointer means copied)
  // (a tuned call's parts scan masks made on the main stream: no early scan)
  ScanPlacement place(*this, sl, !tuned_call && s.uvw != a.uvw && s.vis != vis &&
                                     (a.wgt == nullptr || s.wgt != a.wgt) &&
                                     (a.mask == nullptr || s.mask != a.mask));
  double *img = reinterpret_cast<double *>(b_img.ensure(npix * sizeof(double)));
  if (accumulate) {
    int nb = launch_blocks(npix, 256);
    if (a.dirty_type == WSG_F64)
      k_load_image<double><<<nb, 256, 0, stream>>>(npix, (const double *)din, img, 0);
    else
      k_load_image<float><<<nb, 256, 0, stream>>>(npix, (const float *)din, img, 0);
    cuda_check(cudaGetLastError(), "k_load_image launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  }
  void *dout = ddev ? dirty : sl.out.ensure(npix * dsz);
  bool direct;
  if (tuned_call)
    direct = (a.precision == WSG_PREC_FP64) ? grid_tuned<double>(a, s, img, accumulate != 0, dout)
                                            : grid_tuned<float>(a, s, img, accumulate != 0, dout);
  else
    direct = (a.precision == WSG_PREC_FP64) ? grid_core<double>(a, s, img, accumulate != 0, dout)
                                            : grid_core<float>(a, s, img, accumulate != 0, dout);
  if (!direct) {  // convert/copy out of the FP64 accumulator
    int nb = launch_blocks(npix, 256);
    if (a.dirty_type == WSG_F64)
      k_store_image<double><<<nb, 256, 0, stream>>>(npix, img, (double *)dout);
    else
      k_store_image<float><<<nb, 256, 0, stream>>>(npix, img, (float *)dout);
    cuda_check(cudaGetLastError(), "k_store_image launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  }
  cudaStream_t last = stream;
  if (!ddev) {
    CK(cudaEventRecord(ev_done, stream));
    CK(cudaStreamWaitEvent(d2h, ev_done, 0));
    CK(cudaMemcpyAsync(dirty, dout, npix * dsz, cudaMemcpyDeviceToHost, d2h));
    last = d2h;
  }
  finish_call(a, sl, last);
}

void Context::dirty2ms(const wsg_args &a, const void *dirty, void *vis) {
  validate(a);
  require(vis && dirty, "vis and dirty are required");
  CK(cudaSetDevice(device));
  const size_t nvis = a.nrows * a.nchan;
  const size_t vbytes = nvis * (a.vis_type == WSG_C128 ? 16 : 8);
  const size_t npix = a.npix_x * a.npix_y;
  const size_t dsz = a.dirty_type == WSG_F64 ? 8 : 4;
  Slot &sl = slots[slot_k++ % kSlots];
  CK(cudaEventSynchronize(sl.free_ev));
  Staged s;
  s.uvw = reinterpret_cast<const double *>(stage_in(a.uvw, a.nrows * 3 * sizeof(double), sl.uvw, cpy));
  s.wgt = stage_in(a.wgt, nvis * (a.wgt_type == WSG_F64 ? 8 : 4), sl.wgt, cpy);
  s.mask = reinterpret_cast<const uint8_t *>(stage_in(a.mask, nvis, sl.mask, cpy));
  const void *din = stage_in(dirty, npix * dsz, sl.out, cpy);
  CK(cudaEventRecord(ev_in, cpy));
  CK(cudaStreamWaitEvent(stream, ev_in, 0));
  ScanPlacement place(*this, sl, !tuned_call && s.uvw != a.uvw &&
                                     (a.wgt == nullptr || s.wgt != a.wgt) &&
                                     (a.mask == nullptr || s.mask != a.mask));
  // (the w-screen reads the model image in place: no FP64 copy)
  const bool vdev = is_device_pointer(vis);
  void *vout = vdev ? vis : sl.vis.ensure(vbytes);
  // inactive visibilities are zeroed; with no active ones at all the whole
  // output is zero
  CK(cudaMemsetAsync(vout, 0, vbytes, stream));
  if (tuned_call) {
    if (a.precision == WSG_PREC_FP64)
      degrid_tuned<double>(a, s, nullptr, vout, din);
    else
      degrid_tuned<float>(a, s, nullptr, vout, din);
  } else if (a.precision == WSG_PREC_FP64) {
    degrid_core<double>(a, s, nullptr, vout, din);
  } else {
    degrid_core<float>(a, s, nullptr, vout, din);
  }
  cudaStream_t last = stream;
  if (!vdev) {
    CK(cudaEventRecord(ev_done, stream));
    CK(cudaStreamWaitEvent(d2h, ev_done, 0));
    CK(cudaMemcpyAsync(vis, vout, vbytes, cudaMemcpyDeviceToHost, d2h));
    last = d2h;
  }
  finish_call(a, sl, last);
}

void Context::degrid_from_image(const wsg_args &a, const Staged &s, const double *img, void *vis,
                                size_t vbytes, bool tuned) {
  const bool vdev = is_device_pointer(vis);
  void *vout = vdev ? vis : b_vis.ensure(vbytes);
  // inactive visibilities are zeroed by the scan; with no active ones at all
  // the whole output is zero
  CK(cudaMemsetAsync(vout, 0, vbytes, stream));
  if (tuned) {
    if (a.precision == WSG_PREC_FP64)
      degrid_tuned<double>(a, s, img, vout, nullptr);
    else
      degrid_tuned<float>(a, s, img, vout, nullptr);
  } else if (a.precision == WSG_PREC_FP64) {
    degrid_core<double>(a, s, img, vout);
  } else {
    degrid_core<float>(a, s, img, vout);
  }
  if (!vdev) CK(cudaMemcpyAsync(vis, vout, vbytes, cudaMemcpyDeviceToHost, stream));
  CK(cudaEventRecord(ev[6], stream));
  CK(cudaStreamSynchronize(stream));
  float t;
  CK(cudaEventElapsedTime(&t, ev[0], ev[6]));
  stats.ms_total = t;
  stats.kernel_launches = g_kernel_launches.load();
  stats.nrows = a.nrows;
  stats.nchan = a.nchan;
}

template bool Context::prepare<float>(const wsg_args &, const Staged &, bool, void *, GridPlan &);
template bool Context::prepare<double>(const wsg_args &, const Staged &, bool, void *, GridPlan &);
template bool Context::grid_core<float>(const wsg_args &, const Staged &, double *, bool, void *,
                                        size_t);
template bool Context::grid_core<double>(const wsg_args &, const Staged &, double *, bool, void *,
                                         size_t);
template void Context::degrid_core<float>(const wsg_args &, const Staged &, const double *, void *,
                                          const void *, size_t, bool);
template void Context::degrid_core<double>(const wsg_args &, const Staged &, const double *, void *,
                                           const void *, size_t, bool);

}  // namespace wsg
