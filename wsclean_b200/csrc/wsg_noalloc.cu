// The allocation-free ms2dirty (wsg_ms2dirty_noalloc).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "wsg_host.cuh"

namespace wsg {

// ====================================================================
// Allocation-free ms2dirty.
//
// Some callers cannot allocate device memory while they grid: a plugin whose
// host application reserved the whole device up front for its own memory pool
// (a cudaMalloc there fails or steals from the host's budget), or code that
// runs under a fixed device-memory budget that must not grow after start-up.
// For them wsg_ms2dirty_noalloc runs the same mixed-precision pipeline as
// wsg_ms2dirty but takes every scratch buffer (sort keys, visibility records,
// chunk table, band grid, transformed columns, FP64 image, twiddle and
// correction tables) from one file-scope device array of kNoAllocScratchBytes,
// carves it up per call, and replaces cuFFT (whose plans allocate) by the
// library's own shared-memory FFT, so nv is a power of two (at most 8192).
// Every GPU that loads the library holds the array until the process exits.
//
// In host code the array's name is only a host-side stand-in, so its device
// address is looked up (cudaGetSymbolAddress, with the device current) on the
// first call in each CUDA context -- once per device, unless the device was
// reset and a new context created, in which case the module is loaded again,
// the array may move and the lookup is repeated.  The call synchronises its
// stream while it runs (it reads the visibility scan's statistics back to
// plan the grid).  All
// calls share the one array: calls that overlap on the GPU (different
// streams, or different host threads on one device) race on it and must be
// serialised by the caller.  Each call clears what must start at zero (image,
// grids, counters) itself.
// ====================================================================

constexpr size_t kNoAllocScratchBytes = size_t(96) << 20;  // 96 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
// (device, unique id of its current CUDA context) -> address of g_noalloc_scratch
std::map<std::pair<int, unsigned long long>, unsigned char *> g_noalloc_ptr;

// Unique id of the calling thread's current CUDA context (cuCtxGetId through
// the runtime's driver entry point, so the library needs no link-time driver
// dependency); 0 if the driver cannot tell, which keys the cache by device
// alone.
unsigned long long current_context_id() {
  using GetCurrent = int (*)(void **);
  using GetId = int (*)(void *, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
    cudaGetLastError();
  });
  void *ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
  return 0;
}

// Device address of the scratch array in the current context of device dev
// (dev is current).  Without a context id the address is looked up every time.
unsigned char *noalloc_scratch(int dev) {
  // cudaSetDevice initialises the device's primary context, so that the id
  // below names the context the lookup and the kernels will use
  cuda_check(cudaSetDevice(dev), "cudaSetDevice");
  const unsigned long long id = current_context_id();
  const auto key = std::make_pair(dev, id);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  auto it = g_noalloc_ptr.find(key);
  if (id != 0 && it != g_noalloc_ptr.end()) return it->second;
  void *p = nullptr;
  cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
  if (id != 0) g_noalloc_ptr[key] = reinterpret_cast<unsigned char *>(p);
  return reinterpret_cast<unsigned char *>(p);
}

// Bump allocator over the static scratch array.
struct Arena {
  unsigned char *base;
  size_t cap, off = 0;
  void *take(size_t bytes) {
    off = (off + 255) & ~size_t(255);
    if (off + bytes > cap)
      throw InvalidArgument("problem too large for the allocation-free entry point: needs more "
                            "than its " + std::to_string(cap >> 20) + " MiB of scratch");
    void *p = base + off;
    off += bytes;
    return p;
  }
  size_t left() const { return cap > ((off + 255) & ~size_t(255)) ? cap - ((off + 255) & ~size_t(255)) : 0; }
};

// Per-stage Stockham twiddles of a length-M FFT (same layout as the cached
// tables of the context path), complex float.
std::vector<float> stage_twiddles_f(size_t M) {
  std::vector<float> h(2 * M, 0.0f);
  size_t off = 0;
  for (size_t NS = 1; NS < M;) {
    const size_t R = (M / NS >= 16) ? 16 : M / NS;
    if (NS > 1) {
      for (size_t r = 1; r < R; ++r)
        for (size_t k = 0; k < NS; ++k) {
          const double f = double(r * k) / double(NS * R);
          h[2 * (off + (r - 1) * NS + k)] = float(std::cos(2.0 * M_PI * f));
          h[2 * (off + (r - 1) * NS + k) + 1] = float(std::sin(2.0 * M_PI * f));
        }
      off += (R - 1) * NS;
    }
    NS *= R;
  }
  return h;
}

void row_fft_f(int logM, void *data, long long rows, const void *tw, int sign, cudaStream_t st) {
  auto go = [&](auto lc) {
    constexpr int LOGM = decltype(lc)::value;
    constexpr int M = 1 << LOGM;
    using Cfg = ColCfg<float, M>;
    const size_t smem = ColSmem<float, M>::bytes();
    smem_attr(k_row_fft<float, LOGM>, smem);
    const long long nblk = (rows + Cfg::NB - 1) / Cfg::NB;
    k_row_fft<float, LOGM><<<unsigned(nblk), Cfg::THREADS, smem, st>>>(data, rows, tw, sign);
    cuda_check(cudaGetLastError(), "k_row_fft launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  };
  switch (logM) {
    case 8: go(std::integral_constant<int, 8>{}); break;
    case 9: go(std::integral_constant<int, 9>{}); break;
    case 10: go(std::integral_constant<int, 10>{}); break;
    case 11: go(std::integral_constant<int, 11>{}); break;
    case 12: go(std::integral_constant<int, 12>{}); break;
    case 13: go(std::integral_constant<int, 13>{}); break;
    default: throw InvalidArgument("v grid size outside the allocation-free FFT range (256..8192)");
  }
}

}  // namespace

void ms2dirty_noalloc(const wsg_args &a, const void *vis, void *dirty, cudaStream_t stream) {
  require(a.precision == WSG_PREC_MIXED, "the allocation-free entry point is mixed precision only");
  require(a.uvw && a.freq && vis && dirty, "uvw, freq, vis and dirty are required");
  require(a.nrows * a.nchan < (size_t(1) << 31), "at most 2^31-1 visibilities per call");
  require(a.npix_x % 2 == 0 && a.npix_y % 2 == 0, "nx_dirty and ny_dirty must be even");
  require(a.epsilon > 0 && a.pixsize_x > 0 && a.pixsize_y > 0, "bad epsilon or pixel size");
  for (const void *p : {(const void *)a.uvw, (const void *)a.freq, vis, (const void *)dirty})
    require(is_device_pointer(p), "the allocation-free entry point needs device pointers");
  require(!a.wgt || is_device_pointer(a.wgt), "weights must be device memory");
  require(!a.mask || is_device_pointer(a.mask), "mask must be device memory");
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  int nsm = 148;
  cuda_check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "attribute");
  Arena ar{noalloc_scratch(dev), kNoAllocScratchBytes};
  const size_t nvis_tot = a.nrows * a.nchan;

  // frequencies (checked on the host as in the Baselines ctor)
  std::vector<double> freq(a.nchan), fovc(a.nchan);
  cuda_check(cudaMemcpyAsync(freq.data(), a.freq, a.nchan * sizeof(double),
                             cudaMemcpyDeviceToHost, stream), "freq D2H");
  cuda_check(cudaStreamSynchronize(stream), "sync");
  for (size_t i = 0; i < a.nchan; ++i) {
    require(freq[i] > 0, "negative channel frequency encountered");
    if (i > 0) require(freq[i] >= freq[i - 1], "channel frequencies must be sorted in ascending order");
    fovc[i] = freq[i] / kSpeedOfLight;
  }
  double *d_fovc = reinterpret_cast<double *>(ar.take(a.nchan * sizeof(double)));
  cuda_check(cudaMemcpyAsync(d_fovc, fovc.data(), a.nchan * sizeof(double), cudaMemcpyHostToDevice,
                             stream), "fovc H2D");
  char *small = reinterpret_cast<char *>(ar.take(256));
  ScanOut *d_scan = reinterpret_cast<ScanOut *>(small);
  int *d_nch = reinterpret_cast<int *>(small + 64), *counter = d_nch + 1, *d_err = d_nch + 2;
  Staged st;
  st.uvw = a.uvw;
  st.fovc = d_fovc;
  st.vis = vis;
  st.wgt = a.wgt;
  st.mask = a.mask;

  ScanOut h0{};
  h0.wmin_bits = 0x7ff0000000000000ull;
  cuda_check(cudaMemcpyAsync(d_scan, &h0, sizeof(h0), cudaMemcpyHostToDevice, stream), "scan init");
  cuda_check(cudaMemsetAsync(d_nch, 0, 3 * sizeof(int), stream), "counters");
  {
    int nb = std::min(launch_blocks(a.nrows, 256), nsm * 8);
    with_types(a, [&](auto *tw, auto *tv) {
      using TW = std::remove_pointer_t<decltype(tw)>;
      using TV = std::remove_pointer_t<decltype(tv)>;
      k_scan<TV, TW><<<nb, 256, 0, stream>>>(a.nrows, int(a.nchan), st.uvw, st.fovc,
                                             reinterpret_cast<const TV *>(st.vis),
                                             reinterpret_cast<const TW *>(st.wgt), st.mask, 1,
                                             a.negate_v ? -1.0 : 1.0, d_scan, (TV *)nullptr,
                                             ImgW{});
    });
    cuda_check(cudaGetLastError(), "k_scan launch");
  }
  ScanOut hs;
  cuda_check(cudaMemcpyAsync(&hs, d_scan, sizeof(hs), cudaMemcpyDeviceToHost, stream), "scan D2H");
  cuda_check(cudaStreamSynchronize(stream), "sync");

  const size_t npix = a.npix_x * a.npix_y;
  double *img = reinterpret_cast<double *>(ar.take(npix * sizeof(double)));
  cuda_check(cudaMemsetAsync(img, 0, npix * sizeof(double), stream), "img clear");
  if (hs.nvis > 0) {
    GridPlan gp;
    gp.nx = a.npix_x;
    gp.ny = a.npix_y;
    gp.px = a.pixsize_x;
    gp.py = a.pixsize_y;
    gp.eps = a.epsilon;
    gp.do_w = a.do_wgridding != 0;
    gp.fp32 = true;
    gp.negate_v = a.negate_v != 0;
    gp.divide_by_n = a.divide_by_n != 0;
    gp.lshift = a.center_x;
    gp.mshift = a.negate_v ? -a.center_y : a.center_y;
    gp.nvis = hs.nvis;
    auto bits2d = [](unsigned long long b) {
      double d;
      std::memcpy(&d, &b, 8);
      return d;
    };
    gp.wmin_d = bits2d(hs.wmin_bits);
    gp.wmax_d = bits2d(hs.wmax_bits);
    gp.umax = bits2d(hs.umax_bits);
    gp.vmax = bits2d(hs.vmax_bits);
    choose_grid(gp, a.sigma_min, a.sigma_max, 16, /*pow2_v=*/true);
    limit_key_bits(gp, 31);  // this path sorts 32-bit keys
    int logMv = 0;
    while ((size_t(1) << logMv) < gp.nv) ++logMv;
    const DevGeom g = make_geom(gp);

    // sort
    uint32_t *ka = reinterpret_cast<uint32_t *>(ar.take(nvis_tot * 4));
    uint32_t *kb = reinterpret_cast<uint32_t *>(ar.take(nvis_tot * 4));
    uint32_t *va = reinterpret_cast<uint32_t *>(ar.take(nvis_tot * 4));
    uint32_t *vb = reinterpret_cast<uint32_t *>(ar.take(nvis_tot * 4));
    with_types(a, [&](auto *tw, auto *tv) {
      using TW = std::remove_pointer_t<decltype(tw)>;
      using TV = std::remove_pointer_t<decltype(tv)>;
      k_keys<TV, TW, uint32_t><<<launch_blocks(a.nrows, 256), 256, 0, stream>>>(
          a.nrows, int(a.nchan), st.uvw, st.fovc, reinterpret_cast<const TV *>(st.vis),
          reinterpret_cast<const TW *>(st.wgt), st.mask, 1, g, ka, va, ImgW{});
    });
    cuda_check(cudaGetLastError(), "k_keys launch");
    size_t tmp = 0;
    const int end_bit = gp.key_bits + 1;
    cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ka, kb, va, vb, int(nvis_tot), 0,
                                               end_bit, stream), "sort size");
    void *dtmp = ar.take(tmp);
    cuda_check(cub::DeviceRadixSort::SortPairs(dtmp, tmp, ka, kb, va, vb, int(nvis_tot), 0,
                                               end_bit, stream), "sort");
    void *rec = ar.take(gp.nvis * sizeof(RecF));
    with_types(a, [&](auto *tw, auto *tv) {
      using TW = std::remove_pointer_t<decltype(tw)>;
      using TV = std::remove_pointer_t<decltype(tv)>;
      launch_records<float, TW, TV>(gp.nvis, a, st, true, g, vb, va, rec, stream);
    });
    int *chunks = reinterpret_cast<int *>(ar.take((gp.nvis + 1) * sizeof(int)));
    ChunkStartPred<uint32_t> pred{kb, 2 * gp.lbits, 1024};
    thrust::counting_iterator<int> it(0);
    tmp = 0;
    cuda_check(cub::DeviceSelect::If(nullptr, tmp, it, chunks, d_nch, int(gp.nvis), pred, stream),
               "select size");
    dtmp = ar.take(tmp);
    cuda_check(cub::DeviceSelect::If(dtmp, tmp, it, chunks, d_nch, int(gp.nvis), pred, stream),
               "select");

    // correction and twiddle tables
    KernelTransform tr(gp.kernel);
    double vmax = 0.5 * std::max(double(gp.nx) / gp.nu, double(gp.ny) / gp.nv) * 1.0000001;
    if (gp.do_w) vmax = std::min(std::max(vmax, 0.5 / gp.ofactor * 1.0000001), 1.0);
    const ChebCorr cc = fit_cheb_corr(tr, vmax);
    std::vector<double> cf(gp.nx / 2 + 1 + gp.ny / 2 + 1);
    for (size_t i = 0; i <= gp.nx / 2; ++i) cf[i] = cc(double(i) / gp.nu);
    for (size_t i = 0; i <= gp.ny / 2; ++i) cf[gp.nx / 2 + 1 + i] = cc(double(i) / gp.nv);
    double *d_cf = reinterpret_cast<double *>(ar.take(cf.size() * sizeof(double)));
    cuda_check(cudaMemcpyAsync(d_cf, cf.data(), cf.size() * sizeof(double), cudaMemcpyHostToDevice,
                               stream), "cf H2D");
    const size_t Mu = size_t(1) << gp.logM, Mv = gp.nv;
    const std::vector<double> htwd = col_twiddle_table(Mu, gp.nu, size_t(gp.K));
    const std::vector<float> htw(htwd.begin(), htwd.end());
    const std::vector<float> htwv = stage_twiddles_f(Mv);
    float *d_tw = reinterpret_cast<float *>(ar.take(htw.size() * sizeof(float)));
    float *d_twv = reinterpret_cast<float *>(ar.take(htwv.size() * sizeof(float)));
    cuda_check(cudaMemcpyAsync(d_tw, htw.data(), htw.size() * sizeof(float), cudaMemcpyHostToDevice,
                               stream), "tw H2D");
    cuda_check(cudaMemcpyAsync(d_twv, htwv.data(), htwv.size() * sizeof(float),
                               cudaMemcpyHostToDevice, stream), "twv H2D");

    // grids: as many w planes per pass as fit in what is left
    const size_t per_plane = (gp.band_rows * gp.nv + gp.ny * gp.hrow()) * 8 + 1024;
    const size_t P = std::min(gp.nplanes, ar.left() / per_plane);
    require(P >= 1, "problem too large for the allocation-free entry point (no room for one w plane)");
    char *band = reinterpret_cast<char *>(ar.take(gp.band_rows * P * gp.nv * 8));
    char *H = reinterpret_cast<char *>(ar.take(P * gp.ny * gp.hrow() * 8));
    const DevKernel<float> kc = make_kernel<float>(gp.poly);
    const TileLayout tl = make_layout(gp.T, gp.kernel.W);
    const size_t smem = grid_smem_bytes<float>(tl, gp.kernel.W, true);
    GridArgs ga{};
    ga.err = d_err;
    ga.rec = rec;
    ga.chunk_start = chunks;
    ga.nchunks = d_nch;
    ga.counter = counter;
    ga.nvis = int(gp.nvis);
    ga.grid = band;
    ga.P = int(P);
    ga.tl = tl;
    ga.sb = grid_sb<float>();
    const ColArgs ca = make_col(gp, P, d_tw, band, H);
    for (size_t pb0 = 0; pb0 < gp.nplanes; pb0 += P) {
      const size_t npl = std::min(P, gp.nplanes - pb0);
      cuda_check(cudaMemsetAsync(band, 0, gp.band_rows * P * gp.nv * 8, stream), "band clear");
      cuda_check(cudaMemsetAsync(counter, 0, sizeof(int), stream), "counter clear");
      ga.pb0 = int(pb0);
      ga.pb1 = int(pb0 + npl);
      grid_dispatch<float>(gp.kernel.W, true, nsm, smem, stream, ga, g, kc);
      row_fft_f(logMv, band, (long long)(gp.band_rows * P), d_twv, +1, stream);
      col_run<float>(gp.logM, true, ca, int(npl), stream, d_err);
      ScreenArgs sa = make_screen(gp, d_cf, cc, P);
      sa.pb0 = int(pb0);
      sa.npl = int(npl);
      const dim3 sg = screen_grid(gp);
      launch_screen_add<float>(sg, stream, sa, H, img, nullptr, 0);
    }
    int herr = 0;
    cuda_check(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream), "err D2H");
    cuda_check(cudaStreamSynchronize(stream), "sync");
    if (herr & 2)
      throw std::runtime_error("internal error: a staged copy into shared memory did not complete");
    if (herr) throw std::runtime_error("internal error: a visibility record fell outside its tile");
  }
  const int nb = launch_blocks(npix, 256);
  if (a.dirty_type == WSG_F64)
    k_store_image<double><<<nb, 256, 0, stream>>>(npix, img, (double *)dirty);
  else
    k_store_image<float><<<nb, 256, 0, stream>>>(npix, img, (float *)dirty);
  cuda_check(cudaGetLastError(), "k_store_image launch");
  cuda_check(cudaStreamSynchronize(stream), "sync");
}

}  // namespace wsg
