// Host orchestration of libwsg: execution contexts, buffer cache, cuFFT plans,
// and the ms2dirty / dirty2ms drivers (the analogues of ducc0's
// Params::x2dirty and Params::dirty2x, wgridder.h:1430-1501).
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "wsg_context.h"
#include "wsg_device.cuh"

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
#define CK(x) cuda_check((x), #x)

static void cufft_check(cufftResult r, const char *what) {
  if (r == CUFFT_SUCCESS) return;
  if (r == CUFFT_ALLOC_FAILED) throw OutOfMemory(std::string(what) + ": cuFFT allocation failed");
  throw CufftError(std::string(what) + ": cuFFT error " + std::to_string(int(r)));
}
#define CF(x) cufft_check((x), #x)

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

static int env_int(const char *name, int dflt) {
  const char *s = std::getenv(name);
  return (s && *s) ? std::atoi(s) : dflt;
}

// Bin tile edge asked of the planner (which shrinks it until the W-plane
// tile fits shared memory): measured on the 8.1M-visibility 4096^2 pair,
// 20 is the fastest in mixed precision (3 -> 2 CTAs per SM, but half the
// tile flushes of 16) and 24 in FP64; WSG_TILE overrides it.
static int default_tile(bool fp32) { return env_int("WSG_TILE", fp32 ? 20 : 24); }

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
  int nn = n, inembed = n, onembed = n;
  size_t work = 0;
  CF(cufftMakePlanMany(h, 1, &nn, &inembed, istride, idist, &onembed, ostride, odist,
                       dbl ? CUFFT_Z2Z : CUFFT_C2C, batch, &work));
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

// ------------------------------------------------------------- planning

namespace {

DevGeom make_geom(const GridPlan &g) {
  DevGeom d;
  std::memset(&d, 0, sizeof d);  // padding too: geometries are compared bytewise
  d.nu = int(g.nu);
  d.nv = int(g.nv);
  d.W = g.kernel.W;
  d.nsafe = g.nsafe;
  d.maxiu0 = g.maxiu0;
  d.maxiv0 = g.maxiv0;
  d.px = g.px;
  d.py = g.py;
  d.ushift = g.ushift;
  d.vshift = g.vshift;
  d.wmin = g.wmin;
  d.dw = g.dw;
  d.xdw = g.xdw;
  d.wshift = g.wshift;
  d.nplanes = int(g.nplanes);
  d.do_w = g.do_w;
  d.lshift = g.lshift;
  d.mshift = g.mshift;
  d.nshift = g.nshift;
  d.vfac = g.negate_v ? -1.0 : 1.0;
  d.shifting = g.shifting;
  d.T = g.T;
  d.ntu = g.ntu;
  d.ntv = g.ntv;
  d.nwmin = g.nwmin;
  d.lbits = g.lbits;
  int tb = 0;
  while ((1 << tb) < g.T) ++tb;
  d.qshift = tb - g.lbits;
  d.wide = g.wide_keys ? 1 : 0;
  d.inactive_key = 1ull << g.key_bits;
  d.Lu = int(g.Lu);
  d.band_rows = int(g.band_rows);
  d.band_full = g.band_full;
  return d;
}

template <typename R>
DevKernel<R> make_kernel(const PolyKernel &pk) {
  DevKernel<R> k;
  std::memset(&k, 0, sizeof(k));
  k.D = pk.D;
  for (int j = 0; j <= pk.D; ++j)
    for (int i = 0; i < pk.W; ++i) k.c[j][i] = R(pk.coef[size_t(j) * pk.W + i]);
  return k;
}

TileLayout make_layout(int T, int W) {
  TileLayout tl;
  tl.S = T + W - 1;
  tl.RS = tl.S | 1;  // odd row stride
  int ps = tl.S * tl.RS;
  tl.PS = ps + ((8 - (ps % 32)) + 32) % 32;  // plane stride = 8 mod 32
  return tl;
}

// Before the transposed u transform fills the band grid: it writes every
// band row of the ny image columns (v indices [nv - ny/2, nv) and
// [0, ny/2)), so only the nv - ny columns between them need clearing.
void clear_outside_columns(void *band, size_t rows, size_t nv, size_t ny, size_t cs,
                           cudaStream_t st) {
  if (nv <= ny) return;
  cuda_check(cudaMemset2DAsync(static_cast<char *>(band) + (ny / 2) * cs, nv * cs, 0,
                               (nv - ny) * cs, rows, st),
             "cudaMemset2DAsync");
}

// Half-width in cells of the v columns the spread can write ([0, Lv] and
// [nv - Lv, nv)): the largest |v| plus half a kernel and a margin, as the u
// band (set_band); -1 when that covers the whole row.
long band_v_halfwidth(const GridPlan &g) {
  const double L = std::ceil(g.vmax * g.py * double(g.nv) + 0.5 * g.kernel.W + 2.0);
  if (!(L >= 0) || 2.0 * L + 1.0 >= double(g.nv)) return -1;
  return long(L);
}

int launch_blocks(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  return int(std::min<size_t>(std::max<size_t>(b, 1), 65535 * 8));
}

// Dynamic shared-memory limit of a kernel, set once per (kernel, device):
// every driver call on the launch path costs host time that the GPU waits
// through.
template <typename F>
void smem_attr(F *fn, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> done;
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_pair(reinterpret_cast<const void *>(fn), dev);
  auto it = done.find(key);
  if (it != done.end() && it->second >= smem) return;
  cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
             "smem attribute");
  done[key] = smem;
}

}  // namespace

// Kernel template dispatch over the support W.
template <typename R>
struct GridKernels {
  static constexpr int NWARP = 8;
  static constexpr int SB = sizeof(R) == 4 ? 256 : 64;
  template <int W>
  static constexpr int ppl() {
    return (sizeof(R) == 4 && W * W > 32) ? 2 : 1;
  }
  static size_t smem_bytes(const TileLayout &tl, int W, bool spread) {
    const size_t kst = sizeof(R) == 4 ? ((3 * size_t(W) + 3) & ~size_t(3))
                                      : ((3 * size_t(W) + 1) & ~size_t(1));
    const size_t stage = sizeof(R) * (32 * kst + 64) + 128;  // WarpStage<R, W>::bytes
    size_t tile = ((sizeof(R) * 2 * size_t(W) * tl.PS) + 15) & ~size_t(15);
    (void)spread;
    const size_t b = tile + size_t(NWARP) * stage;
    require(b == tile_smem_bytes(tl.S - W + 1, W, sizeof(R) == 4) && b <= kMaxSmemPerBlock,
            "internal: spread tile exceeds shared memory");
    return b;
  }
  // warps that share one record (more than one when a lane's share of the
  // W x W (plane, u-row) pairs would exceed PPL)
  static int groups(int W) {  // WarpGroups<W, ppl, NWARP>::NG
    const int ppl = (sizeof(R) == 4 && W * W > 32) ? 2 : 1;
    const int ng = (W * W + 32 * ppl - 1) / (32 * ppl);
    return ng > NWARP / 2 ? NWARP : ng;
  }
  template <int W>
  static void run(bool spread, dim3 grid, size_t smem, cudaStream_t st, const GridArgs &a,
                  const DevGeom &g, const DevKernel<R> &kc) {
    constexpr int P = ppl<W>();
    if (spread) {
      auto fn = k_spread<R, W, P, NWARP>;
      smem_attr(fn, smem);
      fn<<<grid, NWARP * 32, smem, st>>>(a, g, kc);
    } else {
      auto fn = k_interp<R, W, P, NWARP>;
      smem_attr(fn, smem);
      fn<<<grid, NWARP * 32, smem, st>>>(a, g, kc);
    }
    cuda_check(cudaGetLastError(), spread ? "k_spread launch" : "k_interp launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  }
  template <int W>
  static int occupancy(bool spread, size_t smem) {
    // cached: the query is a driver call, and plans enqueue launches while
    // a stream is being captured into a graph
    static std::mutex mu;
    static std::map<std::tuple<int, size_t, int>, int> memo;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    const auto key = std::make_tuple(int(spread), smem, dev);
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = memo.find(key);
      if (it != memo.end()) return it->second;
    }
    constexpr int P = ppl<W>();
    int nb = 0;
    if (spread)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_spread<R, W, P, NWARP>, NWARP * 32, smem);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_interp<R, W, P, NWARP>, NWARP * 32, smem);
    nb = std::max(nb, 1);
    std::lock_guard<std::mutex> lk(mu);
    memo[key] = nb;
    return nb;
  }
  static void dispatch(int W, bool spread, int nsm, size_t smem, cudaStream_t st, const GridArgs &a,
                       const DevGeom &g, const DevKernel<R> &kc) {
    auto go = [&](auto wc) {
      constexpr int WW = decltype(wc)::value;
      if constexpr (sizeof(R) == 4 && WW > 8) {
        throw std::runtime_error("support too large for mixed precision");
      } else {
        // set the smem attribute before asking for the occupancy
        constexpr int P = ppl<WW>();
        if (spread)
          smem_attr(k_spread<R, WW, P, NWARP>, smem);
        else
          smem_attr(k_interp<R, WW, P, NWARP>, smem);
        int occ = occupancy<WW>(spread, smem);
        dim3 grid(nsm * occ);
        run<WW>(spread, grid, smem, st, a, g, kc);
      }
    };
    switch (W) {
      case 4: go(std::integral_constant<int, 4>{}); break;
      case 5: go(std::integral_constant<int, 5>{}); break;
      case 6: go(std::integral_constant<int, 6>{}); break;
      case 7: go(std::integral_constant<int, 7>{}); break;
      case 8: go(std::integral_constant<int, 8>{}); break;
      case 9: go(std::integral_constant<int, 9>{}); break;
      case 10: go(std::integral_constant<int, 10>{}); break;
      case 11: go(std::integral_constant<int, 11>{}); break;
      case 12: go(std::integral_constant<int, 12>{}); break;
      case 13: go(std::integral_constant<int, 13>{}); break;
      case 14: go(std::integral_constant<int, 14>{}); break;
      case 15: go(std::integral_constant<int, 15>{}); break;
      case 16: go(std::integral_constant<int, 16>{}); break;
      default: throw std::runtime_error("unsupported kernel support");
    }
  }
};

// Whether `extra` bytes of shared memory fit beside a CTA's `base` bytes
// without lowering the CTAs an SM holds (228 KB a SM, 227 KB a CTA, 1 KB
// reserved a CTA).
// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library has no link-time driver dependency); nullptr if unavailable.
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
    cudaGetLastError();
  });
  return fn;
}

bool twist_tables_fit(size_t base, size_t extra) {
  constexpr size_t kSM = 228 * 1024, kCTA = 227 * 1024, kRes = 1024;
  if (base + extra > kCTA) return false;
  return kSM / (base + extra + kRes) == kSM / (base + kRes);
}

// Pruned u-transform kernels, dispatched over log2(M).
template <typename R>
struct ColKernels {
  // The band-to-image transform with the band columns staged by the tensor
  // memory accelerator (k_ucol_bwd_tma), when its boxes can be used: a box
  // row of NB columns is a multiple of 16 bytes, column groups start on a
  // 16-byte boundary and do not straddle the wrap of the v axis.  Returns
  // false when not used.
  template <int LOGM>
  static bool run_tma(const ColArgs &a, int npl, cudaStream_t st, int *err) {
    constexpr int M = 1 << LOGM;
    using Cfg = TmaCfg<R, M>;
    constexpr int NB = Cfg::NB;
    EncodeTiledFn enc = encode_tiled();
    if (!err || !enc || env_int("WSG_UCOL_TMA", 1) == 0) return false;
    if (NB * 2 * int(sizeof(R)) % 16 != 0 || (a.ny / 2) % NB != 0) return false;
    if (sizeof(R) == 4 && ((a.nv - a.ny / 2) % 2) != 0) return false;
    CUtensorMap map;
    const cuuint64_t dims[2] = {cuuint64_t(2) * cuuint64_t(npl) * cuuint64_t(a.nv),
                                cuuint64_t(a.band_rows)};
    const cuuint64_t strides[1] = {cuuint64_t(a.P) * cuuint64_t(a.nv) * 2 * sizeof(R)};
    const cuuint32_t box[2] = {cuuint32_t(2 * NB), cuuint32_t(Cfg::BR)};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&map, sizeof(R) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
            2, const_cast<void *>(a.band), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    const size_t base = Cfg::stage_bytes() +
                        (size_t(NB) * FftBuf<M>::value + M) * 2 * sizeof(R) + 128;
    // the twist tables go to shared memory too when that costs no resident CTA
    const size_t extra = size_t(a.K) * (M / 16 + 32) * 2 * sizeof(R);
    const bool tws = twist_tables_fit(base, extra);
    const size_t smem = tws ? base + extra : base;
    auto *kern = tws ? k_ucol_bwd_tma<R, LOGM, true> : k_ucol_bwd_tma<R, LOGM, false>;
    smem_attr(kern, smem);
    static int per_sm[2] = {-1, -1};  // resident CTAs per SM of each instantiation
    if (per_sm[tws] < 0) {
      int n = 0;
      cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, ColCfg<R, M>::THREADS,
                                                               smem),
                 "occupancy");
      per_sm[tws] = std::max(n, 1);
    }
    int dev = 0, nsm = 148;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "attribute");
    const long long nitems = (long long)((a.ny + NB - 1) / NB) * npl;
    const int grid = int(std::min<long long>(nitems, (long long)nsm * per_sm[tws]));
    kern<<<grid, ColCfg<R, M>::THREADS, smem, st>>>(a, map, npl, err);
    cuda_check(cudaGetLastError(), "k_ucol_bwd_tma launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return true;
  }
  // The image-to-band transform with each pass's H-row segments staged by
  // bulk copies (k_ucol_fwd_bulk), when its shared memory fits a CTA.
  // Returns false when not used.
  template <int LOGM>
  static bool run_bulk(const ColArgs &a, int npl, cudaStream_t st, int *err) {
    constexpr int M = 1 << LOGM;
    using Cfg = ColCfg<R, M>;
    constexpr int NB = Cfg::NB;
    if (!err || env_int("WSG_UCOL_TMA", 1) == 0) return false;
    const size_t cs = 2 * sizeof(R);
    if ((size_t(a.hseg) * cs) % 16 != 0 || (reinterpret_cast<uintptr_t>(a.H) & 15) != 0)
      return false;
    const size_t base = 128 + (size_t(NB) * a.hseg + size_t(NB) * FftBuf<M>::value + M) * cs;
    if (base > 227 * 1024) return false;
    // the twist tables go to shared memory too when that costs no resident
    // CTA (registers or shared memory, whichever binds)
    const size_t extra = size_t(a.K) * (M / 16 + 32) * cs;
    auto *k0 = k_ucol_fwd_bulk<R, LOGM, false>;
    auto *k1 = k_ucol_fwd_bulk<R, LOGM, true>;
    int n0 = 0, n1 = 0;
    smem_attr(k0, base);
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n0, k0, Cfg::THREADS, base),
               "occupancy");
    if (n0 < 1) return false;
    if (base + extra <= 227 * 1024) {
      smem_attr(k1, base + extra);
      cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n1, k1, Cfg::THREADS,
                                                               base + extra),
                 "occupancy");
    }
    const bool tws = n1 >= n0;
    const size_t smem = tws ? base + extra : base;
    auto *kern = tws ? k1 : k0;
    const int per_sm = tws ? n1 : n0;
    int dev = 0, nsm = 148;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "attribute");
    const long long nitems = (long long)((a.ny + NB - 1) / NB) * npl;
    const int grid = int(std::min<long long>(nitems, (long long)nsm * per_sm));
    kern<<<grid, Cfg::THREADS, smem, st>>>(a, npl, err);
    cuda_check(cudaGetLastError(), "k_ucol_fwd_bulk launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return true;
  }
  template <int LOGM>
  static void run1(bool bwd, const ColArgs &a, int npl, cudaStream_t st, int *err) {
    constexpr int M = 1 << LOGM;
    using Cfg = ColCfg<R, M>;
    if (bwd && run_tma<LOGM>(a, npl, st, err)) return;
    if (!bwd && run_bulk<LOGM>(a, npl, st, err)) return;
    const size_t smem = ColSmem2<R, M>::bytes();
    dim3 grid((a.ny + Cfg::NB - 1) / Cfg::NB, npl);
    if (bwd) {
      smem_attr(k_ucol_bwd<R, LOGM>, smem);
      k_ucol_bwd<R, LOGM><<<grid, Cfg::THREADS, smem, st>>>(a);
    } else {
      // the forward kernel keeps its twist tables in shared memory when they
      // fit without costing a resident CTA
      const size_t extra = size_t(a.K) * (M / 16 + 32) * 2 * sizeof(R);
      if (twist_tables_fit(smem, extra)) {
        smem_attr(k_ucol_fwd<R, LOGM, true>, smem + extra);
        k_ucol_fwd<R, LOGM, true><<<grid, Cfg::THREADS, smem + extra, st>>>(a);
      } else {
        smem_attr(k_ucol_fwd<R, LOGM, false>, smem);
        k_ucol_fwd<R, LOGM, false><<<grid, Cfg::THREADS, smem, st>>>(a);
      }
    }
    cuda_check(cudaGetLastError(), bwd ? "k_ucol_bwd launch" : "k_ucol_fwd launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  }
  // err: the device error word (bit 2: a staged copy did not complete), or
  // nullptr to stay with the plain loads (either direction)
  static void run(int logM, bool bwd, const ColArgs &a, int npl, cudaStream_t st,
                  int *err = nullptr) {
    switch (logM) {
      case 8: run1<8>(bwd, a, npl, st, err); break;
      case 9: run1<9>(bwd, a, npl, st, err); break;
      case 10: run1<10>(bwd, a, npl, st, err); break;
      case 11: run1<11>(bwd, a, npl, st, err); break;
      case 12: run1<12>(bwd, a, npl, st, err); break;
      case 13:
        if constexpr (sizeof(R) == 4) {
          run1<13>(bwd, a, npl, st, err);
          break;
        }
        [[fallthrough]];
      default: throw std::runtime_error("unsupported pruned FFT length");
    }
  }
};

// ------------------------------------------------------------ the driver

namespace {

template <typename TW, typename TV>
void launch_scan(Context &cx, const wsg_args &a, const Staged &s, bool gridding, TV *vis_out,
                 ScanOut *d_out, cudaStream_t st) {
  int nb = launch_blocks(a.nrows, 256);
  nb = std::min(nb, cx.num_sms * 8);
  k_scan<TV, TW><<<nb, 256, 0, st>>>(
      a.nrows, int(a.nchan), s.uvw, s.fovc, reinterpret_cast<const TV *>(s.vis),
      reinterpret_cast<const TW *>(s.wgt), s.mask, gridding ? 1 : 0, a.negate_v ? -1.0 : 1.0,
      d_out, vis_out, s.iw);
  cuda_check(cudaGetLastError(), "k_scan launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

template <typename TW, typename TV, typename K>
void launch_keys(Context &cx, const wsg_args &a, const Staged &s, bool gridding, const DevGeom &g,
                 K *keys, uint32_t *vals) {
  int nb = launch_blocks(a.nrows, 256);
  k_keys<TV, TW, K><<<nb, 256, 0, cx.stream>>>(a.nrows, int(a.nchan), s.uvw, s.fovc,
                                               reinterpret_cast<const TV *>(s.vis),
                                               reinterpret_cast<const TW *>(s.wgt), s.mask,
                                               gridding ? 1 : 0, g, keys, vals, s.iw);
  cuda_check(cudaGetLastError(), "k_keys launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

// Records of the nvis active visibilities in sorted order: the sorted
// positions pos (scratch of nvis_tot entries) from the sort's permutation
// sidx, then the records built in visibility order and scattered to them
// (the inactive visibilities sorted last and are skipped).
template <typename R, typename TW, typename TV>
void launch_records(size_t nvis, const wsg_args &a, const Staged &s, bool gridding,
                    const DevGeom &g, const uint32_t *sidx, uint32_t *pos, void *rec,
                    cudaStream_t st) {
  const size_t nvis_tot = a.nrows * a.nchan;
  k_rank<<<launch_blocks(nvis_tot, 256), 256, 0, st>>>(nvis_tot, sidx, pos);
  cuda_check(cudaGetLastError(), "k_rank launch");
  k_records<R, TV, TW><<<launch_blocks(nvis_tot, 256), 256, 0, st>>>(
      nvis_tot, nvis, int(a.nchan), pos, s.uvw, s.fovc, reinterpret_cast<const TV *>(s.vis),
      reinterpret_cast<const TW *>(s.wgt), gridding ? 1 : 0, g,
      reinterpret_cast<typename RecOf<R>::type *>(rec), s.iw);
  cuda_check(cudaGetLastError(), "k_records launch");
  g_kernel_launches.fetch_add(2, std::memory_order_relaxed);
}

// type-dispatch helpers over (weight type, vis type)
template <typename F>
void with_types(const wsg_args &a, F &&f) {
  bool wd = a.wgt && a.wgt_type == WSG_F64;
  bool vd = a.vis_type == WSG_C128;
  if (wd && vd) f((double *)nullptr, (double2 *)nullptr);
  else if (wd) f((double *)nullptr, (float2 *)nullptr);
  else if (vd) f((float *)nullptr, (double2 *)nullptr);
  else f((float *)nullptr, (float2 *)nullptr);
}

}  // namespace

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

namespace {

ScreenArgs make_screen(const GridPlan &g, const double *d_cf, const ChebCorr &cc, size_t P) {
  ScreenArgs s{};
  s.nx = int(g.nx);
  s.ny = int(g.ny);
  s.nu = int(g.nu);
  s.nv = int(g.nv);
  s.ld = g.ny;
  s.px = g.px;
  s.py = g.py;
  s.x0 = g.lshift - 0.5 * g.nx * g.px;
  s.y0 = g.mshift - 0.5 * g.ny * g.py;
  s.nshift = g.nshift;
  s.dw = g.dw;
  s.wmin = g.wmin;
  s.do_w = g.do_w;
  s.divide_by_n = g.do_w && g.divide_by_n;
  s.P = int(P);
  s.K = g.K;
  s.hseg = int(g.hseg());
  s.hm0 = g.hm0();
  s.nbs = int((g.hseg() + 31) / 32);
  s.cfu = d_cf;
  s.cfv = d_cf + g.nx / 2 + 1;
  s.ncheb = cc.n;
  s.ymax = cc.ymax;
  for (int i = 0; i < cc.n && i < kDMaxCheb; ++i) s.cheb[i] = cc.c[i];
  return s;
}

ColArgs make_col(const GridPlan &g, size_t P, const void *tw, void *band, void *H) {
  ColArgs c{};
  c.nx = int(g.nx);
  c.ny = int(g.ny);
  c.nu = int(g.nu);
  c.nv = int(g.nv);
  c.P = int(P);
  c.L = int(g.Lu);
  c.band_rows = int(g.band_rows);
  c.band_full = g.band_full;
  c.K = g.K;
  const size_t cs = g.fp32 ? 8 : 16;
  const size_t M = size_t(1) << g.logM;
  c.twM = tw;
  c.twB = reinterpret_cast<const char *>(tw) + M * cs;
  c.twQ = reinterpret_cast<const char *>(tw) + (M + size_t(g.K) * (M / 16)) * cs;
  c.band = band;
  c.H = H;
  c.hseg = int(g.hseg());
  c.hm0 = g.hm0();
  return c;
}

// Screen kernel grid: 32-entry blocks of every H-row segment by 32 image
// columns.
dim3 screen_grid(const GridPlan &g) {
  return dim3(unsigned(size_t(g.K) * ((g.hseg() + 31) / 32)), unsigned((g.ny + 31) / 32));
}

}  // namespace

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
static size_t col_table_entries(size_t M, size_t K) { return M + K * (M / 16) + 32 * K; }

static std::vector<double> col_twiddle_table(size_t M, size_t nu, size_t K) {
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
  char *bandf = reinterpret_cast<char *>(b_bandf.ensure(rowsP * nv * cs));
  char *H = reinterpret_cast<char *>(b_H.ensure(P * gp.ny * gp.hrow() * cs));
  const void *tw = upload_twiddles(gp, dbl);
  ColArgs ca = make_col(gp, P, tw, bandf, H);
  const long Lv = band_v_halfwidth(gp);
  const TileLayout tl = make_layout(gp.T, gp.kernel.W);
  const size_t smem = GridKernels<R>::smem_bytes(tl, gp.kernel.W, true);
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
  ga.sb = GridKernels<R>::SB;

  const int dir = CUFFT_INVERSE;
  float t_grid = 0, t_fft = 0, t_screen = 0;
  for (size_t pb0 = 0; pb0 < gp.nplanes; pb0 += P) {
    const size_t npl = std::min(P, gp.nplanes - pb0);
    CK(cudaEventRecord(ev[2], stream));
    clear_band(band, rowsP, nv, cs);
    CK(cudaMemsetAsync(counter, 0, sizeof(int), stream));
    ga.pb0 = int(pb0);
    ga.pb1 = int(pb0 + npl);
    GridKernels<R>::dispatch(gp.kernel.W, true, num_sms, smem, stream, ga, g, kc);
    band_dirty = BandDirty{band, rowsP, nv, cs, Lv};
    CK(cudaEventRecord(ev[3], stream));
    // transform along v: every (band row, plane) is a contiguous row of nv
    {
      cufftHandle h = fft_plan(int(nv), 1, int(nv), 1, int(nv), int(rowsP), dbl);
      fft_exec(h, band, bandf, dir, dbl);
    }
    // pruned transform along u: band rows of the image columns -> image rows
    ColKernels<R>::run(gp.logM, true, ca, int(npl), stream, d_err);
    CK(cudaEventRecord(ev[4], stream));
    ScreenArgs sa = make_screen(gp, cf_cur, cc, P);
    sa.pb0 = int(pb0);
    sa.npl = int(npl);
    sa.ld = ld;
    const dim3 sg = screen_grid(gp);
    k_screen_add<R><<<sg, 256, 0, stream>>>(sa, H, img, direct_out, out_mode);
    cuda_check(cudaGetLastError(), "k_screen_add launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
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
  char *bandi = reinterpret_cast<char *>(b_bandd.ensure(rowsP * nv * cs));
  char *band = reinterpret_cast<char *>(b_bandf.ensure(rowsP * nv * cs));
  char *H = reinterpret_cast<char *>(b_H.ensure(P * gp.ny * gp.hrow() * cs));
  const void *tw = upload_twiddles(gp, dbl);
  ColArgs ca = make_col(gp, P, tw, bandi, H);
  const TileLayout tl = make_layout(gp.T, gp.kernel.W);
  const size_t smem = GridKernels<R>::smem_bytes(tl, gp.kernel.W, false);
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
  ga.sb = GridKernels<R>::SB;
  ga.vis_out = vis_out;
  ga.vis_double = a.vis_type == WSG_C128;
  ga.vis_accumulate = vis_acc ? 1 : 0;
  const bool multi = P < gp.nplanes;
  const bool need_acc = multi || GridKernels<R>::groups(gp.kernel.W) > 1;
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
    k_screen_put<R><<<sg, 256, 0, stream>>>(sa, src, src_f32, H);
    cuda_check(cudaGetLastError(), "k_screen_put launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    CK(cudaEventRecord(ev[3], stream));
    // pruned transform along u (transposed): image rows -> band rows of the
    // image columns; the other columns of the band grid stay zero
    const BandDirty zl{bandi, rowsP, nv, cs, long(gp.ny)};
    if (!(bandd_zero.p == zl.p && bandd_zero.rows == zl.rows && bandd_zero.nv == zl.nv &&
          bandd_zero.cs == zl.cs && bandd_zero.Lv == zl.Lv)) {
      bandd_zero = BandDirty{};
      clear_outside_columns(bandi, rowsP, nv, gp.ny, cs, stream);
      bandd_zero = zl;
    }
    ColKernels<R>::run(gp.logM, false, ca, int(npl), stream, d_err);
    // transform along v
    {
      cufftHandle h = fft_plan(int(nv), 1, int(nv), 1, int(nv), int(rowsP), dbl);
      fft_exec(h, bandi, band, dir, dbl);
    }
    CK(cudaEventRecord(ev[4], stream));
    CK(cudaMemsetAsync(counter, 0, sizeof(int), stream));
    ga.pb0 = int(pb0);
    ga.pb1 = int(pb0 + npl);
    ga.first_pass = pb0 == 0;
    ga.last_pass = pb0 + npl >= gp.nplanes;
    GridKernels<R>::dispatch(gp.kernel.W, false, num_sms, smem, stream, ga, g, kc);
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
  std::printf("  nvis=%zu, w=[%g; %g], dw=%g, planes per pass=%zu, u band rows=%zu\n", g.nvis,
              g.wmin_d, g.wmax_d, g.dw, P, g.band_rows);
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

// ------------------------------------------------- reusable plans, batches
//
// A plan runs prepare() (scan, keys, sort, records) once per job with the
// degridding active set and records (static factor = weight x conjugate
// shift phasor, conjugation bit), copies each job's records and chunk list
// into one concatenated array, and keeps every job's band grid resident.
// Execution is then one persistent spread (or interpolation) launch over
// all chunks of all jobs, the job of a chunk selecting its grid, followed by
// each job's v-FFT, pruned u-transform and w-screen.  Nothing on the
// execution path allocates or synchronises with the host.

Plan::Plan(Context &cx, const wsg_args &a, const wsg_job *jobs, size_t njobs) : cx_(cx), a_(a) {
  cx_.validate(a);
  require(a.nrows * a.nchan < (size_t(1) << 31), "plans index at most 2^31 - 1 visibilities");
  std::vector<wsg_job> js;
  if (jobs == nullptr || njobs == 0) {
    wsg_job j{};
    j.npix_x = a.npix_x;
    j.npix_y = a.npix_y;
    j.center_x = a.center_x;
    j.center_y = a.center_y;
    j.chan_begin = 0;
    j.chan_end = a.nchan;
    js.push_back(j);
  } else {
    js.assign(jobs, jobs + njobs);
  }
  for (const auto &j : js) {
    require(j.npix_x % 2 == 0 && j.npix_y % 2 == 0, "job image sizes must be even");
    require(j.npix_x >= 16 && j.npix_y >= 16, "job images must be at least 16 x 16");
    require(j.chan_begin < j.chan_end && j.chan_end <= a.nchan, "job channel range out of bounds");
  }
  dbl_ = a.precision == WSG_PREC_FP64;
  use_graphs_ = env_int("WSG_PLAN_GRAPHS", 1) != 0;
  CK(cudaSetDevice(cx_.device));
  if (dbl_)
    build<double>(js);
  else
    build<float>(js);
  // registered once built: a plan whose construction failed is never checked
  cx_.plan_err.push_back(reinterpret_cast<int *>(small_.p) + 2);
}

Plan::~Plan() {
  cudaSetDevice(cx_.device);
  cudaStreamSynchronize(cx_.stream);
  auto &pe = cx_.plan_err;
  pe.erase(std::remove(pe.begin(), pe.end(), reinterpret_cast<int *>(small_.p) + 2), pe.end());
  for (auto &g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (auto &j : jobs_)
    if (j.fft) cufftDestroy(j.fft);
  for (DevBuf *b : {&rec_, &chunks_, &chunk_job_, &jobgeom_, &band_, &H_, &img_, &cf_, &tw_, &acc_,
                    &small_, &fftwork_})
    b->release();
}

namespace {
size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
}  // namespace

template <typename R>
void Plan::build(const std::vector<wsg_job> &js) {
  using Rec = typename RecOf<R>::type;
  const size_t cs = 2 * sizeof(R);
  const size_t nchan = a_.nchan, nrows = a_.nrows;
  cudaStream_t st = cx_.stream;
  const int tile = default_tile(sizeof(R) == 4);

  // coordinates on the device (kept only while building)
  Staged s;
  s.uvw = reinterpret_cast<const double *>(cx_.stage_in(a_.uvw, nrows * 3 * sizeof(double), cx_.b_uvw));
  const size_t wsz = a_.wgt_type == WSG_F64 ? 8 : 4;
  const void *wgt_all = cx_.stage_in(a_.wgt, nrows * nchan * wsz, cx_.b_wgt);
  const uint8_t *mask_all =
      reinterpret_cast<const uint8_t *>(cx_.stage_in(a_.mask, nrows * nchan, cx_.b_mask));
  std::vector<double> freq(nchan);
  if (is_device_pointer(a_.freq))
    CK(cudaMemcpy(freq.data(), a_.freq, nchan * sizeof(double), cudaMemcpyDeviceToHost));
  else
    std::memcpy(freq.data(), a_.freq, nchan * sizeof(double));

  // the shared kernel: the one chosen for the largest job with active data
  size_t big = 0;
  for (size_t j = 1; j < js.size(); ++j)
    if (js[j].npix_x * js[j].npix_y > js[big].npix_x * js[big].npix_y) big = j;
  std::vector<size_t> order{big};
  for (size_t j = 0; j < js.size(); ++j)
    if (j != big) order.push_back(j);

  size_t cap = 0;
  for (const auto &j : js) cap += nrows * (j.chan_end - j.chan_begin);
  rec_.ensure(std::max<size_t>(cap, 1) * sizeof(Rec));
  chunks_.ensure((std::max<size_t>(cap, 1) + 1) * sizeof(int));
  chunk_job_.ensure((std::max<size_t>(cap, 1) + 1) * sizeof(int));
  small_.ensure(4096);
  CK(cudaMemsetAsync(small_.p, 0, 4096, cx_.stream));
  DevBuf wsub, msub;
  jobs_.assign(js.size(), PlanJob{});
  int forceW = 0;
  double forceS = 0;
  std::vector<double> cf_host;
  std::vector<char> tw_host;
  for (size_t oi = 0; oi < order.size(); ++oi) {
    const size_t j = order[oi];
    const wsg_job &jd = js[j];
    PlanJob &pj = jobs_[j];
    pj.chan0 = jd.chan_begin;
    pj.chan1 = jd.chan_end;
    const size_t nch = jd.chan_end - jd.chan_begin;
    wsg_args aj = a_;
    aj.nchan = nch;
    aj.freq = freq.data() + jd.chan_begin;
    aj.npix_x = jd.npix_x;
    aj.npix_y = jd.npix_y;
    aj.center_x = jd.center_x;
    aj.center_y = jd.center_y;
    Staged sj = s;
    // the job's channel columns of weights and mask, compacted
    if (a_.wgt) {
      void *d = wsub.ensure(nrows * nch * wsz);
      CK(cudaMemcpy2DAsync(d, nch * wsz, static_cast<const char *>(wgt_all) + jd.chan_begin * wsz,
                           nchan * wsz, nch * wsz, nrows, cudaMemcpyDeviceToDevice, st));
      sj.wgt = d;
      aj.wgt = d;
    }
    if (a_.mask) {
      void *d = msub.ensure(nrows * nch);
      CK(cudaMemcpy2DAsync(d, nch, mask_all + jd.chan_begin, nchan, nch, nrows,
                           cudaMemcpyDeviceToDevice, st));
      sj.mask = reinterpret_cast<const uint8_t *>(d);
      aj.mask = reinterpret_cast<const uint8_t *>(d);
    }
    GridPlan &gp = pj.gp;
    gp.nx = jd.npix_x;
    gp.ny = jd.npix_y;
    gp.px = a_.pixsize_x;
    gp.py = a_.pixsize_y;
    gp.eps = a_.epsilon;
    gp.do_w = a_.do_wgridding != 0;
    gp.fp32 = sizeof(R) == 4;
    gp.gridding = false;
    gp.negate_v = a_.negate_v != 0;
    gp.divide_by_n = a_.divide_by_n != 0;
    gp.lshift = jd.center_x;
    gp.mshift = a_.negate_v ? -jd.center_y : jd.center_y;
    gp.force_W = forceW;
    gp.force_sigma = forceS;
    const bool any = cx_.prepare<R>(aj, sj, false, nullptr, gp);
    if (forceW == 0 && any) {  // the largest job with active visibilities
      forceW = gp.kernel.W;
      forceS = gp.kernel.sigma;
      DevKernel<R> kc = make_kernel<R>(gp.poly);
      kernel_.resize(sizeof(kc));
      std::memcpy(kernel_.data(), &kc, sizeof(kc));
      DevGeom g0 = make_geom(gp);
      geom_.resize(sizeof(g0));
      std::memcpy(geom_.data(), &g0, sizeof(g0));
      W_ = gp.kernel.W;
      T_ = gp.T;
    }
    if (!any) continue;
    require(gp.T == T_ && gp.kernel.W == W_, "internal: jobs must share kernel and tile");
    pj.nrec = gp.nvis;
    int nch_j = 0;
    CK(cudaMemcpyAsync(&nch_j, reinterpret_cast<char *>(cx_.b_small.p) + 1024, sizeof(int),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    pj.rec_off = nrec_;
    CK(cudaMemcpyAsync(static_cast<char *>(rec_.p) + nrec_ * sizeof(Rec), cx_.b_rec.p,
                       pj.nrec * sizeof(Rec), cudaMemcpyDeviceToDevice, st));
    Rec *rj = reinterpret_cast<Rec *>(rec_.p) + nrec_;
    k_plan_remap<Rec><<<launch_blocks(pj.nrec, 256), 256, 0, st>>>(
        pj.nrec, rj, uint32_t(nch), uint32_t(nchan), uint32_t(jd.chan_begin));
    cuda_check(cudaGetLastError(), "k_plan_remap launch");
    k_plan_chunks<<<launch_blocks(size_t(nch_j), 256), 256, 0, st>>>(
        nch_j, reinterpret_cast<const int *>(cx_.b_chunks.p),
        reinterpret_cast<int *>(chunks_.p) + nchunks_, reinterpret_cast<int *>(chunk_job_.p) + nchunks_,
        int(nrec_), int(j));
    cuda_check(cudaGetLastError(), "k_plan_chunks launch");
    g_kernel_launches.fetch_add(2, std::memory_order_relaxed);
    nrec_ += pj.nrec;
    nchunks_ += nch_j;
    // corrections and twiddles of this grid
    pj.cc = cx_.upload_corrections(gp);
    const void *twd = cx_.upload_twiddles(gp, sizeof(R) == 8);
    CK(cudaStreamSynchronize(st));  // the uploads are stream-ordered
    const size_t ncf = gp.nx / 2 + 1 + gp.ny / 2 + 1;
    pj.cf_off = cf_host.size();
    cf_host.resize(cf_host.size() + ncf);
    CK(cudaMemcpy(cf_host.data() + pj.cf_off, cx_.cf_cur, ncf * sizeof(double),
                  cudaMemcpyDeviceToHost));
    const size_t M = size_t(1) << gp.logM;
    const size_t ntw = col_table_entries(M, size_t(gp.K)) * cs;
    pj.tw_off = tw_host.size();
    tw_host.resize(align256(tw_host.size() + ntw));
    CK(cudaMemcpy(tw_host.data() + pj.tw_off, twd, ntw, cudaMemcpyDeviceToHost));
    // the job's band grid with all its planes, and its v-FFT plan
    pj.band_bytes = gp.band_rows * gp.nplanes * gp.nv * cs;
    pj.band_off = band_total_;
    band_total_ = align256(band_total_ + pj.band_bytes);
    max_npix_ = std::max(max_npix_, gp.nx * gp.ny);
  }
  require(nrec_ > 0, "no active visibilities in any job");
  CK(cudaMemcpyAsync(small_.p, &nchunks_, sizeof(int), cudaMemcpyHostToDevice, st));

  size_t hmax = 0, work = 0;
  std::vector<JobGeom> jg(jobs_.size());
  band_.ensure(band_total_);
  for (size_t j = 0; j < jobs_.size(); ++j) {
    PlanJob &pj = jobs_[j];
    if (pj.nrec == 0) continue;
    const GridPlan &gp = pj.gp;
    hmax = std::max(hmax, gp.nplanes * gp.ny * gp.hrow() * cs);
    JobGeom &g = jg[j];
    g.nu = int(gp.nu);
    g.nv = int(gp.nv);
    g.Lu = int(gp.Lu);
    g.band_rows = int(gp.band_rows);
    g.band_full = gp.band_full;
    g.P = int(gp.nplanes);
    g.pb0 = 0;
    g.pb1 = int(gp.nplanes);
    g.grid = static_cast<char *>(band_.p) + pj.band_off;
    CF(cufftCreate(&pj.fft));
    CF(cufftSetAutoAllocation(pj.fft, 0));
    int n = int(gp.nv), inembed = n, onembed = n;
    size_t w = 0;
    CF(cufftMakePlanMany(pj.fft, 1, &n, &inembed, 1, n, &onembed, 1, n,
                         sizeof(R) == 8 ? CUFFT_Z2Z : CUFFT_C2C, int(gp.band_rows * gp.nplanes), &w));
    work = std::max(work, w);
  }
  H_.ensure(hmax);
  img_.ensure(max_npix_ * sizeof(double));
  fftwork_.ensure(std::max<size_t>(work, 256));
  jobgeom_.ensure(jg.size() * sizeof(JobGeom));
  CK(cudaMemcpyAsync(jobgeom_.p, jg.data(), jg.size() * sizeof(JobGeom), cudaMemcpyHostToDevice, st));
  cf_.ensure(std::max<size_t>(cf_host.size(), 1) * sizeof(double));
  CK(cudaMemcpyAsync(cf_.p, cf_host.data(), cf_host.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  tw_.ensure(std::max<size_t>(tw_host.size(), 1));
  CK(cudaMemcpyAsync(tw_.p, tw_host.data(), tw_host.size(), cudaMemcpyHostToDevice, st));
  need_acc_ = GridKernels<R>::groups(W_) > 1;
  if (need_acc_) acc_.ensure(nrec_ * cs);
  CK(cudaStreamSynchronize(st));
}

template <typename R>
void Plan::enqueue_grid(const void *vis, void *const *dirty, int accumulate) {
  const size_t cs = 2 * sizeof(R);
  cudaStream_t st = cx_.stream;
  int *d_nch = reinterpret_cast<int *>(small_.p);
  int *counter = d_nch + 1;
  int *d_err = d_nch + 2;
  CK(cudaMemsetAsync(band_.p, 0, band_total_, st));
  CK(cudaMemsetAsync(counter, 0, sizeof(int), st));  // (the error word stays until read)
  const TileLayout tl = make_layout(T_, W_);
  const size_t smem = GridKernels<R>::smem_bytes(tl, W_, true);
  GridArgs ga{};
  ga.rec = rec_.p;
  ga.chunk_start = reinterpret_cast<const int *>(chunks_.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(nrec_);
  ga.tl = tl;
  ga.sb = GridKernels<R>::SB;
  ga.err = d_err;
  ga.jobs = reinterpret_cast<const JobGeom *>(jobgeom_.p);
  ga.chunk_job = reinterpret_cast<const int *>(chunk_job_.p);
  ga.vis_in = vis;
  ga.vis_in_double = a_.vis_type == WSG_C128;
  DevKernel<R> kc;
  std::memcpy(&kc, kernel_.data(), sizeof(kc));
  DevGeom g0;
  std::memcpy(&g0, geom_.data(), sizeof(g0));
  GridKernels<R>::dispatch(W_, true, cx_.num_sms, smem, st, ga, g0, kc);
  for (size_t j = 0; j < jobs_.size(); ++j) {
    const PlanJob &pj = jobs_[j];
    const GridPlan &gp = pj.gp;
    const size_t npix = gp.nx * gp.ny;
    double *img = reinterpret_cast<double *>(img_.p);
    const int nb = launch_blocks(npix, 256);
    if (pj.nrec == 0) {
      if (!accumulate)
        CK(cudaMemsetAsync(dirty[j], 0, npix * (a_.dirty_type == WSG_F64 ? 8 : 4), st));
      continue;
    }
    char *band = static_cast<char *>(band_.p) + pj.band_off;
    CF(cufftSetStream(pj.fft, st));
    CF(cufftSetWorkArea(pj.fft, fftwork_.p));
    if (sizeof(R) == 8)
      CF(cufftExecZ2Z(pj.fft, reinterpret_cast<cufftDoubleComplex *>(band),
                      reinterpret_cast<cufftDoubleComplex *>(band), CUFFT_INVERSE));
    else
      CF(cufftExecC2C(pj.fft, reinterpret_cast<cufftComplex *>(band),
                      reinterpret_cast<cufftComplex *>(band), CUFFT_INVERSE));
    ColArgs ca = make_col(gp, gp.nplanes, static_cast<char *>(tw_.p) + pj.tw_off, band, H_.p);
    ColKernels<R>::run(gp.logM, true, ca, int(gp.nplanes), st, d_err);
    if (accumulate) {
      if (a_.dirty_type == WSG_F64)
        k_load_image<double><<<nb, 256, 0, st>>>(npix, (const double *)dirty[j], img, 0);
      else
        k_load_image<float><<<nb, 256, 0, st>>>(npix, (const float *)dirty[j], img, 0);
      cuda_check(cudaGetLastError(), "k_load_image launch");
    } else {
      CK(cudaMemsetAsync(img, 0, npix * sizeof(double), st));
    }
    ScreenArgs sa = make_screen(gp, reinterpret_cast<const double *>(cf_.p) + pj.cf_off, pj.cc,
                                gp.nplanes);
    sa.pb0 = 0;
    sa.npl = int(gp.nplanes);
    const dim3 sg = screen_grid(gp);
    k_screen_add<R><<<sg, 256, 0, st>>>(sa, H_.p, img, nullptr, 0);
    cuda_check(cudaGetLastError(), "k_screen_add launch");
    if (a_.dirty_type == WSG_F64)
      k_store_image<double><<<nb, 256, 0, st>>>(npix, img, (double *)dirty[j]);
    else
      k_store_image<float><<<nb, 256, 0, st>>>(npix, img, (float *)dirty[j]);
    cuda_check(cudaGetLastError(), "k_store_image launch");
    g_kernel_launches.fetch_add(accumulate ? 3 : 2, std::memory_order_relaxed);
  }
  (void)cs;
}

template <typename R>
void Plan::enqueue_degrid(const void *const *dirty, void *vis) {
  const size_t cs = 2 * sizeof(R);
  cudaStream_t st = cx_.stream;
  int *d_nch = reinterpret_cast<int *>(small_.p);
  int *counter = d_nch + 1;
  int *d_err = d_nch + 2;
  const size_t vsz = a_.vis_type == WSG_C128 ? 16 : 8;
  const bool multi = jobs_.size() > 1;
  CK(cudaMemsetAsync(vis, 0, a_.nrows * a_.nchan * vsz, st));
  for (size_t j = 0; j < jobs_.size(); ++j) {
    const PlanJob &pj = jobs_[j];
    if (pj.nrec == 0) continue;
    const GridPlan &gp = pj.gp;
    const size_t npix = gp.nx * gp.ny;
    double *img = reinterpret_cast<double *>(img_.p);
    const int nb = launch_blocks(npix, 256);
    if (a_.dirty_type == WSG_F64)
      k_load_image<double><<<nb, 256, 0, st>>>(npix, (const double *)dirty[j], img, 0);
    else
      k_load_image<float><<<nb, 256, 0, st>>>(npix, (const float *)dirty[j], img, 0);
    cuda_check(cudaGetLastError(), "k_load_image launch");
    ScreenArgs sa = make_screen(gp, reinterpret_cast<const double *>(cf_.p) + pj.cf_off, pj.cc,
                                gp.nplanes);
    sa.pb0 = 0;
    sa.npl = int(gp.nplanes);
    const dim3 sg = screen_grid(gp);
    k_screen_put<R><<<sg, 256, 0, st>>>(sa, img, 0, H_.p);
    cuda_check(cudaGetLastError(), "k_screen_put launch");
    char *band = static_cast<char *>(band_.p) + pj.band_off;
    clear_outside_columns(band, gp.band_rows * gp.nplanes, gp.nv, gp.ny, cs, st);
    ColArgs ca = make_col(gp, gp.nplanes, static_cast<char *>(tw_.p) + pj.tw_off, band, H_.p);
    ColKernels<R>::run(gp.logM, false, ca, int(gp.nplanes), st, d_err);
    CF(cufftSetStream(pj.fft, st));
    CF(cufftSetWorkArea(pj.fft, fftwork_.p));
    if (sizeof(R) == 8)
      CF(cufftExecZ2Z(pj.fft, reinterpret_cast<cufftDoubleComplex *>(band),
                      reinterpret_cast<cufftDoubleComplex *>(band), CUFFT_FORWARD));
    else
      CF(cufftExecC2C(pj.fft, reinterpret_cast<cufftComplex *>(band),
                      reinterpret_cast<cufftComplex *>(band), CUFFT_FORWARD));
    g_kernel_launches.fetch_add(2, std::memory_order_relaxed);
  }
  CK(cudaMemsetAsync(counter, 0, sizeof(int), st));  // (the error word stays until read)
  const TileLayout tl = make_layout(T_, W_);
  const size_t smem = GridKernels<R>::smem_bytes(tl, W_, false);
  GridArgs ga{};
  ga.rec = rec_.p;
  ga.chunk_start = reinterpret_cast<const int *>(chunks_.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(nrec_);
  ga.tl = tl;
  ga.sb = GridKernels<R>::SB;
  ga.err = d_err;
  ga.jobs = reinterpret_cast<const JobGeom *>(jobgeom_.p);
  ga.chunk_job = reinterpret_cast<const int *>(chunk_job_.p);
  ga.vis_out = vis;
  ga.vis_double = a_.vis_type == WSG_C128;
  ga.vis_accumulate = multi ? 1 : 0;
  ga.first_pass = ga.last_pass = 1;
  ga.acc = need_acc_ ? acc_.p : nullptr;
  if (need_acc_) CK(cudaMemsetAsync(acc_.p, 0, nrec_ * cs, st));
  DevKernel<R> kc;
  std::memcpy(&kc, kernel_.data(), sizeof(kc));
  DevGeom g0;
  std::memcpy(&g0, geom_.data(), sizeof(g0));
  GridKernels<R>::dispatch(W_, false, cx_.num_sms, smem, st, ga, g0, kc);
  if (need_acc_) {
    k_finalize<R><<<launch_blocks(nrec_, 256), 256, 0, st>>>(int(nrec_), rec_.p, acc_.p, vis,
                                                             ga.vis_double, ga.vis_accumulate);
    cuda_check(cudaGetLastError(), "k_finalize launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void Plan::enqueue(int mode, const void *in, void *const *outs, const void *const *ins, void *out,
                   int accumulate) {
  if (mode == 0) {
    if (dbl_)
      enqueue_grid<double>(in, outs, accumulate);
    else
      enqueue_grid<float>(in, outs, accumulate);
  } else {
    if (dbl_)
      enqueue_degrid<double>(ins, out);
    else
      enqueue_degrid<float>(ins, out);
  }
}

// Runs one execution: directly into a graph being recorded by the caller,
// else through the plan's own graph for these pointers (recorded on the
// second call with them; the first runs eagerly and sets the kernels'
// launch attributes outside any capture).
void Plan::run(int mode, const void *in, void *const *outs, const void *const *ins, void *out,
               int accumulate) {
  CK(cudaSetDevice(cx_.device));
  cudaStream_t st = cx_.stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    enqueue(mode, in, outs, ins, out, accumulate);
    return;
  }
  std::vector<const void *> ptrs{mode == 0 ? in : out};
  for (size_t j = 0; j < jobs_.size(); ++j) ptrs.push_back(mode == 0 ? outs[j] : ins[j]);
  for (const Graph &g : graphs_)
    if (g.mode == mode && g.accumulate == accumulate && g.ptrs == ptrs) {
      CK(cudaGraphLaunch(g.exec, st));
      return;
    }
  for (const void *p : ptrs)
    require(is_device_pointer(p), "plan execution needs device memory for vis and images");
  const auto seen = std::make_pair(mode * 2 + accumulate, ptrs);
  const bool first = std::find(eager_seen_.begin(), eager_seen_.end(), seen) == eager_seen_.end();
  // the legacy default stream cannot be captured
  if (!use_graphs_ || first || st == nullptr || st == cudaStreamLegacy) {
    enqueue(mode, in, outs, ins, out, accumulate);
    if (first) eager_seen_.push_back(seen);
    return;
  }
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue(mode, in, outs, ins, out, accumulate);
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    throw;
  }
  CK(cudaStreamEndCapture(st, &graph));
  Graph g;
  g.mode = mode;
  g.accumulate = accumulate;
  g.ptrs = ptrs;
  cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    // a graph that cannot be instantiated: run eagerly from now on
    cudaGetLastError();
    use_graphs_ = false;
    enqueue(mode, in, outs, ins, out, accumulate);
    return;
  }
  graphs_.push_back(g);
  CK(cudaGraphLaunch(g.exec, st));
}

void Plan::ms2dirty(const void *vis, void *const *dirty, int accumulate) {
  require(vis && dirty, "vis and dirty are required");
  for (size_t j = 0; j < jobs_.size(); ++j) require(dirty[j] != nullptr, "dirty image missing");
  run(0, vis, dirty, nullptr, nullptr, accumulate ? 1 : 0);
}

void Plan::dirty2ms(const void *const *dirty, void *vis) {
  require(vis && dirty, "vis and dirty are required");
  for (size_t j = 0; j < jobs_.size(); ++j) require(dirty[j] != nullptr, "dirty image missing");
  run(1, nullptr, nullptr, dirty, vis, 0);
}

void Plan::stats(size_t job, wsg_stats &o) const {
  require(job < jobs_.size(), "job index out of range");
  const PlanJob &pj = jobs_[job];
  const GridPlan &g = pj.gp;
  std::memset(&o, 0, sizeof(o));
  o.nrows = a_.nrows;
  o.nchan = pj.chan1 - pj.chan0;
  o.nvis = pj.nrec;
  o.nu = g.nu;
  o.nv = g.nv;
  o.nplanes = g.nplanes;
  o.supp = g.kernel.W;
  o.plane_batch = g.nplanes;
  o.band_rows = g.band_rows;
  o.degree = g.poly.D;
  o.sigma = g.ofactor;
  o.beta = g.kernel.beta;
  o.e0 = g.kernel.e0;
  o.kernel_err = g.kernel.err;
  o.wmin = g.wmin_d;
  o.wmax = g.wmax_d;
  o.dw = g.dw;
  o.nshift = g.nshift;
  o.precision = g.fp32 ? WSG_PREC_MIXED : WSG_PREC_FP64;
  o.device_bytes = rec_.n + chunks_.n + chunk_job_.n + band_.n + H_.n + img_.n + acc_.n + fftwork_.n;
  o.kernel_launches = g_kernel_launches.load();
}

// ---------------------------------------- streaming into a resident grid
//
// The whole w-stack stays in HBM between chunks: chunks only scan, sort,
// build records and spread (or interpolate); the FFTs and screens run once
// per image.  Host chunks are staged through two page-locked buffers and a
// copy stream, so the transfer of chunk k+1 proceeds while chunk k is
// sorted and spread.

void *PinnedBuf::ensure(size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (n < bytes) {
    release();
    cuda_check(cudaHostAlloc(&p, bytes, cudaHostAllocDefault), "cudaHostAlloc");
    n = bytes;
  }
  return p;
}

void PinnedBuf::release() {
  if (p) cudaFreeHost(p);
  p = nullptr;
  n = 0;
}

StreamGridder::StreamGridder(Context &cx, const wsg_args &a, double wmin, double wmax,
                             double umax, double vmax, size_t nvis)
    : cx_(cx), a_(a) {
  require(a.freq != nullptr && a.nchan > 0, "freq is required");
  freq_.resize(a.nchan);
  if (is_device_pointer(a.freq))
    CK(cudaMemcpy(freq_.data(), a.freq, a.nchan * sizeof(double), cudaMemcpyDeviceToHost));
  else
    std::memcpy(freq_.data(), a.freq, a.nchan * sizeof(double));
  a_.freq = freq_.data();
  a_.uvw = nullptr;
  a_.wgt = nullptr;
  a_.mask = nullptr;
  wsg_args v = a_;
  v.nrows = 1;  // validate() checks the geometry, not the (absent) rows
  v.uvw = freq_.data();
  cx_.validate(v);
  require(wmin >= 0 && wmax >= wmin && umax > 0 && vmax > 0, "bad data extent");
  dbl_ = a.precision == WSG_PREC_FP64;
  CK(cudaSetDevice(cx_.device));
  GridPlan &g = gp_;
  g.nx = a.npix_x;
  g.ny = a.npix_y;
  g.px = a.pixsize_x;
  g.py = a.pixsize_y;
  g.eps = a.epsilon;
  g.do_w = a.do_wgridding != 0;
  g.fp32 = !dbl_;
  g.negate_v = a.negate_v != 0;
  g.divide_by_n = a.divide_by_n != 0;
  g.lshift = a.center_x;
  g.mshift = a.negate_v ? -a.center_y : a.center_y;
  g.nvis = nvis ? nvis : size_t(1) << 24;
  g.wmin_d = wmin;
  g.wmax_d = wmax;
  g.umax = umax;
  g.vmax = vmax;
  choose_grid(g, a.sigma_min, a.sigma_max, default_tile(!dbl_));
  g.fixed = true;
  const size_t cs = dbl_ ? 16 : 8;
  band_.ensure(g.band_rows * g.nplanes * g.nv * cs);
  img_.ensure(g.nx * g.ny * sizeof(double));
  cc_ = cx_.upload_corrections(g);
  const void *twd = cx_.upload_twiddles(g, dbl_);
  CK(cudaStreamSynchronize(cx_.stream));  // the uploads are stream-ordered
  const size_t ncf = g.nx / 2 + 1 + g.ny / 2 + 1;
  cf_.ensure(ncf * sizeof(double));
  CK(cudaMemcpy(cf_.p, cx_.cf_cur, ncf * sizeof(double), cudaMemcpyDeviceToDevice));
  const size_t M = size_t(1) << g.logM;
  const size_t ntw = col_table_entries(M, size_t(g.K)) * cs;
  tw_.ensure(ntw);
  CK(cudaMemcpy(tw_.p, twd, ntw, cudaMemcpyDeviceToDevice));
  CF(cufftCreate(&fft_));
  CF(cufftSetAutoAllocation(fft_, 0));
  int n = int(g.nv), inembed = n, onembed = n;
  size_t work = 0;
  CF(cufftMakePlanMany(fft_, 1, &n, &inembed, 1, n, &onembed, 1, n, dbl_ ? CUFFT_Z2Z : CUFFT_C2C,
                       int(g.band_rows * g.nplanes), &work));
  fftwork_.ensure(std::max<size_t>(work, 256));
  H_.ensure(plane_batch() * g.hrow() * g.ny * cs);
  CK(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
  for (auto &sl : slots_) {
    CK(cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
  }
  for (auto &b : batch_) {
    CK(cudaEventCreateWithFlags(&b.filled, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&b.spread, cudaEventDisableTiming));
  }
  // a batch holds a third of the expected visibilities (so that the copies
  // of one overlap the spread of another), at least 32M, within 2^31 - 1
  // and with its inputs in at most 1/16 of the device memory
  {
    size_t freeb = 0, total = 0;
    CK(cudaMemGetInfo(&freeb, &total));
    const size_t row_bytes = 24 + a.nchan * ((a.vis_type == WSG_C128 ? 16 : 8) +
                                             (a.wgt_type == WSG_F64 ? 8 : 4) + 1);
    size_t vis = std::max<size_t>(size_t(32) << 20, (nvis ? nvis : 0) / 3);
    vis = std::min(vis, (size_t(1) << 31) - 1);
    size_t rows = vis / a.nchan;
    rows = std::min(rows, (total / 16) / row_bytes);
    batch_rows_ = std::max<size_t>(rows, 1);
  }
  CK(cudaMemsetAsync(band_.p, 0, band_.n, cx_.stream));
  mode_ = 1;
}

StreamGridder::~StreamGridder() {
  cudaSetDevice(cx_.device);
  cudaStreamSynchronize(cx_.stream);
  if (copy_) {
    cudaStreamSynchronize(copy_);
    cudaStreamDestroy(copy_);
  }
  for (auto &sl : slots_) {
    if (sl.copied) cudaEventDestroy(sl.copied);
    if (sl.done) cudaEventDestroy(sl.done);
    for (DevBuf *b : {&sl.uvw, &sl.vis, &sl.wgt, &sl.mask}) b->release();
    for (PinnedBuf *b : {&sl.h_uvw, &sl.h_vis, &sl.h_wgt, &sl.h_mask}) b->release();
  }
  for (auto &b : batch_) {
    if (b.filled) cudaEventDestroy(b.filled);
    if (b.spread) cudaEventDestroy(b.spread);
    for (DevBuf *d : {&b.uvw, &b.vis, &b.wgt, &b.mask}) d->release();
  }
  if (fft_) cufftDestroy(fft_);
  for (DevBuf *b : {&band_, &H_, &img_, &cf_, &tw_, &fftwork_, &vout_, &lambda_}) b->release();
}

// Planes per pass of the final transforms (the u-transformed rows of a pass
// are held in H): all of them when they fit in a quarter of the free memory.
size_t StreamGridder::plane_batch() const {
  size_t freeb = 0, total = 0;
  CK(cudaMemGetInfo(&freeb, &total));
  const size_t per = gp_.hrow() * gp_.ny * (dbl_ ? 16 : 8);
  return std::max<size_t>(1, std::min<size_t>(gp_.nplanes, (freeb / 4) / std::max<size_t>(per, 1)));
}

// Stages a chunk: device pointers are used in place; page-locked host
// memory is copied directly on the copy stream; pageable memory goes
// through the slot's page-locked buffer first.  The compute stream waits
// for the copies.
Staged StreamGridder::stage(Slot &sl, size_t nrows, const double *uvw, const void *vis,
                            const void *wgt, const uint8_t *mask) {
  CK(cudaEventSynchronize(sl.done));  // the slot's previous chunk is finished
  const size_t nvis = nrows * a_.nchan;
  auto put = [&](const void *src, size_t bytes, DevBuf &dev, PinnedBuf &pin) -> const void * {
    if (!src) return nullptr;
    cudaPointerAttributes at;
    cudaMemoryType t = cudaMemoryTypeUnregistered;
    if (cudaPointerGetAttributes(&at, src) == cudaSuccess)
      t = at.type;
    else
      cudaGetLastError();
    if (t == cudaMemoryTypeDevice || t == cudaMemoryTypeManaged) return src;
    const void *from = src;
    if (t != cudaMemoryTypeHost) {
      std::memcpy(pin.ensure(bytes), src, bytes);
      from = pin.p;
    }
    void *d = dev.ensure(bytes);
    CK(cudaMemcpyAsync(d, from, bytes, cudaMemcpyHostToDevice, copy_));
    return d;
  };
  Staged s;
  s.uvw = reinterpret_cast<const double *>(put(uvw, nrows * 3 * sizeof(double), sl.uvw, sl.h_uvw));
  if (vis) s.vis = put(vis, nvis * (a_.vis_type == WSG_C128 ? 16 : 8), sl.vis, sl.h_vis);
  s.wgt = put(wgt, nvis * (a_.wgt_type == WSG_F64 ? 8 : 4), sl.wgt, sl.h_wgt);
  s.mask = reinterpret_cast<const uint8_t *>(put(mask, nvis, sl.mask, sl.h_mask));
  CK(cudaEventRecord(sl.copied, copy_));
  CK(cudaStreamWaitEvent(cx_.stream, sl.copied, 0));
  return s;
}

template <typename R>
void StreamGridder::add_t(const Staged &s, size_t nrows) {
  wsg_args ac = a_;
  ac.nrows = nrows;
  ac.uvw = s.uvw;
  ac.wgt = s.wgt;
  ac.mask = s.mask;
  GridPlan g = gp_;
  if (!cx_.prepare<R>(ac, s, true, nullptr, g)) return;
  cudaStream_t st = cx_.stream;
  const TileLayout tl = make_layout(g.T, g.kernel.W);
  const size_t smem = GridKernels<R>::smem_bytes(tl, g.kernel.W, true);
  int *counter = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 2048);
  int *d_nch = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 1024);
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 3072);
  if (!err_armed_) {  // read back and cleared by finish()
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    err_armed_ = true;
  }
  CK(cudaMemsetAsync(counter, 0, sizeof(int), st));
  GridArgs ga{};
  ga.err = d_err;
  ga.rec = cx_.b_rec.p;
  ga.chunk_start = reinterpret_cast<const int *>(cx_.b_chunks.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(g.nvis);
  ga.grid = band_.p;
  ga.P = int(g.nplanes);
  ga.pb0 = 0;
  ga.pb1 = int(g.nplanes);
  ga.tl = tl;
  ga.sb = GridKernels<R>::SB;
  GridKernels<R>::dispatch(g.kernel.W, true, cx_.num_sms, smem, st, ga, make_geom(g),
                           make_kernel<R>(g.poly));
}

// Enqueues a copy of bytes from src (device, page-locked or pageable host
// memory) to the device buffer dst on the copy stream; pageable memory goes
// through the page-locked buffer pin (the caller synchronises the copy
// stream before pin is reused).
void StreamGridder::copy_into(void *dst, const void *src, size_t bytes, PinnedBuf &pin) {
  cudaPointerAttributes at;
  cudaMemoryType t = cudaMemoryTypeUnregistered;
  if (cudaPointerGetAttributes(&at, src) == cudaSuccess)
    t = at.type;
  else
    cudaGetLastError();
  if (t == cudaMemoryTypeDevice || t == cudaMemoryTypeManaged || t == cudaMemoryTypeHost) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, copy_));
    return;
  }
  std::memcpy(pin.ensure(bytes), src, bytes);
  CK(cudaMemcpyAsync(dst, pin.p, bytes, cudaMemcpyHostToDevice, copy_));
}

// WSClean multiplies each visibility's weight by the imaging weight of its
// uv cell before gridding (MSGridderBase::readAndWeightVisibilities,
// gridding/msgridderbase.cpp:583-590,640-659).  Here the lookup happens in
// the scan and record kernels of each batch, from the finished grid of w.
void StreamGridder::set_imaging_weights(const ImageWeightsGpu *w) {
  if (!w) {
    iw_ = ImgW{};
    return;
  }
  require(w->finished(), "the imaging weights must be finished (wsg_weights_finish)");
  require(w->device() == cx_.device, "the imaging weights live on another device");
  flush_batch();  // rows added so far keep the weights they were added with
  std::vector<double> l(freq_.size());
  for (size_t c = 0; c < l.size(); ++c) l[c] = kSpeedOfLight / freq_[c];
  CK(cudaStreamSynchronize(cx_.stream));  // an earlier table may still be read
  double *d = reinterpret_cast<double *>(lambda_.ensure(l.size() * sizeof(double)));
  CK(cudaMemcpy(d, l.data(), l.size() * sizeof(double), cudaMemcpyHostToDevice));
  iw_.grid = w->grid_ptr();
  iw_.lambda = d;
  iw_.g = w->geometry();
}

// Sorts and spreads the current batch (after its copies) and switches to
// the other one.  The batch's scan checks its rows against the declared
// extent (prepare() with the fixed grid); a batch that fails is dropped.
void StreamGridder::flush_batch() {
  Batch &b = batch_[bcur_];
  if (b.rows == 0) return;
  const size_t rows = b.rows;
  b.rows = 0;
  bcur_ ^= 1;
  CK(cudaEventRecord(b.filled, copy_));
  CK(cudaStreamWaitEvent(cx_.stream, b.filled, 0));
  Staged s;
  s.uvw = reinterpret_cast<const double *>(b.uvw.p);
  s.vis = b.vis.p;
  s.wgt = b.has_wgt ? b.wgt.p : nullptr;
  s.mask = b.has_mask ? reinterpret_cast<const uint8_t *>(b.mask.p) : nullptr;
  s.iw = iw_;
  if (dbl_)
    add_t<double>(s, rows);
  else
    add_t<float>(s, rows);
  CK(cudaEventRecord(b.spread, cx_.stream));
}

void StreamGridder::add(size_t nrows, const double *uvw, const void *vis, const void *wgt,
                        const uint8_t *mask) {
  require(uvw && vis, "uvw and vis are required");
  if (nrows == 0) return;
  CK(cudaSetDevice(cx_.device));
  if (mode_ == 2) {  // after prediction (a major cycle's Predict, then Invert)
    CK(cudaMemsetAsync(band_.p, 0, band_.n, cx_.stream));
    for (auto &b : batch_) b.rows = 0;
    mode_ = 1;
  }
  if (nrows > batch_rows_) {  // a chunk larger than a batch is spread alone
    flush_batch();
    Slot &sl = slots_[k_++ & 1];
    Staged s = stage(sl, nrows, uvw, vis, wgt, mask);
    s.iw = iw_;
    if (dbl_)
      add_t<double>(s, nrows);
    else
      add_t<float>(s, nrows);
    CK(cudaEventRecord(sl.done, cx_.stream));
    return;
  }
  Batch *b = &batch_[bcur_];
  if (b->rows > 0 && (b->rows + nrows > batch_rows_ || (wgt != nullptr) != b->has_wgt ||
                      (mask != nullptr) != b->has_mask)) {
    flush_batch();
    b = &batch_[bcur_];
  }
  const size_t nchan = a_.nchan;
  const size_t vsz = a_.vis_type == WSG_C128 ? 16 : 8, wsz = a_.wgt_type == WSG_F64 ? 8 : 4;
  if (b->rows == 0) {  // the batch's previous spread has read its buffers
    CK(cudaEventSynchronize(b->spread));
    b->has_wgt = wgt != nullptr;
    b->has_mask = mask != nullptr;
    b->uvw.ensure(batch_rows_ * 3 * sizeof(double));
    b->vis.ensure(batch_rows_ * nchan * vsz);
    if (b->has_wgt) b->wgt.ensure(batch_rows_ * nchan * wsz);
    if (b->has_mask) b->mask.ensure(batch_rows_ * nchan);
  }
  // the caller's buffers are free again when add() returns: the copies
  // (not the spread of an earlier batch, which runs meanwhile) are waited for
  Slot &sl = slots_[0];
  const size_t r0 = b->rows;
  copy_into(static_cast<char *>(b->uvw.p) + r0 * 3 * sizeof(double), uvw, nrows * 3 * sizeof(double),
            sl.h_uvw);
  copy_into(static_cast<char *>(b->vis.p) + r0 * nchan * vsz, vis, nrows * nchan * vsz, sl.h_vis);
  if (wgt)
    copy_into(static_cast<char *>(b->wgt.p) + r0 * nchan * wsz, wgt, nrows * nchan * wsz, sl.h_wgt);
  if (mask) copy_into(static_cast<char *>(b->mask.p) + r0 * nchan, mask, nrows * nchan, sl.h_mask);
  CK(cudaStreamSynchronize(copy_));
  b->rows += nrows;
}

template <typename R>
void StreamGridder::finish_t(void *dirty, int accumulate) {
  const GridPlan &g = gp_;
  cudaStream_t st = cx_.stream;
  const size_t cs = 2 * sizeof(R), npix = g.nx * g.ny;
  double *img = reinterpret_cast<double *>(img_.p);
  const bool ddev = is_device_pointer(dirty);
  const size_t dsz = a_.dirty_type == WSG_F64 ? 8 : 4;
  const int nb = launch_blocks(npix, 256);
  if (accumulate) {
    const void *din = ddev ? dirty : cx_.stage_in(dirty, npix * dsz, cx_.b_out);
    if (a_.dirty_type == WSG_F64)
      k_load_image<double><<<nb, 256, 0, st>>>(npix, (const double *)din, img, 0);
    else
      k_load_image<float><<<nb, 256, 0, st>>>(npix, (const float *)din, img, 0);
    cuda_check(cudaGetLastError(), "k_load_image launch");
  } else {
    CK(cudaMemsetAsync(img, 0, npix * sizeof(double), st));
  }
  CF(cufftSetStream(fft_, st));
  CF(cufftSetWorkArea(fft_, fftwork_.p));
  if (sizeof(R) == 8)
    CF(cufftExecZ2Z(fft_, reinterpret_cast<cufftDoubleComplex *>(band_.p),
                    reinterpret_cast<cufftDoubleComplex *>(band_.p), CUFFT_INVERSE));
  else
    CF(cufftExecC2C(fft_, reinterpret_cast<cufftComplex *>(band_.p),
                    reinterpret_cast<cufftComplex *>(band_.p), CUFFT_INVERSE));
  const size_t P = std::max<size_t>(1, H_.n / (npix * cs));
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 3072);
  if (!err_armed_) {
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    err_armed_ = true;
  }
  for (size_t p0 = 0; p0 < g.nplanes; p0 += P) {
    const size_t np = std::min(P, g.nplanes - p0);
    // the band layout is [row][plane][nv]: a pass starts p0 planes into each row
    ColArgs ca = make_col(g, g.nplanes, tw_.p, static_cast<char *>(band_.p) + p0 * g.nv * cs, H_.p);
    ColKernels<R>::run(g.logM, true, ca, int(np), st, d_err);
    ScreenArgs sa = make_screen(g, reinterpret_cast<const double *>(cf_.p), cc_, np);
    sa.pb0 = int(p0);
    sa.npl = int(np);
    const dim3 sg = screen_grid(g);
    k_screen_add<R><<<sg, 256, 0, st>>>(sa, H_.p, img, nullptr, 0);
    cuda_check(cudaGetLastError(), "k_screen_add launch");
  }
  void *dout = ddev ? dirty : cx_.b_out.ensure(npix * dsz);
  if (a_.dirty_type == WSG_F64)
    k_store_image<double><<<nb, 256, 0, st>>>(npix, img, (double *)dout);
  else
    k_store_image<float><<<nb, 256, 0, st>>>(npix, img, (float *)dout);
  cuda_check(cudaGetLastError(), "k_store_image launch");
  if (!ddev) CK(cudaMemcpyAsync(dirty, dout, npix * dsz, cudaMemcpyDeviceToHost, st));
  CK(cudaMemsetAsync(band_.p, 0, band_.n, st));
  err_armed_ = false;
  cx_.check_device_error(d_err);  // synchronises the stream
}

void StreamGridder::finish(void *dirty, int accumulate) {
  require(mode_ == 1, "finish() without a gridding stream");
  require(dirty != nullptr, "dirty is required");
  CK(cudaSetDevice(cx_.device));
  flush_batch();
  if (dbl_)
    finish_t<double>(dirty, accumulate);
  else
    finish_t<float>(dirty, accumulate);
}

template <typename R>
void StreamGridder::predict_begin_t(const double *img) {
  const GridPlan &g = gp_;
  cudaStream_t st = cx_.stream;
  const size_t cs = 2 * sizeof(R), npix = g.nx * g.ny;
  CK(cudaMemsetAsync(band_.p, 0, band_.n, st));
  const size_t P = std::max<size_t>(1, H_.n / (npix * cs));
  for (size_t p0 = 0; p0 < g.nplanes; p0 += P) {
    const size_t np = std::min(P, g.nplanes - p0);
    ScreenArgs sa = make_screen(g, reinterpret_cast<const double *>(cf_.p), cc_, np);
    sa.pb0 = int(p0);
    sa.npl = int(np);
    const dim3 sg = screen_grid(g);
    k_screen_put<R><<<sg, 256, 0, st>>>(sa, img, 0, H_.p);
    cuda_check(cudaGetLastError(), "k_screen_put launch");
    ColArgs ca = make_col(g, g.nplanes, tw_.p, static_cast<char *>(band_.p) + p0 * g.nv * cs, H_.p);
    ColKernels<R>::run(g.logM, false, ca, int(np), st);
  }
  CF(cufftSetStream(fft_, st));
  CF(cufftSetWorkArea(fft_, fftwork_.p));
  if (sizeof(R) == 8)
    CF(cufftExecZ2Z(fft_, reinterpret_cast<cufftDoubleComplex *>(band_.p),
                    reinterpret_cast<cufftDoubleComplex *>(band_.p), CUFFT_FORWARD));
  else
    CF(cufftExecC2C(fft_, reinterpret_cast<cufftComplex *>(band_.p),
                    reinterpret_cast<cufftComplex *>(band_.p), CUFFT_FORWARD));
}

void StreamGridder::predict_begin(const void *dirty) {
  require(dirty != nullptr, "dirty is required");
  CK(cudaSetDevice(cx_.device));
  for (auto &b : batch_) b.rows = 0;  // rows added since the last finish are discarded
  const size_t npix = gp_.nx * gp_.ny, dsz = a_.dirty_type == WSG_F64 ? 8 : 4;
  const void *din = cx_.stage_in(dirty, npix * dsz, cx_.b_out);
  double *img = reinterpret_cast<double *>(img_.p);
  const int nb = launch_blocks(npix, 256);
  if (a_.dirty_type == WSG_F64)
    k_load_image<double><<<nb, 256, 0, cx_.stream>>>(npix, (const double *)din, img, 0);
  else
    k_load_image<float><<<nb, 256, 0, cx_.stream>>>(npix, (const float *)din, img, 0);
  cuda_check(cudaGetLastError(), "k_load_image launch");
  if (dbl_)
    predict_begin_t<double>(img);
  else
    predict_begin_t<float>(img);
  mode_ = 2;
}

template <typename R>
void StreamGridder::predict_t(const Staged &s, size_t nrows, void *vis_dev) {
  wsg_args ac = a_;
  ac.nrows = nrows;
  ac.uvw = s.uvw;
  ac.wgt = s.wgt;
  ac.mask = s.mask;
  GridPlan g = gp_;
  if (!cx_.prepare<R>(ac, s, false, vis_dev, g)) return;
  cudaStream_t st = cx_.stream;
  const size_t cs = 2 * sizeof(R);
  const TileLayout tl = make_layout(g.T, g.kernel.W);
  const size_t smem = GridKernels<R>::smem_bytes(tl, g.kernel.W, false);
  int *counter = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 2048);
  int *d_nch = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 1024);
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 3072);
  CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  CK(cudaMemsetAsync(counter, 0, sizeof(int), st));
  GridArgs ga{};
  ga.err = d_err;
  ga.rec = cx_.b_rec.p;
  ga.chunk_start = reinterpret_cast<const int *>(cx_.b_chunks.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(g.nvis);
  ga.grid = band_.p;
  ga.P = int(g.nplanes);
  ga.pb0 = 0;
  ga.pb1 = int(g.nplanes);
  ga.tl = tl;
  ga.sb = GridKernels<R>::SB;
  ga.vis_out = vis_dev;
  ga.vis_double = a_.vis_type == WSG_C128;
  ga.first_pass = ga.last_pass = 1;
  const bool need_acc = GridKernels<R>::groups(g.kernel.W) > 1;
  ga.acc = need_acc ? cx_.b_acc.ensure(g.nvis * cs) : nullptr;
  if (need_acc) CK(cudaMemsetAsync(ga.acc, 0, g.nvis * cs, st));
  GridKernels<R>::dispatch(g.kernel.W, false, cx_.num_sms, smem, st, ga, make_geom(g),
                           make_kernel<R>(g.poly));
  if (need_acc) {
    k_finalize<R><<<launch_blocks(g.nvis, 256), 256, 0, st>>>(int(g.nvis), cx_.b_rec.p, ga.acc,
                                                             vis_dev, ga.vis_double, 0);
    cuda_check(cudaGetLastError(), "k_finalize launch");
  }
}

void StreamGridder::predict(size_t nrows, const double *uvw, void *vis, const void *wgt,
                            const uint8_t *mask) {
  require(mode_ == 2, "predict() before predict_begin()");
  require(uvw && vis, "uvw and vis are required");
  if (nrows == 0) return;
  CK(cudaSetDevice(cx_.device));
  Slot &sl = slots_[k_++ & 1];
  Staged s = stage(sl, nrows, uvw, nullptr, wgt, mask);
  const size_t vbytes = nrows * a_.nchan * (a_.vis_type == WSG_C128 ? 16 : 8);
  const bool vdev = is_device_pointer(vis);
  void *vout = vdev ? vis : vout_.ensure(vbytes);
  CK(cudaMemsetAsync(vout, 0, vbytes, cx_.stream));
  if (dbl_)
    predict_t<double>(s, nrows, vout);
  else
    predict_t<float>(s, nrows, vout);
  CK(cudaEventRecord(sl.done, cx_.stream));
  if (!vdev) {
    CK(cudaMemcpyAsync(vis, vout, vbytes, cudaMemcpyDeviceToHost, cx_.stream));
    CK(cudaStreamSynchronize(cx_.stream));
  }
}

void StreamGridder::stats(wsg_stats &o) const {
  const GridPlan &g = gp_;
  std::memset(&o, 0, sizeof(o));
  o.nchan = a_.nchan;
  o.nu = g.nu;
  o.nv = g.nv;
  o.nplanes = g.nplanes;
  o.supp = g.kernel.W;
  o.plane_batch = g.nplanes;
  o.band_rows = g.band_rows;
  o.degree = g.poly.D;
  o.sigma = g.ofactor;
  o.beta = g.kernel.beta;
  o.e0 = g.kernel.e0;
  o.kernel_err = g.kernel.err;
  o.wmin = g.wmin_d;
  o.wmax = g.wmax_d;
  o.dw = g.dw;
  o.nshift = g.nshift;
  o.precision = g.fp32 ? WSG_PREC_MIXED : WSG_PREC_FP64;
  o.device_bytes = band_.n + H_.n + img_.n + fftwork_.n;
  o.kernel_launches = g_kernel_launches.load();
}

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
// the array may move and the lookup is repeated.  That first call should come
// before any stream capture.  The call synchronises its stream while it runs
// (it reads the visibility scan's statistics back to plan the grid).  All
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
    const size_t smem = GridKernels<float>::smem_bytes(tl, gp.kernel.W, true);
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
    ga.sb = GridKernels<float>::SB;
    const ColArgs ca = make_col(gp, P, d_tw, band, H);
    for (size_t pb0 = 0; pb0 < gp.nplanes; pb0 += P) {
      const size_t npl = std::min(P, gp.nplanes - pb0);
      cuda_check(cudaMemsetAsync(band, 0, gp.band_rows * P * gp.nv * 8, stream), "band clear");
      cuda_check(cudaMemsetAsync(counter, 0, sizeof(int), stream), "counter clear");
      ga.pb0 = int(pb0);
      ga.pb1 = int(pb0 + npl);
      GridKernels<float>::dispatch(gp.kernel.W, true, nsm, smem, stream, ga, g, kc);
      row_fft_f(logMv, band, (long long)(gp.band_rows * P), d_twv, +1, stream);
      ColKernels<float>::run(gp.logM, true, ca, int(npl), stream, d_err);
      ScreenArgs sa = make_screen(gp, d_cf, cc, P);
      sa.pb0 = int(pb0);
      sa.npl = int(npl);
      const dim3 sg = screen_grid(gp);
      k_screen_add<float><<<sg, 256, 0, stream>>>(sa, H, img, nullptr, 0);
      cuda_check(cudaGetLastError(), "k_screen_add launch");
      g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
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
