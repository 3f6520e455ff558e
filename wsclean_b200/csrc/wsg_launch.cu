// Launchers of the spread / interpolation kernels (dispatched over the
// support W), the pruned u transforms (over log2 M, with their staged
// forms) and the w-screens: the one translation unit that compiles them.

#include "wsg_host.cuh"

namespace wsg {

namespace {

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

// Whether `extra` bytes of shared memory fit beside a CTA's `base` bytes
// without lowering the CTAs an SM holds (228 KB a SM, 227 KB a CTA, 1 KB
// reserved a CTA).
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
    // a CTA of one column (M = 8192 in FP32, 4096 in FP64) waits on each of
    // its copies with nothing else to do: the plain kernel is faster there
    // (config 5's forward transform: 30 ms plain, 65 ms staged)
    if (NB < 2) return false;
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
    // resident CTAs of each instantiation at these sizes, memoised (the
    // query is a driver call, and plans enqueue while a stream is captured)
    static std::mutex mu;
    static std::map<std::tuple<size_t, size_t, int>, std::pair<int, int>> memo;
    int dev0 = 0;
    cuda_check(cudaGetDevice(&dev0), "cudaGetDevice");
    const auto key = std::make_tuple(base, extra, dev0);
    int n0 = 0, n1 = 0;
    smem_attr(k0, base);
    if (base + extra <= 227 * 1024) smem_attr(k1, base + extra);
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = memo.find(key);
      if (it != memo.end()) {
        n0 = it->second.first;
        n1 = it->second.second;
      } else {
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n0, k0, Cfg::THREADS, base),
                   "occupancy");
        if (base + extra <= 227 * 1024)
          cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n1, k1, Cfg::THREADS,
                                                                   base + extra),
                     "occupancy");
        memo[key] = std::make_pair(n0, n1);
      }
    }
    if (n0 < 1) return false;
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
    if constexpr (sizeof(R) == 8 && LOGM == 13) {
      // FP64 8192-point transforms: one column a CTA, the last stage's
      // twiddles from global memory
      const size_t smem = ColBig<M>::bytes();
      auto *kern = bwd ? k_ucol_bwd_big<LOGM> : k_ucol_fwd_big<LOGM>;
      smem_attr(kern, smem);
      dim3 grid(a.ny, npl);
      kern<<<grid, ColBig<M>::TPF, smem, st>>>(a);
      cuda_check(cudaGetLastError(), bwd ? "k_ucol_bwd_big launch" : "k_ucol_fwd_big launch");
      g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    } else {
      run1s<LOGM>(bwd, a, npl, st, err);
    }
  }
  template <int LOGM>
  static void run1s(bool bwd, const ColArgs &a, int npl, cudaStream_t st, int *err) {
    constexpr int M = 1 << LOGM;
    using Cfg = ColCfg<R, M>;
    if (bwd && run_tma<LOGM>(a, npl, st, err)) return;
    if (!bwd && run_bulk<LOGM>(a, npl, st, err)) return;
    if constexpr (sizeof(R) == 4 && Cfg::NB == 1) {
      // one-column CTAs: two columns a CTA, loaded or stored together
      const size_t smem = (2 * size_t(FftBuf<M>::value) + M) * 2 * sizeof(R);
      auto *kern = bwd ? k_ucol_bwd_pair<R, LOGM> : k_ucol_fwd_pair<R, LOGM>;
      smem_attr(kern, smem);
      dim3 grid((a.ny + 1) / 2, npl);
      kern<<<grid, Cfg::THREADS, smem, st>>>(a);
      cuda_check(cudaGetLastError(), bwd ? "k_ucol_bwd_pair launch" : "k_ucol_fwd_pair launch");
      g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
      return;
    }
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
      case 13: run1<13>(bwd, a, npl, st, err); break;
      default: throw std::runtime_error("unsupported pruned FFT length");
    }
  }
};

}  // namespace

template <typename R>
size_t grid_smem_bytes(const TileLayout &tl, int W, bool spread) {
  return GridKernels<R>::smem_bytes(tl, W, spread);
}
template <typename R>
int grid_groups(int W) {
  return GridKernels<R>::groups(W);
}
template <typename R>
bool grid_needs_acc(int W) {
  const int ng = GridKernels<R>::groups(W);
  return ng > 1 && ng < GridKernels<R>::NWARP;
}
template <typename R>
void grid_dispatch(int W, bool spread, int nsm, size_t smem, cudaStream_t st, const GridArgs &a,
                   const DevGeom &g, const DevKernel<R> &kc) {
  static_assert(GridKernels<R>::SB == grid_sb<R>(), "sub-batch size");
  GridKernels<R>::dispatch(W, spread, nsm, smem, st, a, g, kc);
}
template <typename R>
void col_run(int logM, bool bwd, const ColArgs &a, int npl, cudaStream_t st, int *err) {
  ColKernels<R>::run(logM, bwd, a, npl, st, err);
}
template <typename R>
void launch_screen_add(dim3 grid, cudaStream_t st, const ScreenArgs &s, const void *H,
                       double *img, void *out, int out_mode) {
  k_screen_add<R><<<grid, 256, 0, st>>>(s, H, img, out, out_mode);
  cuda_check(cudaGetLastError(), "k_screen_add launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
template <typename R>
void launch_screen_put(dim3 grid, cudaStream_t st, const ScreenArgs &s, const void *img,
                       int in_f32, void *H) {
  k_screen_put<R><<<grid, 256, 0, st>>>(s, img, in_f32, H);
  cuda_check(cudaGetLastError(), "k_screen_put launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

template <typename R>
void launch_screen_add_grid(dim3 grid, cudaStream_t st, const ScreenArgs &s, const void *G,
                            double *img, void *out, int out_mode) {
  k_screen_add_grid<R><<<grid, 256, 0, st>>>(s, G, img, out, out_mode);
  cuda_check(cudaGetLastError(), "k_screen_add_grid launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
template <typename R>
void launch_screen_put_grid(dim3 grid, cudaStream_t st, const ScreenArgs &s, const void *img,
                            int in_f32, void *G) {
  k_screen_put_grid<R><<<grid, 256, 0, st>>>(s, img, in_f32, G);
  cuda_check(cudaGetLastError(), "k_screen_put_grid launch");
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

#define WSG_LAUNCHERS(R)                                                                     \
  template size_t grid_smem_bytes<R>(const TileLayout &, int, bool);                         \
  template int grid_groups<R>(int);                                                          \
  template bool grid_needs_acc<R>(int);                                                      \
  template void grid_dispatch<R>(int, bool, int, size_t, cudaStream_t, const GridArgs &,     \
                                 const DevGeom &, const DevKernel<R> &);                     \
  template void col_run<R>(int, bool, const ColArgs &, int, cudaStream_t, int *);            \
  template void launch_screen_add<R>(dim3, cudaStream_t, const ScreenArgs &, const void *,  \
                                     double *, void *, int);                                 \
  template void launch_screen_put<R>(dim3, cudaStream_t, const ScreenArgs &, const void *,  \
                                     int, void *);                                           \
  template void launch_screen_add_grid<R>(dim3, cudaStream_t, const ScreenArgs &,            \
                                          const void *, double *, void *, int);             \
  template void launch_screen_put_grid<R>(dim3, cudaStream_t, const ScreenArgs &,            \
                                          const void *, int, void *);
WSG_LAUNCHERS(float)
WSG_LAUNCHERS(double)
#undef WSG_LAUNCHERS

}  // namespace wsg
