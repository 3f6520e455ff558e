// Host-side pieces shared by libwsg's translation units: error checks, the
// conversions from a grid plan to kernel arguments, and the launchers of the
// spread / interpolation, pruned u-transform and w-screen kernels, which are
// compiled once, in wsg_launch.cu.  One translation unit per subsystem:
// wsg_context.cu (contexts and the ms2dirty / dirty2ms drivers), wsg_tuned.cu
// (the tuned schedule), wsg_plan.cu (plans), wsg_stream.cu (streams),
// wsg_weights.cu (imaging weights), wsg_autotune.cu, wsg_gridder.cu (the
// stateful gridder) and wsg_noalloc.cu (the allocation-free entry point).
#pragma once

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
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "wsg_context.h"
#include "wsg_device.cuh"

namespace wsg {

// libwsg kernels launched by this process (cuFFT and CUB kernels excluded).
extern std::atomic<size_t> g_kernel_launches;

void cufft_check(cufftResult r, const char *what);
#define CK(x) cuda_check((x), #x)
#define CF(x) cufft_check((x), #x)

// An integer from the environment (tests and debugging), else dflt.
int env_int(const char *name, int dflt);
// Bin tile edge asked of the planner.
int default_tile(bool fp32);

// ------------------------------------------------------------- planning

inline DevGeom make_geom(const GridPlan &g) {
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

inline TileLayout make_layout(int T, int W) {
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
inline void clear_outside_columns(void *band, size_t rows, size_t nv, size_t ny, size_t cs,
                           cudaStream_t st) {
  if (nv <= ny) return;
  cuda_check(cudaMemset2DAsync(static_cast<char *>(band) + (ny / 2) * cs, nv * cs, 0,
                               (nv - ny) * cs, rows, st),
             "cudaMemset2DAsync");
}

// Half-width in cells of the v columns the spread can write ([0, Lv] and
// [nv - Lv, nv)): the largest |v| plus half a kernel and a margin, as the u
// band (set_band); -1 when that covers the whole row.
inline long band_v_halfwidth(const GridPlan &g) {
  const double L = std::ceil(g.vmax * g.py * double(g.nv) + 0.5 * g.kernel.W + 2.0);
  if (!(L >= 0) || 2.0 * L + 1.0 >= double(g.nv)) return -1;
  return long(L);
}

inline int launch_blocks(size_t n, int threads) {
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

inline ScreenArgs make_screen(const GridPlan &g, const double *d_cf, const ChebCorr &cc, size_t P) {
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

inline ColArgs make_col(const GridPlan &g, size_t P, const void *tw, void *band, void *H) {
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
// columns; for the whole-grid screens (GridPlan::ucufft), 32 image columns
// by 8 image rows a block.
inline dim3 screen_grid(const GridPlan &g) {
  if (g.ucufft) return dim3(unsigned((g.ny + 31) / 32), unsigned((g.nx + 7) / 8));
  return dim3(unsigned(size_t(g.K) * ((g.hseg() + 31) / 32)), unsigned((g.ny + 31) / 32));
}

// Twiddle tables of the pruned u transform (wsg_context.cu).
size_t col_table_entries(size_t M, size_t K);
std::vector<double> col_twiddle_table(size_t M, size_t nu, size_t K);

// ------------------------------------------------------------- launchers
//
// Defined in wsg_launch.cu for R = float and double.

// Records staged per sub-batch by the spread / interpolation kernels.
template <typename R>
constexpr int grid_sb() {
  return sizeof(R) == 4 ? 256 : 64;
}
// Shared memory of a spread / interpolation CTA for this tile layout.
template <typename R>
size_t grid_smem_bytes(const TileLayout &tl, int W, bool spread);
// Warps that share one record.
template <typename R>
int grid_groups(int W);
// Whether the interpolation of one plane pass needs the per-record
// accumulator (and k_finalize): when a record is shared by some but not
// all of a CTA's warps (all warps sharing it add their sums in the kernel).
template <typename R>
bool grid_needs_acc(int W);
// One persistent spread (or interpolation) launch over the chunks.
template <typename R>
void grid_dispatch(int W, bool spread, int nsm, size_t smem, cudaStream_t st, const GridArgs &a,
                   const DevGeom &g, const DevKernel<R> &kc);
// The pruned u transform of npl planes (bwd: band to image columns).  err:
// the device error word (bit 2: a staged copy did not complete), or nullptr
// to stay with the plain loads.
template <typename R>
void col_run(int logM, bool bwd, const ColArgs &a, int npl, cudaStream_t st, int *err = nullptr);
// The w-screens (grid: screen_grid).
template <typename R>
void launch_screen_add(dim3 grid, cudaStream_t st, const ScreenArgs &s, const void *H,
                       double *img, void *out, int out_mode);
template <typename R>
void launch_screen_put(dim3 grid, cudaStream_t st, const ScreenArgs &s, const void *img,
                       int in_f32, void *H);
// The screens on the whole grid (GridPlan::ucufft): G is the grid layout
// [nu][P][nv] at the pass's first plane (grid: screen_grid).
template <typename R>
void launch_screen_add_grid(dim3 grid, cudaStream_t st, const ScreenArgs &s, const void *G,
                            double *img, void *out, int out_mode);
template <typename R>
void launch_screen_put_grid(dim3 grid, cudaStream_t st, const ScreenArgs &s, const void *img,
                            int in_f32, void *G);

// ------------------------------------------------------------ the driver

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

}  // namespace wsg
