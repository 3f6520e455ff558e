// Host-side kernel mathematics and grid-parameter choice for libwsg.
//
// Reference counterparts (external/wgridder/ducc0/):
//   es_phi               <- esknew                   math/gridding_kernel.cc:1538-1543
//   available_kernels    <- getAvailableKernels      math/gridding_kernel.h:397-421
//   fit_poly_kernel      <- getCoeffs/PolynomialKernel math/gridding_kernel.cc:28-75
//   KernelTransform      <- GLFullCorrection/corfunc math/gridding_kernel.h:74-126
//   choose_grid          <- Params::getNuNv + countRanges' plane placement
//                           wgridder/wgridder.h:1503-1576, :690-699
// The kernel table itself (es_kernel_db.inc) is generated by
// wsclean_b200/kernel_db.py from an aliasing-error minimisation, and the
// polynomial fit, quadrature and cost model are this library's own.
#include <algorithm>
#include <cmath>
#include <limits>
#include <tuple>
#include <utility>
#include <vector>

#include "wsg_internal.h"

namespace wsg {

namespace {

struct TableRow {
  int W;
  double sigma, err1d, beta, e0;
};

const TableRow kTable[] = {
#include "es_kernel_db.inc"
};

// FP32 arithmetic (kernel values, grid accumulation, FFT) limits the
// achievable accuracy; kernels are never credited with less than this.
constexpr double kFp32ErrFloor = 3e-7;
constexpr int kMaxWFp32 = 8;

// Gauss-Legendre nodes/weights on [-1,1] by Newton iteration on P_n.
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
  x.resize(n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    double dp = 0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = 0.0;
      for (int j = 1; j <= n; ++j) {
        double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      double dz = p0 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Solves the (n x n) system A c = y in long double, partial pivoting.
bool solve_ld(std::vector<long double> A, std::vector<long double> y, int n,
              std::vector<long double> &c) {
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::fabs((double)A[r * n + col]) > std::fabs((double)A[piv * n + col]))
        piv = r;
    if (A[piv * n + col] == 0) return false;
    if (piv != col) {
      for (int k = 0; k < n; ++k) std::swap(A[col * n + k], A[piv * n + k]);
      std::swap(y[col], y[piv]);
    }
    for (int r = col + 1; r < n; ++r) {
      long double f = A[r * n + col] / A[col * n + col];
      if (f == 0) continue;
      for (int k = col; k < n; ++k) A[r * n + k] -= f * A[col * n + k];
      y[r] -= f * y[col];
    }
  }
  c.assign(n, 0);
  for (int r = n - 1; r >= 0; --r) {
    long double s = y[r];
    for (int k = r + 1; k < n; ++k) s -= A[r * n + k] * c[k];
    c[r] = s / A[r * n + r];
  }
  return true;
}

}  // namespace

double es_phi(double t, int W, double beta, double e0) {
  double s = (1.0 - t) * (1.0 + t);
  if (s < 0) return 0.0;
  return std::exp(beta * W * (std::pow(s, e0) - 1.0));
}

std::vector<KernelSpec> available_kernels(double epsilon, int ndim, bool fp32,
                                          double sigma_min, double sigma_max) {
  std::vector<KernelSpec> out;
  const int wmax = fp32 ? kMaxWFp32 : kMaxW;
  for (int W = 4; W <= wmax; ++W) {
    const TableRow *best = nullptr;
    for (const auto &r : kTable) {
      if (r.W != W || r.sigma < sigma_min - 1e-9 || r.sigma > sigma_max + 1e-9)
        continue;
      double err = ndim * r.err1d;
      if (fp32) err = std::max(err, kFp32ErrFloor);
      if (err > epsilon) continue;
      if (!best || r.sigma < best->sigma) best = &r;
    }
    if (best) {
      double err = ndim * best->err1d;
      if (fp32) err = std::max(err, kFp32ErrFloor);
      out.push_back({W, best->sigma, err, best->beta, best->e0});
    }
  }
  require(!out.empty(),
          "no appropriate kernel found for epsilon=" + std::to_string(epsilon) +
              (fp32 ? " in mixed precision (use FP64 for tighter epsilon)" : ""));
  return out;
}

PolyKernel fit_poly_kernel(const KernelSpec &k, double target_err) {
  const int W = k.W;
  PolyKernel best;
  // Test points: 97 per piece, including the piece edges.
  const int ntest = 97;
  // the device evaluates degree W+4 (lower-degree fits are zero-padded)
  for (int D = W + 1; D <= std::min(kMaxDeg, W + 4); ++D) {
    const int n = D + 1;
    std::vector<long double> A(n * n);
    std::vector<double> xs(n);
    for (int i = 0; i < n; ++i) {  // Chebyshev points of the first kind
      xs[i] = std::cos(M_PI * (i + 0.5) / n);
      long double p = 1;
      for (int j = 0; j < n; ++j) {
        A[i * n + j] = p;
        p *= xs[i];
      }
    }
    PolyKernel pk;
    pk.W = W;
    pk.D = D;
    pk.coef.assign((size_t)n * W, 0.0);
    double maxerr = 0;
    bool ok = true;
    for (int piece = 0; piece < W; ++piece) {
      std::vector<long double> y(n), c;
      for (int i = 0; i < n; ++i) {
        double t = -1.0 + (2.0 * piece + 1.0 + xs[i]) / W;
        y[i] = es_phi(t, W, k.beta, k.e0);
      }
      if (!solve_ld(A, y, n, c)) {
        ok = false;
        break;
      }
      for (int j = 0; j < n; ++j) pk.coef[(size_t)j * W + piece] = (double)c[j];
      for (int s = 0; s < ntest; ++s) {
        double x = -1.0 + 2.0 * s / (ntest - 1);
        double t = -1.0 + (2.0 * piece + 1.0 + x) / W;
        double v = 0;
        for (int j = n - 1; j >= 0; --j) v = v * x + pk.coef[(size_t)j * W + piece];
        maxerr = std::max(maxerr, std::fabs(v - es_phi(t, W, k.beta, k.e0)));
      }
    }
    if (!ok) continue;
    pk.max_err = maxerr;
    best = pk;
    if (maxerr <= target_err) break;
  }
  if (best.W == 0) throw std::runtime_error("kernel polynomial fit failed");
  return best;
}

KernelTransform::KernelTransform(const KernelSpec &k) : W_(k.W) {
  // Composite Gauss-Legendre on [0,1]: 8 uniform panels on [0,1/2], then 40
  // panels halving toward t=1, 16 nodes each.  phi has a branch point at t=1;
  // uniform panels resolve it only to ~1e-7 (W=4) .. 1e-11 (W=8) relative,
  // the graded mesh to ~1e-15 for |nu| <= 1.
  std::vector<double> gx, gw;
  gauss_legendre(16, gx, gw);
  std::vector<double> edges;
  for (int i = 0; i <= 8; ++i) edges.push_back(0.0625 * i);
  double a = 0.5;
  for (int i = 0; i < 40; ++i) {
    a = 1.0 - 0.5 * (1.0 - a);
    edges.push_back(a);
  }
  edges.push_back(1.0);
  for (size_t p = 0; p + 1 < edges.size(); ++p) {
    double lo = edges[p], h = edges[p + 1] - edges[p];
    for (size_t i = 0; i < gx.size(); ++i) {
      double t = lo + 0.5 * h * (gx[i] + 1.0);
      t_.push_back(t);
      wphi_.push_back(0.5 * h * gw[i] * es_phi(t, k.W, k.beta, k.e0));
    }
  }
}

double KernelTransform::operator()(double nu) const {
  // (W/2) * 2 * int_0^1 phi(t) cos(pi W nu t) dt
  double s = 0;
  const double f = M_PI * W_ * nu;
  for (size_t i = 0; i < t_.size(); ++i) s += wphi_[i] * std::cos(f * t_[i]);
  return W_ * s;
}

double ChebCorr::operator()(double v) const {
  double x = 2.0 * (v * v) / ymax - 1.0;
  double b1 = 0, b2 = 0;  // Clenshaw
  for (int j = n - 1; j >= 1; --j) {
    double b0 = 2.0 * x * b1 - b2 + c[j];
    b2 = b1;
    b1 = b0;
  }
  return x * b1 - b2 + c[0];
}

ChebCorr fit_cheb_corr(const KernelTransform &tr, double vmax) {
  ChebCorr best;
  double ymax = std::max(vmax * vmax, 1e-30);
  // check points (fixed) with their exact values
  const int ntest = 65;
  std::vector<double> vt(ntest), ref(ntest);
  for (int s = 0; s < ntest; ++s) {
    vt[s] = std::sqrt(ymax * s / (ntest - 1.0));
    ref[s] = tr.corfunc(vt[s]);
  }
  for (int n = 12; n <= kMaxCheb; n += 6) {
    ChebCorr cc;
    cc.ymax = ymax;
    cc.n = n;
    cc.c.assign(n, 0.0);
    std::vector<double> fv(n);
    for (int k = 0; k < n; ++k) {
      double xk = std::cos(M_PI * (k + 0.5) / n);
      fv[k] = tr.corfunc(std::sqrt(0.5 * (xk + 1.0) * ymax));
    }
    for (int j = 0; j < n; ++j) {
      double s = 0;
      for (int k = 0; k < n; ++k) s += fv[k] * std::cos(M_PI * j * (k + 0.5) / n);
      cc.c[j] = (j == 0 ? 1.0 : 2.0) * s / n;
    }
    double maxrel = 0;
    for (int s = 0; s < ntest; ++s)
      maxrel = std::max(maxrel, std::fabs(cc(vt[s]) - ref[s]) / std::fabs(ref[s]));
    cc.max_rel_err = maxrel;
    bool better = best.n == 0 || maxrel < best.max_rel_err;
    if (better) best = cc;
    if (maxrel < 1e-14 || !better) break;
  }
  return best;
}

// Grid height for the v transform (cuFFT): the smallest n' >= n with prime
// factors 2, 3, 5, 7, unless 2^a or 3 * 2^a is at most 8% longer -- cuFFT
// transforms those fastest per point on the B200 (6144 takes 7% less time
// than 6000 = 2^4 * 3 * 5^3 for 2.4% more points).
size_t good_size_v(size_t n) {
  n = std::max<size_t>(n, 2);
  size_t smooth = 2 * n;
  for (size_t f2 = 1; f2 < smooth; f2 *= 2)
    for (size_t f3 = f2; f3 < smooth; f3 *= 3)
      for (size_t f5 = f3; f5 < smooth; f5 *= 5)
        for (size_t f7 = f5; f7 < smooth; f7 *= 7)
          if (f7 >= n) smooth = std::min(smooth, f7);
  size_t p23 = ~size_t(0);
  for (size_t p = 1; p < 4 * n; p *= 2) {
    if (p >= n) p23 = std::min(p23, p);
    if (3 * p >= n) p23 = std::min(p23, 3 * p);
  }
  return (double(p23) <= 1.08 * double(smooth)) ? p23 : smooth;
}

namespace {

int ceil_log2(uint64_t v) {
  int b = 0;
  while ((uint64_t(1) << b) < v) ++b;
  return b;
}

// Occupied u band for a grid size: rows within W/2+2 cells of the largest
// |u| (in cells) hold all footprints.
void set_band(GridPlan &g) {
  double umax_cells = g.umax * g.px * double(g.nu);
  double L = std::ceil(umax_cells + 0.5 * g.kernel.W + 2.0);
  if (!(L >= 0) || 2.0 * L + 1.0 >= double(g.nu)) {
    g.band_full = true;
    g.Lu = g.nu / 2;
    g.band_rows = g.nu;
  } else {
    g.band_full = false;
    g.Lu = size_t(L);
    g.band_rows = 2 * g.Lu + 1;
  }
}

// Every u row of the grid (the library-FFT layout, GridPlan::ucufft).
void set_full_band(GridPlan &g) {
  g.band_full = true;
  g.Lu = g.nu / 2;
  g.band_rows = g.nu;
}

}  // namespace

// Shared memory of one spread / interpolation CTA: the W-plane tile of
// (T + W - 1)^2 cells (odd row stride, plane stride 8 mod 32, real and
// imaginary parts) and 8 warps' record staging (the layout of the device
// kernels, GridKernels::smem_bytes).
size_t tile_smem_bytes(int T, int W, bool fp32) {
  const size_t rs = fp32 ? 4 : 8;
  const size_t S = size_t(T + W - 1), RS = S | 1;
  size_t PS = S * RS;
  PS += ((8 - (PS % 32)) + 32) % 32;
  const size_t kst = fp32 ? ((3 * size_t(W) + 3) & ~size_t(3)) : ((3 * size_t(W) + 1) & ~size_t(1));
  const size_t stage = rs * (32 * kst + 64) + 128;
  return ((rs * 2 * size_t(W) * PS + 15) & ~size_t(15)) + 8 * stage;
}

// nu = K * 2^m with 2^m >= 2L+1, so that the occupied u band fits one pruned
// FFT of length 2^m, 256 <= 2^m <= 8192 (or K = 1, 2^m = nu when the band
// covers the grid); the smallest such nu >= n0.
bool pick_nu(double n0, double umax_px, int W, size_t &nu, int &logM, int &K) {
  size_t best = ~size_t(0);
  for (int m = 8; m <= 13; ++m) {
    const size_t M = size_t(1) << m;
    const size_t k = std::max<size_t>(1, size_t(std::ceil(n0 / double(M))));
    const size_t n = k * M;
    const double L = std::ceil(umax_px * double(n) + 0.5 * W + 2.0);
    const bool full = 2.0 * L + 1.0 >= double(n);
    if (full ? (k != 1) : (2.0 * L + 1.0 > double(M))) continue;
    if (n < best) {
      best = n;
      nu = n;
      logM = m;
      K = int(k);
    }
  }
  return best != ~size_t(0);
}

void choose_grid(GridPlan &g, double sigma_min, double sigma_max, int tile, bool pow2_v) {
  require(g.nx % 2 == 0, "nx_dirty must be even");
  require(g.ny % 2 == 0, "ny_dirty must be even");
  require(g.eps > 0, "epsilon must be positive");
  require(g.px > 0, "pixsize_x must be positive");
  require(g.py > 0, "pixsize_y must be positive");
  // n-1 range over the image corners (and axes crossings), as the reference
  // does in getNuNv (wgridder.h:1507-1525).
  double xmin = g.lshift - 0.5 * g.nx * g.px, xmax = xmin + (g.nx - 1) * g.px;
  double ymin = g.mshift - 0.5 * g.ny * g.py, ymax = ymin + (g.ny - 1) * g.py;
  std::vector<double> xe{xmin, xmax}, ye{ymin, ymax};
  if (xmin * xmax < 0) xe.push_back(0.0);
  if (ymin * ymax < 0) ye.push_back(0.0);
  g.nm1min = 1e300;
  g.nm1max = -1e300;
  for (double xc : xe)
    for (double yc : ye) {
      double r2 = xc * xc + yc * yc;
      double nv = (r2 <= 1.0) ? std::sqrt(1.0 - r2) - 1.0 : -std::sqrt(r2 - 1.0) - 1.0;
      g.nm1min = std::min(g.nm1min, nv);
      g.nm1max = std::max(g.nm1max, nv);
    }
  g.lmshift = (g.lshift != 0) || (g.mshift != 0);
  g.nshift = g.do_w ? -0.5 * (g.nm1max + g.nm1min) : 0.0;
  g.shifting = g.lmshift || (g.nshift != 0);
  double nmax = std::max(std::fabs(g.nm1max + g.nshift), std::fabs(g.nm1min + g.nshift));
  if (g.do_w) require(nmax > 0, "image too small for w-gridding (n-1 range is zero)");

  auto cands = available_kernels(g.eps, g.do_w ? 3 : 2, g.fp32, sigma_min, sigma_max);
  // Cost model (seconds), per w plane: band grid traffic (zero, spread flush,
  // v transform), the pruned u transform (band in, image rows out), the
  // w-screen pass; plus the spreading work nvis * W^3.
  const double cs = g.fp32 ? 8.0 : 16.0;
  const double hbm = 5.0e12;
  const double c_cell = g.fp32 ? 1.0e-13 : 6.0e-13;
  const double c_fftpt = g.fp32 ? 1.5e-12 : 4.0e-12;
  const double umax_px = g.umax * g.px;
  double best = 1e300;
  KernelSpec bestk{};
  size_t bnu = 0, bnv = 0;
  int blogM = 0, bK = 1;
  bool bucufft = false;
  for (const auto &k : cands) {
    if (g.force_W && (k.W != g.force_W || std::fabs(k.sigma - g.force_sigma) > 1e-12)) continue;
    GridPlan t = g;
    t.kernel = k;
    t.ucufft = false;
    if (!pick_nu(g.nx * k.sigma, umax_px, k.W, t.nu, t.logM, t.K)) {
      if (pow2_v) continue;  // (the allocation-free path has no library FFT)
      t.nu = 2 * good_size_v(size_t(g.nx * k.sigma * 0.5) + 1);
      t.logM = 0;
      t.K = 1;
      t.ucufft = true;
    }
    t.nv = 2 * good_size_v(size_t(g.ny * k.sigma * 0.5) + 1);
    if (pow2_v) {
      size_t p2 = 256;
      while (p2 < size_t(g.ny * k.sigma) + 2) p2 *= 2;
      if (p2 > kPow2VMax) continue;  // beyond the shared-memory row FFT
      t.nv = p2;
    }
    set_band(t);
    if (t.ucufft) set_full_band(t);
    double planes = 1;
    if (g.do_w) {
      double of = std::min(double(t.nu) / g.nx, double(t.nv) / g.ny);
      double dw = 0.5 / of / nmax;
      planes = std::floor((g.wmax_d - g.wmin_d) / dw + k.W);
    }
    const double M = double(size_t(1) << t.logM);
    // (the library's column FFT transforms all nv columns, nu points each,
    // and moves the whole grid twice more)
    double per_plane = t.ucufft
        ? cs * (8.0 * t.band_rows * t.nv + 3.0 * g.nx * g.ny) / hbm +
              c_fftpt * t.nv * double(t.nu) * std::log2(double(t.nu)) / 148.0
        : cs * (4.0 * t.band_rows * t.nv + 1.0 * t.band_rows * g.ny + 3.0 * g.nx * g.ny) / hbm +
              c_fftpt * g.ny * t.K * M * t.logM / 148.0;
    double fft = planes * per_plane;
    double grid = double(g.nvis) * k.W * k.W * (g.do_w ? k.W : 1) * c_cell;
    double cost = fft + grid;
    if (cost < best) {
      best = cost;
      bestk = k;
      bnu = t.nu;
      bnv = t.nv;
      blogM = t.logM;
      bK = t.K;
      bucufft = t.ucufft;
    }
  }
  require(bnu > 0, "no grid size satisfies the pruned-FFT layout (image or band too large)");
  g.cost = best;
  g.kernel = bestk;
  g.nu = bnu;
  g.nv = bnv;
  g.logM = blogM;
  g.K = bK;
  g.ucufft = bucufft;
  g.ofactor = std::min(double(g.nu) / g.nx, double(g.nv) / g.ny);
  const int W = bestk.W;
  g.nsafe = (W + 1) / 2;
  g.ushift = W * (-0.5) + 1 + double(g.nu);
  g.vshift = W * (-0.5) + 1 + double(g.nv);
  g.maxiu0 = int(g.nu + g.nsafe) - W;
  g.maxiv0 = int(g.nv + g.nsafe) - W;
  require(g.nu >= size_t(2 * g.nsafe) && g.nv >= size_t(2 * g.nsafe), "grid too small");
  require(g.nu + size_t(g.nsafe) < 65535 && g.nv + size_t(g.nsafe) < 65535, "grid too large");
  if (g.do_w) {
    g.dw = 0.5 / g.ofactor / nmax;
    g.xdw = 1.0 / g.dw;
    g.nplanes = size_t((g.wmax_d - g.wmin_d) / g.dw + W);
    require(g.nplanes < (size_t(1) << 16), "too many w planes");
    g.wmin = (g.wmin_d + g.wmax_d) * 0.5 - 0.5 * (double(g.nplanes) - 1) * g.dw;
    g.wshift = g.dw - (0.5 * W * g.dw) - g.wmin;
  } else {
    g.dw = g.xdw = g.wmin = g.wshift = 0;
    g.nplanes = 1;
  }
  set_band(g);
  if (g.ucufft)
    set_full_band(g);
  else if (g.band_full)
    require(g.K == 1 && (size_t(1) << g.logM) == g.nu, "internal: full band needs K == 1");
  else
    require((size_t(1) << g.logM) >= g.band_rows, "internal: band exceeds the pruned FFT");
  double target = g.fp32 ? std::max(0.02 * g.kernel.err, 2e-8) : 0.02 * g.kernel.err;
  g.poly = fit_poly_kernel(g.kernel, target);

  // a tile row plus halo (T + W - 1 cells) is staged by one warp's lanes,
  // and the tile plus the warps' staging areas must fit in shared memory
  tile = std::max(1, std::min(tile, 33 - W));
  while (tile > 1 && tile_smem_bytes(tile, W, g.fp32) > kMaxSmemPerBlock) --tile;
  g.T = tile;
  g.ntu = int((g.nu + 1) / tile) + 1;
  g.ntv = int((g.nv + 1) / tile) + 1;
  g.nwmin = g.do_w ? int(g.nplanes) - W + 1 : 1;
  uint64_t nbins = uint64_t(g.ntu) * g.ntv * g.nwmin;
  int bin_bits = ceil_log2(nbins);
  require(bin_bits <= 30, "too many (tile, w-plane) bins for the sort keys");
  // the full in-tile position keeps the records of a bin in footprint order
  // (the spread accumulates in registers while the footprint repeats); when
  // it does not fit 31 bits beside the bin, the keys are 64-bit
  g.bin_bits = bin_bits;
  g.lbits = ceil_log2(uint64_t(tile));
  g.key_bits = bin_bits + 2 * g.lbits;
  g.wide_keys = g.key_bits > 31;
}

void limit_key_bits(GridPlan &g, int max_bits) {
  if (g.key_bits <= max_bits) return;
  g.lbits = std::max(0, std::min(g.lbits, (max_bits - 1 - g.bin_bits) / 2));
  g.key_bits = g.bin_bits + 2 * g.lbits;
  g.wide_keys = g.key_bits > 31;
}

std::vector<std::pair<int, double>> rank_kernels(const GridPlan &g, double sigma_min,
                                                 double sigma_max, int tile, size_t n) {
  std::vector<std::tuple<double, int, double>> all;
  for (const auto &k : available_kernels(g.eps, g.do_w ? 3 : 2, g.fp32, sigma_min, sigma_max)) {
    GridPlan t = g;
    t.force_W = k.W;
    t.force_sigma = k.sigma;
    try {
      choose_grid(t, sigma_min, sigma_max, tile);
    } catch (const std::exception &) {
      continue;
    }
    all.emplace_back(t.cost, k.W, k.sigma);
  }
  std::sort(all.begin(), all.end());
  std::vector<std::pair<int, double>> out;
  for (size_t i = 0; i < all.size() && out.size() < n; ++i)
    out.emplace_back(std::get<1>(all[i]), std::get<2>(all[i]));
  return out;
}

// ------------------------------------------------- tuned schedule choice

namespace {
// n-1 range over a rectangle of (l, m), corners and axis crossings
// (get_nminmax_rectangle, wgridder.cc:110-126)
std::pair<double, double> nm1_range(double x0, double x1, double y0, double y1) {
  std::vector<double> xs{x0, x1}, ys{y0, y1};
  if (x0 * x1 < 0) xs.push_back(0.0);
  if (y0 * y1 < 0) ys.push_back(0.0);
  double lo = 1e300, hi = -1e300;
  for (double x : xs)
    for (double y : ys) {
      const double r2 = x * x + y * y;
      const double n = (r2 <= 1.0) ? std::sqrt(1.0 - r2) - 1.0 : -std::sqrt(r2 - 1.0) - 1.0;
      lo = std::min(lo, n);
      hi = std::max(hi, n);
    }
  return {lo, hi};
}
}  // namespace

TuningChoice tuning_choice(size_t nx, size_t ny, double px, double py, double eps, bool do_w,
                           double cx, double cy, size_t nvis_all, double wmin, double wmax,
                           const uint64_t *hist) {
  TuningChoice out;
  out.wmin = wmin;
  out.wmax = wmax;
  if (!do_w || nx < 500 || ny < 500) return out;
  size_t total = 0;
  std::vector<size_t> acc(kTuningBins);
  for (int i = 0; i < kTuningBins; ++i) acc[i] = (total += size_t(hist[i]));
  if (total == 0 || !(wmax > wmin)) return out;
  // the reference's CPU cost model, in seconds: support from epsilon,
  // oversampling 1.5, a per-visibility gridding cost for its 4-wide SIMD
  // kernels, a per-plane FFT cost scaled from a 2048^2 reference transform,
  // and a per-call pass over all visibilities
  const int W = std::max(3, std::min(16, int(2.0 - std::log10(eps))));
  const double sigma = 1.5;
  std::vector<double> wb(kTuningBins + 1);
  for (int i = 0; i <= kTuningBins; ++i) wb[i] = wmin + i * (wmax - wmin) / kTuningBins;
  const double xmin = cx - 0.5 * nx * px, ymin = cy - 0.5 * ny * py;
  const double xmax = xmin + (nx - 1) * px, ymax = ymin + (ny - 1) * py;
  const auto full = nm1_range(xmin, xmax, ymin, ymax);
  const double dw = 1.0 / sigma / std::fabs(full.first - full.second);
  const int nvec = (W + 3) / 4;
  const double grid0 = 2.2e-10 * W * (W * nvec * 4 + (2 * nvec + 1) * (W + 3) * 4);
  const double nu = sigma * nx, nv = sigma * ny;
  const double ref = 2048.0;
  const double fft0 = double(nx) / ref * nv / ref * (std::log(nu * nv) / std::log(ref * ref)) *
                      0.0693 * 1.3;
  const double overhead = 4e-9 * double(nvis_all);
  const double planes_all = (wmax - wmin) / dw + W;
  if (planes_all <= 2 * W || grid0 * total > 2 * fft0 * planes_all) return out;

  double best = 1e300;
  int bnfx = 0, bnfy = 0, bcut = 0;
  for (int icut = 0; icut <= kTuningBins; ++icut) {
    const double wcut = wb[icut];
    const size_t nlo = icut == 0 ? 0 : acc[icut - 1];
    const size_t nhi = total - nlo;
    double cost = 1e300;
    int cfx = 0, cfy = 0;
    if (nhi > 0) {
      for (int fx = 1; fx < 8; ++fx)
        for (int fy = (fx == 1) ? 2 : 1; fy < 8; ++fy) {
          double planes = 0;
          for (int i = 0; i < fx; ++i)
            for (int j = 0; j < fy; ++j) {
              const auto r = nm1_range(xmin + i * (xmax - xmin) / fx, xmin + (i + 1) * (xmax - xmin) / fx,
                                       ymin + j * (ymax - ymin) / fy, ymin + (j + 1) * (ymax - ymin) / fy);
              const double fdw = 1.0 / sigma / std::fabs(r.first - r.second);
              planes += (wmax - wcut) / fdw + W;
            }
          const double nf = double(fx * fy);
          const double c = nf * double(nhi) * grid0 +
                           fft0 * planes / nf * std::log(nu * nv / nf) / std::log(nu * nv) +
                           nf * overhead;
          if (c < cost) {
            cost = c;
            cfx = fx;
            cfy = fy;
          }
        }
    } else {
      cost = 0;
    }
    if (icut != 0) {
      // the reference discounts the low part's transform when nothing is
      // above the cut (its FFT is then typically sparse)
      const double fudge = nhi == 0 ? 0.75 : 1.0;
      cost += fudge * fft0 * ((wcut - wmin) / dw + W) + grid0 * double(nlo) + overhead;
    }
    if (cost < best) {
      best = cost;
      bnfx = cfx;
      bnfy = cfy;
      bcut = icut;
    }
  }
  if (bcut == kTuningBins) return out;  // no facets: the plain operator
  out.nfx = bnfx;
  out.nfy = bnfy;
  out.icut = bcut;
  return out;
}

Facet tuning_facet(size_t nx, size_t ny, int nfx, int nfy, int ifx, int ify, double px, double py,
                   double cx, double cy) {
  size_t is = (nx + nfx - 1) / nfx, js = (ny + nfy - 1) / nfy;
  is += is % 2;
  js += js % 2;
  require(is <= nx && js <= ny, "bad facet step");
  Facet f;
  f.x0 = size_t(ifx) * is;
  f.x1 = std::min(size_t(ifx + 1) * is, nx);
  f.y0 = size_t(ify) * js;
  f.y1 = std::min(size_t(ify + 1) * js, ny);
  require(f.x0 + 32 <= f.x1 && f.x1 % 2 == 0, "bad facet x length");
  require(f.y0 + 32 <= f.y1 && f.y1 % 2 == 0, "bad facet y length");
  f.cx = cx + px * 0.5 * (double(f.x0 + f.x1) - double(nx));
  f.cy = cy + py * 0.5 * (double(f.y0 + f.y1) - double(ny));
  return f;
}

size_t plan_bytes(const GridPlan &g, size_t planes, bool gridding) {
  const size_t cs = g.fp32 ? 8 : 16;
  (void)gridding;
  // the whole-grid layout transforms and screens one grid in place
  if (g.ucufft) return planes * cs * g.band_rows * g.nv;
  // both directions keep the grid and its v transform apart, plus the
  // u-transformed rows
  return planes * cs * (2 * g.band_rows * g.nv + g.ny * g.hrow());
}

}  // namespace wsg
