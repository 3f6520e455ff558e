// Internal host-side declarations of libwsg (not part of the C ABI).
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace wsg {

constexpr double kSpeedOfLight = 299792458.0;  // wgridder.h:297
constexpr int kMaxW = 16;
constexpr int kMaxDeg = 24;
constexpr int kMaxCheb = 48;

// Thrown for invalid arguments (the reference's MR_assert); mapped to
// WSG_ERR_INVALID at the C ABI.
struct InvalidArgument : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct OutOfMemory : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct CufftError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void require(bool ok, const std::string &msg) {
  if (!ok) throw InvalidArgument(msg);
}

// One row of the generated ES kernel table.
struct KernelSpec {
  int W;
  double sigma;   // tabulated oversampling factor
  double err;     // error estimate for the requested dimensionality
  double beta;    // phi(t) = exp(beta*W*((1-t^2)^e0 - 1))
  double e0;
};

// ES kernel value phi(t), |t|<=1.
double es_phi(double t, int W, double beta, double e0);

// Candidate kernels: for every support W allowed by the precision, the
// smallest tabulated sigma in [sigma_min, sigma_max] whose error estimate
// (ndim * err1d, floored for FP32 arithmetic) is <= epsilon.  Throws
// InvalidArgument if none qualifies.
std::vector<KernelSpec> available_kernels(double epsilon, int ndim, bool fp32,
                                          double sigma_min, double sigma_max);

// W pieces of degree D in the local coordinate x in [-1,1]; piece k covers
// t in [-1+2k/W, -1+2(k+1)/W].  coef[j*W + k] multiplies x^j.
struct PolyKernel {
  int W = 0, D = 0;
  std::vector<double> coef;
  double max_err = 0;  // max |poly - phi| on a dense test grid
};
PolyKernel fit_poly_kernel(const KernelSpec &k, double target_err);

// Fourier transform of the kernel in grid-cell units,
// Phi(nu) = (W/2) int_{-1}^{1} phi(t) cos(pi W nu t) dt,
// by composite Gauss-Legendre quadrature (exact to FP64 rounding for
// |nu| <= 2).  The grid correction is 1/Phi.
class KernelTransform {
 public:
  explicit KernelTransform(const KernelSpec &k);
  double operator()(double nu) const;
  double corfunc(double nu) const { return 1.0 / (*this)(nu); }

 private:
  int W_;
  std::vector<double> t_, wphi_;
};

// Chebyshev interpolant of corfunc(v) as a function of y = v^2 on
// [0, ymax]; evaluated on the device by Clenshaw recurrence.
struct ChebCorr {
  double ymax = 0;
  int n = 0;  // number of coefficients
  std::vector<double> c;
  double max_rel_err = 0;
  double operator()(double v) const;
};
ChebCorr fit_cheb_corr(const KernelTransform &tr, double vmax);

// Half grid height for the v transform: the smallest 2,3,5,7-smooth n' >= n,
// or 2^a / 3 * 2^a when that is at most 8% longer (fastest in cuFFT).
size_t good_size_v(size_t n);

// Everything one ms2dirty/dirty2ms call needs to know, in FP64.
struct GridPlan {
  // inputs
  size_t nx = 0, ny = 0;
  double px = 0, py = 0;
  double eps = 0;
  bool do_w = true, fp32 = true, gridding = true;
  bool negate_v = false, divide_by_n = true;
  double lshift = 0, mshift = 0;
  // scan results
  size_t nvis = 0;
  double wmin_d = 0, wmax_d = 0, umax = 0, vmax = 0;
  // chosen kernel and grid
  KernelSpec kernel{};
  PolyKernel poly;
  size_t nu = 0, nv = 0;
  double ofactor = 0;
  double nm1min = 0, nm1max = 0, nshift = 0;
  bool lmshift = false, shifting = false;
  double wmin = 0, dw = 0, xdw = 0, wshift = 0;
  size_t nplanes = 1;
  int nsafe = 0, maxiu0 = 0, maxiv0 = 0;
  double ushift = 0, vshift = 0;
  // occupied u band: rows [0, Lu] and [nu-Lu, nu), or all rows
  size_t Lu = 0, band_rows = 0;
  bool band_full = false;
  // nu = K * 2^logM with 2^logM >= band_rows: the u transform of an image
  // column is K pruned FFTs of length 2^logM
  int logM = 0, K = 1;
  // No pruned layout fits (the occupied u band is wider than the longest
  // column transform, 8192 points): the grid keeps every u row (band_full,
  // K = 1, nu any 2,3,5,7-smooth length) and the u transform is a library
  // FFT over whole grid columns, whose output rows (one per plane and grid
  // column, nu entries) the w-screens read and write in place of the
  // segmented rows below.
  bool ucufft = false;
  // Layout of one u-transformed image row (the array between the u
  // transform and the w-screen): pixel row i, at s = i - nx/2 = K m + k2
  // (0 <= k2 < K), is written by the k2-th pruned FFT as its output m.  The
  // row holds K segments of hseg() entries, one per k2, each ordered by m
  // from hm0(), so that every FFT reads or writes one contiguous run.  With
  // K == 1 this is the natural order, entry i for pixel i.
  int hm0() const { return -int((nx / 2 + K - 1) / K); }
  size_t hseg() const {
    if (K == 1) return nx;
    const size_t nm = size_t(int((nx - 1 - nx / 2) / K) - hm0() + 1);
    return (nm + 31) & ~size_t(31);
  }
  size_t hrow() const { return size_t(K) * hseg(); }
  // bins and sort keys
  int T = 16;
  int ntu = 0, ntv = 0, nwmin = 1;
  int lbits = 0;      // sort bits per axis for the position inside a tile
  int bin_bits = 0;   // sort bits of the (tile, minplane) bin
  int key_bits = 0;   // total key bits
  bool wide_keys = false;  // key_bits > 31: 64-bit sort keys
  // batch plans: every job uses the kernel (W, sigma) of the first one
  int force_W = 0;
  double force_sigma = 0;
  // streams: the grid was planned from a declared data extent; chunks are
  // checked against it instead of re-planning
  bool fixed = false;
  // modelled time of the chosen grid (seconds)
  double cost = 0;
};

// Parameter choice (the analogue of ducc0 Params::getNuNv, wgridder.h:1503-1576,
// and the w-plane placement of countRanges, wgridder.h:690-699).  The cost
// model is this implementation's own, calibrated for the B200 kernels.
// pow2_v: restrict nv to a power of two no larger than kPow2VMax (for the FFT
// along v by the library's own shared-memory kernel instead of cuFFT, whose
// lengths run from 256 to 8192); kernels that would need a longer nv are
// skipped.
constexpr size_t kPow2VMax = 8192;
void choose_grid(GridPlan &g, double sigma_min, double sigma_max, int tile, bool pow2_v = false);

// Caps the sort key at max_bits by quantising the in-tile position (for
// callers that sort 32-bit keys only).
void limit_key_bits(GridPlan &g, int max_bits);

// The n cheapest kernels (W, sigma) for these inputs by the cost model of
// choose_grid, cheapest first (the autotuner times them).
std::vector<std::pair<int, double>> rank_kernels(const GridPlan &g, double sigma_min,
                                                 double sigma_max, int tile, size_t n);

// Shared memory of a spread / interpolation CTA for tile T and support W.
constexpr size_t kMaxSmemPerBlock = 227 * 1024;
size_t tile_smem_bytes(int T, int W, bool fp32);

// The tuned schedule's subdivision (ducc0's ms2dirty_tuning / dirty2ms_tuning,
// wgridder.h:1781-1877, with the choice of get_tuning_parameters,
// wgridder.cc:144-278): either no subdivision, or nfx x nfy facets (each
// gridded with its own phase centre) of the visibilities whose |w| bin is at
// least icut, plus -- when icut > 0 -- the visibilities below the cut gridded
// on the whole image.  The rule is the reference's, restated, so that a tuned
// call subdivides the way the reference does; the results equal the plain
// operator's within epsilon whatever the subdivision.
struct TuningChoice {
  int nfx = 0, nfy = 0;   // 0: no facets
  int icut = 0;           // first |w| bin of the faceted part (0: all of them)
  double wmin = 0, wmax = 0;
  bool split() const { return nfx > 0; }
};
constexpr int kTuningBins = 50;
// hist: visibility counts of the kTuningBins |w| bins over [wmin, wmax]
// (masked-in visibilities only), nvis_all = nrows * nchan.
TuningChoice tuning_choice(size_t npix_x, size_t npix_y, double pixsize_x, double pixsize_y,
                           double epsilon, bool do_w, double center_x, double center_y,
                           size_t nvis_all, double wmin, double wmax, const uint64_t *hist);
// Facet (ifx, ify) of an nfx x nfy subdivision (get_facet_data,
// wgridder.cc:92-108): pixel range [x0, x1) x [y0, y1) and phase centre.
struct Facet {
  size_t x0, y0, x1, y1;
  double cx, cy;
};
Facet tuning_facet(size_t npix_x, size_t npix_y, int nfx, int nfy, int ifx, int ify,
                   double pixsize_x, double pixsize_y, double center_x, double center_y);

// Geometry of an ImageWeights grid (structures/imageweights.h:73-102): the
// grid is W x H/2 cells over the v >= 0 half plane.
struct WeightGrid {
  int W, H;
  double psx, psy;  // pixel scales (radians)
};

// Imaging weights looked up per visibility (device pointers; grid ==
// nullptr: none) while the visibilities are scanned and their records are
// built: the finished ImageWeights grid and each channel's wavelength.  The
// visibility weight becomes weight x imaging weight, rounded to float when
// the weights are float (as wsg_weights_apply would have stored it).
struct ImgW {
  const double *grid = nullptr;
  const double *lambda = nullptr;
  WeightGrid g{};
};

// Nominal device bytes for one pass with `planes` planes resident.
size_t plan_bytes(const GridPlan &g, size_t planes, bool gridding);

}  // namespace wsg
