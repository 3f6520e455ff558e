/* Test infrastructure only: the FP64 direct Fourier transform that the
 * w-gridder approximates.  It is the numerical truth for parity tests and is
 * never linked by the product.
 *
 * Semantics: WSClean's DirectMSGridder (gridding/directmsgridder.cpp:77-114,
 * theta = -2pi(u l + v m + w (n-1))) restated in ducc0's axis and sign
 * convention, which is the one WSClean's wgridder path uses
 * (external/wgridder/ducc0/wgridder/wgridder.h):
 *   - v is negated when negate_v is set (Baselines ctor, wgridder.h:318-322),
 *     and so is the m shift (Params ctor, wgridder.h:1644);
 *   - u,v,w are in wavelengths, f/c with c = 299792458 m/s (wgridder.h:297,309);
 *   - pixel (i,j) sits at l_i = lshift + (i - nx/2) px, m_j = mshift + (j - ny/2) py
 *     (grid2dirty_post2, wgridder.h:432-433);
 *   - n-1 = (-l^2-m^2)/(sqrt(1-l^2-m^2)+1) (phase(), wgridder.h:395-397).
 *
 *   ms2dirty: dirty(i,j) = sum_k Re[ V_k wgt_k exp(+2 pi i (u l + v' m - w (n-1))) ] [/n]
 *   dirty2ms: V_k = wgt_k sum_ij dirty(i,j) exp(-2 pi i (u l + v' m - w (n-1))) [/n]
 *
 * Angles are reduced in turns (t - rint(t)) before sin/cos, so the result is
 * accurate to FP64 rounding for any baseline length.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

#define WSG_C 299792458.0
#define WSG_TWOPI 6.283185307179586476925286766559

static void pix_lm(size_t i, size_t j, size_t nx, size_t ny, double px,
                   double py, double lshift, double mshift, double *l,
                   double *m, double *nm1, double *n) {
  *l = lshift + ((double)i - 0.5 * (double)nx) * px;
  *m = mshift + ((double)j - 0.5 * (double)ny) * py;
  double r2 = (*l) * (*l) + (*m) * (*m);
  double tmp = 1.0 - r2;
  if (tmp >= 0) {
    *nm1 = -r2 / (sqrt(tmp) + 1.0);
    *n = *nm1 + 1.0;
  } else {
    *nm1 = -sqrt(-tmp) - 1.0;
    *n = 0.0;
  }
}

/* Image-side DFT.  vis is complex128 (nrows*nchan*2 doubles), wgt float64 or
 * NULL, mask uint8 or NULL.  If pix != NULL only the npix listed pixels
 * (flat index i*ny+j) are computed into out[0..npix); otherwise out holds the
 * full nx*ny image (x-major, ducc0's dirty(i,j) layout). */
void wsg_dft_ms2dirty(size_t nrows, size_t nchan, const double *uvw,
                      const double *freq, const double *vis, const double *wgt,
                      const uint8_t *mask, size_t nx, size_t ny, double px,
                      double py, int negate_v, int divide_by_n, double center_x,
                      double center_y, size_t npix, const int64_t *pix,
                      double *out) {
  double vfac = negate_v ? -1.0 : 1.0;
  double lshift = center_x, mshift = negate_v ? -center_y : center_y;
  size_t nout = pix ? npix : nx * ny;
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t o = 0; o < nout; ++o) {
    size_t flat = pix ? (size_t)pix[o] : o;
    size_t i = flat / ny, j = flat % ny;
    double l, m, nm1, n;
    pix_lm(i, j, nx, ny, px, py, lshift, mshift, &l, &m, &nm1, &n);
    double acc = 0.0, comp = 0.0;
    for (size_t r = 0; r < nrows; ++r) {
      double u0 = uvw[3 * r], v0 = vfac * uvw[3 * r + 1], w0 = uvw[3 * r + 2];
      for (size_t c = 0; c < nchan; ++c) {
        size_t k = r * nchan + c;
        if (mask && !mask[k]) continue;
        double f = freq[c] / WSG_C;
        double t = (u0 * l + v0 * m - w0 * nm1) * f;
        t -= rint(t);
        double s = sin(WSG_TWOPI * t), co = cos(WSG_TWOPI * t);
        double wk = wgt ? wgt[k] : 1.0;
        double term = wk * (vis[2 * k] * co - vis[2 * k + 1] * s);
        /* Kahan summation keeps the FP64 sum exact to rounding for 1e7 terms */
        double y = term - comp;
        double tt = acc + y;
        comp = (tt - acc) - y;
        acc = tt;
      }
    }
    if (divide_by_n) acc = (n > 0) ? acc / n : 0.0;
    out[o] = acc;
  }
}

/* Visibility-side DFT (adjoint).  Zero pixels are skipped, so a sparse model
 * image (point sources) is cheap.  If sel != NULL only the nsel listed flat
 * visibility indices are computed into out[0..nsel) (complex128 pairs);
 * otherwise out holds all nrows*nchan visibilities. */
void wsg_dft_dirty2ms(size_t nrows, size_t nchan, const double *uvw,
                      const double *freq, const double *dirty,
                      const double *wgt, const uint8_t *mask, size_t nx,
                      size_t ny, double px, double py, int negate_v,
                      int divide_by_n, double center_x, double center_y,
                      size_t nsel, const int64_t *sel, double *out) {
  double vfac = negate_v ? -1.0 : 1.0;
  double lshift = center_x, mshift = negate_v ? -center_y : center_y;
  size_t nout = sel ? nsel : nrows * nchan;
  /* collect the nonzero pixels once */
  size_t nnz = 0;
  for (size_t p = 0; p < nx * ny; ++p)
    if (dirty[p] != 0.0) ++nnz;
  size_t cap = nnz ? nnz : 1;
  double *pl = (double *)malloc(cap * sizeof(double) * 4);
  size_t q = 0;
  for (size_t p = 0; p < nx * ny; ++p) {
    if (dirty[p] == 0.0) continue;
    double l, m, nm1, n;
    pix_lm(p / ny, p % ny, nx, ny, px, py, lshift, mshift, &l, &m, &nm1, &n);
    double val = dirty[p];
    if (divide_by_n) val = (n > 0) ? val / n : 0.0;
    pl[4 * q] = l;
    pl[4 * q + 1] = m;
    pl[4 * q + 2] = nm1;
    pl[4 * q + 3] = val;
    ++q;
  }
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t o = 0; o < nout; ++o) {
    size_t k = sel ? (size_t)sel[o] : o;
    size_t r = k / nchan, c = k % nchan;
    if (mask && !mask[k]) {
      out[2 * o] = out[2 * o + 1] = 0.0;
      continue;
    }
    double f = freq[c] / WSG_C;
    double u0 = uvw[3 * r] * f, v0 = vfac * uvw[3 * r + 1] * f,
           w0 = uvw[3 * r + 2] * f;
    double re = 0.0, im = 0.0;
    for (size_t p = 0; p < nnz; ++p) {
      double t = u0 * pl[4 * p] + v0 * pl[4 * p + 1] - w0 * pl[4 * p + 2];
      t -= rint(t);
      double s = sin(WSG_TWOPI * t), co = cos(WSG_TWOPI * t);
      re += pl[4 * p + 3] * co;
      im -= pl[4 * p + 3] * s;
    }
    double wk = wgt ? wgt[k] : 1.0;
    out[2 * o] = wk * re;
    out[2 * o + 1] = wk * im;
  }
  free(pl);
}
