// Drives WGriddingGridder_B200 the way WGriddingMSGridder does
// (wgridder/wgriddingmsgridder.cpp:214-302): MakeGridder, InitializeInversion,
// AddInversionData per row chunk, FinalizeImage(1/weight), RealImage; then
// InitializePrediction and PredictVisibilities per chunk.  Used by the tests:
//   dropin_demo <in.bin> <out_image.bin> <out_vis.bin>
// in.bin: header of 8 doubles {nrows, nchan, width, height, width_t, height_t,
// pixsize, epsilon}, then l_shift, m_shift, uvw (nrows*3), freq (nchan), vis
// (nrows*nchan complex<float>), model image (width*height float).
#include <complex>
#include <cstdio>
#include <memory>
#include <vector>

#include "wgriddinggridder_b200.h"

template <typename T>
static void rd(FILE *f, T *p, size_t n) {
  if (fread(p, sizeof(T), n, f) != n) throw std::runtime_error("short read");
}

int main(int argc, char **argv) {
  if (argc != 4) return 2;
  try {
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 3;
    double h[10];
    rd(f, h, 10);
    const size_t nrows = size_t(h[0]), nchan = size_t(h[1]), width = size_t(h[2]),
                 height = size_t(h[3]), wt = size_t(h[4]), ht = size_t(h[5]);
    const double px = h[6], eps = h[7], lsh = h[8], msh = h[9];
    std::vector<double> uvw(nrows * 3), freq(nchan);
    std::vector<std::complex<float>> vis(nrows * nchan);
    std::vector<float> model(width * height);
    rd(f, uvw.data(), uvw.size());
    rd(f, freq.data(), freq.size());
    rd(f, vis.data(), vis.size());
    rd(f, model.data(), model.size());
    fclose(f);
    std::unique_ptr<WGriddingGridderBase> g(
        new WGriddingGridder_B200(width, height, wt, ht, px, px, lsh, msh, 8, eps));
    size_t cst = 0, pv = 0;
    g->MemoryUsage(cst, pv);
    const size_t chunk = (nrows + 2) / 3;  // three row chunks, as the memory budget would give
    g->InitializeInversion();
    for (size_t r0 = 0; r0 < nrows; r0 += chunk) {
      const size_t n = std::min(chunk, nrows - r0);
      g->AddInversionData(n, nchan, uvw.data() + 3 * r0, freq.data(), vis.data() + r0 * nchan);
    }
    g->FinalizeImage(0.5);
    std::vector<float> img = g->RealImage();
    g->InitializePrediction(model.data());
    std::vector<std::complex<float>> pred(nrows * nchan);
    for (size_t r0 = 0; r0 < nrows; r0 += chunk) {
      const size_t n = std::min(chunk, nrows - r0);
      g->PredictVisibilities(n, nchan, uvw.data() + 3 * r0, freq.data(), pred.data() + r0 * nchan);
    }
    FILE *o = fopen(argv[2], "wb");
    fwrite(img.data(), sizeof(float), img.size(), o);
    fclose(o);
    o = fopen(argv[3], "wb");
    fwrite(pred.data(), sizeof(std::complex<float>), pred.size(), o);
    fclose(o);
    // error propagation: an odd trimmed size must throw std::runtime_error
    try {
      WGriddingGridder_B200 bad(width, height, wt - 1, ht, px, px, 0, 0, 8, eps);
      return 4;
    } catch (const std::runtime_error &) {
    }
    return 0;
  } catch (const std::exception &e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
