// Device kernels of libwsg (sm_100a).  Host orchestration: the wsg_*.cu units
// listed in wsg_host.cuh; the heavy kernel templates are launched from wsg_launch.cu.
//
// Data flow of one ms2dirty call (dirty2ms runs the transpose in reverse):
//   k_scan      active mask, |w| and |u| ranges, nvis        (ducc0 scanData, wgridder.h:1578-1618)
//   k_keys      (tile_u, tile_v, minplane, in-tile position) sort key per visibility
//                                                             (get_uvwidx/getpix, wgridder.h:660-682)
//   CUB radix sort of (key, index); k_records gathers one 32-byte record per
//   visibility in key order with FP64 pixel coordinates reduced to local kernel
//   coordinates and the shift phasor / weight / conjugation applied
//                                                             (compute_phases, wgridder.h:1126-1140)
//   k_spread    persistent CTAs drain chunks of one (tile, minplane) bin each,
//               accumulate W planes x W x W footprints in registers while the
//               footprint origin repeats, commit to a shared-memory tile, and
//               flush the tile to the u-band grid with vector atomics
//                                                             (x2grid_c_helper/HelperX2g2, wgridder.h:934-1031,1142-1236)
//   cuFFT       backward FFT along v of the occupied u band (all planes of a pass)
//   k_ucol_bwd  pruned backward FFT along u of the image columns only: nu = K M,
//               K twisted M-point FFTs per column, band in, image rows out
//                                                             (grid2dirty_c_overwrite_wscreen_add, :496-534)
//   k_screen    sum over planes of Re(grid * w-screen), FP64, times the grid
//               correction, added into the FP64 image         (grid2dirty_post2 :428-484, apply_global_corrections :1348-1400)
#pragma once

#include <cuda.h>  // CUtensorMap (the type only; no driver-API calls here)
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

namespace wsg {

constexpr int kDMaxW = 16;
constexpr int kDMaxDeg = 24;
constexpr int kDMaxCheb = 48;

// Piecewise polynomial kernel, passed by value (kernel parameter space).
// c[j][k] multiplies x^j in piece k.
template <typename R>
struct DevKernel {
  R c[kDMaxDeg + 1][kDMaxW];
  int D;
};

// FP64 geometry of one call (see GridPlan in wsg_internal.h).
struct DevGeom {
  int nu, nv, W, nsafe, maxiu0, maxiv0;
  double px, py, ushift, vshift;
  double wmin, dw, xdw, wshift;
  int nplanes, do_w;
  double lshift, mshift, nshift, vfac;
  int shifting;
  int T, ntu, ntv, nwmin, lbits, qshift;  // qshift: in-tile bits dropped per axis
  int wide;                               // 64-bit sort keys
  unsigned long long inactive_key;
  int Lu, band_rows, band_full;
};

struct ScanOut {
  unsigned long long wmin_bits, wmax_bits, umax_bits, vmax_bits;
  unsigned long long nvis;
};

// Copies the scan's statistics into mapped pinned host memory (one warp).
static __global__ void k_scan_readback(const ScanOut *src, ScanOut *dst_host) {
  constexpr int N = sizeof(ScanOut) / sizeof(unsigned long long);
  const auto *s = reinterpret_cast<const unsigned long long *>(src);
  auto *d = reinterpret_cast<volatile unsigned long long *>(dst_host);
  if (threadIdx.x < N) d[threadIdx.x] = s[threadIdx.x];
}

// Visibility record, mixed precision (32 bytes, two 128-bit loads).
struct __align__(16) RecF {
  float xu, xv, xw;   // local kernel coordinates in (-1, 1]
  uint32_t iuv;       // (iu0+nsafe) << 16 | (iv0+nsafe)
  float vr, vi;       // gridding: weighted, phase-shifted, conjugated visibility;
                      // degridding: weight * conj shift phasor
  uint32_t mp;        // first w plane of the footprint
  uint32_t idx;       // flat visibility index; bit 31 = conjugate (degridding)
};
// FP64 record (64 bytes).
struct __align__(16) RecD {
  double xu, xv, xw;
  uint32_t iuv, mp, idx, pad;
  double vr, vi;
  double pad2;
};

template <typename R> struct RecOf;
template <> struct RecOf<float> { using type = RecF; };
template <> struct RecOf<double> { using type = RecD; };

template <typename R> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

// ------------------------------------------------------------- helpers

__device__ __forceinline__ double2 cexp_turns(double t) {
  // exp(2 pi i t) with the argument reduced in turns first
  t -= rint(t);
  double s, c;
  sincospi(2.0 * t, &s, &c);
  return make_double2(c, s);
}

// exp(2 pi i t) to FP32 accuracy: the argument reduced in turns in FP64, the
// sine and cosine of the remainder (|t| <= 1/2) in FP32.
__device__ __forceinline__ float2 cexp_turns_f(double t) {
  t -= rint(t);
  float s, c;
  sincospif(2.0f * float(t), &s, &c);
  return make_float2(c, s);
}

// Complex sum and difference: one packed two-lane instruction each in FP32
// (fadd / fma .f32x2), two scalar ones in FP64.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}

// a * s + acc for a complex a and a real s: one packed two-lane FMA in FP32
// (Blackwell's fma.rn.f32x2), two scalar FMAs in FP64.
__device__ __forceinline__ float2 cfma_real(float2 a, float s, float2 acc) {
  return __ffma2_rn(a, make_float2(s, s), acc);
}
__device__ __forceinline__ double2 cfma_real(double2 a, double s, double2 acc) {
  acc.x = fma(a.x, s, acc.x);
  acc.y = fma(a.y, s, acc.y);
  return acc;
}

// FP64 coordinates of one visibility: (u, v', w) already scaled by f/c.
struct VisPix {
  int iu0, iv0, iw;
  double xu, xv, xw;
  bool flip;
};

__device__ __forceinline__ void vis_pixel(const DevGeom &g, double u, double v,
                                          double w, VisPix &o) {
  o.flip = (w < 0);
  if (o.flip) {
    u = -u;
    v = -v;
    w = -w;
  }
  double uf = u * g.px;
  uf = (uf - floor(uf)) * double(g.nu);
  int iu0 = min(int(uf + g.ushift) - g.nu, g.maxiu0);
  double vf = v * g.py;
  vf = (vf - floor(vf)) * double(g.nv);
  int iv0 = min(int(vf + g.vshift) - g.nv, g.maxiv0);
  o.iu0 = iu0;
  o.iv0 = iv0;
  o.xu = double(g.W - 1) - 2.0 * (uf - double(iu0));
  o.xv = double(g.W - 1) - 2.0 * (vf - double(iv0));
  if (g.do_w) {
    // the plane placement guarantees iw <= nwmin-1; the clamp keeps sort keys
    // inside their (tile, minplane) bin even under rounding
    int iw = min(max(0, int((w + g.wshift) * g.xdw)), g.nwmin - 1);
    o.iw = iw;
    o.xw = 2.0 * (double(iw) - (w - g.wmin) * g.xdw) + double(g.W - 1);
  } else {
    o.iw = 0;
    o.xw = 0.0;
  }
}

// Sort key of a visibility: its (tile, minplane) bin, then its position in
// the tile (quantised to lbits per axis), in 32 or -- when the bins and the
// full in-tile position need more than 31 bits -- 64 bits.
template <typename K>
__device__ __forceinline__ K bin_key(const DevGeom &g, const VisPix &p) {
  int a = p.iu0 + g.nsafe, b = p.iv0 + g.nsafe;
  uint32_t tu = uint32_t(a / g.T), tv = uint32_t(b / g.T);
  uint32_t lu = uint32_t(a % g.T), lv = uint32_t(b % g.T);
  uint32_t bin = (tu * uint32_t(g.ntv) + tv) * uint32_t(g.nwmin) + uint32_t(p.iw);
  // in-tile position, quantised to lbits per axis (T <= 32)
  uint32_t q = ((lu >> g.qshift) << g.lbits) | (lv >> g.qshift);
  return (K(bin) << (2 * g.lbits)) | K(q);
}



__device__ __forceinline__ bool weight_cell(const WeightGrid &g, double u, double v, int &x,
                                            int &y) {
  if (v < 0.0) {
    u = -u;
    v = -v;
  }
  x = int(floor(u * double(g.W) * g.psx + double(g.W / 2)));
  y = int(floor(v * double(g.H) * g.psy));
  return x >= 0 && x < g.W && y < g.H / 2;
}

// The visibility weight w (1 when there are none) times the imaging weight
// of row r, channel c (raw uvw: v not negated).
template <typename TW>
__device__ __forceinline__ double weighted(const ImgW &iw, const double *__restrict__ uvw, size_t r,
                                           int c, double w) {
  if (!iw.grid) return w;
  int x, y;
  const double lam = iw.lambda[c];
  const double f = weight_cell(iw.g, uvw[3 * r] / lam, uvw[3 * r + 1] / lam, x, y)
                       ? iw.grid[size_t(x) + size_t(y) * iw.g.W]
                       : 0.0;
  const double p = w * f;
  return sizeof(TW) == 4 ? double(float(p)) : p;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// --------------------------------------------------------------- k_scan

// Active mask, |w| range, max |u|, |v| and the active count of the
// visibilities (scanData, wgridder.h:1578-1618); with KEYS, also the sort
// key of every visibility for the grid geometry g, as k_keys writes it (the
// caller checks afterwards that the planned geometry is g).
template <typename TV, typename TW, bool KEYS, typename K = uint32_t>
__device__ __forceinline__ void scan_rows(size_t nrows, int nchan, const double *__restrict__ uvw,
                                          const double *__restrict__ fovc,
                                          const TV *__restrict__ vis, const TW *__restrict__ wgt,
                                          const uint8_t *__restrict__ mask, int gridding,
                                          double vfac, ScanOut *out, TV *__restrict__ vis_out,
                                          const DevGeom &g, K *__restrict__ keys,
                                          uint32_t *__restrict__ vals, const ImgW &iw) {
  double lwmin = 1e300, lwmax = 0, lumax = 0, lvmax = 0;
  unsigned long long cnt = 0;
  for (size_t r = blockIdx.x * size_t(blockDim.x) + threadIdx.x; r < nrows;
       r += size_t(gridDim.x) * blockDim.x) {
    double u = uvw[3 * r], v = vfac * uvw[3 * r + 1], w = uvw[3 * r + 2];
    for (int c = 0; c < nchan; ++c) {
      size_t k = r * nchan + c;
      bool act;
      if (gridding) {
        TV x = vis[k];
        auto n = x.x * x.x + x.y * x.y;
        if (iw.grid)
          n *= decltype(n)(weighted<TW>(iw, uvw, r, c, wgt ? double(wgt[k]) : 1.0));
        else if (wgt)
          n *= wgt[k];
        if (mask) n *= mask[k];
        act = (n != 0);
      } else {
        act = (!wgt || wgt[k] != 0) && (!mask || mask[k] != 0);
        if (!act && vis_out) vis_out[k] = TV{0, 0};
      }
      K key = KEYS ? K(g.inactive_key) : K(0);
      if (act) {
        double f = fovc[c];
        double aw = fabs(w * f);
        lwmin = fmin(lwmin, aw);
        lwmax = fmax(lwmax, aw);
        lumax = fmax(lumax, fabs(u * f));
        lvmax = fmax(lvmax, fabs(v * f));
        ++cnt;
        if constexpr (KEYS) {
          VisPix p;
          vis_pixel(g, u * f, v * f, w * f, p);
          key = bin_key<K>(g, p);
        }
      }
      if constexpr (KEYS) {
        keys[k] = key;
        vals[k] = uint32_t(k);
      }
    }
  }
  // warp then block reduction
  for (int o = 16; o > 0; o >>= 1) {
    lwmin = fmin(lwmin, __shfl_xor_sync(0xffffffffu, lwmin, o));
    lwmax = fmax(lwmax, __shfl_xor_sync(0xffffffffu, lwmax, o));
    lumax = fmax(lumax, __shfl_xor_sync(0xffffffffu, lumax, o));
    lvmax = fmax(lvmax, __shfl_xor_sync(0xffffffffu, lvmax, o));
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  if ((threadIdx.x & 31) == 0 && cnt > 0) {
    atomicMin(&out->wmin_bits, (unsigned long long)__double_as_longlong(lwmin));
    atomicMax(&out->wmax_bits, (unsigned long long)__double_as_longlong(lwmax));
    atomicMax(&out->umax_bits, (unsigned long long)__double_as_longlong(lumax));
    atomicMax(&out->vmax_bits, (unsigned long long)__double_as_longlong(lvmax));
    atomicAdd(&out->nvis, cnt);
  }
}

template <typename TV, typename TW>
__global__ void k_scan(size_t nrows, int nchan, const double *__restrict__ uvw,
                       const double *__restrict__ fovc, const TV *__restrict__ vis,
                       const TW *__restrict__ wgt, const uint8_t *__restrict__ mask,
                       int gridding, double vfac, ScanOut *out, TV *__restrict__ vis_out,
                       ImgW iw) {
  const DevGeom g{};
  scan_rows<TV, TW, false>(nrows, nchan, uvw, fovc, vis, wgt, mask, gridding, vfac, out, vis_out,
                           g, (uint32_t *)nullptr, nullptr, iw);
}

// The scan with the keys of an expected geometry: when consecutive calls
// plan the same grid (the usual case: the same image and data extent), the
// separate pass of k_keys over uvw and the visibilities is not needed.
template <typename TV, typename TW, typename K>
__global__ void k_scan_keys(size_t nrows, int nchan, const double *__restrict__ uvw,
                            const double *__restrict__ fovc, const TV *__restrict__ vis,
                            const TW *__restrict__ wgt, const uint8_t *__restrict__ mask,
                            int gridding, double vfac, ScanOut *out, TV *__restrict__ vis_out,
                            DevGeom g, K *__restrict__ keys, uint32_t *__restrict__ vals,
                            ImgW iw) {
  scan_rows<TV, TW, true, K>(nrows, nchan, uvw, fovc, vis, wgt, mask, gridding, vfac, out,
                             vis_out, g, keys, vals, iw);
}

// --------------------------------------------------------------- k_keys

template <typename TV, typename TW, typename K>
__global__ void k_keys(size_t nrows, int nchan, const double *__restrict__ uvw,
                       const double *__restrict__ fovc, const TV *__restrict__ vis,
                       const TW *__restrict__ wgt, const uint8_t *__restrict__ mask,
                       int gridding, DevGeom g, K *__restrict__ keys,
                       uint32_t *__restrict__ vals, ImgW iw) {
  for (size_t r = blockIdx.x * size_t(blockDim.x) + threadIdx.x; r < nrows;
       r += size_t(gridDim.x) * blockDim.x) {
    double u = uvw[3 * r], v = g.vfac * uvw[3 * r + 1], w = uvw[3 * r + 2];
    for (int c = 0; c < nchan; ++c) {
      size_t k = r * nchan + c;
      bool act;
      if (gridding) {
        TV x = vis[k];
        auto n = x.x * x.x + x.y * x.y;
        if (iw.grid)
          n *= decltype(n)(weighted<TW>(iw, uvw, r, c, wgt ? double(wgt[k]) : 1.0));
        else if (wgt)
          n *= wgt[k];
        if (mask) n *= mask[k];
        act = (n != 0);
      } else {
        act = (!wgt || wgt[k] != 0) && (!mask || mask[k] != 0);
      }
      K key = K(g.inactive_key);
      if (act) {
        double f = fovc[c];
        VisPix p;
        vis_pixel(g, u * f, v * f, w * f, p);
        key = bin_key<K>(g, p);
      }
      keys[k] = key;
      vals[k] = uint32_t(k);
    }
  }
}

// ------------------------------------------------------------ k_records

// The record of visibility k (row k / nchan, channel k % nchan).
template <typename R, typename TV, typename TW>
__device__ __forceinline__ typename RecOf<R>::type make_record(
    uint32_t k, int nchan, const double *__restrict__ uvw, const double *__restrict__ fovc,
    const TV *__restrict__ vis, const TW *__restrict__ wgt, int gridding, const DevGeom &g,
    const ImgW &iw) {
  using Rec = typename RecOf<R>::type;
  size_t r = k / uint32_t(nchan);
  int c = int(k - r * uint32_t(nchan));
  double f = fovc[c];
  double u = uvw[3 * r], v = g.vfac * uvw[3 * r + 1], w = uvw[3 * r + 2];
  VisPix p;
  vis_pixel(g, u * f, v * f, w * f, p);
  double wk = wgt ? double(wgt[k]) : 1.0;
  if (gridding) wk = weighted<TW>(iw, uvw, r, c, wk);
  double2 ph = make_double2(1.0, 0.0);
  if (g.shifting) ph = cexp_turns((u * g.lshift + v * g.mshift + w * g.nshift) * f);
  Rec o;
  o.xu = R(p.xu);
  o.xv = R(p.xv);
  o.xw = R(p.xw);
  o.iuv = (uint32_t(p.iu0 + g.nsafe) << 16) | uint32_t(p.iv0 + g.nsafe);
  o.mp = uint32_t(p.iw);
  if (gridding) {
    TV x = vis[k];
    double xr = double(x.x), xi = double(x.y);
    double vr = (xr * ph.x - xi * ph.y) * wk;
    double vi = (xr * ph.y + xi * ph.x) * wk;
    if (p.flip) vi = -vi;
    o.vr = R(vr);
    o.vi = R(vi);
    o.idx = k;
  } else {
    // output = wgt * exp(-2 pi i phase) * (flip ? conj(S) : S)
    o.vr = R(wk * ph.x);
    o.vi = R(-wk * ph.y);
    o.idx = k | (p.flip ? 0x80000000u : 0u);
  }
  return o;
}

// Sorted position of every visibility: pos[sidx[s]] = s (the inactive
// ones sort last, at positions >= the active count, and have no record).
static __global__ void k_rank(size_t n, const uint32_t *__restrict__ sidx, uint32_t *__restrict__ pos) {
  for (size_t s = blockIdx.x * size_t(blockDim.x) + threadIdx.x; s < n;
       s += size_t(gridDim.x) * blockDim.x)
    pos[sidx[s]] = uint32_t(s);
}

// Records in visibility order: thread k reads visibility k's coordinates,
// value and weight (coalesced; a row's uvw is shared by its channels) and
// writes its record to the sorted slot pos[k] -- one aligned 32-byte (64 in
// FP64) record per write, so the scatter moves whole sectors, where a
// gather in sorted order would fetch a sector for every 8-byte visibility
// and every 24-byte uvw row.
template <typename R, typename TV, typename TW>
__global__ void k_records(size_t nvis_tot, size_t nvis, int nchan, const uint32_t *__restrict__ pos,
                          const double *__restrict__ uvw, const double *__restrict__ fovc,
                          const TV *__restrict__ vis, const TW *__restrict__ wgt,
                          int gridding, DevGeom g, typename RecOf<R>::type *__restrict__ rec,
                          ImgW iw) {
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < nvis_tot;
       k += size_t(gridDim.x) * blockDim.x) {
    const uint32_t p = pos[k];
    if (p >= nvis) continue;
    rec[p] = make_record<R, TV, TW>(uint32_t(k), nchan, uvw, fovc, vis, wgt, gridding, g, iw);
  }
}

// Batch plans: a job's records index its own channel range; make the index
// flat over the full nrows x nchan_total array (the conjugation bit is kept).
template <typename Rec>
__global__ void k_plan_remap(size_t n, Rec *__restrict__ rec, uint32_t nch, uint32_t nch_total,
                             uint32_t chan0) {
  for (size_t s = blockIdx.x * size_t(blockDim.x) + threadIdx.x; s < n;
       s += size_t(gridDim.x) * blockDim.x) {
    const uint32_t id = rec[s].idx;
    const uint32_t k = id & 0x7fffffffu, r = k / nch, c = k - r * nch;
    rec[s].idx = (id & 0x80000000u) | (r * nch_total + chan0 + c);
  }
}

// Batch plans: append a job's chunk starts (shifted by its record offset)
// and tag the chunks with the job.
static __global__ void k_plan_chunks(int n, const int *__restrict__ in, int *__restrict__ out,
                              int *__restrict__ job_of, int rec_off, int job) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    out[i] = in[i] + rec_off;
    job_of[i] = job;
  }
}

// ----------------------------------------------------- chunk boundaries

// A chunk starts where the (tile, minplane) bin changes or at a multiple of
// the chunk size; chunks therefore never cross bins.
template <typename K>
struct ChunkStartPred {
  const K *keys;
  int shift;
  int chunk;
  __host__ __device__ bool operator()(const int &i) const {
    if (i == 0 || (i % chunk) == 0) return true;
    return (keys[i] >> shift) != (keys[i - 1] >> shift);
  }
};

// ------------------------------------------------------- tile geometry

struct TileLayout {
  int S;    // tile extent incl. halo: T + W - 1
  int RS;   // row stride (elements), odd
  int PS;   // plane stride (elements)
};

// Grid geometry of one gridding job.  A call is one job; a batch plan runs
// many jobs (facets x output channels) sharing one kernel, tile size and
// record array through a single spread / interpolation launch.
struct JobGeom {
  int nu, nv, Lu, band_rows, band_full;
  int P, pb0, pb1;   // planes in the band layout, planes of this pass [pb0, pb1)
  void *grid;        // the job's u-band grid [band_rows][P][nv] complex
};

struct GridArgs {
  const void *rec;
  const int *chunk_start;
  const int *nchunks;
  int *counter;
  int nvis;
  void *grid;        // u-band grid [band_rows][P][nv] complex
  int P;             // planes in the layout
  int pb0, pb1;      // planes of this pass: [pb0, pb1)
  TileLayout tl;
  int sb;            // records per sub-batch
  int *err;          // set to 1 if a record falls outside its chunk's tile
  // degridding outputs
  void *vis_out;     // complex TV
  int vis_double;
  void *acc;         // per-record accumulator (multi-pass), complex R
  int first_pass, last_pass;
  // batch plans: per-job geometry and the job of each chunk (jobs == null:
  // one job, described by DevGeom and the fields above)
  const JobGeom *jobs;
  const int *chunk_job;
  // plan execution (gridding): records hold the static factor c = weight *
  // conj(shift phasor); the visibility is gathered at staging and the
  // spread value is V conj(c), conjugated for flipped w
  const void *vis_in;
  int vis_in_double;
  // degridding: add into vis_out (jobs that predict the same visibilities)
  int vis_accumulate;
};

__device__ __forceinline__ JobGeom load_job(const GridArgs &a, const DevGeom &g, int ch) {
  if (a.jobs) return a.jobs[a.chunk_job ? a.chunk_job[ch] : 0];
  JobGeom j;
  j.nu = g.nu;
  j.nv = g.nv;
  j.Lu = g.Lu;
  j.band_rows = g.band_rows;
  j.band_full = g.band_full;
  j.P = a.P;
  j.pb0 = a.pb0;
  j.pb1 = a.pb1;
  j.grid = a.grid;
  return j;
}


// The job geometry a tile flush or stage needs, copied out of shared memory
// into registers: inside loops that also store to shared memory the compiler
// would otherwise reload every field for every cell.
struct JobRegs {
  int nu, nv, Lu, rows, P, pb0, pb1;
  bool full;
  void *grid;
  __device__ __forceinline__ explicit JobRegs(const JobGeom &j)
      : nu(j.nu), nv(j.nv), Lu(j.Lu), rows(j.band_rows), P(j.P), pb0(j.pb0), pb1(j.pb1),
        full(j.band_full), grid(j.grid) {}
  // band row of grid row u (wrapped into [0, nu)), or -1 outside the band
  __device__ __forceinline__ int band_row(int u) const {
    if (full || u <= Lu) return u;
    return (u >= nu - Lu) ? u - (nu - rows) : -1;
  }
  __device__ __forceinline__ int wrap_u(int u) const {
    u += (u < 0) ? nu : 0;
    return u - ((u >= nu) ? nu : 0);
  }
  __device__ __forceinline__ int wrap_v(int v) const {
    v += (v < 0) ? nv : 0;
    return v - ((v >= nv) ? nv : 0);
  }
};

constexpr uint32_t kSkip = 0xfffffffeu;  // record marker: outside its chunk's tile


// ------------------------------------------------- per-warp record staging
//
// A warp works through its slice of a chunk 32 records at a time: lane l
// loads record l of the batch (coalesced), evaluates its 3W kernel values --
// W pieces per axis by Horner's rule of fixed degree W+4 with the
// coefficients as compile-time constant-bank operands (the host pads
// lower-degree fits with zero leading coefficients) -- and stages them in a
// per-warp shared-memory block; the warp then consumes the batch record by
// record with broadcast reads.
template <int W> struct KDeg { static constexpr int value = W + 4; };
template <typename R, int W> struct KStride {
  // row of 3W values, padded to a 16-byte multiple
  static constexpr int value = sizeof(R) == 4 ? ((3 * W + 3) & ~3) : ((3 * W + 1) & ~1);
};
template <typename R, int W> struct WarpStage {
  static constexpr int KST = KStride<R, W>::value;
  static constexpr size_t bytes = sizeof(R) * (32 * KST + 64) + 128;  // kv, (vr,vi), luv
};

// W consecutive values of a staged row, by 16- or 8-byte vector loads where
// the layout allows: with W even every staged row, and its v block at W,
// starts on a 16-byte boundary (the tile before the staging areas holds
// 2 W planes, and the row stride is a multiple of 16 bytes).
template <int W, typename R>
__device__ __forceinline__ void lds_row(const R *p, R (&out)[W]) {
  if constexpr (sizeof(R) == 4 && W % 4 == 0) {
#pragma unroll
    for (int i = 0; i < W / 4; ++i) {
      const float4 v = reinterpret_cast<const float4 *>(p)[i];
      out[4 * i] = v.x;
      out[4 * i + 1] = v.y;
      out[4 * i + 2] = v.z;
      out[4 * i + 3] = v.w;
    }
  } else if constexpr (W % 2 == 0) {
    using V2 = typename Cplx<R>::type;
#pragma unroll
    for (int i = 0; i < W / 2; ++i) {
      const V2 v = reinterpret_cast<const V2 *>(p)[i];
      out[2 * i] = v.x;
      out[2 * i + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) out[i] = p[i];
  }
}

template <int W, typename R>
__device__ __forceinline__ void eval_const(const DevKernel<R> &k, R x, R *out) {
  constexpr int DEG = KDeg<W>::value;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    R v = k.c[DEG][i];
#pragma unroll
    for (int j = DEG - 1; j >= 0; --j) v = fma(v, x, k.c[j][i]);
    out[i] = v;
  }
}

// The per-record part of staging that is not kernel evaluation: the packed
// in-tile origin (or kSkip when the record lies outside its chunk's tile),
// the bounding box of origins, and the visibility to spread (gathered and
// multiplied by the static factor for plan execution).  Returns false for a
// skipped record.
template <typename R, typename Rec>
__device__ __forceinline__ bool stage_meta(const Rec &rr, int lane, int tu, int tv, int mp,
                                           const DevGeom &g, R *vv, uint32_t *luv, int *err,
                                           int &bb0, int &bb1, int &bb2, int &bb3,
                                           const void *vis_in, int vis_in_double) {
  const int lu = int(rr.iuv >> 16) - tu * g.T;
  const int lv = int(rr.iuv & 0xffffu) - tv * g.T;
  if (lu < 0 || lu >= g.T || lv < 0 || lv >= g.T || int(rr.mp) != mp) {
    atomicOr(err, 1);
    luv[lane] = kSkip;
    vv[2 * lane] = R(0);
    vv[2 * lane + 1] = R(0);
    return false;
  }
  luv[lane] = (uint32_t(lu) << 16) | uint32_t(lv);
  bb0 = min(bb0, lu); bb1 = max(bb1, lu);
  bb2 = min(bb2, lv); bb3 = max(bb3, lv);
  R vr = rr.vr, vi = rr.vi;
  if (vis_in) {
    const uint32_t id = rr.idx & 0x7fffffffu;
    R xr, xi;
    if (vis_in_double) {
      const double2 x = reinterpret_cast<const double2 *>(vis_in)[id];
      xr = R(x.x);
      xi = R(x.y);
    } else {
      const float2 x = reinterpret_cast<const float2 *>(vis_in)[id];
      xr = R(x.x);
      xi = R(x.y);
    }
    vr = xr * rr.vr + xi * rr.vi;
    vi = xi * rr.vr - xr * rr.vi;
    if (rr.idx & 0x80000000u) vi = -vi;
  }
  vv[2 * lane] = vr;
  vv[2 * lane + 1] = vi;
  return true;
}

// Stages records [b0, b0+nb) of the warp's slice; returns via luv the packed
// in-tile origin (or kSkip).  Lanes >= nb do nothing.
template <typename R, int W, typename Rec>
__device__ __forceinline__ void stage_batch(const Rec *recs, int b0, int nb, int lane, int tu,
                                            int tv, int mp, const DevGeom &g,
                                            const DevKernel<R> &kc, R *kv, R *vv, uint32_t *luv,
                                            int *err, int &bb0, int &bb1, int &bb2, int &bb3,
                                            const void *vis_in, int vis_in_double) {
  constexpr int KST = KStride<R, W>::value;
  if (lane < nb) {
    const Rec rr = recs[b0 + lane];
    R *row = kv + lane * KST;
    if (!stage_meta<R>(rr, lane, tu, tv, mp, g, vv, luv, err, bb0, bb1, bb2, bb3, vis_in,
                       vis_in_double)) {
#pragma unroll
      for (int i = 0; i < 3 * W; ++i) row[i] = R(0);
    } else {
      R vals[W];
      eval_const<W>(kc, rr.xu, vals);
#pragma unroll
      for (int i = 0; i < W; ++i) row[i] = vals[i];
      eval_const<W>(kc, rr.xv, vals);
#pragma unroll
      for (int i = 0; i < W; ++i) row[W + i] = vals[i];
      if (g.do_w) {
        eval_const<W>(kc, rr.xw, vals);
#pragma unroll
        for (int i = 0; i < W; ++i) row[2 * W + i] = vals[i];
      } else {
#pragma unroll
        for (int i = 0; i < W; ++i) row[2 * W + i] = R(i == 0);
      }
    }
  }
}

// Staging shared by all NW warps of a CTA that works as one slice (large W
// in FP64): lane l of warp w evaluates kernel values [w Q, (w + 1) Q) of the
// 3W of record l (Q = ceil(3W / NW)), instead of every warp evaluating all of
// them; warp 0 also does the rest of the staging.  The caller brackets it
// with CTA barriers.
template <typename R, int W, int NW, typename Rec>
__device__ __forceinline__ void stage_batch_split(const Rec *recs, int b0, int nb, int lane, int w,
                                                  int tu, int tv, int mp, const DevGeom &g,
                                                  const DevKernel<R> &kc, R *kv, R *vv,
                                                  uint32_t *luv, int *err, int &bb0, int &bb1,
                                                  int &bb2, int &bb3, const void *vis_in,
                                                  int vis_in_double) {
  constexpr int KST = KStride<R, W>::value;
  constexpr int Q = (3 * W + NW - 1) / NW;
  constexpr int DEG = KDeg<W>::value;
  if (lane < nb) {
    const Rec rr = recs[b0 + lane];
    if (w == 0)
      stage_meta<R>(rr, lane, tu, tv, mp, g, vv, luv, err, bb0, bb1, bb2, bb3, vis_in,
                    vis_in_double);
    R *row = kv + lane * KST;
#pragma unroll
    for (int qi = 0; qi < Q; ++qi) {
      const int v = w * Q + qi;  // the same for every lane of the warp
      if (v < 3 * W) {
        const int axis = v / W, piece = v - axis * W;
        R val;
        if (axis == 2 && !g.do_w) {
          val = R(piece == 0);
        } else {
          const R x = axis == 0 ? rr.xu : (axis == 1 ? rr.xv : rr.xw);
          val = kc.c[DEG][piece];
#pragma unroll
          for (int j = DEG - 1; j >= 0; --j) val = fma(val, x, kc.c[j][piece]);
        }
        row[v] = val;
      }
    }
  }
}

// Warps sharing one record's footprint: when more than half the warps would,
// all of them do, as one slice whose warps also share the record staging.
template <int W, int PPL, int NWARP>
struct WarpGroups {
  static constexpr int NG0 = (W * W + 32 * PPL - 1) / (32 * PPL);
  static constexpr int NG = NG0 > NWARP / 2 ? NWARP : NG0;
  static constexpr int NSL = NWARP / NG;
  static constexpr bool SPLIT = (NG == NWARP) && NG > 1;
};

// Warp sums of G complex values at once (G = 1, 2, 4 or 8), as a
// reduce-scatter: at each of the first log2(G) butterfly stages a lane keeps
// the half of its values that its lane bit names and adds the partner's
// copy of that half, so G sums cost about 2G + 2 log2(32/G) shuffles instead
// of 10 G.  On return every lane holds the total of value
// (lane >> (5 - log2 G)) & (G - 1).
template <int G, typename C>
__device__ __forceinline__ C warp_sum_scatter(C (&v)[G], int lane) {
  constexpr int LG = G == 1 ? 0 : G == 2 ? 1 : G == 4 ? 2 : 3;
  static_assert((1 << LG) == G, "warp_sum_scatter: G must be 1, 2, 4 or 8");
#pragma unroll
  for (int st = 0; st < LG; ++st) {
    const int b = 4 - st;
    const int n = G >> st;  // values held before this stage
    const bool hi = (lane >> b) & 1;
#pragma unroll
    for (int i = 0; i < n / 2; ++i) {
      C send = hi ? v[i] : v[n / 2 + i];
      const C keep = hi ? v[n / 2 + i] : v[i];
      send.x = __shfl_xor_sync(0xffffffffu, send.x, 1 << b);
      send.y = __shfl_xor_sync(0xffffffffu, send.y, 1 << b);
      v[i] = cadd(keep, send);
    }
  }
  C t = v[0];
#pragma unroll
  for (int b = 4 - LG; b >= 0; --b) {
    t.x += __shfl_xor_sync(0xffffffffu, t.x, 1 << b);
    t.y += __shfl_xor_sync(0xffffffffu, t.y, 1 << b);
  }
  return t;
}

__device__ __forceinline__ void warp_minmax(int &bb0, int &bb1, int &bb2, int &bb3) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    bb0 = min(bb0, __shfl_xor_sync(0xffffffffu, bb0, o));
    bb1 = max(bb1, __shfl_xor_sync(0xffffffffu, bb1, o));
    bb2 = min(bb2, __shfl_xor_sync(0xffffffffu, bb2, o));
    bb3 = max(bb3, __shfl_xor_sync(0xffffffffu, bb3, o));
  }
}

// ------------------------------------------------------------- k_spread
//
// Persistent CTAs drain chunks; all records of a chunk share one
// (tile, minplane) bin, so the CTA owns a W-plane shared-memory tile
// (structure of arrays: real parts, then imaginary parts) for the chunk.  Each
// warp takes a contiguous slice of the chunk; lane q owns PPL (plane, u-row)
// pairs of the footprint and the W cells along v of each, accumulating in
// registers while consecutive records share the footprint origin (records are
// sorted by position inside the tile), then commits with shared-memory
// atomics.  At the end of the chunk the touched region is added to the u-band
// grid with vector atomics.
// Atomically reads a shared-memory cell and leaves zero in it.
__device__ __forceinline__ float take_zero(float *p) { return atomicExch(p, 0.0f); }
__device__ __forceinline__ double take_zero(double *p) {
  return __longlong_as_double(
      (long long)atomicExch(reinterpret_cast<unsigned long long *>(p), 0ull));
}

// Chunks touching few distinct footprint origins are flushed / staged
// footprint by footprint instead of over their bounding box.
constexpr int kMaxOrig = 64;

template <typename R, int W, int PPL, int NWARP>
__global__ void __launch_bounds__(NWARP * 32, sizeof(R) == 4 ? 3 : 1)
k_spread(GridArgs a, DevGeom g, DevKernel<R> kc) {
  using Rec = typename RecOf<R>::type;
  using C = typename Cplx<R>::type;
  constexpr int NG = WarpGroups<W, PPL, NWARP>::NG;    // warps per record
  constexpr int NSL = WarpGroups<W, PPL, NWARP>::NSL;  // record slices
  constexpr bool SPLIT = WarpGroups<W, PPL, NWARP>::SPLIT;
  constexpr int KST = KStride<R, W>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TileLayout tl = a.tl;
  R *tre = reinterpret_cast<R *>(smem_raw);
  R *tim = tre + W * tl.PS;
  __shared__ int sh_chunk, sh_bb[4], sh_norig;
  __shared__ uint32_t sh_orig[kMaxOrig];
  __shared__ JobGeom sh_job;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = warp % NG, slice = warp / NG;
  // the warp's own staging area, and the one it reads records from (warp 0's
  // when the CTA's warps share the staging)
  unsigned char *wown = smem_raw + size_t(2 * W * tl.PS) * sizeof(R) + warp * WarpStage<R, W>::bytes;
  unsigned char *wbase = SPLIT ? smem_raw + size_t(2 * W * tl.PS) * sizeof(R) : wown;
  R *kv = reinterpret_cast<R *>(wbase);
  R *vv = kv + 32 * KST;
  uint32_t *luvs = reinterpret_cast<uint32_t *>(vv + 64);
  const Rec *recs = reinterpret_cast<const Rec *>(a.rec);

  for (int i = tid; i < 2 * W * tl.PS; i += blockDim.x) tre[i] = R(0);
  int pp[PPL], cu[PPL];
#pragma unroll
  for (int k = 0; k < PPL; ++k) {
    const int q = grp * 32 * PPL + lane + 32 * k;
    pp[k] = q / W;
    cu[k] = q - pp[k] * W;
  }

  for (;;) {
    __syncthreads();
    if (tid == 0) {
      sh_chunk = atomicAdd(a.counter, 1);
      sh_bb[0] = 1 << 30; sh_bb[1] = -1; sh_bb[2] = 1 << 30; sh_bb[3] = -1;
      sh_norig = 0;
      if (sh_chunk < *a.nchunks) sh_job = load_job(a, g, sh_chunk);
    }
    __syncthreads();
    const int ch = sh_chunk;
    if (ch >= *a.nchunks) break;
    const JobGeom &jb = sh_job;  // read from shared memory where used
    const int s0 = a.chunk_start[ch];
    const int s1 = (ch + 1 < *a.nchunks) ? a.chunk_start[ch + 1] : a.nvis;
    const Rec r0 = recs[s0];
    const int tu = int(r0.iuv >> 16) / g.T, tv = int(r0.iuv & 0xffffu) / g.T;
    const int mp = int(r0.mp);
    if (!((mp < jb.pb1) && (mp + W > jb.pb0))) continue;

    if (slice < NSL) {
      const int n = s1 - s0;
      const int j0 = s0 + (n * slice) / NSL, j1 = s0 + (n * (slice + 1)) / NSL;
      bool ok[PPL];
#pragma unroll
      for (int k = 0; k < PPL; ++k)
        ok[k] = (pp[k] < W) && (mp + pp[k] >= jb.pb0) && (mp + pp[k] < jb.pb1);
      // (re, im) accumulators; in FP32 updated with Blackwell's packed
      // two-lane FMA (one instruction per complex cell)
      C acc[PPL][W];
#pragma unroll
      for (int k = 0; k < PPL; ++k)
#pragma unroll
        for (int c = 0; c < W; ++c) acc[k][c].x = acc[k][c].y = R(0);
      uint32_t cur = 0xffffffffu;
      int bb0 = 1 << 30, bb1 = -1, bb2 = 1 << 30, bb3 = -1;
      // the lane's kernel-row indices and tile offsets, fixed for the chunk
      int kwi[PPL], kui[PPL], coff[PPL];
#pragma unroll
      for (int k = 0; k < PPL; ++k) {
        kwi[k] = 2 * W + (ok[k] ? pp[k] : 0);
        kui[k] = ok[k] ? cu[k] : 0;
        coff[k] = pp[k] * tl.PS + cu[k] * tl.RS;
      }
      // When every warp works on the same records (SPLIT), the warps reach
      // each commit together, and for one origin every tile cell belongs to
      // one lane: a barrier before the commit orders it after the previous
      // origin's, and the commit is a plain read-modify-write (FP64 shared
      // atomics cost a quarter of the spread).  Otherwise warps of other
      // slices may commit to the same cells at any time: shared atomics.
      auto commit = [&]() {
        if (cur >= kSkip) return;  // nothing accumulated, or skipped records only (uniform)
        if constexpr (SPLIT) __syncthreads();
        const int o = int(cur >> 16) * tl.RS + int(cur & 0xffffu);
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
          if (!ok[k]) continue;
          const int base = coff[k] + o;
#pragma unroll
          for (int c = 0; c < W; ++c) {
            if constexpr (SPLIT) {
              tre[base + c] += acc[k][c].x;
              tim[base + c] += acc[k][c].y;
            } else {
              atomicAdd(&tre[base + c], acc[k][c].x);
              atomicAdd(&tim[base + c], acc[k][c].y);
            }
            acc[k][c].x = acc[k][c].y = R(0);
          }
        }
      };
      for (int b0 = j0; b0 < j1; b0 += 32) {
        const int nb = min(32, j1 - b0);
        if constexpr (SPLIT) {
          __syncthreads();  // every warp is done with the previous batch
          stage_batch_split<R, W, NWARP>(recs, b0, nb, lane, warp, tu, tv, mp, g, kc, kv, vv,
                                         luvs, a.err, bb0, bb1, bb2, bb3, a.vis_in,
                                         a.vis_in_double);
          __syncthreads();
        } else {
          stage_batch<R, W>(recs, b0, nb, lane, tu, tv, mp, g, kc, kv, vv, luvs, a.err, bb0, bb1,
                            bb2, bb3, a.vis_in, a.vis_in_double);
          __syncwarp();
        }
        if (grp == 0) {
          // the batch's new footprint origins, by a ballot over the staged
          // records (a skipped record counts as one; a repeated origin in the
          // list is harmless, its cells being taken by atomic exchange)
          const uint32_t my = lane < nb ? luvs[lane] : 0u;
          uint32_t prev = __shfl_up_sync(0xffffffffu, my, 1);
          if (lane == 0) prev = cur;
          const unsigned nm = __ballot_sync(0xffffffffu, lane < nb && my != prev && my != kSkip);
          if (nm) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&sh_norig, __popc(nm));
            base = __shfl_sync(0xffffffffu, base, 0);
            const int k = base + __popc(nm & ((1u << lane) - 1u));
            if (((nm >> lane) & 1u) && k < kMaxOrig) sh_orig[k] = my;
          }
        }
        for (int jj = 0; jj < nb; ++jj) {
          const uint32_t luv = luvs[jj];
          if (__any_sync(0xffffffffu, luv != cur)) {  // warp-uniform: luv is one value
            commit();
            cur = luv;
          }
          const R *kb = kv + jj * KST;
          R kvv[W];
          lds_row<W>(kb + W, kvv);
          const C vx = reinterpret_cast<const C *>(vv)[jj];
          const R vr = vx.x, vi = vx.y;
#pragma unroll
          for (int k = 0; k < PPL; ++k) {
            const R f = kb[kwi[k]] * kb[kui[k]];
            C a;
            a.x = vr * f;
            a.y = vi * f;
#pragma unroll
            for (int c = 0; c < W; ++c) acc[k][c] = cfma_real(a, kvv[c], acc[k][c]);
          }
        }
        __syncwarp();
      }
      commit();
      warp_minmax(bb0, bb1, bb2, bb3);
      if (lane == 0 && bb1 >= 0) {
        atomicMin(&sh_bb[0], bb0); atomicMax(&sh_bb[1], bb1);
        atomicMin(&sh_bb[2], bb2); atomicMax(&sh_bb[3], bb3);
      }
    }
    __syncthreads();
    // flush the touched cells of the tile to the band grid: footprint by
    // footprint when few origins were used (a cell shared by two footprints
    // is taken by atomic exchange, so it is added once), else the bounding box
    const int lu0 = sh_bb[0], lv0 = sh_bb[2];
    const int nbu = max(sh_bb[1] + W - lu0, 0), nbv = max(sh_bb[3] + W - lv0, 0);
    const int ucorner = tu * g.T - g.nsafe, vcorner = tv * g.T - g.nsafe;
    const int norig = sh_norig;
    const bool by_list = norig <= kMaxOrig && norig * W * W < nbu * nbv;
    // one (plane, row) line per warp-iteration, lanes along v (no divisions);
    // the line's band row is found once, then each cell only wraps v
    const int nline = by_list ? norig * W * W : W * nbu;
    const int linelen = by_list ? W : nbv;
    const JobRegs jr(jb);
    // bounding-box lines: (plane, row) of line = p nbu + r, stepped without
    // a division
    int bp = 0, br = warp;
    while (!by_list && nbu > 0 && br >= nbu) { br -= nbu; ++bp; }
    for (int line = warp; line < nline; line += NWARP) {
      int p, ia, ib0;
      if (by_list) {
        const int o = line / (W * W), pr = line - o * W * W;
        p = pr / W;
        const uint32_t luv = sh_orig[o];
        ia = int(luv >> 16) + (pr - p * W);
        ib0 = int(luv & 0xffffu);
      } else {
        p = bp;
        ia = lu0 + br;
        ib0 = lv0;
        br += NWARP;
        while (br >= nbu) { br -= nbu; ++bp; }
      }
      const int plane = mp + p;
      const int bi = jr.band_row(jr.wrap_u(ucorner + ia));
      C *const rowp = (plane >= jr.pb0 && plane < jr.pb1 && bi >= 0)
                          ? reinterpret_cast<C *>(jr.grid) +
                                (size_t(bi) * jr.P + (plane - jr.pb0)) * size_t(jr.nv)
                          : nullptr;
      R *const lre = tre + p * tl.PS + ia * tl.RS;
      R *const lim = tim + p * tl.PS + ia * tl.RS;
      for (int c = lane; c < linelen; c += 32) {
        const int ib = ib0 + c;
        R xr, xi;
        if (by_list) {
          xr = take_zero(&lre[ib]);
          xi = take_zero(&lim[ib]);
        } else {
          xr = lre[ib];
          xi = lim[ib];
          lre[ib] = R(0);
          lim[ib] = R(0);
        }
        if (rowp && (xr != R(0) || xi != R(0))) {
          C *dst = rowp + jr.wrap_v(vcorner + ib);
          if constexpr (sizeof(R) == 4) {
            atomicAdd(reinterpret_cast<float2 *>(dst), make_float2(xr, xi));
          } else {
            atomicAdd(&dst->x, xr);
            atomicAdd(&dst->y, xi);
          }
        }
      }
    }
  }
}

// Writes (or, for batch plans, atomically adds) one degridded visibility.
__device__ __forceinline__ void store_vis(void *out, int dbl, int accumulate, uint32_t idx,
                                          double re, double im) {
  if (dbl) {
    double2 *p = reinterpret_cast<double2 *>(out) + idx;
    if (accumulate) {
      atomicAdd(&p->x, re);
      atomicAdd(&p->y, im);
    } else {
      *p = make_double2(re, im);
    }
  } else {
    float2 *p = reinterpret_cast<float2 *>(out) + idx;
    if (accumulate)
      atomicAdd(p, make_float2(float(re), float(im)));
    else
      *p = make_float2(float(re), float(im));
  }
}

// ------------------------------------------------------------- k_interp
//
// Degridding, the exact transpose of k_spread: the chunk's tile region is
// staged from the band grid into shared memory, each lane caches its
// (plane, u-row) x W cells in registers while the footprint origin repeats,
// and the kernel-weighted sum is reduced across the warp.  With one warp per
// record and a single plane pass the result is finalised in place
// (conjugation, conjugate shift phasor and weight); otherwise partial sums
// go to a per-record accumulator finalised by k_finalize.
// IG: records whose warp sums are formed together (4 measured fastest, 8
// close behind, 1 -- a full butterfly per record -- 10% slower overall)
template <typename R, int W, int PPL, int NWARP, int IG = 4>
__global__ void __launch_bounds__(NWARP * 32, sizeof(R) == 4 ? 3 : 1)
k_interp(GridArgs a, DevGeom g, DevKernel<R> kc) {
  using Rec = typename RecOf<R>::type;
  using C = typename Cplx<R>::type;
  constexpr int NG = WarpGroups<W, PPL, NWARP>::NG;
  constexpr int NSL = WarpGroups<W, PPL, NWARP>::NSL;
  constexpr bool SPLIT = WarpGroups<W, PPL, NWARP>::SPLIT;
  constexpr int KST = KStride<R, W>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TileLayout tl = a.tl;
  R *tre = reinterpret_cast<R *>(smem_raw);
  R *tim = tre + W * tl.PS;
  __shared__ int sh_chunk, sh_bb[4], sh_norig;
  __shared__ uint32_t sh_orig[kMaxOrig];
  __shared__ JobGeom sh_job;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = warp % NG, slice = warp / NG;
  // the warp's own staging area, and the one it reads records from (warp 0's
  // when the CTA's warps share the staging)
  unsigned char *wown = smem_raw + size_t(2 * W * tl.PS) * sizeof(R) + warp * WarpStage<R, W>::bytes;
  unsigned char *wbase = SPLIT ? smem_raw + size_t(2 * W * tl.PS) * sizeof(R) : wown;
  R *kv = reinterpret_cast<R *>(wbase);
  R *vv = kv + 32 * KST;
  uint32_t *luvs = reinterpret_cast<uint32_t *>(vv + 64);
  const Rec *recs = reinterpret_cast<const Rec *>(a.rec);
  // finalised in place in a single plane pass, when one warp owns each
  // record or all warps share every record (SPLIT: warp 0 adds their sums)
  const bool direct = a.last_pass && a.first_pass && (NG == 1 || SPLIT);

  int pp[PPL], cu[PPL];
  bool ok[PPL];
#pragma unroll
  for (int k = 0; k < PPL; ++k) {
    const int q = grp * 32 * PPL + lane + 32 * k;
    pp[k] = q / W;
    cu[k] = q - pp[k] * W;
    ok[k] = q < W * W;
  }

  for (;;) {
    __syncthreads();
    if (tid == 0) {
      sh_chunk = atomicAdd(a.counter, 1);
      sh_bb[0] = 1 << 30; sh_bb[1] = -1; sh_bb[2] = 1 << 30; sh_bb[3] = -1;
      sh_norig = 0;
      if (sh_chunk < *a.nchunks) sh_job = load_job(a, g, sh_chunk);
    }
    __syncthreads();
    const int ch = sh_chunk;
    if (ch >= *a.nchunks) break;
    const JobGeom &jb = sh_job;  // read from shared memory where used
    const int s0 = a.chunk_start[ch];
    const int s1 = (ch + 1 < *a.nchunks) ? a.chunk_start[ch + 1] : a.nvis;
    const Rec r0 = recs[s0];
    const int tu = int(r0.iuv >> 16) / g.T, tv = int(r0.iuv & 0xffffu) / g.T;
    const int mp = int(r0.mp);
    if (!((mp < jb.pb1) && (mp + W > jb.pb0))) continue;  // contributes nothing this pass
    // bounding box and distinct footprint origins of the chunk
    for (int s = s0 + tid; s < s1; s += blockDim.x) {
      const uint32_t iuv = recs[s].iuv;
      const int lu = int(iuv >> 16) - tu * g.T, lv = int(iuv & 0xffffu) - tv * g.T;
      if (lu < 0 || lu >= g.T || lv < 0 || lv >= g.T) continue;
      atomicMin(&sh_bb[0], lu); atomicMax(&sh_bb[1], lu);
      atomicMin(&sh_bb[2], lv); atomicMax(&sh_bb[3], lv);
      if (s == s0 || recs[s - 1].iuv != iuv) {
        const int k = atomicAdd(&sh_norig, 1);
        if (k < kMaxOrig) sh_orig[k] = (uint32_t(lu) << 16) | uint32_t(lv);
      }
    }
    __syncthreads();
    {
      // stage the cells the chunk reads: footprint by footprint when few
      // origins are used (cells shared by footprints are written twice with
      // the same value), else the bounding box; eight loads in flight
      const int lu0 = sh_bb[0], lv0 = sh_bb[2];
      const int nbu = max(sh_bb[1] + W - lu0, 0), nbv = max(sh_bb[3] + W - lv0, 0);
      const int ucorner = tu * g.T - g.nsafe, vcorner = tv * g.T - g.nsafe;
      const int norig = sh_norig;
      const bool by_list = norig <= kMaxOrig && norig * W * W < nbu * nbv;
      // (plane, row) lines over warps, lanes along v, eight lines in flight
      const int nline = by_list ? norig * W * W : W * nbu;
      const int linelen = by_list ? W : nbv;
      const JobRegs jr(jb);
      // bounding-box lines: (plane, row) of line = p nbu + r, stepped by
      // NWARP lines without a division
      int bp = 0, br = warp;
      while (!by_list && nbu > 0 && br >= nbu) { br -= nbu; ++bp; }
      for (int l0 = warp; l0 < nline; l0 += 8 * NWARP) {
        C val[8];
        int sidx[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int line = l0 + q * NWARP;
          const int lp = bp, lr = br;
          if (!by_list) {
            br += NWARP;
            while (br >= nbu) { br -= nbu; ++bp; }
          }
          val[q].x = R(0);
          val[q].y = R(0);
          sidx[q] = -1;
          if (line < nline && lane < linelen) {
            int p, ia, ib;
            if (by_list) {
              const int o = line / (W * W), pr = line - o * W * W;
              p = pr / W;
              const uint32_t luv = sh_orig[o];
              ia = int(luv >> 16) + (pr - p * W);
              ib = int(luv & 0xffffu) + lane;
            } else {
              p = lp;
              ia = lu0 + lr;
              ib = lv0 + lane;
            }
            sidx[q] = p * tl.PS + ia * tl.RS + ib;
            const int plane = mp + p;
            if (plane >= jr.pb0 && plane < jr.pb1) {
              const int bi = jr.band_row(jr.wrap_u(ucorner + ia));
              if (bi >= 0)
                val[q] = reinterpret_cast<const C *>(jr.grid)[(size_t(bi) * jr.P + (plane - jr.pb0)) *
                                                                  size_t(jr.nv) +
                                                              jr.wrap_v(vcorner + ib)];
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          if (sidx[q] >= 0) {
            tre[sidx[q]] = val[q].x;
            tim[sidx[q]] = val[q].y;
          }
        }
      }
    }
    __syncthreads();
    if (slice < NSL) {
      const int n = s1 - s0;
      const int j0 = s0 + (n * slice) / NSL, j1 = s0 + (n * (slice + 1)) / NSL;
      C cl[PPL][W];  // the lane's cells (re, im) at the current origin
      uint32_t cur = 0xffffffffu;
      int bb0 = 0, bb1 = 0, bb2 = 0, bb3 = 0;
      for (int b0 = j0; b0 < j1; b0 += 32) {
        const int nb = min(32, j1 - b0);
        if constexpr (SPLIT) {
          __syncthreads();  // every warp is done with the previous batch
          stage_batch_split<R, W, NWARP>(recs, b0, nb, lane, warp, tu, tv, mp, g, kc, kv, vv,
                                         luvs, a.err, bb0, bb1, bb2, bb3, a.vis_in,
                                         a.vis_in_double);
          __syncthreads();
        } else {
          stage_batch<R, W>(recs, b0, nb, lane, tu, tv, mp, g, kc, kv, vv, luvs, a.err, bb0, bb1,
                            bb2, bb3, a.vis_in, a.vis_in_double);
          __syncwarp();
        }
        // record sums of the batch, G records at a time (reduce-scatter);
        // the staged visibility slots of the warp are free here and hold them
        constexpr int G = IG;
        constexpr int LG = G == 1 ? 0 : G == 2 ? 1 : G == 4 ? 2 : 3;
        R *osum = reinterpret_cast<R *>(wown) + 32 * KST;
        for (int g0 = 0; g0 < nb; g0 += G) {
          C part[G];
#pragma unroll
          for (int r = 0; r < G; ++r) {
            part[r].x = part[r].y = R(0);
            const int jj = g0 + r;
            if (jj >= nb) continue;
            const uint32_t luv = luvs[jj];
            if (luv == kSkip) continue;
            if (luv != cur) {
              cur = luv;
              const int lu = int(luv >> 16), lv = int(luv & 0xffffu);
#pragma unroll
              for (int k = 0; k < PPL; ++k) {
                const int base = (ok[k] ? pp[k] * tl.PS + (lu + cu[k]) * tl.RS : 0) + lv;
#pragma unroll
                for (int c = 0; c < W; ++c) {
                  cl[k][c].x = ok[k] ? tre[base + c] : R(0);
                  cl[k][c].y = ok[k] ? tim[base + c] : R(0);
                }
              }
            }
            const R *kb = kv + jj * KST;
            R kvv[W];
            lds_row<W>(kb + W, kvv);
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
              C t;
              t.x = t.y = R(0);
#pragma unroll
              for (int c = 0; c < W; ++c) t = cfma_real(cl[k][c], kvv[c], t);
              const R f = ok[k] ? kb[2 * W + pp[k]] * kb[cu[k]] : R(0);
              part[r] = cfma_real(t, f, part[r]);
            }
          }
          const C tot = warp_sum_scatter<G>(part, lane);
          const int ridx = g0 + ((lane >> (5 - LG)) & (G - 1));
          if ((lane & ((32 >> LG) - 1)) == 0 && ridx < nb) {
            osum[2 * ridx] = tot.x;
            osum[2 * ridx + 1] = tot.y;
          }
        }
        __syncwarp();
        R osr = lane < nb ? osum[2 * lane] : R(0);
        R osi = lane < nb ? osum[2 * lane + 1] : R(0);
        if constexpr (SPLIT) {
          // every warp summed its pairs of the same records: warp 0 adds the
          // warps' sums from their staging areas (free until the next
          // batch's barrier), so each record has one writer
          __syncthreads();
          if (warp == 0 && lane < nb) {
            for (int w = 1; w < NWARP; ++w) {
              const R *os = reinterpret_cast<const R *>(
                                smem_raw + size_t(2 * W * tl.PS) * sizeof(R) +
                                size_t(w) * WarpStage<R, W>::bytes) + 32 * KST;
              osr += os[2 * lane];
              osi += os[2 * lane + 1];
            }
          }
        }
        // lanes finalise their own records of the batch together (one
        // coalesced record load, instead of one lane per record in turn)
        if ((!SPLIT || warp == 0) && lane < nb && luvs[lane] != kSkip) {
          const int s = b0 + lane;
          if (direct) {
            const Rec rr = recs[s];
            const uint32_t idx = rr.idx & 0x7fffffffu;
            const R si = (rr.idx & 0x80000000u) ? -osi : osi;
            const double orr = double(rr.vr) * double(osr) - double(rr.vi) * double(si);
            const double oi = double(rr.vr) * double(si) + double(rr.vi) * double(osr);
            store_vis(a.vis_out, a.vis_double, a.vis_accumulate, idx, orr, oi);
          } else if constexpr (SPLIT) {  // the record's one writer in this pass
            C *accp = reinterpret_cast<C *>(a.acc) + s;
            accp->x += osr;
            accp->y += osi;
          } else {
            C *accp = reinterpret_cast<C *>(a.acc) + s;
            atomicAdd(&accp->x, osr);
            atomicAdd(&accp->y, osi);
          }
        }
        __syncwarp();
      }
    }
  }
}

// Finalises degridded visibilities accumulated over plane passes or warp
// groups: out[idx] = P * (flip ? conj(acc) : acc) (added into out when
// accumulating).
template <typename R>
__global__ void k_finalize(int nvis, const void *recv, const void *accv, void *vis_out,
                           int vis_double, int vis_accumulate) {
  using Rec = typename RecOf<R>::type;
  using C = typename Cplx<R>::type;
  const Rec *recs = reinterpret_cast<const Rec *>(recv);
  const C *acc = reinterpret_cast<const C *>(accv);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nvis; s += gridDim.x * blockDim.x) {
    const Rec rr = recs[s];
    double sr = double(acc[s].x), si = double(acc[s].y);
    if (rr.idx & 0x80000000u) si = -si;
    const uint32_t idx = rr.idx & 0x7fffffffu;
    const double orr = double(rr.vr) * sr - double(rr.vi) * si;
    const double oi = double(rr.vr) * si + double(rr.vi) * sr;
    store_vis(vis_out, vis_double, vis_accumulate, idx, orr, oi);
  }
}

// ------------------------------------------------ shared-memory FFTs
//
// The transform along u of one image column is pruned on both sides: only
// the occupied u band [-L, L] holds data and only the nx image rows are
// needed.  With nu = K*M, M = 2^m >= 2L+1, the length-nu DFT splits into K
// length-M DFTs of the band data twisted by exp(+-2 pi i u k2 / nu):
//     F(K k1 + k2) = sum_u [g(u) e^{2 pi i u k2/nu}] e^{2 pi i u k1/M}.
// Each is a radix-16 Stockham FFT in shared memory by M/16 threads holding 16
// values each; twiddles come from FP64-computed tables.

__host__ __device__ constexpr double cos16(int e) {
  return e == 0 ? 1.0 : e == 1 ? 0.92387953251128673848 : e == 2 ? 0.70710678118654752440
       : e == 3 ? 0.38268343236508977173 : e == 4 ? 0.0 : e == 5 ? -0.38268343236508977173
       : e == 6 ? -0.70710678118654752440 : e == 7 ? -0.92387953251128673848 : -1.0;
}
__host__ __device__ constexpr double sin16(int e) {
  return e == 0 ? 0.0 : e == 1 ? 0.38268343236508977173 : e == 2 ? 0.70710678118654752440
       : e == 3 ? 0.92387953251128673848 : e == 4 ? 1.0 : e == 5 ? 0.92387953251128673848
       : e == 6 ? 0.70710678118654752440 : e == 7 ? 0.38268343236508977173 : 0.0;
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

// In-register DFT of N <= 16 points: v[q] <- sum_r v[r] exp(sign 2 pi i r q / N),
// as radix-2 Stockham stages (natural order in and out, so every register
// index is a compile-time constant once the loops are unrolled).
template <int N, typename C>
__device__ __forceinline__ void dft_reg(C *v, int sign) {
  using R = decltype(v[0].x);
  constexpr int LOG = N == 2 ? 1 : N == 4 ? 2 : N == 8 ? 3 : 4;
  static_assert((1 << LOG) == N, "dft_reg: N must be 2, 4, 8 or 16");
#pragma unroll
  for (int s = 0; s < LOG; ++s) {
    const int NS = 1 << s;
    C y[N];
#pragma unroll
    for (int j = 0; j < N / 2; ++j) {
      const int k = j & (NS - 1);
      const C a = v[j];
      C b = v[j + N / 2];
      const int e = k * (8 / NS);  // twiddle exp(sign 2 pi i k / (2 NS)) in 16ths of a turn
      if (e == 4) {  // w = sign * i
        const R bx = b.x;
        b.x = sign > 0 ? -b.y : b.y;
        b.y = sign > 0 ? bx : -bx;
      } else if (e == 2 || e == 6) {  // w = (+-1 + sign i) / sqrt(2)
        const R h = R(0.70710678118654752440);
        const R c = (e == 2) ? h : -h, sn = sign > 0 ? h : -h;
        const R bx = b.x;
        b.x = c * bx - sn * b.y;
        b.y = c * b.y + sn * bx;
      } else if (e != 0) {
        C w;
        w.x = R(cos16(e));
        w.y = R(sign * sin16(e));
        b = cmul(b, w);
      }
      const int d = (j / NS) * 2 * NS + k;
      y[d] = cadd(a, b);
      y[d + NS] = csub(a, b);
    }
#pragma unroll
    for (int j = 0; j < N; ++j) v[j] = y[j];
  }
}

// Buffer index with one padding slot per 16 elements: the first radix-16
// stage writes at a stride of 16 elements, which without padding puts every
// lane of a warp on the same shared-memory banks.
__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }
template <int M> struct FftBuf { static constexpr int value = M + M / 16; };

// Per-stage twiddle tables: the stage with stride NS > 1 and radix R needs
// exp(+2 pi i r k / (NS R)) for r in [1, R), k in [0, NS); stored [r-1][k]
// (consecutive lanes read consecutive k), concatenated in stage order.
// (every stage before the last has radix 16, so the stage with stride NS
// starts after the tables of strides 16, 256, ..., NS/16).
template <int NS>
struct TwOffset {
  static constexpr int value = (NS <= 16) ? 0 : TwOffset<NS / 16>::value + 15 * (NS / 16);
};
template <>
struct TwOffset<1> {
  static constexpr int value = 0;
};

// Stockham autosort stages on buf (in place: each stage reads all its inputs
// before a barrier, then writes).  tw: the per-stage tables above.
template <typename C, int M, int NS, int TPF>
struct FftStages {
  static __device__ __forceinline__ void run(C *buf, const C *tw, int t, int sign) {
    if constexpr (NS < M) {
      constexpr int R = (M / NS >= 16) ? 16 : M / NS;
      constexpr int ITEMS = (M / R) / TPF;
      C v[ITEMS][R];
#pragma unroll
      for (int it = 0; it < ITEMS; ++it) {
        const int j = t + TPF * it;
#pragma unroll
        for (int r = 0; r < R; ++r) v[it][r] = buf[fpad(j + r * (M / R))];
      }
      __syncthreads();
#pragma unroll
      for (int it = 0; it < ITEMS; ++it) {
        const int j = t + TPF * it;
        const int k = j & (NS - 1);
        if constexpr (NS > 1) {
          constexpr int off = TwOffset<NS>::value;
#pragma unroll
          for (int r = 1; r < R; ++r) {
            C w = tw[off + (r - 1) * NS + k];
            if (sign < 0) w.y = -w.y;
            v[it][r] = cmul(v[it][r], w);
          }
        }
        dft_reg<R>(v[it], sign);
        const int d = (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[fpad(d + r * NS)] = v[it][r];
      }
      __syncthreads();
      FftStages<C, M, NS * R, TPF>::run(buf, tw, t, sign);
    }
  }
};

struct ColArgs {
  int nx, ny, nu, nv;
  int P, npl;           // planes in the band layout, planes in this pass
  int L, band_rows, band_full, K;
  const void *twM;      // per-stage FFT twiddles, M entries
  const void *twB;      // exp(+2 pi i t k2 / nu), [k2][t], K x M/16 entries
  const void *twQ;      // exp(+2 pi i (M/16 q - neg M) k2 / nu), [k2][q][neg], K x 32
  void *band;           // [band_rows][P][nv] complex
  void *H;              // [P][ny][K * hseg] complex: u-transformed image columns
  int hseg, hm0;        // row layout of H (GridPlan::hseg / hm0)
};

// Offset in an H row of output q of thread t in pass k2 (m = t + TPF q, the
// upper half of the outputs being the negative frequencies m - M), and
// whether that output is one of the nx image rows kept.
template <int TPF>
__device__ __forceinline__ int h_pos(const ColArgs &a, int k2, int t, int q, bool &keep) {
  const int mq = t + TPF * (q < 8 ? q : q - 16);
  const int i = a.K * mq + k2 + a.nx / 2;
  keep = unsigned(i) < unsigned(a.nx);
  return k2 * a.hseg + (mq - a.hm0);
}

// u of buffer slot b (b in [0, M)), or a value > nu if the slot is empty.
__device__ __forceinline__ int slot_u(const ColArgs &a, int b, int M) {
  if (a.band_full) return b;           // K == 1, M == nu: every row
  if (b <= a.L) return b;
  if (b >= M - a.L) return b - M;      // negative u
  return 1 << 30;
}
__device__ __forceinline__ int slot_bi(const ColArgs &a, int u) {
  return (a.band_full || u >= 0) ? u : u + a.band_rows;
}

// Columns per CTA (NB) and threads: M/16 threads per column, up to 512
// threads per CTA in mixed precision and 256 in FP64 (register budget).
template <typename R, int M>
struct ColCfg {
  static constexpr int TPF = M / 16;
  static constexpr int MAXT = 256;
  static constexpr int NB = (MAXT / TPF) > 8 ? 8 : ((MAXT / TPF) < 1 ? 1 : MAXT / TPF);
  static constexpr int THREADS = NB * TPF;
  // resident CTAs asked of the register allocator (128 registers a thread
  // for FP32 at 256 threads)
  static constexpr int MINB = (sizeof(R) == 4 && THREADS <= 256) ? 2 : 1;
};

// Shared memory of a column CTA: NB padded buffers, then the M twiddles.
template <typename R, int M>
struct ColSmem {
  static constexpr size_t bytes() {
    return (size_t(ColCfg<R, M>::NB) * FftBuf<M>::value + M) * 2 * sizeof(R);
  }
};

// ---- column transforms with register-resident first and last stages ----
//
// The M-point transform runs as Stockham stages (radix 16, the last one of
// radix M/NS) but keeps the first stage's inputs and the last stage's outputs
// in registers: thread t of a column group holds positions t + TPF q
// (q = 0..15) on both ends, which are exactly the first radix-16 stage's
// inputs and (for every power-of-two M) the last stage's outputs.  Only the
// exchanges between stages go through shared memory, ping-ponging between two
// buffers so that each stage needs one barrier.

// Stages after the first, from stride NS on: `cur` holds the data; middle
// stages write `oth` and swap.  The last stage leaves its outputs in o[q] =
// X[t + TPF q].
template <typename C, int M, int NS, int TPF, int SIGN>
__device__ __forceinline__ void col_tail(C *cur, C *oth, const C *tw, int t, C (&o)[16]) {
  if constexpr (M / NS > 16) {
    C v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = cur[fpad(t + r * TPF)];
    const int k = t & (NS - 1);
    constexpr int off = TwOffset<NS>::value;
#pragma unroll
    for (int r = 1; r < 16; ++r) {
      C w = tw[off + (r - 1) * NS + k];
      if (SIGN < 0) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    dft_reg<16>(v, SIGN);
    const int d = (t / NS) * NS * 16 + k;
#pragma unroll
    for (int r = 0; r < 16; ++r) oth[fpad(d + r * NS)] = v[r];
    __syncthreads();
    col_tail<C, M, NS * 16, TPF, SIGN>(oth, cur, tw, t, o);
  } else {
    constexpr int RL = M / NS, IT = 16 / RL;
    constexpr int off = TwOffset<NS>::value;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int j = t + TPF * it;  // < NS: the stage's k is j itself
      C v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) v[r] = cur[fpad(j + r * NS)];
#pragma unroll
      for (int r = 1; r < RL; ++r) {
        C w = tw[off + (r - 1) * NS + j];
        if (SIGN < 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
      dft_reg<RL>(v, SIGN);
#pragma unroll
      for (int r = 0; r < RL; ++r) o[it + r * IT] = v[r];
    }
  }
}

// In-place col_tail: the data in buf, each middle stage reading all its
// inputs before a barrier and writing back in place; the last stage leaves
// its outputs in o[q] = X[t + TPF q].
template <typename C, int M, int NS, int TPF, int SIGN>
__device__ __forceinline__ void col_tail_inplace(C *buf, const C *tw, int t, C (&o)[16]) {
  if constexpr (M / NS > 16) {
    C v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = buf[fpad(t + r * TPF)];
    const int k = t & (NS - 1);
    constexpr int off = TwOffset<NS>::value;
#pragma unroll
    for (int r = 1; r < 16; ++r) {
      C w = tw[off + (r - 1) * NS + k];
      if (SIGN < 0) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    dft_reg<16>(v, SIGN);
    const int d = (t / NS) * NS * 16 + k;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 16; ++r) buf[fpad(d + r * NS)] = v[r];
    __syncthreads();
    col_tail_inplace<C, M, NS * 16, TPF, SIGN>(buf, tw, t, o);
  } else {
    constexpr int RL = M / NS, IT = 16 / RL;
    constexpr int off = TwOffset<NS>::value;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int j = t + TPF * it;
      C v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) v[r] = buf[fpad(j + r * NS)];
#pragma unroll
      for (int r = 1; r < RL; ++r) {
        C w = tw[off + (r - 1) * NS + j];
        if (SIGN < 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
      dft_reg<RL>(v, SIGN);
#pragma unroll
      for (int r = 0; r < RL; ++r) o[it + r * IT] = v[r];
    }
  }
}

// Number of middle (radix-16, not last) stages of an M-point transform.
template <int M>
struct ColMid {
  static constexpr int count() {
    int n = 0;
    for (int NS = 16; M / NS > 16; NS *= 16) ++n;
    return n;
  }
  static constexpr int value = count();
};

// v[q] = x[t + TPF q] -> o[q] = X[t + TPF q].  S and O are the group's two
// buffers; with an even number of middle stages the last stage reads S, so
// the caller alternates S between consecutive transforms.
template <typename C, int M, int TPF, int SIGN>
__device__ __forceinline__ void col_fft(C (&v)[16], C *S, C *O, const C *tw, int t, C (&o)[16]) {
  dft_reg<16>(v, SIGN);
#pragma unroll
  for (int r = 0; r < 16; ++r) S[fpad(16 * t + r)] = v[r];
  __syncthreads();
  col_tail<C, M, 16, TPF, SIGN>(S, O, tw, t, o);
}

// Twist factor exp(+2 pi i u k2 / nu) of slot b = t + TPF q, u = b or b - M
// (the negative half of the band), as base(k2, t) * tq(k2, q, neg); both
// tables are exact FP64 values rounded to R.
template <typename C, int TPF>
__device__ __forceinline__ C col_twist(const ColArgs &a, const C *twB, const C *twQ, int k2,
                                       int t, int q, int M, C base) {
  const int b = t + TPF * q;
  const int neg = (!a.band_full && b >= M - a.L) ? 1 : 0;
  return cmul(__ldg(&twQ[(k2 * 16 + q) * 2 + neg]), base);
}

// Copies N table entries to shared memory with all of a thread's loads in
// flight together (a strided copy loop would wait for each load in turn).
template <typename C, int N, int THREADS>
__device__ __forceinline__ void fill_table(C *dst, const C *src) {
  constexpr int NF = (N + THREADS - 1) / THREADS;
  C tmp[NF];
#pragma unroll
  for (int n = 0; n < NF; ++n) {
    const int i = threadIdx.x + n * THREADS;
    if (i < N) tmp[n] = __ldg(&src[i]);
  }
#pragma unroll
  for (int n = 0; n < NF; ++n) {
    const int i = threadIdx.x + n * THREADS;
    if (i < N) dst[i] = tmp[n];
  }
}

// Shared memory of a column CTA: two padded buffers per column, then the
// M stage twiddles.
template <typename R, int M>
struct ColSmem2 {
  static constexpr size_t bytes() {
    return (size_t(2) * ColCfg<R, M>::NB * FftBuf<M>::value + M) * 2 * sizeof(R);
  }
};

// ms2dirty direction: band rows (after the v transform) -> H image rows,
// backward (+) transform along u, for NB adjacent image columns j and plane lp.
template <typename R, int LOGM>
__global__ void __launch_bounds__(ColCfg<R, (1 << LOGM)>::THREADS, ColCfg<R, (1 << LOGM)>::MINB)
k_ucol_bwd(ColArgs a) {
  using C = typename Cplx<R>::type;
  constexpr int M = 1 << LOGM, TPF = ColCfg<R, M>::TPF, NB = ColCfg<R, M>::NB;
  constexpr int BL = FftBuf<M>::value;
  constexpr bool kFlip = (ColMid<M>::value % 2) == 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *bufall = reinterpret_cast<C *>(smem_raw);
  C *tws = bufall + 2 * NB * BL;
  const int grp = threadIdx.x / TPF, t = threadIdx.x - grp * TPF;
  C *A = bufall + 2 * grp * BL, *B = A + BL;
  const int lp = blockIdx.y;
  const int j = blockIdx.x * NB + grp;
  const bool jv = j < a.ny;
  const C *band = reinterpret_cast<const C *>(a.band);
  const C *twB = reinterpret_cast<const C *>(a.twB);
  const C *twQ = reinterpret_cast<const C *>(a.twQ);
  C *H = reinterpret_cast<C *>(a.H);
  fill_table<C, M, ColCfg<R, M>::THREADS>(tws, reinterpret_cast<const C *>(a.twM));
  // coalesced load (slot-major, adjacent image columns innermost) into the
  // A buffers, all sixteen loads of a thread in flight together
  constexpr int ITEMS = NB * M / ColCfg<R, M>::THREADS;  // 16
  {
    C val[ITEMS];
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int item = threadIdx.x + q * blockDim.x;
      const int c = item % NB, b = item / NB;
      const int jj = blockIdx.x * NB + c;
      val[q].x = R(0);
      val[q].y = R(0);
      const int u = slot_u(a, b, M);
      if (jj < a.ny && u < (1 << 29)) {
        int jx = jj + a.nv - a.ny / 2;
        jx -= (jx >= a.nv) ? a.nv : 0;
        val[q] = band[(size_t(slot_bi(a, u)) * a.P + lp) * a.nv + jx];
      }
    }
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int item = threadIdx.x + q * blockDim.x;
      bufall[(item % NB) * 2 * BL + fpad(item / NB)] = val[q];
    }
  }
  __syncthreads();
  C g[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) g[q] = A[fpad(t + TPF * q)];
  __syncthreads();
  C *rowp = H + (size_t(lp) * a.ny + j) * (size_t(a.K) * a.hseg);
  for (int k2 = 0; k2 < a.K; ++k2) {
    C v[16];
    if (k2 == 0) {
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = g[q];
    } else {
      const C base = __ldg(&twB[k2 * TPF + t]);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = cmul(g[q], col_twist<C, TPF>(a, twB, twQ, k2, t, q, M, base));
    }
    C *S = (kFlip && (k2 & 1)) ? B : A;
    C *O = (kFlip && (k2 & 1)) ? A : B;
    C o[16];
    col_fft<C, M, TPF, +1>(v, S, O, tws, t, o);
    if (jv) {
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        bool keep;
        const int pos = h_pos<TPF>(a, k2, t, q, keep);
        if (keep) rowp[pos] = o[q];
      }
    }
  }
}

// ---- the band columns staged by the tensor memory accelerator ----
//
// k_ucol_bwd_tma is k_ucol_bwd made persistent: each CTA loops over (plane,
// column group) items, and while it transforms one, the tensor memory
// accelerator (cp.async.bulk.tensor, 2-D boxes of NB adjacent columns by up
// to 256 band rows, no multicast) copies the next item's band columns into a
// shared staging buffer, completing on an mbarrier.  The band loads then
// overlap the FFTs instead of stalling each CTA at its start, and the stage
// twiddles are loaded once per CTA instead of once per column group.  The
// transforms run in place in one buffer per column (the staging buffer
// takes the place of the second one).

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return uint32_t(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// One bounded attempt; true once the phase of the given parity completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Waits for the phase with an iteration limit; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Staging of one item: NB adjacent columns of the band rows, in two regions
// that start on box boundaries (every box lands 4 KB-aligned): rows [0, L]
// (u >= 0) in region 1, rows (L, 2L] (u = -L..-1) in region 2 after it; the
// last box of a region may run past its rows (the copy engine fills rows
// past the band with zeros) into the region's pad.  With the full band,
// region 1 holds all M rows.
template <typename R, int M>
struct TmaCfg {
  static constexpr int NB = ColCfg<R, M>::NB;
  static constexpr int BR = 256;                 // rows per box (M >= 256)
  static constexpr int ROWS = M + 2 * BR;        // staging rows
  static constexpr int BOX_BYTES = BR * NB * 2 * int(sizeof(R));
  static constexpr size_t stage_bytes() { return size_t(ROWS) * NB * 2 * sizeof(R); }
};

// Boxes of region 1 (rows [0, L] or all rows with the full band).
__device__ __forceinline__ int tma_boxes1(const ColArgs &a, int M, int BR) {
  return a.band_full ? M / BR : (a.L + 1 + BR - 1) / BR;
}

// Issues the boxes of one item (plane lp, first column j0) into the staging
// buffer and arms the barrier with their bytes (one thread).
template <typename R, int M>
__device__ __forceinline__ void tma_issue_item(const ColArgs &a, const CUtensorMap *map,
                                               typename Cplx<R>::type *stage, uint64_t *bar,
                                               int lp, int j0) {
  using Cfg = TmaCfg<R, M>;
  int jx = j0 + a.nv - a.ny / 2;
  jx -= (jx >= a.nv) ? a.nv : 0;
  const int x = 2 * (lp * a.nv + jx);
  const int n1 = tma_boxes1(a, M, Cfg::BR);
  const int n2 = a.band_full ? 0 : (a.L + Cfg::BR - 1) / Cfg::BR;
  mbar_expect_tx(bar, uint32_t((n1 + n2) * Cfg::BOX_BYTES));
  for (int k = 0; k < n1; ++k)
    tma_load_2d(stage + size_t(k * Cfg::BR) * Cfg::NB, map, x, k * Cfg::BR, bar);
  for (int k = 0; k < n2; ++k)
    tma_load_2d(stage + size_t((n1 + k) * Cfg::BR) * Cfg::NB, map, x, a.L + 1 + k * Cfg::BR, bar);
}

// In-place variant of col_fft: v[q] = x[t + TPF q] -> o[q] = X[t + TPF q],
// every exchange through the one buffer buf, with a barrier between the
// reads and the writes of each stage.
template <typename C, int M, int TPF, int SIGN>
__device__ __forceinline__ void col_fft_inplace(C (&v)[16], C *buf, const C *tw, int t,
                                                C (&o)[16]) {
  dft_reg<16>(v, SIGN);
  __syncthreads();  // earlier readers of buf are done
#pragma unroll
  for (int r = 0; r < 16; ++r) buf[fpad(16 * t + r)] = v[r];
  __syncthreads();
  col_tail_inplace<C, M, 16, TPF, SIGN>(buf, tw, t, o);
}

// One-column geometries (M = 4096 and 8192 in FP32, where a CTA of M/16
// threads takes one image column): k_ucol_bwd_pair gives a CTA two adjacent
// columns, loads both -- 16 bytes a band row instead of 8, half the sectors
// fetched for the data used -- and transforms them in turn, each in place in
// its own buffer (the band values of the column in hand stay in registers
// across the twist passes).
template <typename R, int LOGM>
__global__ void __launch_bounds__(ColCfg<R, (1 << LOGM)>::THREADS, 1)
k_ucol_bwd_pair(ColArgs a) {
  using C = typename Cplx<R>::type;
  constexpr int M = 1 << LOGM, TPF = ColCfg<R, M>::TPF;
  static_assert(ColCfg<R, M>::NB == 1, "for one-column CTAs");
  constexpr int THREADS = TPF;
  constexpr int BL = FftBuf<M>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);  // [2][BL]
  C *tws = buf + 2 * BL;                     // [M]
  const int t = threadIdx.x;
  const int lp = blockIdx.y, j0 = blockIdx.x * 2;
  const C *band = reinterpret_cast<const C *>(a.band);
  const C *twB = reinterpret_cast<const C *>(a.twB);
  const C *twQ = reinterpret_cast<const C *>(a.twQ);
  fill_table<C, M, THREADS>(tws, reinterpret_cast<const C *>(a.twM));
  // both columns, slot-major with the column pair innermost (adjacent threads
  // read the two columns of one band row), eight loads in flight a thread
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    C val[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int item = t + (h * 8 + q) * THREADS;
      const int c = item & 1, b = item >> 1;
      const int jj = j0 + c;
      val[q].x = R(0);
      val[q].y = R(0);
      const int u = slot_u(a, b, M);
      if (jj < a.ny && u < (1 << 29)) {
        int jx = jj + a.nv - a.ny / 2;
        jx -= (jx >= a.nv) ? a.nv : 0;
        val[q] = band[(size_t(slot_bi(a, u)) * a.P + lp) * a.nv + jx];
      }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int item = t + (h * 8 + q) * THREADS;
      buf[(item & 1) * BL + fpad(item >> 1)] = val[q];
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int c = 0; c < 2; ++c) {
    const int j = j0 + c;
    const bool jv = j < a.ny;
    C *A = buf + c * BL;
    C g[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) g[q] = A[fpad(t + TPF * q)];
    C *rowp = reinterpret_cast<C *>(a.H) + (size_t(lp) * a.ny + (jv ? j : 0)) * (size_t(a.K) * a.hseg);
    for (int k2 = 0; k2 < a.K; ++k2) {
      C v[16];
      if (k2 == 0) {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = g[q];
      } else {
        const C base = __ldg(&twB[k2 * TPF + t]);
#pragma unroll
        for (int q = 0; q < 16; ++q)
          v[q] = cmul(g[q], col_twist<C, TPF>(a, twB, twQ, k2, t, q, M, base));
      }
      C o[16];
      // (its first barrier keeps the in-place writes after every thread's reads of A)
      col_fft_inplace<C, M, TPF, +1>(v, A, tws, t, o);
      if (jv) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          bool keep;
          const int pos = h_pos<TPF>(a, k2, t, q, keep);
          if (keep) rowp[pos] = o[q];
        }
      }
    }
  }
}

// The forward transform of one-column geometries, as k_ucol_bwd_pair: two
// adjacent columns a CTA, each transformed and accumulated in its own buffer
// in turn, then both stored together -- 16 bytes a band row instead of 8.
template <typename R, int LOGM>
__global__ void __launch_bounds__(ColCfg<R, (1 << LOGM)>::THREADS, 1)
k_ucol_fwd_pair(ColArgs a) {
  using C = typename Cplx<R>::type;
  constexpr int M = 1 << LOGM, TPF = ColCfg<R, M>::TPF;
  static_assert(ColCfg<R, M>::NB == 1, "for one-column CTAs");
  constexpr int THREADS = TPF;
  constexpr int BL = FftBuf<M>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);  // [2][BL]
  C *tws = buf + 2 * BL;                     // [M]
  const int t = threadIdx.x;
  const int lp = blockIdx.y, j0 = blockIdx.x * 2;
  C *band = reinterpret_cast<C *>(a.band);
  const C *twB = reinterpret_cast<const C *>(a.twB);
  const C *twQ = reinterpret_cast<const C *>(a.twQ);
  fill_table<C, M, THREADS>(tws, reinterpret_cast<const C *>(a.twM));
  __syncthreads();  // the stage table is in place
#pragma unroll 1
  for (int c = 0; c < 2; ++c) {
    const int j = j0 + c;
    const bool jv = j < a.ny;
    C *A = buf + c * BL;
    const C *rowp = reinterpret_cast<const C *>(a.H) +
                    (size_t(lp) * a.ny + (jv ? j : 0)) * (size_t(a.K) * a.hseg);
    C acc[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc[q].x = acc[q].y = R(0);
    for (int k2 = 0; k2 < a.K; ++k2) {
      C v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        bool keep;
        const int pos = h_pos<TPF>(a, k2, t, q, keep);
        v[q].x = R(0);
        v[q].y = R(0);
        if (jv && keep) v[q] = rowp[pos];
      }
      C o[16];
      col_fft_inplace<C, M, TPF, -1>(v, A, tws, t, o);
      if (k2 == 0) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          acc[q].x += o[q].x;
          acc[q].y += o[q].y;
        }
      } else {
        const C base = __ldg(&twB[k2 * TPF + t]);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          C w = col_twist<C, TPF>(a, twB, twQ, k2, t, q, M, base);
          w.y = -w.y;
          const C val = cmul(o[q], w);
          acc[q].x += val.x;
          acc[q].y += val.y;
        }
      }
    }
    __syncthreads();  // the last transform's reads of A are done
#pragma unroll
    for (int q = 0; q < 16; ++q) A[fpad(t + TPF * q)] = acc[q];
  }
  __syncthreads();
  // both columns, the pair innermost: adjacent threads store one band row's
  // two columns
  for (int item = t; item < 2 * M; item += THREADS) {
    const int c = item & 1, b = item >> 1;
    const int jj = j0 + c;
    const int u = slot_u(a, b, M);
    if (jj < a.ny && u < (1 << 29)) {
      int jx = jj + a.nv - a.ny / 2;
      jx -= (jx >= a.nv) ? a.nv : 0;
      band[(size_t(slot_bi(a, u)) * a.P + lp) * a.nv + jx] = buf[c * BL + fpad(b)];
    }
  }
}

// ---- FP64 transforms of 8192 points ----
//
// One column a CTA of M/16 = 512 threads, transformed in place in one padded
// buffer (139 KB).  The stage tables of every stage but the last (4080
// entries, 65 KB) are in shared memory; the last stage (radix 2, stride
// 4096) reads its 4096 twiddles from global memory, where every CTA reads
// the same 64 KB (L1/L2-resident).  Outputs leave the last stage through
// emit(q, X[t + TPF q]) as they are made, so no register array of outputs
// outlives the transform (512 threads leave 128 registers a thread).

// Stride of the last stage of an M-point transform (radix-16 stages before it).
template <int M>
struct ColLastNS {
  static constexpr int get() {
    int ns = 1;
    while (M / ns > 16) ns *= 16;
    return ns;
  }
  static constexpr int value = get();
};

template <typename C, int M, int NS, int TPF, int SIGN, typename Emit>
__device__ __forceinline__ void col_tail_emit(C *buf, const C *tws, const C *twg, int t,
                                              Emit &emit) {
  if constexpr (M / NS > 16) {
    C v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = buf[fpad(t + r * TPF)];
    const int k = t & (NS - 1);
    constexpr int off = TwOffset<NS>::value;
#pragma unroll
    for (int r = 1; r < 16; ++r) {
      C w = tws[off + (r - 1) * NS + k];
      if (SIGN < 0) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    dft_reg<16>(v, SIGN);
    const int d = (t / NS) * NS * 16 + k;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 16; ++r) buf[fpad(d + r * NS)] = v[r];
    __syncthreads();
    col_tail_emit<C, M, NS * 16, TPF, SIGN>(buf, tws, twg, t, emit);
  } else {
    constexpr int RL = M / NS, IT = 16 / RL;
    constexpr int off = TwOffset<NS>::value;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int j = t + TPF * it;
      C v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) v[r] = buf[fpad(j + r * NS)];
#pragma unroll
      for (int r = 1; r < RL; ++r) {
        C w = __ldg(&twg[off + (r - 1) * NS + j]);
        if (SIGN < 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
      dft_reg<RL>(v, SIGN);
#pragma unroll
      for (int r = 0; r < RL; ++r) emit(it + r * IT, v[r]);
    }
  }
}

// v[q] = x[t + TPF q] -> emit(q, X[t + TPF q]); tws: the shared stage tables
// before the last stage's, twg: the full table in global memory.
template <typename C, int M, int TPF, int SIGN, typename Emit>
__device__ __forceinline__ void col_fft_emit(C (&v)[16], C *buf, const C *tws, const C *twg,
                                             int t, Emit &emit) {
  dft_reg<16>(v, SIGN);
  __syncthreads();  // earlier readers of buf are done
#pragma unroll
  for (int r = 0; r < 16; ++r) buf[fpad(16 * t + r)] = v[r];
  __syncthreads();
  col_tail_emit<C, M, 16, TPF, SIGN>(buf, tws, twg, t, emit);
}

template <int M>
struct ColBig {
  static constexpr int TPF = M / 16;
  static constexpr int NTAB = TwOffset<ColLastNS<M>::value>::value;  // shared table entries
  static constexpr size_t bytes() { return (size_t(FftBuf<M>::value) + NTAB) * 2 * sizeof(double); }
};

// ms2dirty direction (band rows -> H image rows, backward transform), one
// image column j = blockIdx.x of plane lp = blockIdx.y.  The band column is
// read again for each twisted pass (from L2 after the first).
template <int LOGM>
__global__ void __launch_bounds__(ColBig<(1 << LOGM)>::TPF, 1) k_ucol_bwd_big(ColArgs a) {
  using C = double2;
  constexpr int M = 1 << LOGM, TPF = ColBig<M>::TPF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  C *tws = buf + FftBuf<M>::value;
  const int t = threadIdx.x, j = blockIdx.x, lp = blockIdx.y;
  const C *band = reinterpret_cast<const C *>(a.band);
  const C *twB = reinterpret_cast<const C *>(a.twB);
  const C *twQ = reinterpret_cast<const C *>(a.twQ);
  const C *twg = reinterpret_cast<const C *>(a.twM);
  C *rowp = reinterpret_cast<C *>(a.H) + (size_t(lp) * a.ny + j) * (size_t(a.K) * a.hseg);
  int jx = j + a.nv - a.ny / 2;
  jx -= (jx >= a.nv) ? a.nv : 0;
  // (ordered before its first use by the transform's barriers)
  fill_table<C, ColBig<M>::NTAB, TPF>(tws, twg);
  for (int k2 = 0; k2 < a.K; ++k2) {
    C v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int u = slot_u(a, t + TPF * q, M);
      v[q].x = v[q].y = 0.0;
      if (u < (1 << 29)) v[q] = band[(size_t(slot_bi(a, u)) * a.P + lp) * a.nv + jx];
    }
    if (k2 > 0) {
      const C base = __ldg(&twB[k2 * TPF + t]);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = cmul(v[q], col_twist<C, TPF>(a, twB, twQ, k2, t, q, M, base));
    }
    auto emit = [&](int q, C val) {
      bool keep;
      const int pos = h_pos<TPF>(a, k2, t, q, keep);
      if (keep) rowp[pos] = val;
    };
    col_fft_emit<C, M, TPF, +1>(v, buf, tws, twg, t, emit);
  }
}

// dirty2ms direction (H image rows -> band rows, forward transform).  Each
// pass's twisted outputs are summed in the band array itself: every thread
// owns the same band slots in every pass, so the read-modify-write needs no
// synchronisation.
template <int LOGM>
__global__ void __launch_bounds__(ColBig<(1 << LOGM)>::TPF, 1) k_ucol_fwd_big(ColArgs a) {
  using C = double2;
  constexpr int M = 1 << LOGM, TPF = ColBig<M>::TPF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  C *tws = buf + FftBuf<M>::value;
  const int t = threadIdx.x, j = blockIdx.x, lp = blockIdx.y;
  C *band = reinterpret_cast<C *>(a.band);
  const C *twB = reinterpret_cast<const C *>(a.twB);
  const C *twQ = reinterpret_cast<const C *>(a.twQ);
  const C *twg = reinterpret_cast<const C *>(a.twM);
  const C *rowp = reinterpret_cast<const C *>(a.H) + (size_t(lp) * a.ny + j) * (size_t(a.K) * a.hseg);
  int jx = j + a.nv - a.ny / 2;
  jx -= (jx >= a.nv) ? a.nv : 0;
  fill_table<C, ColBig<M>::NTAB, TPF>(tws, twg);
  for (int k2 = 0; k2 < a.K; ++k2) {
    C v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      bool keep;
      const int pos = h_pos<TPF>(a, k2, t, q, keep);
      v[q].x = v[q].y = 0.0;
      if (keep) v[q] = rowp[pos];
    }
    const C base = k2 > 0 ? __ldg(&twB[k2 * TPF + t]) : make_double2(1.0, 0.0);
    auto emit = [&](int q, C val) {
      const int u = slot_u(a, t + TPF * q, M);
      if (u >= (1 << 29)) return;
      C *dst = &band[(size_t(slot_bi(a, u)) * a.P + lp) * a.nv + jx];
      if (k2 > 0) {
        C w = col_twist<C, TPF>(a, twB, twQ, k2, t, q, M, base);
        w.y = -w.y;
        val = cmul(val, w);
        const C old = *dst;
        val.x += old.x;
        val.y += old.y;
      }
      *dst = val;
    };
    col_fft_emit<C, M, TPF, -1>(v, buf, tws, twg, t, emit);
  }
}

template <typename R, int LOGM, bool TWS>
__global__ void __launch_bounds__(ColCfg<R, (1 << LOGM)>::THREADS, ColCfg<R, (1 << LOGM)>::MINB)
k_ucol_bwd_tma(ColArgs a, const __grid_constant__ CUtensorMap tmap, int npl, int *err) {
  using C = typename Cplx<R>::type;
  constexpr int M = 1 << LOGM, TPF = ColCfg<R, M>::TPF;
  using Cfg = TmaCfg<R, M>;
  constexpr int NB = Cfg::NB;
  constexpr int BL = FftBuf<M>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the staging buffer starts on a 128-byte boundary (the host adds 128 bytes)
  const uint32_t mis = smem_u32(smem_raw) & 127u;
  C *stage = reinterpret_cast<C *>(smem_raw + (mis ? 128u - mis : 0u));   // [ROWS][NB]
  C *bufall = stage + size_t(Cfg::ROWS) * NB;                               // [NB][BL]
  C *tws = bufall + size_t(NB) * BL;                                        // [M]
  __shared__ __align__(8) uint64_t bar;
  const int grp = threadIdx.x / TPF, t = threadIdx.x - grp * TPF;
  C *A = bufall + size_t(grp) * BL;
  const int npairs = (a.ny + NB - 1) / NB;
  const int nitems = npairs * npl;
  const C *twB = reinterpret_cast<const C *>(a.twB);
  const C *twQ = reinterpret_cast<const C *>(a.twQ);
  const int reg2 = tma_boxes1(a, M, Cfg::BR) * Cfg::BR;  // first staging row of region 2
  fill_table<C, M, ColCfg<R, M>::THREADS>(tws, reinterpret_cast<const C *>(a.twM));
  if constexpr (TWS) {  // the twist tables after the stage table (barrier below)
    C *twBs = tws + M, *twQs = twBs + a.K * TPF;
    for (int i = threadIdx.x; i < a.K * TPF; i += blockDim.x) twBs[i] = twB[i];
    for (int i = threadIdx.x; i < a.K * 32; i += blockDim.x) twQs[i] = twQ[i];
    twB = twBs;
    twQ = twQs;
  }
  int item = blockIdx.x;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (item < nitems)
      tma_issue_item<R, M>(a, &tmap, stage, &bar, item / npairs, (item % npairs) * NB);
  }
  __syncthreads();  // the barrier is initialised before anyone waits on it
  for (uint32_t parity = 0; item < nitems; item += gridDim.x, parity ^= 1u) {
    const int lp = item / npairs, j = (item % npairs) * NB + grp;
    if (!mbar_wait(&bar, parity)) {  // the copy did not complete: report and stop
      if (threadIdx.x == 0) atomicOr(err, 2);
      mbar_wait(&bar, parity);
      return;
    }
    // the untwisted band values at slots t + TPF q (zero between the halves)
    C g[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int b = t + TPF * q;
      g[q].x = R(0);
      g[q].y = R(0);
      if (a.band_full || b <= a.L)
        g[q] = stage[size_t(b) * NB + grp];
      else if (b >= M - a.L)
        g[q] = stage[size_t(reg2 + b - (M - a.L)) * NB + grp];
    }
    __syncthreads();  // the staging buffer is free for the next item's boxes
    const int next = item + gridDim.x;
    if (threadIdx.x == 0 && next < nitems) {
      // order the reads above (generic proxy) before the copy engine's
      // writes to the same buffer (async proxy)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tma_issue_item<R, M>(a, &tmap, stage, &bar, next / npairs, (next % npairs) * NB);
    }
    const bool jv = j < a.ny;
    C *rowp = reinterpret_cast<C *>(a.H) + (size_t(lp) * a.ny + (jv ? j : 0)) * (size_t(a.K) * a.hseg);
    for (int k2 = 0; k2 < a.K; ++k2) {
      C v[16];
      if (k2 == 0) {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = g[q];
      } else if constexpr (TWS) {
        const C base = twB[k2 * TPF + t];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int b = t + TPF * q;
          const int neg = (!a.band_full && b >= M - a.L) ? 1 : 0;
          v[q] = cmul(g[q], cmul(twQ[(k2 * 16 + q) * 2 + neg], base));
        }
      } else {
        const C base = __ldg(&twB[k2 * TPF + t]);
#pragma unroll
        for (int q = 0; q < 16; ++q)
          v[q] = cmul(g[q], col_twist<C, TPF>(a, twB, twQ, k2, t, q, M, base));
      }
      C o[16];
      col_fft_inplace<C, M, TPF, +1>(v, A, tws, t, o);
      if (jv) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          bool keep;
          const int pos = h_pos<TPF>(a, k2, t, q, keep);
          if (keep) rowp[pos] = o[q];
        }
      }
    }
  }
}

// dirty2ms direction, the exact transpose: H image rows -> band rows of the
// image columns, forward (-) transform along u.  Band entries of other
// columns are left untouched (zeroed by the caller).  TWS: the twist tables
// are copied to shared memory after the stage twiddles (K (M/16 + 32) more
// entries), where the host finds room for them without losing a resident CTA.
template <typename R, int LOGM, bool TWS>
__global__ void __launch_bounds__(ColCfg<R, (1 << LOGM)>::THREADS, ColCfg<R, (1 << LOGM)>::MINB)
k_ucol_fwd(ColArgs a) {
  using C = typename Cplx<R>::type;
  constexpr int M = 1 << LOGM, TPF = ColCfg<R, M>::TPF, NB = ColCfg<R, M>::NB;
  constexpr int BL = FftBuf<M>::value;
  constexpr bool kFlip = (ColMid<M>::value % 2) == 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *bufall = reinterpret_cast<C *>(smem_raw);
  C *tws = bufall + 2 * NB * BL;
  const int grp = threadIdx.x / TPF, t = threadIdx.x - grp * TPF;
  C *A = bufall + 2 * grp * BL, *B = A + BL;
  const int lp = blockIdx.y;
  const int j = blockIdx.x * NB + grp;
  const bool jv = j < a.ny;
  C *band = reinterpret_cast<C *>(a.band);
  const C *twB = reinterpret_cast<const C *>(a.twB);
  const C *twQ = reinterpret_cast<const C *>(a.twQ);
  if constexpr (TWS) {  // ordered before use by the first transform's barriers
    C *twBs = tws + M, *twQs = twBs + a.K * TPF;
    for (int i = threadIdx.x; i < a.K * TPF; i += blockDim.x) twBs[i] = twB[i];
    for (int i = threadIdx.x; i < a.K * 32; i += blockDim.x) twQs[i] = twQ[i];
    twB = twBs;
    twQ = twQs;
  }
  const C *rowp = reinterpret_cast<const C *>(a.H) +
                  (size_t(lp) * a.ny + (jv ? j : 0)) * (size_t(a.K) * a.hseg);
  fill_table<C, M, ColCfg<R, M>::THREADS>(tws, reinterpret_cast<const C *>(a.twM));
  C acc[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) acc[q].x = acc[q].y = R(0);
  for (int k2 = 0; k2 < a.K; ++k2) {
    C v[16];
    // input q is image row K m + k2 + nx/2, m = t + TPF q for q < 8 and
    // t + TPF q - M for q >= 8 (nu = 16 K TPF: the wrap at nu/2 falls at q = 8)
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      bool keep;
      const int pos = h_pos<TPF>(a, k2, t, q, keep);
      v[q].x = R(0);
      v[q].y = R(0);
      if (jv && keep) v[q] = rowp[pos];
    }
    C *S = (kFlip && (k2 & 1)) ? B : A;
    C *O = (kFlip && (k2 & 1)) ? A : B;
    if (k2 == 0) __syncthreads();  // the stage table is in place
    C o[16];
    col_fft<C, M, TPF, -1>(v, S, O, tws, t, o);
    if (k2 == 0) {
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        acc[q].x += o[q].x;
        acc[q].y += o[q].y;
      }
    } else {
      const C base = TWS ? twB[k2 * TPF + t] : __ldg(&twB[k2 * TPF + t]);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        C w;
        if constexpr (TWS) {
          const int b = t + TPF * q;
          const int neg = (!a.band_full && b >= M - a.L) ? 1 : 0;
          w = cmul(twQ[(k2 * 16 + q) * 2 + neg], base);
        } else {
          w = col_twist<C, TPF>(a, twB, twQ, k2, t, q, M, base);
        }
        w.y = -w.y;
        const C val = cmul(o[q], w);
        acc[q].x += val.x;
        acc[q].y += val.y;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 16; ++q) A[fpad(t + TPF * q)] = acc[q];
  __syncthreads();
  for (int item = threadIdx.x; item < NB * M; item += blockDim.x) {
    const int c = item % NB, b = item / NB;
    const int jj = blockIdx.x * NB + c;
    const int u = slot_u(a, b, M);
    if (jj < a.ny && u < (1 << 29)) {
      int jx = jj + a.nv - a.ny / 2;
      jx -= (jx >= a.nv) ? a.nv : 0;
      band[(size_t(slot_bi(a, u)) * a.P + lp) * a.nv + jx] = bufall[c * 2 * BL + fpad(b)];
    }
  }
}

// ---- the image rows staged by bulk copies ----
//
// k_ucol_fwd_bulk is k_ucol_fwd made persistent over (plane, column group)
// items.  The input of each pass -- one contiguous segment of hseg entries
// per column of the segmented H row -- is brought into shared memory by 1-D
// bulk copies (cp.async.bulk, completing on an mbarrier, no multicast).  The
// next segment (the next pass, or the first pass of the CTA's next item) is
// requested as soon as the current one has been read into registers, so it
// lands while the current pass transforms.  The transforms run in place in
// one buffer per column.

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Requests segment k2 of the H rows of columns [j0, j0 + NB) of plane lp
// into the staging buffer and arms the barrier with their bytes (one thread).
template <typename C, int NB>
__device__ __forceinline__ void fwd_issue(const ColArgs &a, C *stage, uint64_t *bar, int lp,
                                          int j0, int k2) {
  const size_t hrow = size_t(a.K) * a.hseg;
  const uint32_t bytes = uint32_t(a.hseg) * uint32_t(sizeof(C));
  const int nc = min(NB, a.ny - j0);
  mbar_expect_tx(bar, uint32_t(nc) * bytes);
  const C *src = reinterpret_cast<const C *>(a.H) + (size_t(lp) * a.ny + j0) * hrow +
                 size_t(k2) * a.hseg;
  for (int c = 0; c < nc; ++c) bulk_load(stage + size_t(c) * a.hseg, src + c * hrow, bytes, bar);
}

template <typename R, int LOGM, bool TWS>
__global__ void __launch_bounds__(ColCfg<R, (1 << LOGM)>::THREADS, ColCfg<R, (1 << LOGM)>::MINB)
k_ucol_fwd_bulk(ColArgs a, int npl, int *err) {
  using C = typename Cplx<R>::type;
  constexpr int M = 1 << LOGM, TPF = ColCfg<R, M>::TPF, NB = ColCfg<R, M>::NB;
  constexpr int BL = FftBuf<M>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the staging buffer starts on a 128-byte boundary (the host adds 128 bytes)
  const uint32_t mis = smem_u32(smem_raw) & 127u;
  C *stage = reinterpret_cast<C *>(smem_raw + (mis ? 128u - mis : 0u));  // [NB][hseg]
  C *bufall = stage + size_t(NB) * a.hseg;                                 // [NB][BL]
  C *tws = bufall + size_t(NB) * BL;                                       // [M]
  __shared__ __align__(8) uint64_t bar;
  const int grp = threadIdx.x / TPF, t = threadIdx.x - grp * TPF;
  C *A = bufall + size_t(grp) * BL;
  C *band = reinterpret_cast<C *>(a.band);
  const C *twB = reinterpret_cast<const C *>(a.twB);
  const C *twQ = reinterpret_cast<const C *>(a.twQ);
  const int npairs = (a.ny + NB - 1) / NB;
  const int nitems = npairs * npl;
  fill_table<C, M, ColCfg<R, M>::THREADS>(tws, reinterpret_cast<const C *>(a.twM));
  if constexpr (TWS) {  // the twist tables after the stage table (barrier below)
    C *twBs = tws + M, *twQs = twBs + a.K * TPF;
    for (int i = threadIdx.x; i < a.K * TPF; i += blockDim.x) twBs[i] = twB[i];
    for (int i = threadIdx.x; i < a.K * 32; i += blockDim.x) twQs[i] = twQ[i];
    twB = twBs;
    twQ = twQs;
  }
  int item = blockIdx.x;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (item < nitems) fwd_issue<C, NB>(a, stage, &bar, item / npairs, (item % npairs) * NB, 0);
  }
  __syncthreads();  // the barrier and the tables are in place
  uint32_t parity = 0;
  for (; item < nitems; item += gridDim.x) {
    const int lp = item / npairs, jb = (item % npairs) * NB;
    const bool jv = jb + grp < a.ny;
    C acc[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc[q].x = acc[q].y = R(0);
    for (int k2 = 0; k2 < a.K; ++k2, parity ^= 1u) {
      if (!mbar_wait(&bar, parity)) {  // the copy did not complete: report and stop
        if (threadIdx.x == 0) atomicOr(err, 2);
        mbar_wait(&bar, parity);
        return;
      }
      C v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        bool keep;
        const int pos = h_pos<TPF>(a, k2, t, q, keep) - k2 * a.hseg;
        v[q].x = R(0);
        v[q].y = R(0);
        if (jv && keep) v[q] = stage[size_t(grp) * a.hseg + pos];
      }
      __syncthreads();  // the staging buffer is free for the next segment
      if (threadIdx.x == 0) {
        int ni = item, nk = k2 + 1;
        if (nk == a.K) {
          ni = item + gridDim.x;
          nk = 0;
        }
        if (ni < nitems) {
          // order the reads above (generic proxy) before the copy engine's
          // writes to the same buffer (async proxy)
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          fwd_issue<C, NB>(a, stage, &bar, ni / npairs, (ni % npairs) * NB, nk);
        }
      }
      C o[16];
      col_fft_inplace<C, M, TPF, -1>(v, A, tws, t, o);
      if (k2 == 0) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          acc[q].x += o[q].x;
          acc[q].y += o[q].y;
        }
      } else {
        const C base = TWS ? twB[k2 * TPF + t] : __ldg(&twB[k2 * TPF + t]);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          C w;
          if constexpr (TWS) {
            const int b = t + TPF * q;
            const int neg = (!a.band_full && b >= M - a.L) ? 1 : 0;
            w = cmul(twQ[(k2 * 16 + q) * 2 + neg], base);
          } else {
            w = col_twist<C, TPF>(a, twB, twQ, k2, t, q, M, base);
          }
          w.y = -w.y;
          const C val = cmul(o[q], w);
          acc[q].x += val.x;
          acc[q].y += val.y;
        }
      }
    }
    __syncthreads();  // the last transform's reads of A are done
#pragma unroll
    for (int q = 0; q < 16; ++q) A[fpad(t + TPF * q)] = acc[q];
    __syncthreads();
    for (int it = threadIdx.x; it < NB * M; it += blockDim.x) {
      const int c = it % NB, b = it / NB;
      const int jj = jb + c;
      const int u = slot_u(a, b, M);
      if (jj < a.ny && u < (1 << 29)) {
        int jx = jj + a.nv - a.ny / 2;
        jx -= (jx >= a.nv) ? a.nv : 0;
        band[(size_t(slot_bi(a, u)) * a.P + lp) * a.nv + jx] = bufall[c * BL + fpad(b)];
      }
    }
    // (the next item's first transform writes A only after a barrier)
  }
}

// In-place FFT of `rows` contiguous rows of length M = 2^LOGM in global
// memory (the transform along v when cuFFT cannot be used), sign +1 backward.
template <typename R, int LOGM>
__global__ void __launch_bounds__(ColCfg<R, (1 << LOGM)>::THREADS)
k_row_fft(void *data, long long rows, const void *twv, int sign) {
  using C = typename Cplx<R>::type;
  constexpr int M = 1 << LOGM, TPF = ColCfg<R, M>::TPF, NB = ColCfg<R, M>::NB;
  constexpr int BL = FftBuf<M>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *bufall = reinterpret_cast<C *>(smem_raw);
  C *tws = bufall + NB * BL;
  const int grp = threadIdx.x / TPF, t = threadIdx.x - grp * TPF;
  C *d = reinterpret_cast<C *>(data);
  for (int i = threadIdx.x; i < M; i += blockDim.x) tws[i] = reinterpret_cast<const C *>(twv)[i];
  const long long row = (long long)blockIdx.x * NB + grp;
  const bool rv = row < rows;
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    C v;
    v.x = R(0);
    v.y = R(0);
    if (rv) v = d[row * M + t + TPF * r];
    bufall[grp * BL + fpad(t + TPF * r)] = v;
  }
  __syncthreads();
  FftStages<C, M, 1, TPF>::run(bufall + grp * BL, tws, t, sign);
#pragma unroll
  for (int r = 0; r < 16; ++r)
    if (rv) d[row * M + t + TPF * r] = bufall[grp * BL + fpad(t + TPF * r)];
}

// ------------------------------------------------------- image weights
//
// WSClean's ImageWeights (structures/imageweights.h:36-100,
// structures/imageweights.cpp:78-143) on the device: a width x height/2 grid
// of summed visibility weights over the v >= 0 half plane, finished into
// natural, uniform or Briggs imaging weights, then looked up per visibility.
// (u, v) are in wavelengths, u / lambda with lambda = c / f per channel.

static __global__ void k_weights_grid(size_t nrows, int nchan, int npol, const double *__restrict__ uvw,
                               const double *__restrict__ lambda, const float *__restrict__ wgt,
                               int as_taper, WeightGrid g, double *__restrict__ grid,
                               double *__restrict__ total) {
  double sum = 0.0;
  for (size_t r = blockIdx.x * size_t(blockDim.x) + threadIdx.x; r < nrows;
       r += size_t(gridDim.x) * blockDim.x) {
    for (int c = 0; c < nchan; ++c) {
      const double u = uvw[3 * r] / lambda[c], v = uvw[3 * r + 1] / lambda[c];
      int x, y;
      const bool in = weight_cell(g, u, v, x, y);
      for (int p = 0; p < npol; ++p) {
        float w = wgt ? wgt[(r * nchan + c) * npol + p] : 1.0f;
        if (as_taper && w != 0.0f) w = 1.0f;
        if (in) {
          atomicAdd(&grid[size_t(x) + size_t(y) * g.W], double(w));
          sum += double(w);
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31) == 0 && sum != 0.0) atomicAdd(total, sum);
}

static __global__ void k_weights_sumsq(size_t n, const double *__restrict__ grid, double *__restrict__ out) {
  double s = 0.0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    s += grid[i] * grid[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(out, s);
}

// mode 0 natural, 1 uniform, 2 Briggs (s2 = (5 * 10^-robust)^2 / (sum W^2 / sum W))
static __global__ void k_weights_finish(size_t n, double *__restrict__ grid, int mode,
                                 const double *__restrict__ sums, double num_sq) {
  const double s2 = mode == 2 ? num_sq / (sums[1] / sums[0]) : 0.0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const double v = grid[i];
    if (mode == 2)
      grid[i] = 1.0 / (1.0 + v * s2);
    else if (mode == 1)
      grid[i] = v != 0.0 ? 1.0 / v : 0.0;
    else
      grid[i] = v != 0.0 ? 1.0 : v;
  }
}

// out = in * imaging weight of the visibility's cell (0 outside the grid)
static __global__ void k_weights_apply(size_t nrows, int nchan, int npol, const double *__restrict__ uvw,
                                const double *__restrict__ lambda, WeightGrid g,
                                const double *__restrict__ grid, const float *__restrict__ in,
                                float *__restrict__ out) {
  for (size_t r = blockIdx.x * size_t(blockDim.x) + threadIdx.x; r < nrows;
       r += size_t(gridDim.x) * blockDim.x) {
    for (int c = 0; c < nchan; ++c) {
      const double u = uvw[3 * r] / lambda[c], v = uvw[3 * r + 1] / lambda[c];
      int x, y;
      const double iw = weight_cell(g, u, v, x, y) ? grid[size_t(x) + size_t(y) * g.W] : 0.0;
      for (int p = 0; p < npol; ++p) {
        const size_t k = (r * nchan + c) * npol + p;
        out[k] = float(double(in ? in[k] : 1.0f) * iw);
      }
    }
  }
}

// ------------------------------------------------- tuned schedule (w split)
//
// The |w| statistics behind the tuned schedule's choice of a w cut and
// facets (get_winfo, wgridder.cc:28-89): the range of |w f/c| over the
// masked-in visibilities, a histogram of NBIN equal bins over that range,
// and the split of the mask into the visibilities below and at or above the
// cut bin.  A visibility's bin is min(floor((|w f/c| - wmin) * xdw), NBIN-1)
// with xdw = NBIN / (wmax - wmin), as the reference computes it.

static __global__ void k_wrange(size_t nrows, int nchan, const double *__restrict__ uvw,
                         const double *__restrict__ fovc, const uint8_t *__restrict__ mask,
                         unsigned long long *out /* [0] min bits, [1] max bits, [2] count */) {
  double lo = 1e300, hi = 0;
  unsigned long long cnt = 0;
  for (size_t r = blockIdx.x * size_t(blockDim.x) + threadIdx.x; r < nrows;
       r += size_t(gridDim.x) * blockDim.x) {
    const double w = uvw[3 * r + 2];
    for (int c = 0; c < nchan; ++c) {
      if (mask && !mask[r * nchan + c]) continue;
      const double aw = fabs(w * fovc[c]);
      lo = fmin(lo, aw);
      hi = fmax(hi, aw);
      ++cnt;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  if ((threadIdx.x & 31) == 0 && cnt > 0) {
    atomicMin(&out[0], (unsigned long long)__double_as_longlong(lo));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(hi));
    atomicAdd(&out[2], cnt);
  }
}

constexpr int kTuneBins = 50;

__device__ __forceinline__ int w_bin(double aw, double wmin, double xdw) {
  const double x = (aw - wmin) * xdw;
  const unsigned long long b = (unsigned long long)x;  // x >= 0
  return int(b < (unsigned long long)(kTuneBins - 1) ? b : (unsigned long long)(kTuneBins - 1));
}

static __global__ void k_whist(size_t nrows, int nchan, const double *__restrict__ uvw,
                        const double *__restrict__ fovc, const uint8_t *__restrict__ mask,
                        double wmin, double xdw, unsigned long long *hist) {
  __shared__ unsigned int h[kTuneBins];
  for (int i = threadIdx.x; i < kTuneBins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (size_t r = blockIdx.x * size_t(blockDim.x) + threadIdx.x; r < nrows;
       r += size_t(gridDim.x) * blockDim.x) {
    const double w = uvw[3 * r + 2];
    for (int c = 0; c < nchan; ++c) {
      if (mask && !mask[r * nchan + c]) continue;
      atomicAdd(&h[w_bin(fabs(w * fovc[c]), wmin, xdw)], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kTuneBins; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

// hi[k] = mask_k and bin >= icut; lo[k] = mask_k and bin < icut
static __global__ void k_wsplit(size_t nrows, int nchan, const double *__restrict__ uvw,
                         const double *__restrict__ fovc, const uint8_t *__restrict__ mask,
                         double wmin, double xdw, int icut, uint8_t *__restrict__ hi,
                         uint8_t *__restrict__ lo) {
  for (size_t r = blockIdx.x * size_t(blockDim.x) + threadIdx.x; r < nrows;
       r += size_t(gridDim.x) * blockDim.x) {
    const double w = uvw[3 * r + 2];
    for (int c = 0; c < nchan; ++c) {
      const size_t k = r * nchan + c;
      const bool in = !mask || mask[k];
      const bool up = in && w_bin(fabs(w * fovc[c]), wmin, xdw) >= icut;
      hi[k] = up ? 1 : 0;
      lo[k] = (in && !up) ? 1 : 0;
    }
  }
}

// ------------------------------------------------------------- screens

struct ScreenArgs {
  int nx, ny, nu, nv;
  size_t ld;                // row stride of the x-major image (ny, or the full
                            // image's ny for a facet inside a larger image)
  double px, py, x0, y0;
  double nshift, dw, wmin;
  int do_w, divide_by_n;
  int P, pb0, npl;          // layout planes, first plane, planes in this pass
  int K, hseg, hm0, nbs;    // H row layout (ColArgs), 32-entry blocks per segment
  const double *cfu, *cfv;  // nx/2+1, ny/2+1 grid-correction factors
  double cheb[kDMaxCheb];   // corfunc(v) as Chebyshev series in y=v^2
  int ncheb;
  double ymax;
};

__device__ __forceinline__ double cheb_corr(const ScreenArgs &s, double v) {
  double x = 2.0 * (v * v) / s.ymax - 1.0;
  double b1 = 0, b2 = 0;
  for (int j = s.ncheb - 1; j >= 1; --j) {
    double b0 = 2.0 * x * b1 - b2 + s.cheb[j];
    b2 = b1;
    b1 = b0;
  }
  return x * b1 - b2 + s.cheb[0];
}

// FP64 grid correction and the n-1 term of pixel (i,j)
// (apply_global_corrections, wgridder.h:1348-1400; phase(), :393-404).
__device__ __forceinline__ void pixel_terms(const ScreenArgs &s, int i, int j,
                                            double &corr, double &q, bool &inside) {
  double l = s.x0 + i * s.px, m = s.y0 + j * s.py;
  double fx = l * l, fy = m * m;
  double tmp = 1.0 - fx - fy;
  double fct;
  inside = tmp > 0;  // phase() drops the screen for tmp <= 0
  double nm1 = 0;
  if (tmp >= 0) {
    nm1 = (-fx - fy) / (sqrt(tmp) + 1.0);
    fct = s.do_w ? cheb_corr(s, (nm1 + s.nshift) * s.dw) : 1.0;
    if (s.divide_by_n) fct /= nm1 + 1.0;
  } else {
    fct = s.divide_by_n ? 0.0 : (s.do_w ? cheb_corr(s, (sqrt(-tmp) - 1.0) * s.dw) : 1.0);
  }
  int iu = abs(s.nx / 2 - i), iv = abs(s.ny / 2 - j);
  corr = fct * s.cfu[iu] * s.cfv[iv];
  q = nm1 + s.nshift;
}

// Offset in H, [P][ny][K hseg], of pixel (i, j)'s entry -- image row i
// being entry mm of segment k2 -- in the first plane, and the stride between
// planes.
__device__ __forceinline__ size_t screen_h_off(const ScreenArgs &s, int i, int j, int k2, int mm,
                                               size_t &pstride) {
  (void)i;
  const size_t hrow = size_t(s.K) * s.hseg;
  pstride = size_t(s.ny) * hrow;
  return size_t(j) * hrow + (size_t(k2) * s.hseg + mm);
}

// The w-screen phase factor exp(2 pi i t) in the precision of the grid: in
// mixed precision the argument is reduced in FP64 and the rest is FP32
// (phases good to ~1e-7 turns, far inside the 1e-5 accuracy that mixed
// precision serves); FP64 throughout otherwise.
template <typename R>
__device__ __forceinline__ auto screen_phase(double t) {
  if constexpr (sizeof(R) == 4)
    return cexp_turns_f(t);
  else
    return cexp_turns(t);
}

// Image row of entry mm of H-row segment k2, or -1 for an entry that holds
// no image row.  A screen CTA covers 32 consecutive entries of one segment
// (blockIdx.x = k2 * nbs + block) by 32 image columns, so that its H
// accesses are contiguous; its image rows are every K-th.
__device__ __forceinline__ int screen_row(const ScreenArgs &s, int k2, int mm) {
  const int i = s.K * (mm + s.hm0) + k2 + s.nx / 2;
  return (mm < s.hseg && unsigned(i) < unsigned(s.nx)) ? i : -1;
}

// ms2dirty: img(i,j) += corr(i,j) * sum_p Re(H[p][j][pos(i)] * exp(-2 pi i w_p q)),
// FP64 pixel terms, the phases by a recurrence over planes in the grid's
// precision (screen_phase), FP64 accumulation of the per-block sums.
template <typename R>
// out_mode 0: img += the sum (FP64 accumulator); 1 / 2: out = the sum as
// FP32 / FP64 (the caller's image, when one pass covers all planes and
// nothing is accumulated)
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 3) k_screen_add(ScreenArgs s, const void *Hv, double *img,
                                                    void *out, int out_mode) {
  using C = typename Cplx<R>::type;
  const C *H = reinterpret_cast<const C *>(Hv);
  __shared__ double tile[32][33];
  const int k2 = blockIdx.x / s.nbs, mm0 = (blockIdx.x - k2 * s.nbs) * 32;
  const int j0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const int i = screen_row(s, k2, mm0 + tx);
  // planes loaded together; the first batch is in flight while the pixel's
  // FP64 terms are computed
  constexpr int PB = sizeof(R) == 4 ? 16 : 8;
  for (int k = 0; k < 4; ++k) {
    const int j = j0 + ty + 8 * k;
    double val = 0;
    if (i >= 0 && j < s.ny) {
      size_t pstride;
      const C *hp = H + screen_h_off(s, i, j, k2, mm0 + tx, pstride);
      C hb[PB];
#pragma unroll
      for (int u = 0; u < PB; ++u)
        if (u < s.npl) hb[u] = hp[u * pstride];
      double corr, q;
      bool inside;
      pixel_terms(s, i, j, corr, q, inside);
      const bool screen = s.do_w && inside;
      using SC = typename std::conditional<sizeof(R) == 4, float2, double2>::type;
      SC sc, st;
      sc.x = st.x = 1;
      sc.y = st.y = 0;
      const double w0 = s.wmin + s.pb0 * s.dw;
      if (screen) st = screen_phase<R>(-s.dw * q);
      double acc = 0;
      for (int p0 = 0; p0 < s.npl; p0 += PB) {
        if (p0 > 0) {
#pragma unroll
          for (int u = 0; u < PB; ++u)
            if (p0 + u < s.npl) hb[u] = hp[(p0 + u) * pstride];
        }
        if (screen) {
          // in FP32 each block of PB planes starts from its exact phase, so
          // that the recurrence's rounding does not build up over many planes
          if (sizeof(R) == 4 || p0 == 0) sc = screen_phase<R>(-(w0 + p0 * s.dw) * q);
          R part = 0;
#pragma unroll
          for (int u = 0; u < PB; ++u) {
            if (p0 + u < s.npl) {
              part += hb[u].x * sc.x - hb[u].y * sc.y;
              const auto nr = sc.x * st.x - sc.y * st.y;
              sc.y = sc.x * st.y + sc.y * st.x;
              sc.x = nr;
            }
          }
          acc += double(part);
        } else {
#pragma unroll
          for (int u = 0; u < PB; ++u)
            if (p0 + u < s.npl) acc += double(hb[u].x);
        }
      }
      val = acc * corr;
    }
    tile[ty + 8 * k][tx] = val;
  }
  __syncthreads();
  for (int k = 0; k < 4; ++k) {
    const int ii = screen_row(s, k2, mm0 + ty + 8 * k), jj = j0 + tx;
    if (ii >= 0 && jj < s.ny) {
      const size_t o = size_t(ii) * s.ld + jj;
      const double x = tile[tx][ty + 8 * k];
      if (out_mode == 0)
        img[o] += x;
      else if (out_mode == 1)
        reinterpret_cast<float *>(out)[o] = float(x);
      else
        reinterpret_cast<double *>(out)[o] = x;
    }
  }
}

// dirty2ms: H[p][j][pos(i)] = dirty(i,j) * corr(i,j) * exp(+2 pi i w_p q)
template <typename R>
// in_f32: img points to the caller's FP32 image instead of the FP64 copy
__global__ void __launch_bounds__(256) k_screen_put(ScreenArgs s, const void *img, int in_f32,
                                                    void *Hv) {
  using C = typename Cplx<R>::type;
  C *H = reinterpret_cast<C *>(Hv);
  __shared__ double tile[32][33];
  const int k2 = blockIdx.x / s.nbs, mm0 = (blockIdx.x - k2 * s.nbs) * 32;
  const int j0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int k = 0; k < 4; ++k) {  // coalesced read along j
    const int ii = screen_row(s, k2, mm0 + ty + 8 * k), jj = j0 + tx;
    double x = 0.0;
    if (ii >= 0 && jj < s.ny) {
      const size_t o = size_t(ii) * s.ld + jj;
      x = in_f32 ? double(reinterpret_cast<const float *>(img)[o])
                 : reinterpret_cast<const double *>(img)[o];
    }
    tile[tx][ty + 8 * k] = x;
  }
  __syncthreads();
  const int i = screen_row(s, k2, mm0 + tx);
  for (int k = 0; k < 4; ++k) {
    const int j = j0 + ty + 8 * k;
    if (i < 0 || j >= s.ny) continue;
    double corr, q;
    bool inside;
    pixel_terms(s, i, j, corr, q, inside);
    const double val = tile[ty + 8 * k][tx] * corr;
    size_t pstride;
    C *hp = H + screen_h_off(s, i, j, k2, mm0 + tx, pstride);
    if (s.do_w && inside) {
      const double w0 = s.wmin + s.pb0 * s.dw;
      const auto st = screen_phase<R>(s.dw * q);
      const R rv = R(val);
      auto sc = st;
      for (int p0 = 0; p0 < s.npl; p0 += 16) {
        // (in FP32 the exact phase at the start of every 16 planes, as in
        // k_screen_add)
        if (sizeof(R) == 4 || p0 == 0) sc = screen_phase<R>((w0 + p0 * s.dw) * q);
        const int pe = min(s.npl, p0 + 16);
        for (int p = p0; p < pe; ++p) {
          C o;
          o.x = rv * sc.x;
          o.y = rv * sc.y;
          hp[p * pstride] = o;
          const auto nr = sc.x * st.x - sc.y * st.y;
          sc.y = sc.x * st.y + sc.y * st.x;
          sc.x = nr;
        }
      }
    } else {
      for (int p = 0; p < s.npl; ++p) {
        C o;
        o.x = R(val);
        o.y = R(0);
        hp[p * pstride] = o;
      }
    }
  }
}

// ---- screens on the whole grid (GridPlan::ucufft) ----
//
// When the grid keeps every u row, the 2-D transform of a plane runs in
// place in the grid layout [nu][P][nv], and the screens read or write that
// layout directly: pixel (i, j) of plane p is grid entry (u, p, jx) with
// u = i - nx/2 (mod nu) and jx = j - ny/2 (mod nv).  Threads run along j,
// which is contiguous in both the grid and the x-major image.
__device__ __forceinline__ size_t grid_cell(const ScreenArgs &s, int i, int j) {
  int jx = j + s.nv - s.ny / 2;
  jx -= (jx >= s.nv) ? s.nv : 0;
  int u = i - s.nx / 2;
  u += (u < 0) ? s.nu : 0;
  return size_t(u) * size_t(s.P) * size_t(s.nv) + size_t(jx);
}

// ms2dirty: img(i,j) (+)= corr(i,j) * sum_p Re(G[u][p][jx] * exp(-2 pi i w_p q))
// (out_mode as k_screen_add).  G points at the pass's first plane.
template <typename R>
__global__ void __launch_bounds__(256) k_screen_add_grid(ScreenArgs s, const void *Gv, double *img,
                                                         void *out, int out_mode) {
  using C = typename Cplx<R>::type;
  const C *G = reinterpret_cast<const C *>(Gv);
  const int j = blockIdx.x * 32 + (threadIdx.x & 31);
  const int i = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (i >= s.nx || j >= s.ny) return;
  constexpr int PB = sizeof(R) == 4 ? 16 : 8;
  const C *gp = G + grid_cell(s, i, j);
  C hb[PB];
#pragma unroll
  for (int u = 0; u < PB; ++u)
    if (u < s.npl) hb[u] = gp[size_t(u) * s.nv];
  double corr, q;
  bool inside;
  pixel_terms(s, i, j, corr, q, inside);
  const bool screen = s.do_w && inside;
  using SC = typename std::conditional<sizeof(R) == 4, float2, double2>::type;
  SC sc, st;
  sc.x = st.x = 1;
  sc.y = st.y = 0;
  const double w0 = s.wmin + s.pb0 * s.dw;
  if (screen) st = screen_phase<R>(-s.dw * q);
  double acc = 0;
  for (int p0 = 0; p0 < s.npl; p0 += PB) {
    if (p0 > 0) {
#pragma unroll
      for (int u = 0; u < PB; ++u)
        if (p0 + u < s.npl) hb[u] = gp[size_t(p0 + u) * s.nv];
    }
    R part = 0;
    if (screen) {
      if (sizeof(R) == 4 || p0 == 0) sc = screen_phase<R>(-(w0 + p0 * s.dw) * q);
#pragma unroll
      for (int u = 0; u < PB; ++u) {
        if (p0 + u < s.npl) {
          part += hb[u].x * sc.x - hb[u].y * sc.y;
          const auto nr = sc.x * st.x - sc.y * st.y;
          sc.y = sc.x * st.y + sc.y * st.x;
          sc.x = nr;
        }
      }
    } else {
#pragma unroll
      for (int u = 0; u < PB; ++u)
        if (p0 + u < s.npl) part += hb[u].x;
    }
    acc += double(part);
  }
  const double x = acc * corr;
  const size_t o = size_t(i) * s.ld + j;
  if (out_mode == 0)
    img[o] += x;
  else if (out_mode == 1)
    reinterpret_cast<float *>(out)[o] = float(x);
  else
    reinterpret_cast<double *>(out)[o] = x;
}

// dirty2ms: G[u][p][jx] = dirty(i,j) * corr(i,j) * exp(+2 pi i w_p q) for the
// pass's planes (the grid's other entries are left as they are: zero).
template <typename R>
__global__ void __launch_bounds__(256) k_screen_put_grid(ScreenArgs s, const void *img, int in_f32,
                                                         void *Gv) {
  using C = typename Cplx<R>::type;
  C *G = reinterpret_cast<C *>(Gv);
  const int j = blockIdx.x * 32 + (threadIdx.x & 31);
  const int i = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (i >= s.nx || j >= s.ny) return;
  const size_t o = size_t(i) * s.ld + j;
  const double x = in_f32 ? double(reinterpret_cast<const float *>(img)[o])
                          : reinterpret_cast<const double *>(img)[o];
  double corr, q;
  bool inside;
  pixel_terms(s, i, j, corr, q, inside);
  const R rv = R(x * corr);
  C *gp = G + grid_cell(s, i, j);
  if (s.do_w && inside) {
    const double w0 = s.wmin + s.pb0 * s.dw;
    const auto st = screen_phase<R>(s.dw * q);
    auto sc = st;
    for (int p0 = 0; p0 < s.npl; p0 += 16) {
      if (sizeof(R) == 4 || p0 == 0) sc = screen_phase<R>((w0 + p0 * s.dw) * q);
      const int pe = min(s.npl, p0 + 16);
      for (int p = p0; p < pe; ++p) {
        C v;
        v.x = rv * sc.x;
        v.y = rv * sc.y;
        gp[size_t(p) * s.nv] = v;
        const auto nr = sc.x * st.x - sc.y * st.y;
        sc.y = sc.x * st.y + sc.y * st.x;
        sc.x = nr;
      }
    }
  } else {
    for (int p = 0; p < s.npl; ++p) {
      C v;
      v.x = rv;
      v.y = R(0);
      gp[size_t(p) * s.nv] = v;
    }
  }
}

// ---------------------------------------------------------- small kernels

template <typename TI>
__global__ void k_load_image(size_t n, const TI *__restrict__ in, double *__restrict__ out,
                             int accumulate) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    out[i] = accumulate ? out[i] + double(in[i]) : double(in[i]);
}

template <typename TO>
__global__ void k_store_image(size_t n, const double *__restrict__ in, TO *__restrict__ out) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    out[i] = TO(in[i]);
}

static __global__ void k_scale(size_t n, double *__restrict__ x, double f) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    x[i] *= f;
}

// trimmed x-major FP64 image <- untrimmed float image (index x + y*width)
static __global__ void k_untrim(int wt, int ht, int width, int dx, int dy, const float *__restrict__ in,
                         double *__restrict__ out) {
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < size_t(wt) * ht;
       t += size_t(gridDim.x) * blockDim.x) {
    int i = int(t / ht), j = int(t % ht);
    out[t] = double(in[(size_t(i) + dx) + (size_t(j) + dy) * width]);
  }
}

// untrimmed float image (NaN outside) <- trimmed x-major FP64 image
static __global__ void k_retrim(int wt, int ht, int width, int height, int dx, int dy,
                         const double *__restrict__ in, float *__restrict__ out) {
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < size_t(width) * height;
       t += size_t(gridDim.x) * blockDim.x) {
    int x = int(t % width), y = int(t / width);
    int i = x - dx, j = y - dy;
    out[t] = (i >= 0 && i < wt && j >= 0 && j < ht) ? float(in[size_t(i) * ht + j])
                                                     : __int_as_float(0x7fc00000);
  }
}

}  // namespace wsg
