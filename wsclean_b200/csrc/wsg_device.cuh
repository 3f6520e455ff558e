// Device kernels of libwsg (sm_100a).  Host orchestration is in wsg_context.cu.
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
//   cuFFT       pruned 2-D backward FFT per plane (band rows along v, image
//               columns along u)                              (grid2dirty_c_overwrite_wscreen_add, :496-534)
//   k_screen    sum over planes of Re(grid * w-screen), FP64, times the grid
//               correction, added into the FP64 image         (grid2dirty_post2 :428-484, apply_global_corrections :1348-1400)
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

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
  uint32_t inactive_key;
  int Lu, band_rows, band_full;
};

struct ScanOut {
  unsigned long long wmin_bits, wmax_bits, umax_bits, vmax_bits;
  unsigned long long nvis;
};

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

__device__ __forceinline__ uint32_t bin_key(const DevGeom &g, const VisPix &p) {
  int a = p.iu0 + g.nsafe, b = p.iv0 + g.nsafe;
  uint32_t tu = uint32_t(a / g.T), tv = uint32_t(b / g.T);
  uint32_t lu = uint32_t(a % g.T), lv = uint32_t(b % g.T);
  uint32_t bin = (tu * uint32_t(g.ntv) + tv) * uint32_t(g.nwmin) + uint32_t(p.iw);
  // in-tile position, quantised to lbits per axis (T <= 32)
  uint32_t q = ((lu >> g.qshift) << g.lbits) | (lv >> g.qshift);
  return (bin << (2 * g.lbits)) | q;
}

template <int W, typename R>
__device__ __forceinline__ void eval_pieces(const DevKernel<R> &k, R x, R *out) {
#pragma unroll
  for (int i = 0; i < W; ++i) out[i] = k.c[k.D][i];
  for (int j = k.D - 1; j >= 0; --j) {
#pragma unroll
    for (int i = 0; i < W; ++i) out[i] = fma(out[i], x, k.c[j][i]);
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// --------------------------------------------------------------- k_scan

template <typename TV, typename TW>
__global__ void k_scan(size_t nrows, int nchan, const double *__restrict__ uvw,
                       const double *__restrict__ fovc, const TV *__restrict__ vis,
                       const TW *__restrict__ wgt, const uint8_t *__restrict__ mask,
                       int gridding, double vfac, ScanOut *out, TV *__restrict__ vis_out) {
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
        if (wgt) n *= wgt[k];
        if (mask) n *= mask[k];
        act = (n != 0);
      } else {
        act = (!wgt || wgt[k] != 0) && (!mask || mask[k] != 0);
        if (!act && vis_out) vis_out[k] = TV{0, 0};
      }
      if (act) {
        double f = fovc[c];
        double aw = fabs(w * f);
        lwmin = fmin(lwmin, aw);
        lwmax = fmax(lwmax, aw);
        lumax = fmax(lumax, fabs(u * f));
        lvmax = fmax(lvmax, fabs(v * f));
        ++cnt;
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

// --------------------------------------------------------------- k_keys

template <typename TV, typename TW>
__global__ void k_keys(size_t nrows, int nchan, const double *__restrict__ uvw,
                       const double *__restrict__ fovc, const TV *__restrict__ vis,
                       const TW *__restrict__ wgt, const uint8_t *__restrict__ mask,
                       int gridding, DevGeom g, uint32_t *__restrict__ keys,
                       uint32_t *__restrict__ vals) {
  for (size_t r = blockIdx.x * size_t(blockDim.x) + threadIdx.x; r < nrows;
       r += size_t(gridDim.x) * blockDim.x) {
    double u = uvw[3 * r], v = g.vfac * uvw[3 * r + 1], w = uvw[3 * r + 2];
    for (int c = 0; c < nchan; ++c) {
      size_t k = r * nchan + c;
      bool act;
      if (gridding) {
        TV x = vis[k];
        auto n = x.x * x.x + x.y * x.y;
        if (wgt) n *= wgt[k];
        if (mask) n *= mask[k];
        act = (n != 0);
      } else {
        act = (!wgt || wgt[k] != 0) && (!mask || mask[k] != 0);
      }
      uint32_t key = g.inactive_key;
      if (act) {
        double f = fovc[c];
        VisPix p;
        vis_pixel(g, u * f, v * f, w * f, p);
        key = bin_key(g, p);
      }
      keys[k] = key;
      vals[k] = uint32_t(k);
    }
  }
}

// ------------------------------------------------------------ k_records

template <typename R, typename TV, typename TW>
__global__ void k_records(size_t nvis, int nchan, const uint32_t *__restrict__ sidx,
                          const double *__restrict__ uvw, const double *__restrict__ fovc,
                          const TV *__restrict__ vis, const TW *__restrict__ wgt,
                          int gridding, DevGeom g, typename RecOf<R>::type *__restrict__ rec) {
  using Rec = typename RecOf<R>::type;
  for (size_t s = blockIdx.x * size_t(blockDim.x) + threadIdx.x; s < nvis;
       s += size_t(gridDim.x) * blockDim.x) {
    uint32_t k = sidx[s];
    size_t r = k / uint32_t(nchan);
    int c = int(k - r * uint32_t(nchan));
    double f = fovc[c];
    double u = uvw[3 * r], v = g.vfac * uvw[3 * r + 1], w = uvw[3 * r + 2];
    VisPix p;
    vis_pixel(g, u * f, v * f, w * f, p);
    double wk = wgt ? double(wgt[k]) : 1.0;
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
    rec[s] = o;
  }
}

// ----------------------------------------------------- chunk boundaries

// A chunk starts where the (tile, minplane) bin changes or at a multiple of
// the chunk size; chunks therefore never cross bins.
struct ChunkStartPred {
  const uint32_t *keys;
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
};

constexpr uint32_t kSkip = 0xfffffffeu;  // record marker: outside its chunk's tile

__device__ __forceinline__ int band_index(const DevGeom &g, int u) {
  if (g.band_full) return u;
  if (u <= g.Lu) return u;
  if (u >= g.nu - g.Lu) return u - (g.nu - g.band_rows);
  return -1;
}

// ------------------------------------------------------------- k_spread
//
// One CTA drains chunks; all records of a chunk share one (tile, minplane)
// bin, so the CTA owns a W-plane shared-memory tile (structure of arrays:
// real parts then imaginary parts) for the chunk.  Warps take contiguous
// slices of each sub-batch; lane q of a warp owns PPL (plane, u-row) pairs of
// the footprint and W cells along v for each, accumulating in registers while
// consecutive records share the footprint origin.
template <typename R, int W, int PPL, int NWARP>
__global__ void __launch_bounds__(NWARP * 32)
k_spread(GridArgs a, DevGeom g, DevKernel<R> kc) {
  using Rec = typename RecOf<R>::type;
  constexpr int NG = (W * W + 32 * PPL - 1) / (32 * PPL);  // warps per record
  constexpr int NSL = NWARP / NG;                          // record slices
  constexpr int KST = 3 * W + 1;                           // kernel values per record
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TileLayout tl = a.tl;
  R *tre = reinterpret_cast<R *>(smem_raw);
  R *tim = tre + W * tl.PS;
  R *kv_s = tim + W * tl.PS;             // [sb][KST]
  R *vv_s = kv_s + a.sb * KST;           // [sb][2]
  uint32_t *luv_s = reinterpret_cast<uint32_t *>(vv_s + 2 * a.sb);  // [sb]
  __shared__ int sh_chunk, sh_bb[4];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = warp % NG, slice = warp / NG;
  const Rec *recs = reinterpret_cast<const Rec *>(a.rec);
  using C = typename Cplx<R>::type;
  C *grid = reinterpret_cast<C *>(a.grid);

  for (int i = tid; i < 2 * W * tl.PS; i += blockDim.x) tre[i] = R(0);
  __syncthreads();

  for (;;) {
    if (tid == 0) {
      sh_chunk = atomicAdd(a.counter, 1);
      sh_bb[0] = 1 << 30; sh_bb[1] = -1; sh_bb[2] = 1 << 30; sh_bb[3] = -1;
    }
    __syncthreads();
    const int ch = sh_chunk;
    if (ch >= *a.nchunks) break;
    const int s0 = a.chunk_start[ch];
    const int s1 = (ch + 1 < *a.nchunks) ? a.chunk_start[ch + 1] : a.nvis;
    const Rec r0 = recs[s0];
    const int a0 = int(r0.iuv >> 16), b0 = int(r0.iuv & 0xffffu);
    const int tu = a0 / g.T, tv = b0 / g.T;
    const int mp = int(r0.mp);
    const bool any_plane = (mp < a.pb1) && (mp + W > a.pb0);

    if (any_plane) {
      for (int sb0 = s0; sb0 < s1; sb0 += a.sb) {
        const int n = min(a.sb, s1 - sb0);
        // kernel values: one (record, axis) per thread
        for (int t = tid; t < 3 * n; t += blockDim.x) {
          const int j = t / 3, ax = t - 3 * j;
          const Rec rr = recs[sb0 + j];
          R vals[W];
          R x = ax == 0 ? rr.xu : (ax == 1 ? rr.xv : rr.xw);
          if (ax < 2 || g.do_w) {
            eval_pieces<W, R>(kc, x, vals);
          } else {
#pragma unroll
            for (int i = 0; i < W; ++i) vals[i] = R(i == 0);
          }
#pragma unroll
          for (int i = 0; i < W; ++i) kv_s[j * KST + ax * W + i] = vals[i];
          if (ax == 0) {
            vv_s[2 * j] = rr.vr;
            vv_s[2 * j + 1] = rr.vi;
            const int lu = int(rr.iuv >> 16) - tu * g.T;
            const int lv = int(rr.iuv & 0xffffu) - tv * g.T;
            if (lu < 0 || lu >= g.T || lv < 0 || lv >= g.T || int(rr.mp) != mp) {
              atomicOr(a.err, 1);
              luv_s[j] = kSkip;
            } else {
              luv_s[j] = (uint32_t(lu) << 16) | uint32_t(lv);
              atomicMin(&sh_bb[0], lu); atomicMax(&sh_bb[1], lu);
              atomicMin(&sh_bb[2], lv); atomicMax(&sh_bb[3], lv);
            }
          }
        }
        __syncthreads();
        if (slice < NSL) {
          const int j0 = (n * slice) / NSL, j1 = (n * (slice + 1)) / NSL;
          R accr[PPL][W], acci[PPL][W];
          int pp[PPL], cu[PPL];
          bool ok[PPL];
#pragma unroll
          for (int k = 0; k < PPL; ++k) {
            const int q = grp * 32 * PPL + lane + 32 * k;
            pp[k] = q / W;
            cu[k] = q - pp[k] * W;
            ok[k] = (q < W * W) && (mp + pp[k] >= a.pb0) && (mp + pp[k] < a.pb1);
#pragma unroll
            for (int c = 0; c < W; ++c) accr[k][c] = acci[k][c] = R(0);
          }
          uint32_t cur = 0xffffffffu;
          auto commit = [&]() {
            if (cur == 0xffffffffu) return;
            const int lu = int(cur >> 16), lv = int(cur & 0xffffu);
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
              if (!ok[k]) continue;
              const int base = pp[k] * tl.PS + (lu + cu[k]) * tl.RS + lv;
#pragma unroll
              for (int c = 0; c < W; ++c) {
                atomicAdd(&tre[base + c], accr[k][c]);
                atomicAdd(&tim[base + c], acci[k][c]);
                accr[k][c] = acci[k][c] = R(0);
              }
            }
          };
          for (int j = j0; j < j1; ++j) {
            const uint32_t luv = luv_s[j];
            if (luv == kSkip) continue;
            if (luv != cur) {
              commit();
              cur = luv;
            }
            const R vr = vv_s[2 * j], vi = vv_s[2 * j + 1];
            const R *kj = kv_s + j * KST;
            R kvv[W];
#pragma unroll
            for (int c = 0; c < W; ++c) kvv[c] = kj[W + c];
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
              const int pk = ok[k] ? pp[k] : 0, ck = ok[k] ? cu[k] : 0;
              const R f = kj[2 * W + pk] * kj[ck];
              const R ar = vr * f, ai = vi * f;
#pragma unroll
              for (int c = 0; c < W; ++c) {
                accr[k][c] = fma(ar, kvv[c], accr[k][c]);
                acci[k][c] = fma(ai, kvv[c], acci[k][c]);
              }
            }
          }
          commit();
        }
        __syncthreads();
      }
      // flush the touched region of the tile to the band grid
      const int lu0 = sh_bb[0], lu1 = sh_bb[1] + W, lv0 = sh_bb[2], lv1 = sh_bb[3] + W;
      const int nbu = max(lu1 - lu0, 0), nbv = max(lv1 - lv0, 0);
      const int ucorner = tu * g.T - g.nsafe, vcorner = tv * g.T - g.nsafe;
      const int ncell = W * nbu * nbv;
      for (int t = tid; t < ncell; t += blockDim.x) {
        const int p = t / (nbu * nbv);
        const int rem = t - p * nbu * nbv;
        const int ia = lu0 + rem / nbv, ib = lv0 + rem % nbv;
        const int sidx = p * tl.PS + ia * tl.RS + ib;
        const R xr = tre[sidx], xi = tim[sidx];
        const int plane = mp + p;
        if ((xr != R(0) || xi != R(0)) && plane >= a.pb0 && plane < a.pb1) {
          int u = ucorner + ia;
          u += (u < 0) ? g.nu : 0;
          u -= (u >= g.nu) ? g.nu : 0;
          int v = vcorner + ib;
          v += (v < 0) ? g.nv : 0;
          v -= (v >= g.nv) ? g.nv : 0;
          const int bi = band_index(g, u);
          if (bi >= 0) {
            C *dst = grid + (size_t(bi) * a.P + (plane - a.pb0)) * size_t(g.nv) + v;
            if constexpr (sizeof(R) == 4) {
              atomicAdd(reinterpret_cast<float2 *>(dst), make_float2(xr, xi));
            } else {
              atomicAdd(&dst->x, xr);
              atomicAdd(&dst->y, xi);
            }
          }
        }
        tre[sidx] = R(0);
        tim[sidx] = R(0);
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------- k_interp
//
// Degridding, the exact transpose of k_spread: the chunk's tile region is
// staged from the band grid into shared memory, each lane caches its
// (plane, u-row) x W cells in registers while the footprint origin repeats,
// and the kernel-weighted sum is reduced across the warp.
template <typename R, int W, int PPL, int NWARP>
__global__ void __launch_bounds__(NWARP * 32)
k_interp(GridArgs a, DevGeom g, DevKernel<R> kc) {
  using Rec = typename RecOf<R>::type;
  using C = typename Cplx<R>::type;
  constexpr int NG = (W * W + 32 * PPL - 1) / (32 * PPL);
  constexpr int NSL = NWARP / NG;
  constexpr int KST = 3 * W + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TileLayout tl = a.tl;
  R *tre = reinterpret_cast<R *>(smem_raw);
  R *tim = tre + W * tl.PS;
  R *kv_s = tim + W * tl.PS;
  R *res_s = kv_s + a.sb * KST;                                     // [sb][2]
  uint32_t *luv_s = reinterpret_cast<uint32_t *>(res_s + 2 * a.sb);  // [sb]
  __shared__ int sh_chunk, sh_bb[4];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = warp % NG, slice = warp / NG;
  const Rec *recs = reinterpret_cast<const Rec *>(a.rec);
  const C *grid = reinterpret_cast<const C *>(a.grid);

  for (;;) {
    if (tid == 0) {
      sh_chunk = atomicAdd(a.counter, 1);
      sh_bb[0] = 1 << 30; sh_bb[1] = -1; sh_bb[2] = 1 << 30; sh_bb[3] = -1;
    }
    __syncthreads();
    const int ch = sh_chunk;
    if (ch >= *a.nchunks) break;
    const int s0 = a.chunk_start[ch];
    const int s1 = (ch + 1 < *a.nchunks) ? a.chunk_start[ch + 1] : a.nvis;
    const Rec r0 = recs[s0];
    const int tu = int(r0.iuv >> 16) / g.T, tv = int(r0.iuv & 0xffffu) / g.T;
    const int mp = int(r0.mp);
    const bool any_plane = (mp < a.pb1) && (mp + W > a.pb0);
    // bounding box of the chunk's footprints
    for (int s = s0 + tid; s < s1; s += blockDim.x) {
      const uint32_t iuv = recs[s].iuv;
      const int lu = int(iuv >> 16) - tu * g.T, lv = int(iuv & 0xffffu) - tv * g.T;
      if (lu < 0 || lu >= g.T || lv < 0 || lv >= g.T) continue;
      atomicMin(&sh_bb[0], lu); atomicMax(&sh_bb[1], lu);
      atomicMin(&sh_bb[2], lv); atomicMax(&sh_bb[3], lv);
    }
    __syncthreads();
    const int lu0 = sh_bb[0], lv0 = sh_bb[2];
    const int nbu = max(sh_bb[1] + W - lu0, 0), nbv = max(sh_bb[3] + W - lv0, 0);
    const int ucorner = tu * g.T - g.nsafe, vcorner = tv * g.T - g.nsafe;
    const int ncell = W * nbu * nbv;
    for (int t = tid; t < ncell; t += blockDim.x) {
      const int p = t / (nbu * nbv);
      const int rem = t - p * nbu * nbv;
      const int ia = lu0 + rem / nbv, ib = lv0 + rem % nbv;
      const int plane = mp + p;
      C val;
      val.x = R(0);
      val.y = R(0);
      if (any_plane && plane >= a.pb0 && plane < a.pb1) {
        int u = ucorner + ia;
        u += (u < 0) ? g.nu : 0;
        u -= (u >= g.nu) ? g.nu : 0;
        int v = vcorner + ib;
        v += (v < 0) ? g.nv : 0;
        v -= (v >= g.nv) ? g.nv : 0;
        const int bi = band_index(g, u);
        if (bi >= 0) val = grid[(size_t(bi) * a.P + (plane - a.pb0)) * size_t(g.nv) + v];
      }
      const int sidx = p * tl.PS + ia * tl.RS + ib;
      tre[sidx] = val.x;
      tim[sidx] = val.y;
    }
    __syncthreads();

    for (int sb0 = s0; sb0 < s1; sb0 += a.sb) {
      const int n = min(a.sb, s1 - sb0);
      for (int t = tid; t < 3 * n; t += blockDim.x) {
        const int j = t / 3, ax = t - 3 * j;
        const Rec rr = recs[sb0 + j];
        R vals[W];
        R x = ax == 0 ? rr.xu : (ax == 1 ? rr.xv : rr.xw);
        if (ax < 2 || g.do_w) {
          eval_pieces<W, R>(kc, x, vals);
        } else {
#pragma unroll
          for (int i = 0; i < W; ++i) vals[i] = R(i == 0);
        }
#pragma unroll
        for (int i = 0; i < W; ++i) kv_s[j * KST + ax * W + i] = vals[i];
        if (ax == 0) {
          res_s[2 * j] = R(0);
          res_s[2 * j + 1] = R(0);
          const int lu = int(rr.iuv >> 16) - tu * g.T;
          const int lv = int(rr.iuv & 0xffffu) - tv * g.T;
          if (lu < 0 || lu >= g.T || lv < 0 || lv >= g.T || int(rr.mp) != mp) {
            atomicOr(a.err, 1);
            luv_s[j] = kSkip;
          } else {
            luv_s[j] = (uint32_t(lu) << 16) | uint32_t(lv);
          }
        }
      }
      __syncthreads();
      if (slice < NSL && any_plane) {
        const int j0 = (n * slice) / NSL, j1 = (n * (slice + 1)) / NSL;
        R cr[PPL][W], ci[PPL][W];
        int pp[PPL], cu[PPL];
        bool ok[PPL];
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
          const int q = grp * 32 * PPL + lane + 32 * k;
          pp[k] = q / W;
          cu[k] = q - pp[k] * W;
          ok[k] = (q < W * W);
        }
        uint32_t cur = 0xffffffffu;
        for (int j = j0; j < j1; ++j) {
          const uint32_t luv = luv_s[j];
          if (luv == kSkip) continue;
          if (luv != cur) {
            cur = luv;
            const int lu = int(luv >> 16), lv = int(luv & 0xffffu);
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
              const int base = (ok[k] ? pp[k] * tl.PS + (lu + cu[k]) * tl.RS : 0) + lv;
#pragma unroll
              for (int c = 0; c < W; ++c) {
                cr[k][c] = ok[k] ? tre[base + c] : R(0);
                ci[k][c] = ok[k] ? tim[base + c] : R(0);
              }
            }
          }
          const R *kj = kv_s + j * KST;
          R kvv[W];
#pragma unroll
          for (int c = 0; c < W; ++c) kvv[c] = kj[W + c];
          R sr = R(0), si = R(0);
#pragma unroll
          for (int k = 0; k < PPL; ++k) {
            R tr = R(0), ti = R(0);
#pragma unroll
            for (int c = 0; c < W; ++c) {
              tr = fma(cr[k][c], kvv[c], tr);
              ti = fma(ci[k][c], kvv[c], ti);
            }
            const int pk = ok[k] ? pp[k] : 0, ck = ok[k] ? cu[k] : 0;
            const R f = ok[k] ? kj[2 * W + pk] * kj[ck] : R(0);
            sr = fma(tr, f, sr);
            si = fma(ti, f, si);
          }
          sr = warp_sum(sr);
          si = warp_sum(si);
          if (lane == 0) {
            if (NG == 1) {
              res_s[2 * j] = sr;
              res_s[2 * j + 1] = si;
            } else {
              atomicAdd(&res_s[2 * j], sr);
              atomicAdd(&res_s[2 * j + 1], si);
            }
          }
        }
      }
      __syncthreads();
      // finalize this sub-batch's records
      for (int j = tid; j < n; j += blockDim.x) {
        const int s = sb0 + j;
        R sr = res_s[2 * j], si = res_s[2 * j + 1];
        C *accp = reinterpret_cast<C *>(a.acc);
        if (!a.first_pass) {
          sr += accp[s].x;
          si += accp[s].y;
        }
        if (a.last_pass) {
          const Rec rr = recs[s];
          const uint32_t idx = rr.idx & 0x7fffffffu;
          if (rr.idx & 0x80000000u) si = -si;
          const double orr = double(rr.vr) * double(sr) - double(rr.vi) * double(si);
          const double oi = double(rr.vr) * double(si) + double(rr.vi) * double(sr);
          if (a.vis_double) {
            reinterpret_cast<double2 *>(a.vis_out)[idx] = make_double2(orr, oi);
          } else {
            reinterpret_cast<float2 *>(a.vis_out)[idx] = make_float2(float(orr), float(oi));
          }
        } else {
          C o;
          o.x = sr;
          o.y = si;
          accp[s] = o;
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------- screens

struct ScreenArgs {
  int nx, ny, nu, nv;
  double px, py, x0, y0;
  double nshift, dw, wmin;
  int do_w, divide_by_n;
  int P, pb0, npl;          // layout planes, first plane, planes in this pass
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

// ms2dirty: img(i,j) += corr(i,j) * sum_p Re(H[p][j][ix] * exp(-2 pi i w_p q))
// H holds the u-transformed image columns, [P][ny][nu].
template <typename R>
__global__ void __launch_bounds__(256) k_screen_add(ScreenArgs s, const void *Hv, double *img) {
  using C = typename Cplx<R>::type;
  const C *H = reinterpret_cast<const C *>(Hv);
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const int i = i0 + tx;
  for (int k = 0; k < 4; ++k) {
    const int j = j0 + ty + 8 * k;
    double val = 0;
    if (i < s.nx && j < s.ny) {
      double corr, q;
      bool inside;
      pixel_terms(s, i, j, corr, q, inside);
      int ix = s.nu - s.nx / 2 + i;
      if (ix >= s.nu) ix -= s.nu;
      double acc = 0;
      if (s.do_w && inside) {
        const double w0 = s.wmin + s.pb0 * s.dw;
        double2 sc = cexp_turns(-w0 * q);
        const double2 st = cexp_turns(-s.dw * q);
        for (int p = 0; p < s.npl; ++p) {
          const C h = H[(size_t(p) * s.ny + j) * s.nu + ix];
          acc += double(h.x) * sc.x - double(h.y) * sc.y;
          const double nr = sc.x * st.x - sc.y * st.y;
          sc.y = sc.x * st.y + sc.y * st.x;
          sc.x = nr;
        }
      } else {
        for (int p = 0; p < s.npl; ++p) acc += double(H[(size_t(p) * s.ny + j) * s.nu + ix].x);
      }
      val = acc * corr;
    }
    tile[ty + 8 * k][tx] = val;
  }
  __syncthreads();
  for (int k = 0; k < 4; ++k) {
    const int ii = i0 + ty + 8 * k, jj = j0 + tx;
    if (ii < s.nx && jj < s.ny) img[size_t(ii) * s.ny + jj] += tile[tx][ty + 8 * k];
  }
}

// dirty2ms: H[p][j][ix] = dirty(i,j) * corr(i,j) * exp(+2 pi i w_p q)
template <typename R>
__global__ void __launch_bounds__(256) k_screen_put(ScreenArgs s, const double *img, void *Hv) {
  using C = typename Cplx<R>::type;
  C *H = reinterpret_cast<C *>(Hv);
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int k = 0; k < 4; ++k) {  // coalesced read along j
    const int ii = i0 + ty + 8 * k, jj = j0 + tx;
    tile[tx][ty + 8 * k] = (ii < s.nx && jj < s.ny) ? img[size_t(ii) * s.ny + jj] : 0.0;
  }
  __syncthreads();
  const int i = i0 + tx;
  for (int k = 0; k < 4; ++k) {
    const int j = j0 + ty + 8 * k;
    if (i >= s.nx || j >= s.ny) continue;
    double corr, q;
    bool inside;
    pixel_terms(s, i, j, corr, q, inside);
    const double val = tile[ty + 8 * k][tx] * corr;
    int ix = s.nu - s.nx / 2 + i;
    if (ix >= s.nu) ix -= s.nu;
    if (s.do_w && inside) {
      const double w0 = s.wmin + s.pb0 * s.dw;
      double2 sc = cexp_turns(w0 * q);
      const double2 st = cexp_turns(s.dw * q);
      for (int p = 0; p < s.npl; ++p) {
        C o;
        o.x = R(val * sc.x);
        o.y = R(val * sc.y);
        H[(size_t(p) * s.ny + j) * s.nu + ix] = o;
        const double nr = sc.x * st.x - sc.y * st.y;
        sc.y = sc.x * st.y + sc.y * st.x;
        sc.x = nr;
      }
    } else {
      for (int p = 0; p < s.npl; ++p) {
        C o;
        o.x = R(val);
        o.y = R(0);
        H[(size_t(p) * s.ny + j) * s.nu + ix] = o;
      }
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

__global__ void k_scale(size_t n, double *__restrict__ x, double f) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    x[i] *= f;
}

// trimmed x-major FP64 image <- untrimmed float image (index x + y*width)
__global__ void k_untrim(int wt, int ht, int width, int dx, int dy, const float *__restrict__ in,
                         double *__restrict__ out) {
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < size_t(wt) * ht;
       t += size_t(gridDim.x) * blockDim.x) {
    int i = int(t / ht), j = int(t % ht);
    out[t] = double(in[(size_t(i) + dx) + (size_t(j) + dy) * width]);
  }
}

// untrimmed float image (NaN outside) <- trimmed x-major FP64 image
__global__ void k_retrim(int wt, int ht, int width, int height, int dx, int dy,
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
