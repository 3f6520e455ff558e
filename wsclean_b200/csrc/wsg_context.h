// Execution context and stateful gridder of libwsg (host side, internal).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <chrono>
#include <array>
#include <map>
#include <utility>
#include <tuple>
#include <vector>

#include "../../include/wsg.h"
#include "wsg_internal.h"

namespace wsg {

void cuda_check(cudaError_t e, const char *what);
bool is_device_pointer(const void *p);

// Grow-only device buffer.
struct DevBuf {
  void *p = nullptr;
  size_t n = 0;
  void *ensure(size_t bytes);
  void release();
};

struct Layout {
  size_t nu = 0, nv = 0, P = 0, cs = 0;
  bool operator==(const Layout &o) const {
    return nu == o.nu && nv == o.nv && P == o.P && cs == o.cs;
  }
};

class Plan;
class StreamGridder;

// A timed kernel / tile choice of the autotuner.
struct TuneChoice {
  int W = 0;
  double sigma = 0;
  int tile = 0;
  double ms = 0;
};
bool tuned_choice(const wsg_args &a, size_t nvis, TuneChoice &out);
void store_tuned(const wsg_args &a, size_t nvis, const TuneChoice &c);

// Device pointers of one call's inputs (and the imaging weights to fold
// into the visibility weights while gridding them).
struct Staged {
  const double *uvw = nullptr;
  const double *fovc = nullptr;
  const void *vis = nullptr;
  const void *wgt = nullptr;
  const uint8_t *mask = nullptr;
  ImgW iw;
};

class Context {
 public:
  explicit Context(int device);
  ~Context();
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;

  void ms2dirty(const wsg_args &a, const void *vis, void *dirty, int accumulate);
  void dirty2ms(const wsg_args &a, const void *dirty, void *vis);
  void release_buffers();
  void synchronize();
  // Times the pair (ms2dirty + dirty2ms) on these data for the `candidates`
  // cheapest kernels of the cost model and the tile sizes, and keeps the
  // fastest for later calls of the same image size, precision, accuracy and
  // visibility count (within a factor of two).
  void autotune(const wsg_args &a, const void *vis, int candidates, wsg_stats &best);
  size_t device_bytes();
  void validate(const wsg_args &a);

  const void *stage_in(const void *p, size_t bytes, DevBuf &buf, cudaStream_t st = nullptr);
  template <typename R>
  // Grids into the FP64 accumulator img (+= with accumulate, else =), or --
  // when direct_out is given, nothing is accumulated and one pass covers all
  // planes -- writes the image of type a.dirty_type to direct_out and
  // returns true.  ld: row stride of img (0: a.npix_y), for an image that is
  // a facet of a larger one.
  bool grid_core(const wsg_args &a, const Staged &s, double *img, bool accumulate,
                 void *direct_out = nullptr, size_t ld = 0);
  template <typename R>
  // Degrids the FP64 image img, or the caller's image direct_in (of type
  // a.dirty_type) when given; ld: their row stride (0: a.npix_y).  With
  // vis_acc the visibilities are added to vis_out (inactive ones untouched)
  // instead of overwriting it.
  void degrid_core(const wsg_args &a, const Staged &s, const double *img, void *vis_out,
                   const void *direct_in = nullptr, size_t ld = 0, bool vis_acc = false);
  void degrid_from_image(const wsg_args &a, const Staged &s, const double *img, void *vis,
                         size_t vbytes, bool tuned = false);

  // The tuned schedule (ducc0's ms2dirty_tuning / dirty2ms_tuning,
  // wgridder.h:1781-1877): the subdivision of tuning_choice, each part run
  // through grid_core / degrid_core into its facet of the image.  Odd image
  // sizes are accepted as the reference's tuned calls accept them.
  void ms2dirty_tuning(const wsg_args &a, const void *vis, void *dirty, int accumulate);
  void dirty2ms_tuning(const wsg_args &a, const void *dirty, void *vis);
  template <typename R>
  bool grid_tuned(const wsg_args &a, const Staged &s, double *img, bool accumulate,
                  void *direct_out);
  template <typename R>
  void degrid_tuned(const wsg_args &a, const Staged &s, const double *img, void *vis_out,
                    const void *direct_in);
  TuningChoice last_tuning;  // the subdivision of the last tuned call
  bool tuned_call = false;   // ms2dirty / dirty2ms run the tuned schedule
  // odd image sizes: the field centre the reference's subdivision rule sees
  // for the padded image (it differs from the centre used for gridding)
  bool tune_center_set = false;
  double tune_center_x = 0, tune_center_y = 0;

  // Pipelined raw operators (wsg_ctx_set_async): wsg_ms2dirty / wsg_dirty2ms
  // stage their inputs through three slots on a copy stream and write host
  // outputs back on a third stream, so that consecutive calls overlap their
  // transfers with each other's kernels; in asynchronous mode they return
  // without waiting (wsg_ctx_synchronize waits and reports deferred errors).
  struct Slot {
    DevBuf uvw, vis, wgt, mask, out, fovc;
    cudaEvent_t free_ev = nullptr;  // the slot's last use has finished
  };
  bool async_mode = false;
  static constexpr int kSlots = 3;
  Slot slots[kSlots];
  size_t slot_k = 0;
  cudaStream_t cpy = nullptr, d2h = nullptr;
  cudaEvent_t ev_start = nullptr, ev_in = nullptr, ev_done = nullptr, ev_scan = nullptr;
  // the last use of the sort buffers (keys, indices, ranks) by the previous
  // prepare(): a scan on the copy stream, which writes the next call's keys,
  // waits for it
  cudaEvent_t ev_keys = nullptr;
  // where prepare() scans (nullptr: the main stream) and puts f/c
  cudaStream_t scan_st = nullptr;
  DevBuf *fovc_buf = nullptr;
  bool err_pending = false;  // a device-side consistency check not yet read
  // error words of the plans on this context, read (and cleared) by
  // synchronize(): plan executions are asynchronous and may be graph-recorded
  std::vector<int *> plan_err;
  // the scan's statistics come back through mapped pinned memory written by
  // a kernel: a copy-engine read-back would queue behind the previous call's
  // device-to-host copy of its output
  void *h_scan = nullptr, *h_scan_dev = nullptr;  // ScanOut
  // pinned staging of the scan's small uploads (f/c, initial statistics): a
  // pageable copy can wait behind a download in flight; reused once the
  // previous call's scan stream was synchronized
  void *h_small = nullptr;
  size_t h_small_cap = 0;
  void finish_call(const wsg_args &a, Slot &sl, cudaStream_t last);

  int device = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  int num_sms = 148;
  int verbosity = 0;
  int chunk_size = 2048;  // records per chunk at most (a bin may take several)
  wsg_stats stats;
  double cheb_err = 0;

  // buffers
  DevBuf b_uvw, b_fovc, b_vis, b_wgt, b_mask;
  DevBuf b_keys_a, b_keys_b, b_vals_a, b_vals_b, b_cub, b_rec, b_chunks, b_small;
  // spread grid, v-transformed grid, degridding input grid, u-transformed rows
  DevBuf b_band, b_bandf, b_bandd, b_H;
  // the part of b_band the last spread may have written: columns [0, Lv]
  // and [nv - Lv, nv) of its rows (Lv < 0: unknown)
  struct BandDirty {
    void *p = nullptr;
    size_t rows = 0, nv = 0, cs = 0;
    long Lv = -1;
  };
  BandDirty band_dirty;
  // b_bandd's layout whose columns outside the ny image columns are known to
  // be zero (Lv holds ny; p == nullptr: unknown)
  BandDirty bandd_zero;
  void clear_band(void *band, size_t rows, size_t nv, size_t cs);
  void grid_fft(void *grid, const GridPlan &g, size_t P, size_t npl, int dir, bool dbl);
  DevBuf b_img, b_img2, b_acc, b_fftwork, b_out;

 private:
  friend class Plan;
  friend class StreamGridder;
  std::vector<DevBuf *> all_buffers();
  template <typename R>
  bool prepare(const wsg_args &a, const Staged &s, bool gridding, void *vis_out_dev, GridPlan &gp);
  ChebCorr upload_corrections(const GridPlan &g);
  const void *upload_twiddles(const GridPlan &g, bool dbl);
  size_t choose_planes(const GridPlan &g, bool gridding);
  cufftHandle fft_plan(int n, int istride, int idist, int ostride, int odist, int batch, bool dbl);
  void fft_exec(cufftHandle h, void *in, void *out, int dir, bool dbl);
  void record_stats(const GridPlan &g, bool gridding, size_t P);
  void check_device_error(const int *d_err);
  // the |w| histogram of the masked-in visibilities and the subdivision it
  // gives; for a w cut, the masks of the two parts in b_mhi / b_mlo
  TuningChoice tuning_for(const wsg_args &a, const Staged &s);
  DevBuf b_tune, b_tfovc, b_mhi, b_mlo, b_pad;
  void print_report(const GridPlan &g, bool gridding, size_t P);
  void mark(const char *what);
  void print_marks(const char *title);
  std::vector<std::pair<const char *, std::chrono::steady_clock::time_point>> marks;

  // autotuner: a forced (W, sigma, tile) while candidates are timed
  int tune_W = 0, tune_tile = 0;
  double tune_sigma = 0;

  cudaEvent_t ev[8];
  std::map<std::tuple<int, int, int, int, int, int, int>, cufftHandle> fft_plans;
  size_t fft_work_need = 0;
  // last plane-batch choice (choose_planes)
  struct PlanesMemo {
    std::tuple<size_t, size_t, int> key;
    size_t P = 0;
    bool valid = false;
  };
  PlanesMemo planes_memo[2];  // degridding, gridding
  // last grid plan per direction, keyed by the arguments and data statistics
  struct GridMemo {
    std::array<double, 22> key{};
    GridPlan plan;
    bool valid = false;
  };
  GridMemo grid_memo[2];
  // device geometry (DevGeom bytes) of the last planned grid: the next scan
  // writes sort keys for it, used when the next plan comes out the same
  std::vector<unsigned char> spec_geom;
  // correction and column-twiddle tables, two of each cached on the device
  // (ms2dirty and dirty2ms plan their grids apart, so alternating calls
  // would otherwise upload both every call -- from pageable memory, which
  // holds the host until the main stream has drained); the least recently
  // used entry is replaced
  struct CorrEntry {
    std::tuple<int, double, double, size_t, size_t, size_t, size_t, double> key;
    ChebCorr cc;
    DevBuf buf;
    uint64_t used = 0;
    bool valid = false;
  };
  struct TwEntry {
    std::tuple<size_t, size_t, int> key;
    DevBuf buf;
    uint64_t used = 0;
    bool valid = false;
  };
  CorrEntry corr_cache[2];
  TwEntry tw_cache[2];
  uint64_t cache_tick = 0;
  const double *cf_cur = nullptr;  // the tables the last upload_corrections chose
  void invalidate_tables();
};

// One job of a plan (see wsg_plan_create).
// The 2-D transform of one plane in place in the grid layout [nu][P][nv]
// (the whole-grid layout, GridPlan::ucufft), and its execution over npl
// consecutive planes (wsg_context.cu).
cufftHandle make_grid_fft_plan(size_t nu, size_t nv, size_t P, bool dbl, size_t &work);
void exec_grid_fft(cufftHandle h, void *grid, size_t nv, size_t npl, int dir, bool dbl,
                   cudaStream_t st, void *work);

struct PlanJob {
  GridPlan gp;              // the job's grid (shared kernel)
  size_t chan0 = 0, chan1 = 0;
  size_t rec_off = 0, nrec = 0;
  size_t band_off = 0, band_bytes = 0;  // bytes in the plan's band buffer
  size_t cf_off = 0;        // doubles in the plan's correction buffer
  size_t tw_off = 0;        // bytes in the plan's twiddle buffer
  ChebCorr cc;
  cufftHandle fft = 0;
  cufftHandle gfft = 0;      // the whole-grid layout's plane transform (GridPlan::ucufft)
};

// Reusable plan over one or more jobs sharing the visibilities.
class Plan {
 public:
  Plan(Context &cx, const wsg_args &a, const wsg_job *jobs, size_t njobs);
  ~Plan();
  Plan(const Plan &) = delete;
  Plan &operator=(const Plan &) = delete;
  void ms2dirty(const void *vis, void *const *dirty, int accumulate);
  void dirty2ms(const void *const *dirty, void *vis);
  void stats(size_t job, wsg_stats &out) const;
  size_t njobs() const { return jobs_.size(); }

 private:
  template <typename R>
  void build(const std::vector<wsg_job> &jobs);
  template <typename R>
  void enqueue_grid(const void *vis, void *const *dirty, int accumulate);
  template <typename R>
  void enqueue_degrid(const void *const *dirty, void *vis);
  void enqueue(int mode, const void *in, void *const *outs, const void *const *ins, void *out,
               int accumulate);
  void run(int mode, const void *in, void *const *outs, const void *const *ins, void *out,
           int accumulate);

  Context &cx_;
  wsg_args a_;
  bool dbl_ = false;
  std::vector<PlanJob> jobs_;
  DevBuf rec_, chunks_, chunk_job_, jobgeom_, band_, H_, img_, cf_, tw_, acc_, small_, fftwork_;
  size_t nrec_ = 0, band_total_ = 0, max_npix_ = 0;
  int nchunks_ = 0;
  std::vector<unsigned char> kernel_;  // DevKernel<R> bytes
  std::vector<unsigned char> geom_;    // DevGeom of the first job (kernel, tile: shared)
  int W_ = 0, T_ = 0;
  bool need_acc_ = false;
  // graphs recorded per (mode, pointers, accumulate)
  struct Graph {
    int mode = 0, accumulate = 0;
    std::vector<const void *> ptrs;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<Graph> graphs_;
  std::vector<std::pair<int, std::vector<const void *>>> eager_seen_;
  bool use_graphs_ = true;
};

// Host buffer in page-locked memory (grow-only).
struct PinnedBuf {
  void *p = nullptr;
  size_t n = 0;
  void *ensure(size_t bytes);
  void release();
};

// Streaming into a resident grid (see wsg_stream_create).
class StreamGridder {
 public:
  StreamGridder(Context &cx, const wsg_args &a, double wmin, double wmax, double umax,
                double vmax, size_t nvis);
  ~StreamGridder();
  StreamGridder(const StreamGridder &) = delete;
  StreamGridder &operator=(const StreamGridder &) = delete;
  void add(size_t nrows, const double *uvw, const void *vis, const void *wgt, const uint8_t *mask);
  void finish(void *dirty, int accumulate);
  void predict_begin(const void *dirty);
  void predict(size_t nrows, const double *uvw, void *vis, const void *wgt, const uint8_t *mask);
  void stats(wsg_stats &out) const;
  // Imaging weights folded into every later add (nullptr: none).
  void set_imaging_weights(const class ImageWeightsGpu *w);

 private:
  struct Slot {
    DevBuf uvw, vis, wgt, mask;
    PinnedBuf h_uvw, h_vis, h_wgt, h_mask;
    cudaEvent_t copied = nullptr, done = nullptr;
    // pipelined prediction into page-locked host memory: the slot's device
    // output and the end of its copy back
    DevBuf vout;
    cudaEvent_t vcopied = nullptr;
  };
  template <typename R>
  void add_t(const Staged &s, size_t nrows);
  template <typename R>
  void finish_t(void *dirty, int accumulate);
  template <typename R>
  void predict_begin_t(const double *img);
  template <typename R>
  void predict_t(const Staged &s, size_t nrows, void *vis_dev);
  Staged stage(Slot &sl, size_t nrows, const double *uvw, const void *vis, const void *wgt,
               const uint8_t *mask);
  size_t plane_batch() const;
  size_t row_plane_bytes() const;
  // Gridding batches: the chunks passed to add() are gathered on the device
  // and sorted and spread together, so that a (tile, w-plane) bin holds the
  // records of many chunks and its tile is flushed to the grid once for all
  // of them; two batches alternate, so that the copies into one overlap the
  // spread of the other.
  struct Batch {
    DevBuf uvw, vis, wgt, mask;
    size_t rows = 0;
    bool has_wgt = false, has_mask = false;
    cudaEvent_t filled = nullptr, spread = nullptr;
  };
  Batch batch_[2];
  int bcur_ = 0;
  size_t batch_rows_ = 0;
  DevBuf lambda_;  // channel wavelengths of the imaging-weight lookup
  ImgW iw_;
  bool err_armed_ = false;  // the device error word was cleared for this gridding
  void copy_into(void *dst, const void *src, size_t bytes, PinnedBuf &pin);
  void flush_batch();

  Context &cx_;
  wsg_args a_;
  std::vector<double> freq_;  // the channels, copied at creation
  GridPlan gp_;
  bool dbl_ = false;
  int mode_ = 0;  // 0 idle, 1 gridding, 2 predicting
  DevBuf band_, H_, img_, cf_, tw_, fftwork_, vout_;
  ChebCorr cc_;
  cufftHandle fft_ = 0;
  cudaStream_t copy_ = nullptr;
  Slot slots_[2];
  size_t k_ = 0;
};

// ImageWeights on the device (see wsg_weights_create).
class ImageWeightsGpu {
 public:
  ImageWeightsGpu(Context &cx, int mode, double robust, size_t width, size_t height, double psx,
                  double psy, bool as_taper, double super_weight);
  ~ImageWeightsGpu();
  void grid(size_t nrows, size_t nchan, size_t npol, const double *uvw, const double *freq,
            const float *w);
  void finish();
  void apply(size_t nrows, size_t nchan, size_t npol, const double *uvw, const double *freq,
             const float *in, float *out);
  void get(double *grid, size_t *width, size_t *height, double *total);
  // the finished grid, for lookups while visibilities are gridded
  bool finished() const { return finished_; }
  const double *grid_ptr() const { return reinterpret_cast<const double *>(grid_.p); }
  WeightGrid geometry() const { return WeightGrid{int(W_), int(H_), psx_, psy_}; }
  int device() const { return cx_.device; }

 private:
  const double *lambdas(size_t nchan, const double *freq);
  Context &cx_;
  int mode_;
  double robust_;
  size_t W_, H_;
  double psx_, psy_;
  bool as_taper_, finished_ = false;
  DevBuf grid_, sums_, lambda_, in_, out_;
};

// Allocation-free mixed-precision ms2dirty (scratch in a static device array).
void ms2dirty_noalloc(const wsg_args &a, const void *vis, void *dirty, cudaStream_t stream);

// WGriddingGridder_Simple replacement (wgridder/wgriddinggridder_simple.h:34-144).
class Gridder {
 public:
  explicit Gridder(const wsg_gridder_params &p);
  void memory_usage(size_t &constant, size_t &per_vis) const;
  void initialize_inversion();
  void add_inversion_data(size_t nrows, size_t nchan, const double *uvw, const double *freq,
                          const void *vis);
  void finalize_image(double f);
  void real_image(float *out);
  void initialize_prediction(const float *image);
  void predict_visibilities(size_t nrows, size_t nchan, const double *uvw, const double *freq,
                            void *vis);
  Context &context() { return ctx; }

 private:
  wsg_args args(size_t nrows, size_t nchan, const double *uvw, const double *freq) const;
  wsg_gridder_params prm;
  Context ctx;
  bool have_img = false;
};

}  // namespace wsg
