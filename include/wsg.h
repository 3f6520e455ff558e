/* wsg.h -- C ABI of libwsg, the B200 (sm_100a) w-gridder for WSClean.
 *
 * Two layers, both plain C (no CUDA or torch types in any signature):
 *
 *  1. The stateful gridder that replaces WSClean's WGriddingGridder_Simple<NumT>
 *     behind its WGriddingGridderBase interface
 *     (wgridder/wgriddinggridder_simple.h:8-22, ctor :64-68).  One
 *     wsg_gridder_* entry point per virtual method; the C++ adapter
 *     wsclean_b200/host/wgriddinggridder_b200.h turns the status codes back into
 *     std::runtime_error so WSClean's ThreadedScheduler rethrow path
 *     (scheduling/threadedscheduler.cpp:63-67) keeps working.
 *
 *  2. The raw operators ms2dirty / dirty2ms with ducc0's full argument set
 *     (external/wgridder/ducc0/wgridder/wgridder.h:1696-1729): negate_v,
 *     divide_by_n, sigma range, center_x/center_y, weights and mask.
 *
 * Pointers may be host (pageable or pinned) or device (cudaMalloc / managed)
 * memory; the library asks the CUDA runtime which one it got and stages host
 * buffers through the context's stream.  The caller owns every buffer for the
 * duration of the call.  Every function returns WSG_OK (0) or an error code;
 * wsg_last_error() gives the message for the calling thread.
 *
 * Thread safety: a context (wsg_ctx) or gridder is used by one thread at a
 * time; different contexts are independent (each owns its stream, buffers and
 * cuFFT plans), matching one gridder per -parallel-gridding worker
 * (scheduling/threadedscheduler.cpp:54-58).
 */
#ifndef WSG_H
#define WSG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WSG_ABI_VERSION 1

/* Status codes.  WSG_ERR_INVALID covers the reference's MR_assert checks
 * (odd image size, unsorted or non-positive frequencies, too many channels or
 * w planes, no kernel for the requested epsilon). */
enum {
  WSG_OK = 0,
  WSG_ERR_INVALID = 1,
  WSG_ERR_CUDA = 2,
  WSG_ERR_NOMEM = 3,
  WSG_ERR_CUFFT = 4,
  WSG_ERR_STATE = 5,
  WSG_ERR_INTERNAL = 7
};

/* Arithmetic forms.  MIXED: FP32 kernel evaluation, spreading, grid and FFT;
 * FP64 uvw->pixel scaling, phases, w-screen, image accumulation and
 * correction.  FP64: everything in FP64 (the plain form). */
enum { WSG_PREC_MIXED = 0, WSG_PREC_FP64 = 1 };
/* element types */
enum { WSG_C64 = 0, WSG_C128 = 1 };   /* complex<float>, complex<double> */
enum { WSG_F32 = 0, WSG_F64 = 1 };    /* float, double */

typedef struct wsg_ctx wsg_ctx;
typedef struct wsg_gridder wsg_gridder;

/* ---------------------------------------------------------------- context */

/* An execution context on one CUDA device: its own stream, buffer cache and
 * cuFFT plans.  device < 0 selects the current device. */
int wsg_ctx_create(int device, wsg_ctx **out);
int wsg_ctx_destroy(wsg_ctx *ctx);
/* Optional: run on a caller-provided cudaStream_t (passed as void*); NULL
 * returns to the context's own stream (pass cudaStreamLegacy for the legacy
 * default stream).  Work on the stream before a call is ordered before it. */
int wsg_ctx_set_stream(wsg_ctx *ctx, void *stream);
/* Releases the cached device buffers and cuFFT plans (they regrow on demand). */
int wsg_ctx_release_buffers(wsg_ctx *ctx);
/* Pipelined mode for wsg_ms2dirty / wsg_dirty2ms (0: off, the default).
 * Every call stages its inputs through one of three buffer slots on a copy
 * stream and writes host outputs back on a third stream, so consecutive
 * calls overlap their transfers with each other's kernels; with async != 0
 * the calls return once their work is enqueued (after the short planning
 * read-back of the visibility scan), outputs are valid after
 * wsg_ctx_synchronize, which also reports errors detected on the device,
 * and host outputs should be page-locked for the copies to overlap.  Not
 * for a gridder's context (wsg_gridder_ctx).  Extension of the reference
 * interface, whose calls are synchronous. */
int wsg_ctx_set_async(wsg_ctx *ctx, int async);

/* ------------------------------------------------------- raw operators */

/* ducc0's argument set (wgridder.h:1696-1729).  uvw: nrows x 3 doubles in
 * metres; freq: nchan doubles in Hz, ascending; wgt: nrows x nchan of
 * wgt_type or NULL (all ones); mask: nrows x nchan uint8 or NULL.  The dirty
 * image is npix_x x npix_y, x-major (index i*npix_y + j, ducc0's dirty(i,j)). */
typedef struct {
  size_t nrows, nchan;
  const double *uvw;
  const double *freq;
  const void *wgt;
  int wgt_type;          /* WSG_F32 / WSG_F64 */
  const uint8_t *mask;
  size_t npix_x, npix_y;
  double pixsize_x, pixsize_y;
  double epsilon;
  int do_wgridding;
  int negate_v;
  int divide_by_n;
  double sigma_min, sigma_max;
  double center_x, center_y;
  int precision;         /* WSG_PREC_MIXED / WSG_PREC_FP64 */
  int vis_type;          /* WSG_C64 / WSG_C128 */
  int dirty_type;        /* WSG_F32 / WSG_F64 */
} wsg_args;

/* Fills a wsg_args with ducc0's defaults (negate_v=0, divide_by_n=1,
 * sigma 1.1..2.6, no shift, MIXED, c64, f32). */
void wsg_args_init(wsg_args *a);

/* Replaces ducc0::ms2dirty (wgridder.h:1696-1710): dirty = gridded image of
 * vis (nrows x nchan of vis_type).  If accumulate != 0 the result is added to
 * dirty instead of overwriting it.  Limits beyond the reference's checks: at
 * most 2^31 - 1 visibilities a call, and an oversampled grid below 65535
 * cells a side (WSG_ERR_INVALID otherwise). */
int wsg_ms2dirty(wsg_ctx *ctx, const wsg_args *a, const void *vis, void *dirty,
                 int accumulate);
/* Replaces ducc0::dirty2ms (wgridder.h:1712-1729), the exact adjoint. */
int wsg_dirty2ms(wsg_ctx *ctx, const wsg_args *a, const void *dirty, void *vis);

/* Replace ducc0::ms2dirty_tuning / dirty2ms_tuning (wgridder.h:1781-1877),
 * the calls behind WSClean's -gridder tuned-wgridder
 * (wgriddinggridder_simple.cpp:59-63, :109-113): the same operators, with
 * the work subdivided when the |w| statistics of the masked-in visibilities
 * say it pays -- facets (each a smaller image with its own phase centre, so
 * fewer w planes) for the visibilities at or above a |w| cut, the whole
 * image for those below it.  The subdivision follows the reference's rule
 * (get_tuning_parameters, wgridder.cc:144-278) and the results equal
 * wsg_ms2dirty / wsg_dirty2ms within epsilon.  Odd image sizes are accepted,
 * as the reference's tuned calls accept them (wgridder.h:1789-1801,
 * :1829-1838).  The calls synchronise with the host between parts. */
int wsg_ms2dirty_tuning(wsg_ctx *ctx, const wsg_args *a, const void *vis, void *dirty,
                        int accumulate);
int wsg_dirty2ms_tuning(wsg_ctx *ctx, const wsg_args *a, const void *dirty, void *vis);
/* The subdivision of the last tuned call on ctx: nfx x nfy facets (0 x 0: the
 * plain operator), their visibilities from |w| bin icut of 50 on, i.e. from
 * |w| = wcut wavelengths (-1 without subdivision; icut 0: every visibility is
 * faceted).  Extension of the reference interface (its verbosity report). */
int wsg_get_tuning(const wsg_ctx *ctx, int *nfx, int *nfy, int *icut, double *wcut);
/* Host-only: the subdivision the tuned calls choose for these arguments and
 * |w| statistics -- hist[50]: counts of the masked-in visibilities in 50 equal
 * |w| bins over [wmin, wmax] wavelengths, nvis_all = nrows x nchan. */
int wsg_tuning_choice(const wsg_args *a, size_t nvis_all, double wmin, double wmax,
                      const uint64_t *hist, int *nfx, int *nfy, int *icut);

/* Allocation-free variant of wsg_ms2dirty, for callers that cannot allocate
 * device memory while they grid: a plugin inside a host application that
 * reserved the whole device for its own memory pool at start-up (where a
 * cudaMalloc fails, or takes memory the host has promised elsewhere), or a
 * service that must run within a device-memory budget fixed when it started.
 * It calls no cudaMalloc, cudaFree or allocating library routine (no cuFFT
 * plans; its own FFT kernels instead): all scratch comes from one static
 * device array of 96 MiB that every GPU loading the library holds until the
 * process exits.  This entry point has no counterpart in the reference.
 *
 * Limits: mixed precision only; uvw, freq, vis, dirty (and wgt/mask when
 * given) must be device memory; the whole problem's scratch (about 40 bytes
 * per visibility plus the FP64 image plus at least one w plane of the band
 * grid and of the transformed columns) must fit in the 96 MiB, otherwise
 * WSG_ERR_INVALID with a message; nv is a power of two of at most 8192 (an
 * image whose kernels all need a longer grid is rejected), so the grid can
 * differ from wsg_ms2dirty's; results agree within epsilon.
 * The first call in a CUDA context (once per device, again after a device
 * reset) looks up the array's device address.  The call synchronises its
 * stream: it reads the visibility
 * scan's statistics back to the host to plan the grid.  All calls share the
 * array: calls that overlap on the GPU race and must be serialised by the
 * caller.  stream may be NULL (the legacy default stream).  The image is
 * overwritten. */
int wsg_ms2dirty_noalloc(const wsg_args *a, const void *vis, void *dirty, void *stream);

/* -------------------------------------- WGriddingGridder_Simple replacement */

typedef struct {
  size_t width, height;       /* untrimmed image (ActualInversionWidth/Height) */
  size_t width_t, height_t;   /* trimmed image that is gridded */
  double pixel_size_x, pixel_size_y;
  double l_shift, m_shift;
  size_t nthreads;            /* accepted for interface parity; unused */
  double epsilon;
  size_t verbosity;           /* 0..2 as in the reference */
  int tuning;                 /* nonzero: the tuned schedule (wsg_ms2dirty_tuning) */
  int precision;              /* WSG_PREC_MIXED (NumT=float) / WSG_PREC_FP64 (NumT=double) */
  int device;                 /* CUDA device, <0 = current */
} wsg_gridder_params;

/* WGriddingGridder_Simple ctor (wgriddinggridder_simple.h:64-68). */
int wsg_gridder_create(const wsg_gridder_params *p, wsg_gridder **out);
int wsg_gridder_destroy(wsg_gridder *g);
/* MemoryUsage (wgriddinggridder_simple.cpp:27-40): host-side budget figures
 * WSClean uses to size its row chunks. */
int wsg_gridder_memory_usage(const wsg_gridder *g, size_t *constant, size_t *per_vis);
/* InitializeInversion (wgriddinggridder_simple.cpp:42-44): zero the image. */
int wsg_gridder_initialize_inversion(wsg_gridder *g);
/* AddInversionData (wgriddinggridder_simple.cpp:46-65): grid nrows x nchan
 * complex<float> visibilities and add the image to the accumulator. */
int wsg_gridder_add_inversion_data(wsg_gridder *g, size_t nrows, size_t nchan,
                                   const double *uvw, const double *freq,
                                   const void *vis);
/* FinalizeImage (wgriddinggridder_simple.cpp:67-70). */
int wsg_gridder_finalize_image(wsg_gridder *g, double factor);
/* RealImage (wgriddinggridder_simple.cpp:72-83): writes width x height floats,
 * index x + y*width, NaN outside the trimmed box. */
int wsg_gridder_real_image(wsg_gridder *g, float *image);
/* InitializePrediction (wgriddinggridder_simple.cpp:85-94): image is
 * width x height floats, index x + y*width. */
int wsg_gridder_initialize_prediction(wsg_gridder *g, const float *image);
/* PredictVisibilities (wgriddinggridder_simple.cpp:96-115): writes nrows x
 * nchan complex<float>. */
int wsg_gridder_predict_visibilities(wsg_gridder *g, size_t nrows, size_t nchan,
                                     const double *uvw, const double *freq,
                                     void *vis);
/* The gridder's execution context (for stats). */
wsg_ctx *wsg_gridder_ctx(wsg_gridder *g);

/* ------------------------------------------------------ stats / errors */

/* Parameters and per-phase timings of the last operator call on a context
 * (the analogue of ducc0's verbosity report and TimerHierarchy,
 * wgridder.h:1535-1576 and infra/timers.h:69). Times are CUDA-event ms. */
typedef struct {
  size_t nrows, nchan, nvis;          /* nvis = active visibilities */
  size_t nu, nv, nplanes, supp;       /* grid, w planes, kernel support W */
  size_t plane_batch;                 /* planes resident per pass */
  size_t band_rows;                   /* u rows that hold data (FFT pruning) */
  size_t degree;                      /* kernel polynomial degree */
  double sigma, beta, e0, kernel_err; /* chosen kernel and its error estimate */
  double wmin, wmax, dw, nshift;
  double ms_prep, ms_sort, ms_grid, ms_fft, ms_screen, ms_total;
  size_t device_bytes;                /* device memory held by the context */
  int gridding;                       /* 1 ms2dirty, 0 dirty2ms */
  int precision;
  size_t kernel_launches;             /* libwsg kernels launched by this process so far
                                         (cuFFT/CUB library kernels not counted) */
} wsg_stats;

int wsg_get_stats(const wsg_ctx *ctx, wsg_stats *out);
/* Host-only planning query: the grid, kernel and w-plane choice the library
 * would make for these arguments and data statistics (active visibility
 * count, |w| range and max |u|,|v| in wavelengths), without touching a GPU
 * (ducc0 reports the same parameters at verbosity 1, wgridder.h:1535-1560).
 * Fills nu, nv, nplanes, supp, band_rows, degree, sigma, beta, e0,
 * kernel_err, wmin, wmax, dw, nshift and precision. */
int wsg_plan_grid(const wsg_args *a, size_t nvis, double wmin, double wmax, double umax,
                  double vmax, wsg_stats *out);
/* Autotuner: times ms2dirty + dirty2ms on these arguments and data for the
 * `candidates` cheapest kernel choices (support W, oversampling sigma, hence
 * grid size and w-plane count) of the cost model and the bin tile sizes,
 * and keeps the fastest for later calls on any context of this process with
 * the same image size, precision, epsilon, w-gridding flag and number of
 * visibilities within a factor of two.  best: the chosen grid (ms_total =
 * its time per pair in ms).  Accuracy is unaffected: every candidate meets
 * epsilon.  Extension of the reference interface. */
int wsg_autotune(wsg_ctx *ctx, const wsg_args *a, const void *vis, int candidates,
                 wsg_stats *best);
/* Message of the last failed call on this thread ("" if none). */
const char *wsg_last_error(void);
int wsg_abi_version(void);

/* ------------------------------------------ reusable plans, batched jobs */

/* A plan fixes everything that depends only on the coordinates -- uvw,
 * freq, weights and mask -- for repeated ms2dirty / dirty2ms calls on new
 * visibilities or images: the grid and kernel choice, the sort of the
 * visibilities into uv-tile bins and the per-visibility records (pixel
 * coordinates, shift phasor and weight).  This is WSClean's major cycle,
 * which grids (Invert) and degrids (Predict) the same rows many times
 * (wgridder/wgriddingmsgridder.cpp:135-137,179-181).
 *
 * A plan holds one or more jobs sharing the visibilities: facets (each with
 * its own image size and phase centre, the per-facet direction-dependent
 * shift of WSClean's faceting) times output channels (each gridding a range
 * of the input channels).  All jobs share one kernel (W, sigma), chosen for
 * the largest; their records are drained by a single persistent spread or
 * interpolation launch, followed by each job's FFTs and w-screen.
 *
 * Execution enqueues work on the context's stream and returns without
 * waiting (wsg_ctx_synchronize waits).  It performs no allocation and no
 * host synchronisation, so it can be recorded into a CUDA graph by the
 * caller; when the stream is not being captured, the plan records its own
 * graph per set of pointers on the second call and replays it afterwards.
 * vis, dirty and the outputs must be device memory.  A visibility whose
 * weight or mask is zero contributes nothing (the active set of dirty2ms;
 * zero-valued visibilities are gridded as zeros).  These entry points
 * extend the reference's interface; ducc0 re-plans on every call. */
typedef struct wsg_plan wsg_plan;

typedef struct {
  size_t npix_x, npix_y;      /* image (facet) size, both even */
  double center_x, center_y;  /* phase centre of the image, as wsg_args */
  size_t chan_begin, chan_end;/* input channels [chan_begin, chan_end) */
} wsg_job;

/* Builds a plan.  a: the common arguments (uvw, freq, nrows, nchan, wgt,
 * mask, pixel sizes, epsilon, flags, sigma range, precision, vis_type,
 * dirty_type).  jobs: njobs job descriptions, or NULL for one job over all
 * channels with a->npix_x, npix_y, center_x, center_y.  The coordinate
 * arrays are read during the call only. */
int wsg_plan_create(wsg_ctx *ctx, const wsg_args *a, const wsg_job *jobs, size_t njobs,
                    wsg_plan **out);
int wsg_plan_destroy(wsg_plan *p);
/* dirty[j] = image of job j (npix_x x npix_y of dirty_type, x-major), or
 * dirty[j] += image when accumulate != 0.  vis: nrows x nchan of vis_type. */
int wsg_plan_ms2dirty(wsg_plan *p, const void *vis, void *const *dirty, int accumulate);
/* vis = sum over jobs of the prediction of dirty[j] (each job writes its
 * channel range; facets of the same channels add up). */
int wsg_plan_dirty2ms(wsg_plan *p, const void *const *dirty, void *vis);
/* Grid, kernel and plane choice of job `job` (timings are zero). */
int wsg_plan_get_stats(const wsg_plan *p, size_t job, wsg_stats *out);
/* Waits for the work enqueued on the context's stream. */
int wsg_ctx_synchronize(wsg_ctx *ctx);

/* --------------------------------------- streaming into a resident grid */

/* Streaming gridding of data larger than one call -- WSClean's chunked
 * AddInversionData / PredictVisibilities loop (wgridder/wgriddingmsgridder.cpp:80-193)
 * -- with the w-stack of the whole observation resident on the GPU: the grid
 * is planned once from the declared data extent; the chunks of rows passed
 * to wsg_stream_add are copied into device batches of about a third of the
 * expected visibilities (nvis) and each batch is sorted and spread into the
 * same grid (so that a tile of the grid collects the records of many chunks
 * before it is flushed; two batches alternate, so the copies into one
 * overlap the spread of the other); the FFTs, w-screens and correction run
 * once, in wsg_stream_finish.  wsg_stream_add returns once its chunk has
 * been copied (the caller's buffers are free again).  Prediction runs the transpose: the model image is
 * transformed once (wsg_stream_predict_begin) and each chunk is interpolated.
 * Extension of the reference interface, which re-plans and re-transforms per
 * chunk.
 *
 * a: pixel sizes, image size, epsilon, flags, sigma range, centre,
 * precision, vis_type, dirty_type, wgt_type, freq/nchan (the channels of
 * every chunk); nrows, uvw, wgt, mask are ignored.  wmin, wmax: |w| range
 * and umax, vmax: max |u|, |v| in wavelengths over all chunks (a chunk
 * outside is rejected); nvis: expected number of visibilities (kernel
 * choice only).  The stream holds every w plane of its grid: with an
 * occupied u band wider than 8192 grid rows that is the whole nu x nv grid
 * a plane. */
typedef struct wsg_stream wsg_stream;
int wsg_stream_create(wsg_ctx *ctx, const wsg_args *a, double wmin, double wmax, double umax,
                      double vmax, size_t nvis, wsg_stream **out);
int wsg_stream_destroy(wsg_stream *s);
/* Adds nrows rows (uvw nrows x 3, vis nrows x nchan, wgt/mask or NULL).
 * After a prediction (wsg_stream_predict_begin) the first add starts a new
 * gridding on a cleared grid, as a major cycle's Invert follows its Predict.
 * Rows are checked against the declared extent when their batch is sorted:
 * a chunk with an active visibility outside it makes the wsg_stream_add
 * that spreads its batch, or wsg_stream_finish, fail with WSG_ERR_INVALID,
 * and that batch is dropped. */
int wsg_stream_add(wsg_stream *s, size_t nrows, const double *uvw, const void *vis,
                   const void *wgt, const uint8_t *mask);
/* Transforms the accumulated grid into dirty (or adds it when accumulate);
 * the stream is then empty again. */
int wsg_stream_finish(wsg_stream *s, void *dirty, int accumulate);
/* Loads a model image for prediction (rows added since the last
 * wsg_stream_finish are discarded). */
int wsg_stream_predict_begin(wsg_stream *s, const void *dirty);
/* Predicts nrows rows into vis (nrows x nchan of vis_type).  The call
 * returns with vis in place, except with the context in pipelined mode
 * (wsg_ctx_set_async) and vis in page-locked host memory: the chunk is then
 * copied back while the next chunk is computed, and vis is in place after
 * wsg_ctx_synchronize. */
int wsg_stream_predict(wsg_stream *s, size_t nrows, const double *uvw, void *vis,
                       const void *wgt, const uint8_t *mask);
/* Grid choice of the stream (timings are zero). */
int wsg_stream_get_stats(const wsg_stream *s, wsg_stats *out);

/* -------------------------------------------------- imaging weights */

/* WSClean's ImageWeights (structures/imageweights.h:30-100,
 * structures/imageweights.cpp:36-143) on the GPU: visibility weights are
 * summed on a width x height/2 grid over the v >= 0 half plane
 * (x = floor(u W psx + W/2), y = floor(v H psy), u, v in wavelengths with
 * lambda = c / f), finished into natural, uniform or Briggs weights, and
 * looked up per visibility -- the imaging weight that
 * MSGridderBase::readAndWeightVisibilities multiplies into each visibility
 * weight (gridding/msgridderbase.cpp:583-590,642-659). */
enum { WSG_WEIGHT_NATURAL = 0, WSG_WEIGHT_UNIFORM = 1, WSG_WEIGHT_BRIGGS = 2 };
typedef struct wsg_weights wsg_weights;
/* width, height, pixel scales: of the image; super_weight divides the grid
 * size (rounded, made even); weights_as_taper: grid 1 for every nonzero
 * weight. */
int wsg_weights_create(wsg_ctx *ctx, int mode, double briggs_robust, size_t width, size_t height,
                       double pixel_scale_x, double pixel_scale_y, int weights_as_taper,
                       double super_weight, wsg_weights **out);
int wsg_weights_destroy(wsg_weights *w);
/* Adds nrows x nchan x npol visibility weights (NULL: all ones). */
int wsg_weights_grid(wsg_weights *w, size_t nrows, size_t nchan, size_t npol, const double *uvw,
                     const double *freq, const float *weights);
/* FinishGridding (imageweights.cpp:113-143). */
int wsg_weights_finish(wsg_weights *w);
/* out[k] = in[k] (1 if in is NULL) x imaging weight of the visibility's cell. */
int wsg_weights_apply(wsg_weights *w, size_t nrows, size_t nchan, size_t npol, const double *uvw,
                      const double *freq, const float *in, float *out);
/* The grid (width x height/2 doubles, index x + y*width; NULL to skip), its
 * size and the sum of gridded weights. */
int wsg_weights_get(wsg_weights *w, double *grid, size_t *width, size_t *height, double *total);
/* Folds the imaging weights of w (finished by wsg_weights_finish, on the
 * stream's device) into every later wsg_stream_add: each visibility is
 * gridded with weight x imaging weight of its uv cell -- the product that
 * MSGridderBase::readAndWeightVisibilities forms on the host
 * (gridding/msgridderbase.cpp:583-590,640-659) -- looked up while the
 * device scans the batch and builds its records, so no weighted copy of the
 * weights is made or uploaded; a visibility outside the weight grid is
 * inactive.  The product is rounded to float for float weights, as
 * wsg_weights_apply stores it.  Predictions are not weighted.  w must stay
 * alive while set; NULL turns the lookup off.  Extension of the reference
 * interface. */
int wsg_stream_set_imaging_weights(wsg_stream *s, const wsg_weights *w);

#ifdef __cplusplus
}
#endif

#endif /* WSG_H */
