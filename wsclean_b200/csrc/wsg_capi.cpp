// extern "C" layer of libwsg: maps C++ exceptions to status codes and keeps
// a per-thread error message (the reference throws std::runtime_error from
// MR_assert; the C++ adapter in wsclean_b200/host rethrows from the codes).
#include <cstring>
#include <new>
#include <string>

#include "../../include/wsg.h"
#include "wsg_context.h"

#include <memory>

// A context handle either owns its Context or views the one inside a gridder.
struct wsg_ctx {
  std::unique_ptr<wsg::Context> own;
  wsg::Context *ctx = nullptr;
  int plans = 0;  // live plans on this context (it must outlive them)
};
struct wsg_plan {
  std::unique_ptr<wsg::Plan> impl;
  wsg_ctx *ctx = nullptr;
};
struct wsg_weights {
  std::unique_ptr<wsg::ImageWeightsGpu> impl;
  wsg_ctx *ctx = nullptr;
};
struct wsg_stream {
  std::unique_ptr<wsg::StreamGridder> impl;
  wsg_ctx *ctx = nullptr;
};
struct wsg_gridder {
  wsg::Gridder impl;
  wsg_ctx view;
  explicit wsg_gridder(const wsg_gridder_params &p) : impl(p) { view.ctx = &impl.context(); }
};

namespace {
thread_local std::string g_last_error;

template <typename F>
int guarded(F &&f) {
  try {
    f();
    g_last_error.clear();
    return WSG_OK;
  } catch (const wsg::InvalidArgument &e) {
    g_last_error = e.what();
    return WSG_ERR_INVALID;
  } catch (const wsg::OutOfMemory &e) {
    g_last_error = e.what();
    return WSG_ERR_NOMEM;
  } catch (const std::bad_alloc &e) {
    g_last_error = "host allocation failed";
    return WSG_ERR_NOMEM;
  } catch (const wsg::CufftError &e) {
    g_last_error = e.what();
    return WSG_ERR_CUFFT;
  } catch (const wsg::CudaError &e) {
    g_last_error = e.what();
    return WSG_ERR_CUDA;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return WSG_ERR_INTERNAL;
  }
}
}  // namespace

extern "C" {

int wsg_abi_version(void) { return WSG_ABI_VERSION; }

const char *wsg_last_error(void) { return g_last_error.c_str(); }

void wsg_args_init(wsg_args *a) {
  std::memset(a, 0, sizeof(*a));
  a->wgt_type = WSG_F32;
  a->do_wgridding = 1;
  a->negate_v = 0;
  a->divide_by_n = 1;
  a->sigma_min = 1.1;
  a->sigma_max = 2.6;
  a->precision = WSG_PREC_MIXED;
  a->vis_type = WSG_C64;
  a->dirty_type = WSG_F32;
}

int wsg_ctx_create(int device, wsg_ctx **out) {
  return guarded([&] {
    wsg::require(out != nullptr, "out is NULL");
    auto *h = new wsg_ctx;
    try {
      h->own.reset(new wsg::Context(device));
    } catch (...) {
      delete h;
      throw;
    }
    h->ctx = h->own.get();
    *out = h;
  });
}

int wsg_ctx_destroy(wsg_ctx *ctx) {
  if (ctx && ctx->plans > 0) {
    g_last_error = "destroy the context's plans first";
    return WSG_ERR_STATE;
  }
  return guarded([&] {
    wsg::require(ctx == nullptr || ctx->own != nullptr, "a gridder's context is destroyed with the gridder");
    delete ctx;
  });
}

int wsg_ctx_set_stream(wsg_ctx *ctx, void *stream) {
  return guarded([&] {
    wsg::require(ctx != nullptr, "ctx is NULL");
    ctx->ctx->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->ctx->own_stream;
  });
}

int wsg_ctx_set_async(wsg_ctx *ctx, int async) {
  return guarded([&] {
    wsg::require(ctx != nullptr, "ctx is NULL");
    wsg::require(ctx->own != nullptr, "a gridder's context stays synchronous");
    if (!async && ctx->ctx->async_mode) ctx->ctx->synchronize();
    ctx->ctx->async_mode = async != 0;
  });
}

int wsg_ctx_release_buffers(wsg_ctx *ctx) {
  return guarded([&] {
    wsg::require(ctx != nullptr, "ctx is NULL");
    ctx->ctx->release_buffers();
  });
}

int wsg_ms2dirty(wsg_ctx *ctx, const wsg_args *a, const void *vis, void *dirty, int accumulate) {
  return guarded([&] {
    wsg::require(ctx && a, "ctx and args are required");
    ctx->ctx->ms2dirty(*a, vis, dirty, accumulate);
  });
}

int wsg_dirty2ms(wsg_ctx *ctx, const wsg_args *a, const void *dirty, void *vis) {
  return guarded([&] {
    wsg::require(ctx && a, "ctx and args are required");
    ctx->ctx->dirty2ms(*a, dirty, vis);
  });
}

int wsg_ms2dirty_tuning(wsg_ctx *ctx, const wsg_args *a, const void *vis, void *dirty,
                        int accumulate) {
  return guarded([&] {
    wsg::require(ctx && a, "ctx and args are required");
    ctx->ctx->ms2dirty_tuning(*a, vis, dirty, accumulate);
  });
}

int wsg_dirty2ms_tuning(wsg_ctx *ctx, const wsg_args *a, const void *dirty, void *vis) {
  return guarded([&] {
    wsg::require(ctx && a, "ctx and args are required");
    ctx->ctx->dirty2ms_tuning(*a, dirty, vis);
  });
}

int wsg_get_tuning(const wsg_ctx *ctx, int *nfx, int *nfy, int *icut, double *wcut) {
  return guarded([&] {
    wsg::require(ctx && nfx && nfy && icut && wcut, "NULL argument");
    const wsg::TuningChoice &t = ctx->ctx->last_tuning;
    *nfx = t.nfx;
    *nfy = t.nfy;
    *icut = t.icut;
    *wcut = t.split() ? t.wmin + t.icut * (t.wmax - t.wmin) / wsg::kTuningBins : -1.0;
  });
}

int wsg_tuning_choice(const wsg_args *a, size_t nvis_all, double wmin, double wmax,
                      const uint64_t *hist, int *nfx, int *nfy, int *icut) {
  return guarded([&] {
    wsg::require(a && hist && nfx && nfy && icut, "NULL argument");
    const size_t nx = a->npix_x + (a->npix_x & 1), ny = a->npix_y + (a->npix_y & 1);
    const wsg::TuningChoice t =
        wsg::tuning_choice(nx, ny, a->pixsize_x, a->pixsize_y, a->epsilon, a->do_wgridding != 0,
                           a->center_x, a->center_y, nvis_all, wmin, wmax, hist);
    *nfx = t.nfx;
    *nfy = t.nfy;
    *icut = t.icut;
  });
}

int wsg_get_stats(const wsg_ctx *ctx, wsg_stats *out) {
  return guarded([&] {
    wsg::require(ctx && out, "ctx and out are required");
    *out = ctx->ctx->stats;
  });
}

int wsg_gridder_create(const wsg_gridder_params *p, wsg_gridder **out) {
  return guarded([&] {
    wsg::require(p && out, "params and out are required");
    *out = new wsg_gridder(*p);
  });
}

int wsg_gridder_destroy(wsg_gridder *g) {
  return guarded([&] { delete g; });
}

int wsg_gridder_memory_usage(const wsg_gridder *g, size_t *constant, size_t *per_vis) {
  return guarded([&] {
    wsg::require(g && constant && per_vis, "NULL argument");
    g->impl.memory_usage(*constant, *per_vis);
  });
}

int wsg_gridder_initialize_inversion(wsg_gridder *g) {
  return guarded([&] {
    wsg::require(g, "gridder is NULL");
    g->impl.initialize_inversion();
  });
}

int wsg_gridder_add_inversion_data(wsg_gridder *g, size_t nrows, size_t nchan, const double *uvw,
                                   const double *freq, const void *vis) {
  return guarded([&] {
    wsg::require(g, "gridder is NULL");
    g->impl.add_inversion_data(nrows, nchan, uvw, freq, vis);
  });
}

int wsg_gridder_finalize_image(wsg_gridder *g, double factor) {
  return guarded([&] {
    wsg::require(g, "gridder is NULL");
    g->impl.finalize_image(factor);
  });
}

int wsg_gridder_real_image(wsg_gridder *g, float *image) {
  return guarded([&] {
    wsg::require(g && image, "NULL argument");
    g->impl.real_image(image);
  });
}

int wsg_gridder_initialize_prediction(wsg_gridder *g, const float *image) {
  return guarded([&] {
    wsg::require(g, "gridder is NULL");
    g->impl.initialize_prediction(image);
  });
}

int wsg_gridder_predict_visibilities(wsg_gridder *g, size_t nrows, size_t nchan,
                                     const double *uvw, const double *freq, void *vis) {
  return guarded([&] {
    wsg::require(g && vis, "NULL argument");
    g->impl.predict_visibilities(nrows, nchan, uvw, freq, vis);
  });
}

wsg_ctx *wsg_gridder_ctx(wsg_gridder *g) { return g ? &g->view : nullptr; }

int wsg_ms2dirty_noalloc(const wsg_args *a, const void *vis, void *dirty, void *stream) {
  return guarded([&] {
    wsg::require(a != nullptr, "args are required");
    wsg::ms2dirty_noalloc(*a, vis, dirty, reinterpret_cast<cudaStream_t>(stream));
  });
}

int wsg_plan_grid(const wsg_args *a, size_t nvis, double wmin, double wmax, double umax,
                  double vmax, wsg_stats *out) {
  return guarded([&] {
    wsg::require(a && out, "NULL argument");
    wsg::GridPlan g;
    g.nx = a->npix_x;
    g.ny = a->npix_y;
    g.px = a->pixsize_x;
    g.py = a->pixsize_y;
    g.eps = a->epsilon;
    g.do_w = a->do_wgridding != 0;
    g.fp32 = a->precision != WSG_PREC_FP64;
    g.negate_v = a->negate_v != 0;
    g.divide_by_n = a->divide_by_n != 0;
    g.lshift = a->center_x;
    g.mshift = a->negate_v ? -a->center_y : a->center_y;
    g.nvis = nvis;
    g.wmin_d = wmin;
    g.wmax_d = wmax;
    g.umax = umax;
    g.vmax = vmax;
    wsg::choose_grid(g, a->sigma_min, a->sigma_max, g.fp32 ? 16 : 8);
    std::memset(out, 0, sizeof(*out));
    out->nvis = nvis;
    out->nu = g.nu;
    out->nv = g.nv;
    out->nplanes = g.nplanes;
    out->supp = g.kernel.W;
    out->band_rows = g.band_rows;
    out->degree = g.poly.D;
    out->sigma = g.ofactor;
    out->beta = g.kernel.beta;
    out->e0 = g.kernel.e0;
    out->kernel_err = g.kernel.err;
    out->wmin = wmin;
    out->wmax = wmax;
    out->dw = g.dw;
    out->nshift = g.nshift;
    out->precision = g.fp32 ? WSG_PREC_MIXED : WSG_PREC_FP64;
  });
}

int wsg_plan_create(wsg_ctx *ctx, const wsg_args *a, const wsg_job *jobs, size_t njobs,
                    wsg_plan **out) {
  return guarded([&] {
    wsg::require(ctx != nullptr && a != nullptr && out != nullptr, "ctx, args and out are required");
    auto *h = new wsg_plan;
    try {
      h->impl.reset(new wsg::Plan(*ctx->ctx, *a, jobs, njobs));
    } catch (...) {
      delete h;
      throw;
    }
    h->ctx = ctx;
    ++ctx->plans;
    *out = h;
  });
}

int wsg_plan_destroy(wsg_plan *p) {
  return guarded([&] {
    if (!p) return;
    if (p->ctx) --p->ctx->plans;
    delete p;
  });
}

int wsg_plan_ms2dirty(wsg_plan *p, const void *vis, void *const *dirty, int accumulate) {
  return guarded([&] {
    wsg::require(p != nullptr, "plan is NULL");
    p->impl->ms2dirty(vis, dirty, accumulate);
  });
}

int wsg_plan_dirty2ms(wsg_plan *p, const void *const *dirty, void *vis) {
  return guarded([&] {
    wsg::require(p != nullptr, "plan is NULL");
    p->impl->dirty2ms(dirty, vis);
  });
}

int wsg_plan_get_stats(const wsg_plan *p, size_t job, wsg_stats *out) {
  return guarded([&] {
    wsg::require(p != nullptr && out != nullptr, "plan and out are required");
    p->impl->stats(job, *out);
  });
}

int wsg_ctx_synchronize(wsg_ctx *ctx) {
  return guarded([&] {
    wsg::require(ctx != nullptr, "ctx is NULL");
    ctx->ctx->synchronize();
  });
}

int wsg_stream_create(wsg_ctx *ctx, const wsg_args *a, double wmin, double wmax, double umax,
                      double vmax, size_t nvis, wsg_stream **out) {
  return guarded([&] {
    wsg::require(ctx != nullptr && a != nullptr && out != nullptr, "ctx, args and out are required");
    auto *h = new wsg_stream;
    try {
      h->impl.reset(new wsg::StreamGridder(*ctx->ctx, *a, wmin, wmax, umax, vmax, nvis));
    } catch (...) {
      delete h;
      throw;
    }
    h->ctx = ctx;
    ++ctx->plans;
    *out = h;
  });
}

int wsg_stream_destroy(wsg_stream *s) {
  return guarded([&] {
    if (!s) return;
    if (s->ctx) --s->ctx->plans;
    delete s;
  });
}

int wsg_stream_add(wsg_stream *s, size_t nrows, const double *uvw, const void *vis,
                   const void *wgt, const uint8_t *mask) {
  return guarded([&] {
    wsg::require(s != nullptr, "stream is NULL");
    s->impl->add(nrows, uvw, vis, wgt, mask);
  });
}

int wsg_stream_finish(wsg_stream *s, void *dirty, int accumulate) {
  return guarded([&] {
    wsg::require(s != nullptr, "stream is NULL");
    s->impl->finish(dirty, accumulate);
  });
}

int wsg_stream_predict_begin(wsg_stream *s, const void *dirty) {
  return guarded([&] {
    wsg::require(s != nullptr, "stream is NULL");
    s->impl->predict_begin(dirty);
  });
}

int wsg_stream_predict(wsg_stream *s, size_t nrows, const double *uvw, void *vis,
                       const void *wgt, const uint8_t *mask) {
  return guarded([&] {
    wsg::require(s != nullptr, "stream is NULL");
    s->impl->predict(nrows, uvw, vis, wgt, mask);
  });
}

int wsg_stream_get_stats(const wsg_stream *s, wsg_stats *out) {
  return guarded([&] {
    wsg::require(s != nullptr && out != nullptr, "stream and out are required");
    s->impl->stats(*out);
  });
}

int wsg_weights_create(wsg_ctx *ctx, int mode, double briggs_robust, size_t width, size_t height,
                       double pixel_scale_x, double pixel_scale_y, int weights_as_taper,
                       double super_weight, wsg_weights **out) {
  return guarded([&] {
    wsg::require(ctx != nullptr && out != nullptr, "ctx and out are required");
    auto *h = new wsg_weights;
    try {
      h->impl.reset(new wsg::ImageWeightsGpu(*ctx->ctx, mode, briggs_robust, width, height,
                                             pixel_scale_x, pixel_scale_y, weights_as_taper != 0,
                                             super_weight));
    } catch (...) {
      delete h;
      throw;
    }
    h->ctx = ctx;
    ++ctx->plans;
    *out = h;
  });
}

int wsg_stream_set_imaging_weights(wsg_stream *s, const wsg_weights *w) {
  return guarded([&] {
    wsg::require(s != nullptr, "stream is NULL");
    s->impl->set_imaging_weights(w ? w->impl.get() : nullptr);
  });
}

int wsg_weights_destroy(wsg_weights *w) {
  return guarded([&] {
    if (!w) return;
    if (w->ctx) --w->ctx->plans;
    delete w;
  });
}

int wsg_weights_grid(wsg_weights *w, size_t nrows, size_t nchan, size_t npol, const double *uvw,
                     const double *freq, const float *weights) {
  return guarded([&] {
    wsg::require(w != nullptr, "weights handle is NULL");
    w->impl->grid(nrows, nchan, npol, uvw, freq, weights);
  });
}

int wsg_weights_finish(wsg_weights *w) {
  return guarded([&] {
    wsg::require(w != nullptr, "weights handle is NULL");
    w->impl->finish();
  });
}

int wsg_weights_apply(wsg_weights *w, size_t nrows, size_t nchan, size_t npol, const double *uvw,
                      const double *freq, const float *in, float *out) {
  return guarded([&] {
    wsg::require(w != nullptr, "weights handle is NULL");
    w->impl->apply(nrows, nchan, npol, uvw, freq, in, out);
  });
}

int wsg_weights_get(wsg_weights *w, double *grid, size_t *width, size_t *height, double *total) {
  return guarded([&] {
    wsg::require(w != nullptr, "weights handle is NULL");
    w->impl->get(grid, width, height, total);
  });
}

int wsg_autotune(wsg_ctx *ctx, const wsg_args *a, const void *vis, int candidates,
                 wsg_stats *best) {
  return guarded([&] {
    wsg::require(ctx != nullptr && a != nullptr && best != nullptr, "ctx, args and best are required");
    ctx->ctx->autotune(*a, vis, candidates, *best);
  });
}

}  // extern "C"
