// Streaming chunks into a resident grid (wsg_stream_*).
#include "wsg_host.cuh"

namespace wsg {

// ---------------------------------------- streaming into a resident grid
//
// The whole w-stack stays in HBM between chunks: chunks only scan, sort,
// build records and spread (or interpolate); the FFTs and screens run once
// per image.  Host chunks are staged through two page-locked buffers and a
// copy stream, so the transfer of chunk k+1 proceeds while chunk k is
// sorted and spread.

void *PinnedBuf::ensure(size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (n < bytes) {
    release();
    cuda_check(cudaHostAlloc(&p, bytes, cudaHostAllocDefault), "cudaHostAlloc");
    n = bytes;
  }
  return p;
}

void PinnedBuf::release() {
  if (p) cudaFreeHost(p);
  p = nullptr;
  n = 0;
}

StreamGridder::StreamGridder(Context &cx, const wsg_args &a, double wmin, double wmax,
                             double umax, double vmax, size_t nvis)
    : cx_(cx), a_(a) {
  require(a.freq != nullptr && a.nchan > 0, "freq is required");
  freq_.resize(a.nchan);
  if (is_device_pointer(a.freq))
    CK(cudaMemcpy(freq_.data(), a.freq, a.nchan * sizeof(double), cudaMemcpyDeviceToHost));
  else
    std::memcpy(freq_.data(), a.freq, a.nchan * sizeof(double));
  a_.freq = freq_.data();
  a_.uvw = nullptr;
  a_.wgt = nullptr;
  a_.mask = nullptr;
  wsg_args v = a_;
  v.nrows = 1;  // validate() checks the geometry, not the (absent) rows
  v.uvw = freq_.data();
  cx_.validate(v);
  require(wmin >= 0 && wmax >= wmin && umax > 0 && vmax > 0, "bad data extent");
  dbl_ = a.precision == WSG_PREC_FP64;
  CK(cudaSetDevice(cx_.device));
  GridPlan &g = gp_;
  g.nx = a.npix_x;
  g.ny = a.npix_y;
  g.px = a.pixsize_x;
  g.py = a.pixsize_y;
  g.eps = a.epsilon;
  g.do_w = a.do_wgridding != 0;
  g.fp32 = !dbl_;
  g.negate_v = a.negate_v != 0;
  g.divide_by_n = a.divide_by_n != 0;
  g.lshift = a.center_x;
  g.mshift = a.negate_v ? -a.center_y : a.center_y;
  g.nvis = nvis ? nvis : size_t(1) << 24;
  g.wmin_d = wmin;
  g.wmax_d = wmax;
  g.umax = umax;
  g.vmax = vmax;
  choose_grid(g, a.sigma_min, a.sigma_max, default_tile(!dbl_));
  g.fixed = true;
  const size_t cs = dbl_ ? 16 : 8;
  band_.ensure(g.band_rows * g.nplanes * g.nv * cs);
  img_.ensure(g.nx * g.ny * sizeof(double));
  cc_ = cx_.upload_corrections(g);
  const void *twd = g.ucufft ? nullptr : cx_.upload_twiddles(g, dbl_);
  CK(cudaStreamSynchronize(cx_.stream));  // the uploads are stream-ordered
  const size_t ncf = g.nx / 2 + 1 + g.ny / 2 + 1;
  cf_.ensure(ncf * sizeof(double));
  CK(cudaMemcpy(cf_.p, cx_.cf_cur, ncf * sizeof(double), cudaMemcpyDeviceToDevice));
  if (!g.ucufft) {  // (whole-column transforms use the library FFT, no tables)
    const size_t M = size_t(1) << g.logM;
    const size_t ntw = col_table_entries(M, size_t(g.K)) * cs;
    tw_.ensure(ntw);
    CK(cudaMemcpy(tw_.p, twd, ntw, cudaMemcpyDeviceToDevice));
  }
  CF(cufftCreate(&fft_));
  CF(cufftSetAutoAllocation(fft_, 0));
  int n = int(g.nv), inembed = n, onembed = n;
  size_t work = 0;
  CF(cufftMakePlanMany(fft_, 1, &n, &inembed, 1, n, &onembed, 1, n, dbl_ ? CUFFT_Z2Z : CUFFT_C2C,
                       int(g.band_rows * g.nplanes), &work));
  fftwork_.ensure(std::max<size_t>(work, 256));
  if (!g.ucufft) H_.ensure(plane_batch() * row_plane_bytes());
  CK(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
  for (auto &sl : slots_) {
    CK(cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&sl.vcopied, cudaEventDisableTiming));
  }
  for (auto &b : batch_) {
    CK(cudaEventCreateWithFlags(&b.filled, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&b.spread, cudaEventDisableTiming));
  }
  // a batch holds a third of the expected visibilities (so that the copies
  // of one overlap the spread of another), at least 32M, within 2^31 - 1
  // and with its inputs in at most 1/16 of the device memory
  {
    size_t freeb = 0, total = 0;
    CK(cudaMemGetInfo(&freeb, &total));
    const size_t row_bytes = 24 + a.nchan * ((a.vis_type == WSG_C128 ? 16 : 8) +
                                             (a.wgt_type == WSG_F64 ? 8 : 4) + 1);
    size_t vis = std::max<size_t>(size_t(32) << 20, (nvis ? nvis : 0) / 3);
    vis = std::min(vis, (size_t(1) << 31) - 1);
    size_t rows = vis / a.nchan;
    rows = std::min(rows, (total / 16) / row_bytes);
    batch_rows_ = std::max<size_t>(rows, 1);
  }
  CK(cudaMemsetAsync(band_.p, 0, band_.n, cx_.stream));
  mode_ = 1;
}

StreamGridder::~StreamGridder() {
  cudaSetDevice(cx_.device);
  cudaStreamSynchronize(cx_.stream);
  cudaStreamSynchronize(cx_.d2h);  // pipelined predictions still copying back
  if (copy_) {
    cudaStreamSynchronize(copy_);
    cudaStreamDestroy(copy_);
  }
  for (auto &sl : slots_) {
    if (sl.copied) cudaEventDestroy(sl.copied);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.vcopied) cudaEventDestroy(sl.vcopied);
    for (DevBuf *b : {&sl.uvw, &sl.vis, &sl.wgt, &sl.mask, &sl.vout}) b->release();
    for (PinnedBuf *b : {&sl.h_uvw, &sl.h_vis, &sl.h_wgt, &sl.h_mask}) b->release();
  }
  for (auto &b : batch_) {
    if (b.filled) cudaEventDestroy(b.filled);
    if (b.spread) cudaEventDestroy(b.spread);
    for (DevBuf *d : {&b.uvw, &b.vis, &b.wgt, &b.mask}) d->release();
  }
  if (fft_) cufftDestroy(fft_);
  for (DevBuf *b : {&band_, &H_, &img_, &cf_, &tw_, &fftwork_, &vout_, &lambda_}) b->release();
}

// Bytes of one plane's u-transformed rows: ny segmented rows of hrow
// entries (none with the whole-grid layout, which is screened in place).
size_t StreamGridder::row_plane_bytes() const {
  const size_t cs = dbl_ ? 16 : 8;
  return gp_.ucufft ? 0 : gp_.hrow() * gp_.ny * cs;
}

// Planes per pass of the final transforms (the u-transformed rows of a pass
// are held in H): all of them when they fit in a quarter of the free memory.
size_t StreamGridder::plane_batch() const {
  size_t freeb = 0, total = 0;
  CK(cudaMemGetInfo(&freeb, &total));
  const size_t per = row_plane_bytes();
  size_t P = std::max<size_t>(1, std::min<size_t>(gp_.nplanes, (freeb / 4) / std::max<size_t>(per, 1)));
  const int lim = env_int("WSG_MAX_PLANES", 0);  // a test and debugging limit
  if (lim > 0) P = std::min<size_t>(P, size_t(lim));
  return P;
}

// Stages a chunk: device pointers are used in place; page-locked host
// memory is copied directly on the copy stream; pageable memory goes
// through the slot's page-locked buffer first.  The compute stream waits
// for the copies.
Staged StreamGridder::stage(Slot &sl, size_t nrows, const double *uvw, const void *vis,
                            const void *wgt, const uint8_t *mask) {
  CK(cudaEventSynchronize(sl.done));  // the slot's previous chunk is finished
  const size_t nvis = nrows * a_.nchan;
  auto put = [&](const void *src, size_t bytes, DevBuf &dev, PinnedBuf &pin) -> const void * {
    if (!src) return nullptr;
    cudaPointerAttributes at;
    cudaMemoryType t = cudaMemoryTypeUnregistered;
    if (cudaPointerGetAttributes(&at, src) == cudaSuccess)
      t = at.type;
    else
      cudaGetLastError();
    if (t == cudaMemoryTypeDevice || t == cudaMemoryTypeManaged) return src;
    const void *from = src;
    if (t != cudaMemoryTypeHost) {
      std::memcpy(pin.ensure(bytes), src, bytes);
      from = pin.p;
    }
    void *d = dev.ensure(bytes);
    CK(cudaMemcpyAsync(d, from, bytes, cudaMemcpyHostToDevice, copy_));
    return d;
  };
  Staged s;
  s.uvw = reinterpret_cast<const double *>(put(uvw, nrows * 3 * sizeof(double), sl.uvw, sl.h_uvw));
  if (vis) s.vis = put(vis, nvis * (a_.vis_type == WSG_C128 ? 16 : 8), sl.vis, sl.h_vis);
  s.wgt = put(wgt, nvis * (a_.wgt_type == WSG_F64 ? 8 : 4), sl.wgt, sl.h_wgt);
  s.mask = reinterpret_cast<const uint8_t *>(put(mask, nvis, sl.mask, sl.h_mask));
  CK(cudaEventRecord(sl.copied, copy_));
  CK(cudaStreamWaitEvent(cx_.stream, sl.copied, 0));
  return s;
}

template <typename R>
void StreamGridder::add_t(const Staged &s, size_t nrows) {
  wsg_args ac = a_;
  ac.nrows = nrows;
  ac.uvw = s.uvw;
  ac.wgt = s.wgt;
  ac.mask = s.mask;
  GridPlan g = gp_;
  if (!cx_.prepare<R>(ac, s, true, nullptr, g)) return;
  cudaStream_t st = cx_.stream;
  const TileLayout tl = make_layout(g.T, g.kernel.W);
  const size_t smem = grid_smem_bytes<R>(tl, g.kernel.W, true);
  int *counter = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 2048);
  int *d_nch = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 1024);
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 3072);
  if (!err_armed_) {  // read back and cleared by finish()
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    err_armed_ = true;
  }
  CK(cudaMemsetAsync(counter, 0, sizeof(int), st));
  GridArgs ga{};
  ga.err = d_err;
  ga.rec = cx_.b_rec.p;
  ga.chunk_start = reinterpret_cast<const int *>(cx_.b_chunks.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(g.nvis);
  ga.grid = band_.p;
  ga.P = int(g.nplanes);
  ga.pb0 = 0;
  ga.pb1 = int(g.nplanes);
  ga.tl = tl;
  ga.sb = grid_sb<R>();
  grid_dispatch<R>(g.kernel.W, true, cx_.num_sms, smem, st, ga, make_geom(g),
                           make_kernel<R>(g.poly));
}

// Enqueues a copy of bytes from src (device, page-locked or pageable host
// memory) to the device buffer dst on the copy stream; pageable memory goes
// through the page-locked buffer pin (the caller synchronises the copy
// stream before pin is reused).
void StreamGridder::copy_into(void *dst, const void *src, size_t bytes, PinnedBuf &pin) {
  cudaPointerAttributes at;
  cudaMemoryType t = cudaMemoryTypeUnregistered;
  if (cudaPointerGetAttributes(&at, src) == cudaSuccess)
    t = at.type;
  else
    cudaGetLastError();
  if (t == cudaMemoryTypeDevice || t == cudaMemoryTypeManaged || t == cudaMemoryTypeHost) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, copy_));
    return;
  }
  std::memcpy(pin.ensure(bytes), src, bytes);
  CK(cudaMemcpyAsync(dst, pin.p, bytes, cudaMemcpyHostToDevice, copy_));
}

// WSClean multiplies each visibility's weight by the imaging weight of its
// uv cell before gridding (MSGridderBase::readAndWeightVisibilities,
// gridding/msgridderbase.cpp:583-590,640-659).  Here the lookup happens in
// the scan and record kernels of each batch, from the finished grid of w.
void StreamGridder::set_imaging_weights(const ImageWeightsGpu *w) {
  if (!w) {
    iw_ = ImgW{};
    return;
  }
  require(w->finished(), "the imaging weights must be finished (wsg_weights_finish)");
  require(w->device() == cx_.device, "the imaging weights live on another device");
  flush_batch();  // rows added so far keep the weights they were added with
  std::vector<double> l(freq_.size());
  for (size_t c = 0; c < l.size(); ++c) l[c] = kSpeedOfLight / freq_[c];
  CK(cudaStreamSynchronize(cx_.stream));  // an earlier table may still be read
  double *d = reinterpret_cast<double *>(lambda_.ensure(l.size() * sizeof(double)));
  CK(cudaMemcpy(d, l.data(), l.size() * sizeof(double), cudaMemcpyHostToDevice));
  iw_.grid = w->grid_ptr();
  iw_.lambda = d;
  iw_.g = w->geometry();
}

// Sorts and spreads the current batch (after its copies) and switches to
// the other one.  The batch's scan checks its rows against the declared
// extent (prepare() with the fixed grid); a batch that fails is dropped.
void StreamGridder::flush_batch() {
  Batch &b = batch_[bcur_];
  if (b.rows == 0) return;
  const size_t rows = b.rows;
  b.rows = 0;
  bcur_ ^= 1;
  CK(cudaEventRecord(b.filled, copy_));
  CK(cudaStreamWaitEvent(cx_.stream, b.filled, 0));
  Staged s;
  s.uvw = reinterpret_cast<const double *>(b.uvw.p);
  s.vis = b.vis.p;
  s.wgt = b.has_wgt ? b.wgt.p : nullptr;
  s.mask = b.has_mask ? reinterpret_cast<const uint8_t *>(b.mask.p) : nullptr;
  s.iw = iw_;
  if (dbl_)
    add_t<double>(s, rows);
  else
    add_t<float>(s, rows);
  CK(cudaEventRecord(b.spread, cx_.stream));
}

void StreamGridder::add(size_t nrows, const double *uvw, const void *vis, const void *wgt,
                        const uint8_t *mask) {
  require(uvw && vis, "uvw and vis are required");
  if (nrows == 0) return;
  CK(cudaSetDevice(cx_.device));
  if (mode_ == 2) {  // after prediction (a major cycle's Predict, then Invert)
    CK(cudaMemsetAsync(band_.p, 0, band_.n, cx_.stream));
    for (auto &b : batch_) b.rows = 0;
    mode_ = 1;
  }
  if (nrows > batch_rows_) {  // a chunk larger than a batch is spread alone
    flush_batch();
    Slot &sl = slots_[k_++ & 1];
    Staged s = stage(sl, nrows, uvw, vis, wgt, mask);
    s.iw = iw_;
    if (dbl_)
      add_t<double>(s, nrows);
    else
      add_t<float>(s, nrows);
    CK(cudaEventRecord(sl.done, cx_.stream));
    return;
  }
  Batch *b = &batch_[bcur_];
  if (b->rows > 0 && (b->rows + nrows > batch_rows_ || (wgt != nullptr) != b->has_wgt ||
                      (mask != nullptr) != b->has_mask)) {
    flush_batch();
    b = &batch_[bcur_];
  }
  const size_t nchan = a_.nchan;
  const size_t vsz = a_.vis_type == WSG_C128 ? 16 : 8, wsz = a_.wgt_type == WSG_F64 ? 8 : 4;
  if (b->rows == 0) {  // the batch's previous spread has read its buffers
    CK(cudaEventSynchronize(b->spread));
    b->has_wgt = wgt != nullptr;
    b->has_mask = mask != nullptr;
    b->uvw.ensure(batch_rows_ * 3 * sizeof(double));
    b->vis.ensure(batch_rows_ * nchan * vsz);
    if (b->has_wgt) b->wgt.ensure(batch_rows_ * nchan * wsz);
    if (b->has_mask) b->mask.ensure(batch_rows_ * nchan);
  }
  // the caller's buffers are free again when add() returns: the copies
  // (not the spread of an earlier batch, which runs meanwhile) are waited for
  Slot &sl = slots_[0];
  const size_t r0 = b->rows;
  copy_into(static_cast<char *>(b->uvw.p) + r0 * 3 * sizeof(double), uvw, nrows * 3 * sizeof(double),
            sl.h_uvw);
  copy_into(static_cast<char *>(b->vis.p) + r0 * nchan * vsz, vis, nrows * nchan * vsz, sl.h_vis);
  if (wgt)
    copy_into(static_cast<char *>(b->wgt.p) + r0 * nchan * wsz, wgt, nrows * nchan * wsz, sl.h_wgt);
  if (mask) copy_into(static_cast<char *>(b->mask.p) + r0 * nchan, mask, nrows * nchan, sl.h_mask);
  CK(cudaStreamSynchronize(copy_));
  b->rows += nrows;
}

template <typename R>
void StreamGridder::finish_t(void *dirty, int accumulate) {
  const GridPlan &g = gp_;
  cudaStream_t st = cx_.stream;
  const size_t cs = 2 * sizeof(R), npix = g.nx * g.ny;
  double *img = reinterpret_cast<double *>(img_.p);
  const bool ddev = is_device_pointer(dirty);
  const size_t dsz = a_.dirty_type == WSG_F64 ? 8 : 4;
  const int nb = launch_blocks(npix, 256);
  if (accumulate) {
    const void *din = ddev ? dirty : cx_.stage_in(dirty, npix * dsz, cx_.b_out);
    if (a_.dirty_type == WSG_F64)
      k_load_image<double><<<nb, 256, 0, st>>>(npix, (const double *)din, img, 0);
    else
      k_load_image<float><<<nb, 256, 0, st>>>(npix, (const float *)din, img, 0);
    cuda_check(cudaGetLastError(), "k_load_image launch");
  } else {
    CK(cudaMemsetAsync(img, 0, npix * sizeof(double), st));
  }
  if (g.ucufft) {
    // the whole grid: each plane's 2-D transform in place, screened in place
    cx_.grid_fft(band_.p, g, g.nplanes, g.nplanes, CUFFT_INVERSE, sizeof(R) == 8);
  } else {
    CF(cufftSetStream(fft_, st));
    CF(cufftSetWorkArea(fft_, fftwork_.p));
    if (sizeof(R) == 8)
      CF(cufftExecZ2Z(fft_, reinterpret_cast<cufftDoubleComplex *>(band_.p),
                      reinterpret_cast<cufftDoubleComplex *>(band_.p), CUFFT_INVERSE));
    else
      CF(cufftExecC2C(fft_, reinterpret_cast<cufftComplex *>(band_.p),
                      reinterpret_cast<cufftComplex *>(band_.p), CUFFT_INVERSE));
  }
  // planes per pass: as many planes of u-transformed rows as H holds (all of
  // them with the whole-grid layout)
  const size_t P = g.ucufft ? g.nplanes : std::max<size_t>(1, H_.n / row_plane_bytes());
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 3072);
  if (!err_armed_) {
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    err_armed_ = true;
  }
  for (size_t p0 = 0; p0 < g.nplanes; p0 += P) {
    const size_t np = std::min(P, g.nplanes - p0);
    // the band layout is [row][plane][nv]: a pass starts p0 planes into each row
    char *band_p0 = static_cast<char *>(band_.p) + p0 * g.nv * cs;
    ScreenArgs sa = make_screen(g, reinterpret_cast<const double *>(cf_.p), cc_, g.nplanes);
    sa.pb0 = int(p0);
    sa.npl = int(np);
    const dim3 sg = screen_grid(g);
    if (g.ucufft) {
      launch_screen_add_grid<R>(sg, st, sa, band_p0, img, nullptr, 0);
    } else {
      ColArgs ca = make_col(g, g.nplanes, tw_.p, band_p0, H_.p);
      col_run<R>(g.logM, true, ca, int(np), st, d_err);
      launch_screen_add<R>(sg, st, sa, H_.p, img, nullptr, 0);
    }
  }
  void *dout = ddev ? dirty : cx_.b_out.ensure(npix * dsz);
  if (a_.dirty_type == WSG_F64)
    k_store_image<double><<<nb, 256, 0, st>>>(npix, img, (double *)dout);
  else
    k_store_image<float><<<nb, 256, 0, st>>>(npix, img, (float *)dout);
  cuda_check(cudaGetLastError(), "k_store_image launch");
  if (!ddev) CK(cudaMemcpyAsync(dirty, dout, npix * dsz, cudaMemcpyDeviceToHost, st));
  CK(cudaMemsetAsync(band_.p, 0, band_.n, st));
  err_armed_ = false;
  cx_.check_device_error(d_err);  // synchronises the stream
}

void StreamGridder::finish(void *dirty, int accumulate) {
  require(mode_ == 1, "finish() without a gridding stream");
  require(dirty != nullptr, "dirty is required");
  CK(cudaSetDevice(cx_.device));
  flush_batch();
  if (dbl_)
    finish_t<double>(dirty, accumulate);
  else
    finish_t<float>(dirty, accumulate);
}

template <typename R>
void StreamGridder::predict_begin_t(const double *img) {
  const GridPlan &g = gp_;
  cudaStream_t st = cx_.stream;
  const size_t cs = 2 * sizeof(R);
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.ensure(4096)) + 3072);
  CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  CK(cudaMemsetAsync(band_.p, 0, band_.n, st));
  if (g.ucufft) {
    // the whole grid (zero outside the image, as cleared above): screened
    // in place, then each plane's 2-D transform in place
    ScreenArgs sa = make_screen(g, reinterpret_cast<const double *>(cf_.p), cc_, g.nplanes);
    sa.pb0 = 0;
    sa.npl = int(g.nplanes);
    launch_screen_put_grid<R>(screen_grid(g), st, sa, img, 0, band_.p);
    cx_.grid_fft(band_.p, g, g.nplanes, g.nplanes, CUFFT_FORWARD, sizeof(R) == 8);
    cx_.check_device_error(d_err);
    return;
  }
  // planes per pass: as many planes of u-transformed rows as H holds
  const size_t P = std::max<size_t>(1, H_.n / row_plane_bytes());
  for (size_t p0 = 0; p0 < g.nplanes; p0 += P) {
    const size_t np = std::min(P, g.nplanes - p0);
    ScreenArgs sa = make_screen(g, reinterpret_cast<const double *>(cf_.p), cc_, np);
    sa.pb0 = int(p0);
    sa.npl = int(np);
    const dim3 sg = screen_grid(g);
    launch_screen_put<R>(sg, st, sa, img, 0, H_.p);
    ColArgs ca = make_col(g, g.nplanes, tw_.p, static_cast<char *>(band_.p) + p0 * g.nv * cs, H_.p);
    col_run<R>(g.logM, false, ca, int(np), st, d_err);  // (the staged forms report on d_err)
  }
  CF(cufftSetStream(fft_, st));
  CF(cufftSetWorkArea(fft_, fftwork_.p));
  if (sizeof(R) == 8)
    CF(cufftExecZ2Z(fft_, reinterpret_cast<cufftDoubleComplex *>(band_.p),
                    reinterpret_cast<cufftDoubleComplex *>(band_.p), CUFFT_FORWARD));
  else
    CF(cufftExecC2C(fft_, reinterpret_cast<cufftComplex *>(band_.p),
                    reinterpret_cast<cufftComplex *>(band_.p), CUFFT_FORWARD));
  // a staged copy of the u transform that did not complete (once per model;
  // synchronises the stream)
  cx_.check_device_error(d_err);
}

void StreamGridder::predict_begin(const void *dirty) {
  require(dirty != nullptr, "dirty is required");
  CK(cudaSetDevice(cx_.device));
  for (auto &b : batch_) b.rows = 0;  // rows added since the last finish are discarded
  const size_t npix = gp_.nx * gp_.ny, dsz = a_.dirty_type == WSG_F64 ? 8 : 4;
  const void *din = cx_.stage_in(dirty, npix * dsz, cx_.b_out);
  double *img = reinterpret_cast<double *>(img_.p);
  const int nb = launch_blocks(npix, 256);
  if (a_.dirty_type == WSG_F64)
    k_load_image<double><<<nb, 256, 0, cx_.stream>>>(npix, (const double *)din, img, 0);
  else
    k_load_image<float><<<nb, 256, 0, cx_.stream>>>(npix, (const float *)din, img, 0);
  cuda_check(cudaGetLastError(), "k_load_image launch");
  if (dbl_)
    predict_begin_t<double>(img);
  else
    predict_begin_t<float>(img);
  mode_ = 2;
}

template <typename R>
void StreamGridder::predict_t(const Staged &s, size_t nrows, void *vis_dev) {
  wsg_args ac = a_;
  ac.nrows = nrows;
  ac.uvw = s.uvw;
  ac.wgt = s.wgt;
  ac.mask = s.mask;
  GridPlan g = gp_;
  if (!cx_.prepare<R>(ac, s, false, vis_dev, g)) return;
  cudaStream_t st = cx_.stream;
  const size_t cs = 2 * sizeof(R);
  const TileLayout tl = make_layout(g.T, g.kernel.W);
  const size_t smem = grid_smem_bytes<R>(tl, g.kernel.W, false);
  int *counter = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 2048);
  int *d_nch = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 1024);
  int *d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(cx_.b_small.p) + 3072);
  CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  CK(cudaMemsetAsync(counter, 0, sizeof(int), st));
  GridArgs ga{};
  ga.err = d_err;
  ga.rec = cx_.b_rec.p;
  ga.chunk_start = reinterpret_cast<const int *>(cx_.b_chunks.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(g.nvis);
  ga.grid = band_.p;
  ga.P = int(g.nplanes);
  ga.pb0 = 0;
  ga.pb1 = int(g.nplanes);
  ga.tl = tl;
  ga.sb = grid_sb<R>();
  ga.vis_out = vis_dev;
  ga.vis_double = a_.vis_type == WSG_C128;
  ga.first_pass = ga.last_pass = 1;
  const bool need_acc = grid_needs_acc<R>(g.kernel.W);
  ga.acc = need_acc ? cx_.b_acc.ensure(g.nvis * cs) : nullptr;
  if (need_acc) CK(cudaMemsetAsync(ga.acc, 0, g.nvis * cs, st));
  grid_dispatch<R>(g.kernel.W, false, cx_.num_sms, smem, st, ga, make_geom(g),
                           make_kernel<R>(g.poly));
  if (need_acc) {
    k_finalize<R><<<launch_blocks(g.nvis, 256), 256, 0, st>>>(int(g.nvis), cx_.b_rec.p, ga.acc,
                                                             vis_dev, ga.vis_double, 0);
    cuda_check(cudaGetLastError(), "k_finalize launch");
  }
}

void StreamGridder::predict(size_t nrows, const double *uvw, void *vis, const void *wgt,
                            const uint8_t *mask) {
  require(mode_ == 2, "predict() before predict_begin()");
  require(uvw && vis, "uvw and vis are required");
  if (nrows == 0) return;
  CK(cudaSetDevice(cx_.device));
  Slot &sl = slots_[k_++ & 1];
  Staged s = stage(sl, nrows, uvw, nullptr, wgt, mask);
  const size_t vbytes = nrows * a_.nchan * (a_.vis_type == WSG_C128 ? 16 : 8);
  const bool vdev = is_device_pointer(vis);
  // pipelined (wsg_ctx_set_async) into page-locked host memory: the chunk is
  // predicted into the slot's own device buffer and copied back on the
  // context's read-back stream while the next chunk is computed; the caller
  // finds vis in place after wsg_ctx_synchronize
  bool pinned = false;
  if (!vdev && cx_.async_mode) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, vis) == cudaSuccess)
      pinned = at.type == cudaMemoryTypeHost;
    else
      cudaGetLastError();
  }
  void *vout = vdev ? vis : pinned ? sl.vout.ensure(vbytes) : vout_.ensure(vbytes);
  if (pinned) CK(cudaStreamWaitEvent(cx_.stream, sl.vcopied, 0));  // the slot's last copy is out
  CK(cudaMemsetAsync(vout, 0, vbytes, cx_.stream));
  if (dbl_)
    predict_t<double>(s, nrows, vout);
  else
    predict_t<float>(s, nrows, vout);
  CK(cudaEventRecord(sl.done, cx_.stream));
  if (pinned) {
    CK(cudaStreamWaitEvent(cx_.d2h, sl.done, 0));
    CK(cudaMemcpyAsync(vis, vout, vbytes, cudaMemcpyDeviceToHost, cx_.d2h));
    CK(cudaEventRecord(sl.vcopied, cx_.d2h));
  } else if (!vdev) {
    CK(cudaMemcpyAsync(vis, vout, vbytes, cudaMemcpyDeviceToHost, cx_.stream));
    CK(cudaStreamSynchronize(cx_.stream));
  }
}

void StreamGridder::stats(wsg_stats &o) const {
  const GridPlan &g = gp_;
  std::memset(&o, 0, sizeof(o));
  o.nchan = a_.nchan;
  o.nu = g.nu;
  o.nv = g.nv;
  o.nplanes = g.nplanes;
  o.supp = g.kernel.W;
  o.plane_batch = g.nplanes;
  o.band_rows = g.band_rows;
  o.degree = g.poly.D;
  o.sigma = g.ofactor;
  o.beta = g.kernel.beta;
  o.e0 = g.kernel.e0;
  o.kernel_err = g.kernel.err;
  o.wmin = g.wmin_d;
  o.wmax = g.wmax_d;
  o.dw = g.dw;
  o.nshift = g.nshift;
  o.precision = g.fp32 ? WSG_PREC_MIXED : WSG_PREC_FP64;
  o.device_bytes = band_.n + H_.n + img_.n + fftwork_.n;
  o.kernel_launches = g_kernel_launches.load();
}

}  // namespace wsg
