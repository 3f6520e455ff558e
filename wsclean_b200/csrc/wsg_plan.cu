// Reusable plans: batched jobs (facets x output channels) over one record set.
#include "wsg_host.cuh"

namespace wsg {

// ------------------------------------------------- reusable plans, batches
//
// A plan runs prepare() (scan, keys, sort, records) once per job with the
// degridding active set and records (static factor = weight x conjugate
// shift phasor, conjugation bit), copies each job's records and chunk list
// into one concatenated array, and keeps every job's band grid resident.
// Execution is then one persistent spread (or interpolation) launch over
// all chunks of all jobs, the job of a chunk selecting its grid, followed by
// each job's v-FFT, pruned u-transform and w-screen.  Nothing on the
// execution path allocates or synchronises with the host.

Plan::Plan(Context &cx, const wsg_args &a, const wsg_job *jobs, size_t njobs) : cx_(cx), a_(a) {
  cx_.validate(a);
  require(a.nrows * a.nchan < (size_t(1) << 31), "plans index at most 2^31 - 1 visibilities");
  std::vector<wsg_job> js;
  if (jobs == nullptr || njobs == 0) {
    wsg_job j{};
    j.npix_x = a.npix_x;
    j.npix_y = a.npix_y;
    j.center_x = a.center_x;
    j.center_y = a.center_y;
    j.chan_begin = 0;
    j.chan_end = a.nchan;
    js.push_back(j);
  } else {
    js.assign(jobs, jobs + njobs);
  }
  for (const auto &j : js) {
    require(j.npix_x % 2 == 0 && j.npix_y % 2 == 0, "job image sizes must be even");
    require(j.npix_x >= 16 && j.npix_y >= 16, "job images must be at least 16 x 16");
    require(j.chan_begin < j.chan_end && j.chan_end <= a.nchan, "job channel range out of bounds");
  }
  dbl_ = a.precision == WSG_PREC_FP64;
  use_graphs_ = env_int("WSG_PLAN_GRAPHS", 1) != 0;
  CK(cudaSetDevice(cx_.device));
  if (dbl_)
    build<double>(js);
  else
    build<float>(js);
  // registered once built: a plan whose construction failed is never checked
  cx_.plan_err.push_back(reinterpret_cast<int *>(small_.p) + 2);
}

Plan::~Plan() {
  cudaSetDevice(cx_.device);
  cudaStreamSynchronize(cx_.stream);
  auto &pe = cx_.plan_err;
  pe.erase(std::remove(pe.begin(), pe.end(), reinterpret_cast<int *>(small_.p) + 2), pe.end());
  for (auto &g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (auto &j : jobs_)
    for (cufftHandle h : {j.fft, j.gfft})
      if (h) cufftDestroy(h);
  for (DevBuf *b : {&rec_, &chunks_, &chunk_job_, &jobgeom_, &band_, &H_, &img_, &cf_, &tw_, &acc_,
                    &small_, &fftwork_})
    b->release();
}

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
}  // namespace

template <typename R>
void Plan::build(const std::vector<wsg_job> &js) {
  using Rec = typename RecOf<R>::type;
  const size_t cs = 2 * sizeof(R);
  const size_t nchan = a_.nchan, nrows = a_.nrows;
  cudaStream_t st = cx_.stream;
  const int tile = default_tile(sizeof(R) == 4);

  // coordinates on the device (kept only while building)
  Staged s;
  s.uvw = reinterpret_cast<const double *>(cx_.stage_in(a_.uvw, nrows * 3 * sizeof(double), cx_.b_uvw));
  const size_t wsz = a_.wgt_type == WSG_F64 ? 8 : 4;
  const void *wgt_all = cx_.stage_in(a_.wgt, nrows * nchan * wsz, cx_.b_wgt);
  const uint8_t *mask_all =
      reinterpret_cast<const uint8_t *>(cx_.stage_in(a_.mask, nrows * nchan, cx_.b_mask));
  std::vector<double> freq(nchan);
  if (is_device_pointer(a_.freq))
    CK(cudaMemcpy(freq.data(), a_.freq, nchan * sizeof(double), cudaMemcpyDeviceToHost));
  else
    std::memcpy(freq.data(), a_.freq, nchan * sizeof(double));

  // the shared kernel: the one chosen for the largest job with active data
  size_t big = 0;
  for (size_t j = 1; j < js.size(); ++j)
    if (js[j].npix_x * js[j].npix_y > js[big].npix_x * js[big].npix_y) big = j;
  std::vector<size_t> order{big};
  for (size_t j = 0; j < js.size(); ++j)
    if (j != big) order.push_back(j);

  size_t cap = 0;
  for (const auto &j : js) cap += nrows * (j.chan_end - j.chan_begin);
  rec_.ensure(std::max<size_t>(cap, 1) * sizeof(Rec));
  chunks_.ensure((std::max<size_t>(cap, 1) + 1) * sizeof(int));
  chunk_job_.ensure((std::max<size_t>(cap, 1) + 1) * sizeof(int));
  small_.ensure(4096);
  CK(cudaMemsetAsync(small_.p, 0, 4096, cx_.stream));
  DevBuf wsub, msub;
  jobs_.assign(js.size(), PlanJob{});
  int forceW = 0;
  double forceS = 0;
  std::vector<double> cf_host;
  std::vector<char> tw_host;
  for (size_t oi = 0; oi < order.size(); ++oi) {
    const size_t j = order[oi];
    const wsg_job &jd = js[j];
    PlanJob &pj = jobs_[j];
    pj.chan0 = jd.chan_begin;
    pj.chan1 = jd.chan_end;
    const size_t nch = jd.chan_end - jd.chan_begin;
    wsg_args aj = a_;
    aj.nchan = nch;
    aj.freq = freq.data() + jd.chan_begin;
    aj.npix_x = jd.npix_x;
    aj.npix_y = jd.npix_y;
    aj.center_x = jd.center_x;
    aj.center_y = jd.center_y;
    Staged sj = s;
    // the job's channel columns of weights and mask, compacted
    if (a_.wgt) {
      void *d = wsub.ensure(nrows * nch * wsz);
      CK(cudaMemcpy2DAsync(d, nch * wsz, static_cast<const char *>(wgt_all) + jd.chan_begin * wsz,
                           nchan * wsz, nch * wsz, nrows, cudaMemcpyDeviceToDevice, st));
      sj.wgt = d;
      aj.wgt = d;
    }
    if (a_.mask) {
      void *d = msub.ensure(nrows * nch);
      CK(cudaMemcpy2DAsync(d, nch, mask_all + jd.chan_begin, nchan, nch, nrows,
                           cudaMemcpyDeviceToDevice, st));
      sj.mask = reinterpret_cast<const uint8_t *>(d);
      aj.mask = reinterpret_cast<const uint8_t *>(d);
    }
    GridPlan &gp = pj.gp;
    gp.nx = jd.npix_x;
    gp.ny = jd.npix_y;
    gp.px = a_.pixsize_x;
    gp.py = a_.pixsize_y;
    gp.eps = a_.epsilon;
    gp.do_w = a_.do_wgridding != 0;
    gp.fp32 = sizeof(R) == 4;
    gp.gridding = false;
    gp.negate_v = a_.negate_v != 0;
    gp.divide_by_n = a_.divide_by_n != 0;
    gp.lshift = jd.center_x;
    gp.mshift = a_.negate_v ? -jd.center_y : jd.center_y;
    gp.force_W = forceW;
    gp.force_sigma = forceS;
    const bool any = cx_.prepare<R>(aj, sj, false, nullptr, gp);
    if (forceW == 0 && any) {  // the largest job with active visibilities
      forceW = gp.kernel.W;
      forceS = gp.kernel.sigma;
      DevKernel<R> kc = make_kernel<R>(gp.poly);
      kernel_.resize(sizeof(kc));
      std::memcpy(kernel_.data(), &kc, sizeof(kc));
      DevGeom g0 = make_geom(gp);
      geom_.resize(sizeof(g0));
      std::memcpy(geom_.data(), &g0, sizeof(g0));
      W_ = gp.kernel.W;
      T_ = gp.T;
    }
    if (!any) continue;
    require(gp.T == T_ && gp.kernel.W == W_, "internal: jobs must share kernel and tile");
    pj.nrec = gp.nvis;
    int nch_j = 0;
    CK(cudaMemcpyAsync(&nch_j, reinterpret_cast<char *>(cx_.b_small.p) + 1024, sizeof(int),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    pj.rec_off = nrec_;
    CK(cudaMemcpyAsync(static_cast<char *>(rec_.p) + nrec_ * sizeof(Rec), cx_.b_rec.p,
                       pj.nrec * sizeof(Rec), cudaMemcpyDeviceToDevice, st));
    Rec *rj = reinterpret_cast<Rec *>(rec_.p) + nrec_;
    k_plan_remap<Rec><<<launch_blocks(pj.nrec, 256), 256, 0, st>>>(
        pj.nrec, rj, uint32_t(nch), uint32_t(nchan), uint32_t(jd.chan_begin));
    cuda_check(cudaGetLastError(), "k_plan_remap launch");
    k_plan_chunks<<<launch_blocks(size_t(nch_j), 256), 256, 0, st>>>(
        nch_j, reinterpret_cast<const int *>(cx_.b_chunks.p),
        reinterpret_cast<int *>(chunks_.p) + nchunks_, reinterpret_cast<int *>(chunk_job_.p) + nchunks_,
        int(nrec_), int(j));
    cuda_check(cudaGetLastError(), "k_plan_chunks launch");
    g_kernel_launches.fetch_add(2, std::memory_order_relaxed);
    nrec_ += pj.nrec;
    nchunks_ += nch_j;
    // corrections and twiddles of this grid
    pj.cc = cx_.upload_corrections(gp);
    const void *twd = gp.ucufft ? nullptr : cx_.upload_twiddles(gp, sizeof(R) == 8);
    CK(cudaStreamSynchronize(st));  // the uploads are stream-ordered
    const size_t ncf = gp.nx / 2 + 1 + gp.ny / 2 + 1;
    pj.cf_off = cf_host.size();
    cf_host.resize(cf_host.size() + ncf);
    CK(cudaMemcpy(cf_host.data() + pj.cf_off, cx_.cf_cur, ncf * sizeof(double),
                  cudaMemcpyDeviceToHost));
    if (!gp.ucufft) {  // (whole-column transforms use the library FFT, no tables)
      const size_t M = size_t(1) << gp.logM;
      const size_t ntw = col_table_entries(M, size_t(gp.K)) * cs;
      pj.tw_off = tw_host.size();
      tw_host.resize(align256(tw_host.size() + ntw));
      CK(cudaMemcpy(tw_host.data() + pj.tw_off, twd, ntw, cudaMemcpyDeviceToHost));
    }
    // the job's band grid with all its planes, and its v-FFT plan
    pj.band_bytes = gp.band_rows * gp.nplanes * gp.nv * cs;
    pj.band_off = band_total_;
    band_total_ = align256(band_total_ + pj.band_bytes);
    max_npix_ = std::max(max_npix_, gp.nx * gp.ny);
  }
  require(nrec_ > 0, "no active visibilities in any job");
  CK(cudaMemcpyAsync(small_.p, &nchunks_, sizeof(int), cudaMemcpyHostToDevice, st));

  size_t hmax = 0, work = 0;
  std::vector<JobGeom> jg(jobs_.size());
  band_.ensure(band_total_);
  for (size_t j = 0; j < jobs_.size(); ++j) {
    PlanJob &pj = jobs_[j];
    if (pj.nrec == 0) continue;
    const GridPlan &gp = pj.gp;
    if (!gp.ucufft) hmax = std::max(hmax, gp.nplanes * gp.ny * gp.hrow() * cs);
    JobGeom &g = jg[j];
    g.nu = int(gp.nu);
    g.nv = int(gp.nv);
    g.Lu = int(gp.Lu);
    g.band_rows = int(gp.band_rows);
    g.band_full = gp.band_full;
    g.P = int(gp.nplanes);
    g.pb0 = 0;
    g.pb1 = int(gp.nplanes);
    g.grid = static_cast<char *>(band_.p) + pj.band_off;
    size_t w = 0;
    if (gp.ucufft) {  // the whole grid: each plane's 2-D transform in place
      pj.gfft = make_grid_fft_plan(gp.nu, gp.nv, gp.nplanes, sizeof(R) == 8, w);
    } else {
      CF(cufftCreate(&pj.fft));
      CF(cufftSetAutoAllocation(pj.fft, 0));
      int n = int(gp.nv), inembed = n, onembed = n;
      CF(cufftMakePlanMany(pj.fft, 1, &n, &inembed, 1, n, &onembed, 1, n,
                           sizeof(R) == 8 ? CUFFT_Z2Z : CUFFT_C2C, int(gp.band_rows * gp.nplanes),
                           &w));
    }
    work = std::max(work, w);
  }
  H_.ensure(hmax);
  img_.ensure(max_npix_ * sizeof(double));
  fftwork_.ensure(std::max<size_t>(work, 256));
  jobgeom_.ensure(jg.size() * sizeof(JobGeom));
  CK(cudaMemcpyAsync(jobgeom_.p, jg.data(), jg.size() * sizeof(JobGeom), cudaMemcpyHostToDevice, st));
  cf_.ensure(std::max<size_t>(cf_host.size(), 1) * sizeof(double));
  CK(cudaMemcpyAsync(cf_.p, cf_host.data(), cf_host.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  tw_.ensure(std::max<size_t>(tw_host.size(), 1));
  CK(cudaMemcpyAsync(tw_.p, tw_host.data(), tw_host.size(), cudaMemcpyHostToDevice, st));
  need_acc_ = grid_needs_acc<R>(W_);
  if (need_acc_) acc_.ensure(nrec_ * cs);
  CK(cudaStreamSynchronize(st));
}

template <typename R>
void Plan::enqueue_grid(const void *vis, void *const *dirty, int accumulate) {
  const size_t cs = 2 * sizeof(R);
  cudaStream_t st = cx_.stream;
  int *d_nch = reinterpret_cast<int *>(small_.p);
  int *counter = d_nch + 1;
  int *d_err = d_nch + 2;
  CK(cudaMemsetAsync(band_.p, 0, band_total_, st));
  CK(cudaMemsetAsync(counter, 0, sizeof(int), st));  // (the error word stays until read)
  const TileLayout tl = make_layout(T_, W_);
  const size_t smem = grid_smem_bytes<R>(tl, W_, true);
  GridArgs ga{};
  ga.rec = rec_.p;
  ga.chunk_start = reinterpret_cast<const int *>(chunks_.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(nrec_);
  ga.tl = tl;
  ga.sb = grid_sb<R>();
  ga.err = d_err;
  ga.jobs = reinterpret_cast<const JobGeom *>(jobgeom_.p);
  ga.chunk_job = reinterpret_cast<const int *>(chunk_job_.p);
  ga.vis_in = vis;
  ga.vis_in_double = a_.vis_type == WSG_C128;
  DevKernel<R> kc;
  std::memcpy(&kc, kernel_.data(), sizeof(kc));
  DevGeom g0;
  std::memcpy(&g0, geom_.data(), sizeof(g0));
  grid_dispatch<R>(W_, true, cx_.num_sms, smem, st, ga, g0, kc);
  for (size_t j = 0; j < jobs_.size(); ++j) {
    const PlanJob &pj = jobs_[j];
    const GridPlan &gp = pj.gp;
    const size_t npix = gp.nx * gp.ny;
    double *img = reinterpret_cast<double *>(img_.p);
    const int nb = launch_blocks(npix, 256);
    if (pj.nrec == 0) {
      if (!accumulate)
        CK(cudaMemsetAsync(dirty[j], 0, npix * (a_.dirty_type == WSG_F64 ? 8 : 4), st));
      continue;
    }
    char *band = static_cast<char *>(band_.p) + pj.band_off;
    if (gp.ucufft) {
      exec_grid_fft(pj.gfft, band, gp.nv, gp.nplanes, CUFFT_INVERSE, sizeof(R) == 8, st,
                    fftwork_.p);
    } else {
      CF(cufftSetStream(pj.fft, st));
      CF(cufftSetWorkArea(pj.fft, fftwork_.p));
      if (sizeof(R) == 8)
        CF(cufftExecZ2Z(pj.fft, reinterpret_cast<cufftDoubleComplex *>(band),
                        reinterpret_cast<cufftDoubleComplex *>(band), CUFFT_INVERSE));
      else
        CF(cufftExecC2C(pj.fft, reinterpret_cast<cufftComplex *>(band),
                        reinterpret_cast<cufftComplex *>(band), CUFFT_INVERSE));
      ColArgs ca = make_col(gp, gp.nplanes, static_cast<char *>(tw_.p) + pj.tw_off, band, H_.p);
      col_run<R>(gp.logM, true, ca, int(gp.nplanes), st, d_err);
    }
    if (accumulate) {
      if (a_.dirty_type == WSG_F64)
        k_load_image<double><<<nb, 256, 0, st>>>(npix, (const double *)dirty[j], img, 0);
      else
        k_load_image<float><<<nb, 256, 0, st>>>(npix, (const float *)dirty[j], img, 0);
      cuda_check(cudaGetLastError(), "k_load_image launch");
    } else {
      CK(cudaMemsetAsync(img, 0, npix * sizeof(double), st));
    }
    ScreenArgs sa = make_screen(gp, reinterpret_cast<const double *>(cf_.p) + pj.cf_off, pj.cc,
                                gp.nplanes);
    sa.pb0 = 0;
    sa.npl = int(gp.nplanes);
    const dim3 sg = screen_grid(gp);
    if (gp.ucufft)
      launch_screen_add_grid<R>(sg, st, sa, band, img, nullptr, 0);
    else
      launch_screen_add<R>(sg, st, sa, H_.p, img, nullptr, 0);
    if (a_.dirty_type == WSG_F64)
      k_store_image<double><<<nb, 256, 0, st>>>(npix, img, (double *)dirty[j]);
    else
      k_store_image<float><<<nb, 256, 0, st>>>(npix, img, (float *)dirty[j]);
    cuda_check(cudaGetLastError(), "k_store_image launch");
    g_kernel_launches.fetch_add(accumulate ? 3 : 2, std::memory_order_relaxed);
  }
  (void)cs;
}

template <typename R>
void Plan::enqueue_degrid(const void *const *dirty, void *vis) {
  const size_t cs = 2 * sizeof(R);
  cudaStream_t st = cx_.stream;
  int *d_nch = reinterpret_cast<int *>(small_.p);
  int *counter = d_nch + 1;
  int *d_err = d_nch + 2;
  const size_t vsz = a_.vis_type == WSG_C128 ? 16 : 8;
  const bool multi = jobs_.size() > 1;
  CK(cudaMemsetAsync(vis, 0, a_.nrows * a_.nchan * vsz, st));
  for (size_t j = 0; j < jobs_.size(); ++j) {
    const PlanJob &pj = jobs_[j];
    if (pj.nrec == 0) continue;
    const GridPlan &gp = pj.gp;
    const size_t npix = gp.nx * gp.ny;
    double *img = reinterpret_cast<double *>(img_.p);
    const int nb = launch_blocks(npix, 256);
    if (a_.dirty_type == WSG_F64)
      k_load_image<double><<<nb, 256, 0, st>>>(npix, (const double *)dirty[j], img, 0);
    else
      k_load_image<float><<<nb, 256, 0, st>>>(npix, (const float *)dirty[j], img, 0);
    cuda_check(cudaGetLastError(), "k_load_image launch");
    ScreenArgs sa = make_screen(gp, reinterpret_cast<const double *>(cf_.p) + pj.cf_off, pj.cc,
                                gp.nplanes);
    sa.pb0 = 0;
    sa.npl = int(gp.nplanes);
    const dim3 sg = screen_grid(gp);
    char *band = static_cast<char *>(band_.p) + pj.band_off;
    if (gp.ucufft) {
      // the whole grid, zero outside the image, screened and transformed in place
      CK(cudaMemsetAsync(band, 0, pj.band_bytes, st));
      launch_screen_put_grid<R>(sg, st, sa, img, 0, band);
      exec_grid_fft(pj.gfft, band, gp.nv, gp.nplanes, CUFFT_FORWARD, sizeof(R) == 8, st,
                    fftwork_.p);
    } else {
      launch_screen_put<R>(sg, st, sa, img, 0, H_.p);
      clear_outside_columns(band, gp.band_rows * gp.nplanes, gp.nv, gp.ny, cs, st);
      ColArgs ca = make_col(gp, gp.nplanes, static_cast<char *>(tw_.p) + pj.tw_off, band, H_.p);
      col_run<R>(gp.logM, false, ca, int(gp.nplanes), st, d_err);
      CF(cufftSetStream(pj.fft, st));
      CF(cufftSetWorkArea(pj.fft, fftwork_.p));
      if (sizeof(R) == 8)
        CF(cufftExecZ2Z(pj.fft, reinterpret_cast<cufftDoubleComplex *>(band),
                        reinterpret_cast<cufftDoubleComplex *>(band), CUFFT_FORWARD));
      else
        CF(cufftExecC2C(pj.fft, reinterpret_cast<cufftComplex *>(band),
                        reinterpret_cast<cufftComplex *>(band), CUFFT_FORWARD));
    }
    g_kernel_launches.fetch_add(2, std::memory_order_relaxed);
  }
  CK(cudaMemsetAsync(counter, 0, sizeof(int), st));  // (the error word stays until read)
  const TileLayout tl = make_layout(T_, W_);
  const size_t smem = grid_smem_bytes<R>(tl, W_, false);
  GridArgs ga{};
  ga.rec = rec_.p;
  ga.chunk_start = reinterpret_cast<const int *>(chunks_.p);
  ga.nchunks = d_nch;
  ga.counter = counter;
  ga.nvis = int(nrec_);
  ga.tl = tl;
  ga.sb = grid_sb<R>();
  ga.err = d_err;
  ga.jobs = reinterpret_cast<const JobGeom *>(jobgeom_.p);
  ga.chunk_job = reinterpret_cast<const int *>(chunk_job_.p);
  ga.vis_out = vis;
  ga.vis_double = a_.vis_type == WSG_C128;
  ga.vis_accumulate = multi ? 1 : 0;
  ga.first_pass = ga.last_pass = 1;
  ga.acc = need_acc_ ? acc_.p : nullptr;
  if (need_acc_) CK(cudaMemsetAsync(acc_.p, 0, nrec_ * cs, st));
  DevKernel<R> kc;
  std::memcpy(&kc, kernel_.data(), sizeof(kc));
  DevGeom g0;
  std::memcpy(&g0, geom_.data(), sizeof(g0));
  grid_dispatch<R>(W_, false, cx_.num_sms, smem, st, ga, g0, kc);
  if (need_acc_) {
    k_finalize<R><<<launch_blocks(nrec_, 256), 256, 0, st>>>(int(nrec_), rec_.p, acc_.p, vis,
                                                             ga.vis_double, ga.vis_accumulate);
    cuda_check(cudaGetLastError(), "k_finalize launch");
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void Plan::enqueue(int mode, const void *in, void *const *outs, const void *const *ins, void *out,
                   int accumulate) {
  if (mode == 0) {
    if (dbl_)
      enqueue_grid<double>(in, outs, accumulate);
    else
      enqueue_grid<float>(in, outs, accumulate);
  } else {
    if (dbl_)
      enqueue_degrid<double>(ins, out);
    else
      enqueue_degrid<float>(ins, out);
  }
}

// Runs one execution: directly into a graph being recorded by the caller,
// else through the plan's own graph for these pointers (recorded on the
// second call with them; the first runs eagerly and sets the kernels'
// launch attributes outside any capture).
void Plan::run(int mode, const void *in, void *const *outs, const void *const *ins, void *out,
               int accumulate) {
  CK(cudaSetDevice(cx_.device));
  cudaStream_t st = cx_.stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    enqueue(mode, in, outs, ins, out, accumulate);
    return;
  }
  std::vector<const void *> ptrs{mode == 0 ? in : out};
  for (size_t j = 0; j < jobs_.size(); ++j) ptrs.push_back(mode == 0 ? outs[j] : ins[j]);
  for (const Graph &g : graphs_)
    if (g.mode == mode && g.accumulate == accumulate && g.ptrs == ptrs) {
      CK(cudaGraphLaunch(g.exec, st));
      return;
    }
  for (const void *p : ptrs)
    require(is_device_pointer(p), "plan execution needs device memory for vis and images");
  const auto seen = std::make_pair(mode * 2 + accumulate, ptrs);
  const bool first = std::find(eager_seen_.begin(), eager_seen_.end(), seen) == eager_seen_.end();
  // the legacy default stream cannot be captured
  if (!use_graphs_ || first || st == nullptr || st == cudaStreamLegacy) {
    enqueue(mode, in, outs, ins, out, accumulate);
    if (first) eager_seen_.push_back(seen);
    return;
  }
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue(mode, in, outs, ins, out, accumulate);
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    throw;
  }
  CK(cudaStreamEndCapture(st, &graph));
  Graph g;
  g.mode = mode;
  g.accumulate = accumulate;
  g.ptrs = ptrs;
  cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    // a graph that cannot be instantiated: run eagerly from now on
    cudaGetLastError();
    use_graphs_ = false;
    enqueue(mode, in, outs, ins, out, accumulate);
    return;
  }
  graphs_.push_back(g);
  CK(cudaGraphLaunch(g.exec, st));
}

void Plan::ms2dirty(const void *vis, void *const *dirty, int accumulate) {
  require(vis && dirty, "vis and dirty are required");
  for (size_t j = 0; j < jobs_.size(); ++j) require(dirty[j] != nullptr, "dirty image missing");
  run(0, vis, dirty, nullptr, nullptr, accumulate ? 1 : 0);
}

void Plan::dirty2ms(const void *const *dirty, void *vis) {
  require(vis && dirty, "vis and dirty are required");
  for (size_t j = 0; j < jobs_.size(); ++j) require(dirty[j] != nullptr, "dirty image missing");
  run(1, nullptr, nullptr, dirty, vis, 0);
}

void Plan::stats(size_t job, wsg_stats &o) const {
  require(job < jobs_.size(), "job index out of range");
  const PlanJob &pj = jobs_[job];
  const GridPlan &g = pj.gp;
  std::memset(&o, 0, sizeof(o));
  o.nrows = a_.nrows;
  o.nchan = pj.chan1 - pj.chan0;
  o.nvis = pj.nrec;
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
  o.device_bytes = rec_.n + chunks_.n + chunk_job_.n + band_.n + H_.n + img_.n + acc_.n + fftwork_.n;
  o.kernel_launches = g_kernel_launches.load();
}

}  // namespace wsg
