"""Python face of the B200 w-gridder.

* ``ms2dirty`` / ``dirty2ms`` mirror ducc0's operators
  (external/wgridder/ducc0/wgridder/wgridder.h:1696-1729) with the same
  argument names and meaning; arrays may be numpy arrays (host) or torch
  tensors (host or CUDA).  CUDA tensors are used in place; host arrays are
  staged by the library.
* ``WGriddingGridder`` mirrors WSClean's WGriddingGridder_Simple
  (wgridder/wgriddinggridder_simple.h:34-144): MemoryUsage,
  InitializeInversion, AddInversionData, FinalizeImage, RealImage,
  InitializePrediction, PredictVisibilities.

Errors from the library raise ``WsgError`` (``InvalidArgument`` for the
reference's MR_assert cases).  Nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib as L

try:
    import torch
except Exception:  # pragma: no cover - torch is part of the image
    torch = None

_NP_C = {np.dtype(np.complex64): L.WSG_C64, np.dtype(np.complex128): L.WSG_C128}
_NP_F = {np.dtype(np.float32): L.WSG_F32, np.dtype(np.float64): L.WSG_F64}


# cudaStreamLegacy: the handle of the legacy default stream (a NULL stream
# argument would select the context's own stream instead)
_CUDA_STREAM_LEGACY = 1


def _is_torch(x):
    return torch is not None and isinstance(x, torch.Tensor)


def _prep(x, dtype=None):
    """-> (object kept alive, pointer, numpy dtype, is_cuda)."""
    if x is None:
        return None, None, None, False
    if _is_torch(x):
        if dtype is not None:
            tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
                   np.dtype(np.complex64): torch.complex64,
                   np.dtype(np.complex128): torch.complex128,
                   np.dtype(np.uint8): torch.uint8}[np.dtype(dtype)]
            if x.dtype != tdt:
                x = x.to(tdt)
        x = x.contiguous()
        npdt = {torch.float32: np.float32, torch.float64: np.float64,
                torch.complex64: np.complex64, torch.complex128: np.complex128,
                torch.uint8: np.uint8, torch.bool: np.uint8}[x.dtype]
        if x.dtype == torch.bool:
            x = x.to(torch.uint8)
        return x, x.data_ptr(), np.dtype(npdt), x.is_cuda
    a = np.ascontiguousarray(x, dtype=dtype)
    return a, a.ctypes.data, a.dtype, False


class Context:
    """An execution context (CUDA stream, buffers, cuFFT plans) on one device."""

    def __init__(self, device=-1):
        h = ctypes.c_void_p()
        L.check(L.lib().wsg_ctx_create(int(device), ctypes.byref(h)))
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            L.lib().wsg_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def release_buffers(self):
        L.check(L.lib().wsg_ctx_release_buffers(self._h))

    def set_async(self, flag=True):
        """Pipelined mode (``wsg_ctx_set_async``): ms2dirty / dirty2ms return
        once enqueued and overlap their transfers with each other's kernels;
        results are valid after ``synchronize()``.  Host inputs and outputs
        must stay alive (and should be page-locked) until then."""
        L.check(L.lib().wsg_ctx_set_async(self._h, int(bool(flag))))
        self._async = bool(flag)
        if not flag:
            self._pending = []

    def synchronize(self):
        """Waits for the context's work; raises errors detected on the device."""
        L.check(L.lib().wsg_ctx_synchronize(self._h))
        self._pending = []

    def _bind_stream(self, *tensors):
        """Run the call on torch's current stream of the tensors' device when
        any operand is a CUDA tensor, so that it is ordered after the torch
        work that produced its inputs (the context's own stream otherwise)."""
        dev = next((t.device for t in tensors if _is_torch(t) and t.is_cuda), None)
        s = torch.cuda.current_stream(dev).cuda_stream if dev is not None else None
        if dev is not None and s == 0:
            s = _CUDA_STREAM_LEGACY   # torch's default stream is the legacy NULL stream
        L.check(L.lib().wsg_ctx_set_stream(self._h, s))

    def stats(self):
        s = L.WsgStats()
        L.check(L.lib().wsg_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

    def last_tuning(self):
        """Subdivision of the last tuned call: dict(nfx, nfy, icut, wcut);
        nfx == 0 when the plain operator ran (wsg_get_tuning)."""
        return _tuning_of(self._h)

    def _args(self, uvw, freq, nrows, nchan, wgt, mask, npix_x, npix_y, pixsize_x, pixsize_y,
              epsilon, do_wgridding, negate_v, divide_by_n, sigma_min, sigma_max, center_x,
              center_y, precision, vis_type, dirty_type, keep):
        a = L.WsgArgs()
        L.lib().wsg_args_init(ctypes.byref(a))
        u, up, _, _ = _prep(uvw, np.float64)
        f, fp, _, _ = _prep(freq, np.float64)
        keep += [u, f]
        a.nrows, a.nchan = nrows, nchan
        a.uvw, a.freq = up, fp
        if wgt is not None:
            w, wp, wdt, _ = _prep(wgt)
            if wdt not in _NP_F:
                w, wp, wdt, _ = _prep(wgt, np.float32)
            keep.append(w)
            a.wgt, a.wgt_type = wp, _NP_F[wdt]
        if mask is not None:
            m, mp, _, _ = _prep(mask, np.uint8)
            keep.append(m)
            a.mask = mp
        a.npix_x, a.npix_y = int(npix_x), int(npix_y)
        a.pixsize_x, a.pixsize_y = float(pixsize_x), float(pixsize_y)
        a.epsilon = float(epsilon)
        a.do_wgridding = int(bool(do_wgridding))
        a.negate_v = int(bool(negate_v))
        a.divide_by_n = int(bool(divide_by_n))
        a.sigma_min, a.sigma_max = float(sigma_min), float(sigma_max)
        a.center_x, a.center_y = float(center_x), float(center_y)
        a.precision = _precision(precision)
        a.vis_type, a.dirty_type = vis_type, dirty_type
        return a

    def ms2dirty(self, uvw, freq, vis, npix_x, npix_y, pixsize_x, pixsize_y, epsilon,
                 do_wgridding=True, wgt=None, mask=None, negate_v=False, divide_by_n=True,
                 sigma_min=1.1, sigma_max=2.6, center_x=0.0, center_y=0.0,
                 precision="mixed", dirty=None, accumulate=False, dirty_dtype=None,
                 tuning=False):
        """ducc0::ms2dirty (tuning=True: ms2dirty_tuning, the subdivided
        schedule of -gridder tuned-wgridder; odd image sizes allowed)."""
        keep = []
        v, vp, vdt, vcuda = _prep(vis)
        if vdt not in _NP_C:
            v, vp, vdt, vcuda = _prep(vis, np.complex64)
        keep.append(v)
        nrows, nchan = v.shape
        if dirty is None:
            ddt = np.dtype(dirty_dtype) if dirty_dtype is not None else (
                np.dtype(np.float64) if _precision(precision) == L.WSG_PREC_FP64 else np.dtype(np.float32))
            if vcuda:
                tdt = torch.float64 if ddt == np.float64 else torch.float32
                dirty = torch.zeros((npix_x, npix_y), dtype=tdt, device=v.device)
            else:
                dirty = np.zeros((npix_x, npix_y), dtype=ddt)
        d, dp, ddt, _ = _prep(dirty)
        if d is not dirty and not _is_torch(dirty):
            raise ValueError("dirty must be a C-contiguous float32/float64 array")
        a = self._args(uvw, freq, nrows, nchan, wgt, mask, npix_x, npix_y, pixsize_x, pixsize_y,
                       epsilon, do_wgridding, negate_v, divide_by_n, sigma_min, sigma_max,
                       center_x, center_y, precision, _NP_C[vdt], _NP_F[ddt], keep)
        self._bind_stream(v, d, *keep)
        fn = L.lib().wsg_ms2dirty_tuning if tuning else L.lib().wsg_ms2dirty
        L.check(fn(self._h, ctypes.byref(a), vp, dp, int(bool(accumulate))))
        if getattr(self, "_async", False):
            self._pending = (getattr(self, "_pending", []) + [(keep, d)])[-4:]
        return d

    def autotune(self, uvw, freq, vis, npix_x, npix_y, pixsize_x, pixsize_y, epsilon,
                 candidates=4, do_wgridding=True, wgt=None, mask=None, negate_v=False,
                 divide_by_n=True, sigma_min=1.1, sigma_max=2.6, center_x=0.0, center_y=0.0,
                 precision="mixed", dirty_dtype=None):
        """Times the pair on these data for the `candidates` cheapest kernel
        choices and tile sizes and keeps the fastest for later calls with the
        same image size, precision and epsilon (``wsg_autotune``).  Returns the
        chosen grid's stats (ms_total = ms per pair)."""
        keep = []
        v, vp, vdt, _ = _prep(vis)
        if vdt not in _NP_C:
            v, vp, vdt, _ = _prep(vis, np.complex64)
        keep.append(v)
        nrows, nchan = v.shape
        ddt = np.dtype(dirty_dtype) if dirty_dtype is not None else (
            np.dtype(np.float64) if _precision(precision) == L.WSG_PREC_FP64 else np.dtype(np.float32))
        a = self._args(uvw, freq, nrows, nchan, wgt, mask, npix_x, npix_y, pixsize_x, pixsize_y,
                       epsilon, do_wgridding, negate_v, divide_by_n, sigma_min, sigma_max,
                       center_x, center_y, precision, _NP_C[vdt], _NP_F[ddt], keep)
        self._bind_stream(v, *keep)
        s = L.WsgStats()
        L.check(L.lib().wsg_autotune(self._h, ctypes.byref(a), vp, int(candidates), ctypes.byref(s)))
        return s.as_dict()

    def dirty2ms(self, uvw, freq, dirty, pixsize_x, pixsize_y, epsilon, do_wgridding=True,
                 wgt=None, mask=None, negate_v=False, divide_by_n=True, sigma_min=1.1,
                 sigma_max=2.6, center_x=0.0, center_y=0.0, precision="mixed",
                 vis=None, vis_dtype=np.complex64, tuning=False):
        """ducc0::dirty2ms (tuning=True: dirty2ms_tuning)."""
        keep = []
        d, dp, ddt, dcuda = _prep(dirty)
        if ddt not in _NP_F:
            d, dp, ddt, dcuda = _prep(dirty, np.float64)
        keep.append(d)
        npix_x, npix_y = d.shape
        nrows = int(uvw.shape[0])
        nchan = int(freq.shape[0])
        if vis is None:
            if dcuda:
                tdt = torch.complex128 if np.dtype(vis_dtype) == np.complex128 else torch.complex64
                vis = torch.zeros((nrows, nchan), dtype=tdt, device=d.device)
            else:
                vis = np.zeros((nrows, nchan), dtype=vis_dtype)
        v, vp, vdt, _ = _prep(vis)
        a = self._args(uvw, freq, nrows, nchan, wgt, mask, npix_x, npix_y, pixsize_x, pixsize_y,
                       epsilon, do_wgridding, negate_v, divide_by_n, sigma_min, sigma_max,
                       center_x, center_y, precision, _NP_C[vdt], _NP_F[ddt], keep)
        self._bind_stream(d, v, *keep)
        fn = L.lib().wsg_dirty2ms_tuning if tuning else L.lib().wsg_dirty2ms
        L.check(fn(self._h, ctypes.byref(a), dp, vp))
        if getattr(self, "_async", False):
            self._pending = (getattr(self, "_pending", []) + [(keep, v)])[-4:]
        return v


def _tuning_of(ctx_handle):
    nfx, nfy, icut, wcut = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    L.check(L.lib().wsg_get_tuning(ctx_handle, ctypes.byref(nfx), ctypes.byref(nfy),
                                   ctypes.byref(icut), ctypes.byref(wcut)))
    return dict(nfx=nfx.value, nfy=nfy.value, icut=icut.value, wcut=wcut.value)


def _precision(p):
    if isinstance(p, int):
        return p
    p = str(p).lower()
    if p in ("mixed", "fp32", "float", "single"):
        return L.WSG_PREC_MIXED
    if p in ("fp64", "double"):
        return L.WSG_PREC_FP64
    raise ValueError(f"unknown precision {p!r}")


_tls = threading.local()


def default_context(device=-1):
    """One context per (thread, device), created on first use."""
    d = getattr(_tls, "ctx", None)
    if d is None:
        d = _tls.ctx = {}
    if device not in d:
        d[device] = Context(device)
    return d[device]


def ms2dirty(uvw, freq, vis, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, do_wgridding=True,
             **kw):
    """ducc0::ms2dirty on the GPU (see Context.ms2dirty for the keywords)."""
    dev = kw.pop("device", -1)
    return default_context(dev).ms2dirty(uvw, freq, vis, npix_x, npix_y, pixsize_x, pixsize_y,
                                         epsilon, do_wgridding, **kw)


def dirty2ms(uvw, freq, dirty, pixsize_x, pixsize_y, epsilon, do_wgridding=True, **kw):
    """ducc0::dirty2ms on the GPU (see Context.dirty2ms for the keywords)."""
    dev = kw.pop("device", -1)
    return default_context(dev).dirty2ms(uvw, freq, dirty, pixsize_x, pixsize_y, epsilon,
                                         do_wgridding, **kw)


class WGriddingGridder:
    """WGriddingGridder_Simple<NumT> on the GPU (wgriddinggridder_simple.h:34-144).

    precision "mixed" stands for NumT=float, "fp64" for NumT=double; WSClean
    picks FP64 when the accuracy is <= 1.01e-5 (wgriddingmsgridder.cpp:41-51),
    which ``for_accuracy`` reproduces.
    """

    def __init__(self, width, height, width_t, height_t, pixel_size_x, pixel_size_y,
                 l_shift, m_shift, nthreads=1, epsilon=1e-4, verbosity=0, tuning=False,
                 precision="mixed", device=-1):
        p = L.WsgGridderParams(width, height, width_t, height_t, pixel_size_x, pixel_size_y,
                               l_shift, m_shift, nthreads, epsilon, verbosity, int(tuning),
                               _precision(precision), int(device))
        h = ctypes.c_void_p()
        L.check(L.lib().wsg_gridder_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.width, self.height = width, height
        self.width_t, self.height_t = width_t, height_t

    @staticmethod
    def for_accuracy(*args, epsilon=1e-4, **kw):
        kw["precision"] = "fp64" if epsilon <= 1.01e-5 else "mixed"
        return WGriddingGridder(*args, epsilon=epsilon, **kw)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().wsg_gridder_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def MemoryUsage(self):
        c, p = ctypes.c_size_t(), ctypes.c_size_t()
        L.check(L.lib().wsg_gridder_memory_usage(self._h, ctypes.byref(c), ctypes.byref(p)))
        return c.value, p.value

    def InitializeInversion(self):
        L.check(L.lib().wsg_gridder_initialize_inversion(self._h))

    def AddInversionData(self, uvw, freq, vis):
        v, vp, _, _ = _prep(vis, np.complex64)
        u, up, _, _ = _prep(uvw, np.float64)
        f, fp, _, _ = _prep(freq, np.float64)
        nrows, nchan = v.shape
        L.check(L.lib().wsg_gridder_add_inversion_data(self._h, nrows, nchan, up, fp, vp))

    def FinalizeImage(self, factor):
        L.check(L.lib().wsg_gridder_finalize_image(self._h, float(factor)))

    def RealImage(self):
        """width x height float32, index [y, x] (x + y*width), NaN outside the trimmed box."""
        out = np.empty((self.height, self.width), dtype=np.float32)
        L.check(L.lib().wsg_gridder_real_image(self._h, out.ctypes.data))
        return out

    def InitializePrediction(self, image):
        im, ip, _, _ = _prep(image, np.float32)
        L.check(L.lib().wsg_gridder_initialize_prediction(self._h, ip))

    def PredictVisibilities(self, uvw, freq):
        u, up, _, _ = _prep(uvw, np.float64)
        f, fp, _, _ = _prep(freq, np.float64)
        nrows, nchan = u.shape[0], f.shape[0]
        out = np.zeros((nrows, nchan), dtype=np.complex64)
        L.check(L.lib().wsg_gridder_predict_visibilities(self._h, nrows, nchan, up, fp,
                                                         out.ctypes.data))
        return out

    def stats(self):
        s = L.WsgStats()
        L.check(L.lib().wsg_get_stats(L.lib().wsg_gridder_ctx(self._h), ctypes.byref(s)))
        return s.as_dict()

    def last_tuning(self):
        """Subdivision of the last tuned call (gridders made with tuning=True)."""
        return _tuning_of(L.lib().wsg_gridder_ctx(self._h))


def plan_grid(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, nvis, wmin, wmax, umax, vmax=None,
              do_wgridding=True, precision="mixed", negate_v=True, divide_by_n=False,
              sigma_min=1.1, sigma_max=2.0, center_x=0.0, center_y=0.0):
    """The grid/kernel/w-plane choice for given data statistics (host only,
    no GPU): |w| range and max |u|, |v| in wavelengths."""
    a = L.WsgArgs()
    L.lib().wsg_args_init(ctypes.byref(a))
    a.npix_x, a.npix_y = int(npix_x), int(npix_y)
    a.pixsize_x, a.pixsize_y = float(pixsize_x), float(pixsize_y)
    a.epsilon = float(epsilon)
    a.do_wgridding = int(bool(do_wgridding))
    a.precision = _precision(precision)
    a.negate_v, a.divide_by_n = int(bool(negate_v)), int(bool(divide_by_n))
    a.sigma_min, a.sigma_max = float(sigma_min), float(sigma_max)
    a.center_x, a.center_y = float(center_x), float(center_y)
    s = L.WsgStats()
    L.check(L.lib().wsg_plan_grid(ctypes.byref(a), int(nvis), float(wmin), float(wmax),
                                  float(umax), float(umax if vmax is None else vmax),
                                  ctypes.byref(s)))
    return s.as_dict()


class Plan:
    """A reusable plan (``wsg_plan_create``): the grid choice, visibility sort
    and per-visibility records for fixed uvw / freq / weights / mask, over one
    job or a batch of jobs (facets x output channels) sharing the
    visibilities.  ``jobs`` is a list of dicts with npix_x, npix_y and
    optionally center_x, center_y (phase centre, radians) and chan_begin,
    chan_end (input channel range); without it there is one job of
    npix_x x npix_y over all channels.

    Execution takes torch CUDA tensors, runs on torch's current stream and
    returns without waiting, so a major cycle built from these calls can be
    recorded with ``torch.cuda.graph``.  On a non-default stream the plan
    records and replays its own graph from the second call with the same
    tensors on."""

    def __init__(self, uvw, freq, pixsize_x, pixsize_y, epsilon, npix_x=None, npix_y=None,
                 jobs=None, wgt=None, mask=None, do_wgridding=True, negate_v=False,
                 divide_by_n=True, sigma_min=1.1, sigma_max=2.6, center_x=0.0, center_y=0.0,
                 precision="mixed", vis_dtype=np.complex64, dirty_dtype=None, context=None,
                 device=-1):
        self.ctx = context if context is not None else Context(device)
        self._own_ctx = context is None
        nrows, nchan = int(np.shape(uvw)[0]), int(np.shape(freq)[0])
        self.nrows, self.nchan = nrows, nchan
        self.vis_dtype = np.dtype(vis_dtype)
        pr = _precision(precision)
        self.dirty_dtype = np.dtype(dirty_dtype) if dirty_dtype is not None else (
            np.dtype(np.float64) if pr == L.WSG_PREC_FP64 else np.dtype(np.float32))
        keep = []
        a = self.ctx._args(uvw, freq, nrows, nchan, wgt, mask, npix_x or 16, npix_y or 16,
                           pixsize_x, pixsize_y, epsilon, do_wgridding, negate_v, divide_by_n,
                           sigma_min, sigma_max, center_x, center_y, precision,
                           _NP_C[self.vis_dtype], _NP_F[self.dirty_dtype], keep)
        if jobs is None:
            if npix_x is None or npix_y is None:
                raise ValueError("npix_x and npix_y are required without jobs")
            jobs = [dict(npix_x=npix_x, npix_y=npix_y, center_x=center_x, center_y=center_y)]
        self.jobs = [dict(j) for j in jobs]
        arr = (L.WsgJob * len(jobs))()
        for k, j in enumerate(jobs):
            arr[k].npix_x, arr[k].npix_y = int(j["npix_x"]), int(j["npix_y"])
            arr[k].center_x = float(j.get("center_x", 0.0))
            arr[k].center_y = float(j.get("center_y", 0.0))
            arr[k].chan_begin = int(j.get("chan_begin", 0))
            arr[k].chan_end = int(j.get("chan_end", nchan))
        h = ctypes.c_void_p()
        self.ctx._bind_stream(*[x for x in keep if _is_torch(x)])
        L.check(L.lib().wsg_plan_create(self.ctx._h, ctypes.byref(a), arr, len(jobs),
                                        ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            L.lib().wsg_plan_destroy(self._h)
            self._h = None
        if getattr(self, "_own_ctx", False) and self.ctx is not None:
            self.ctx.close()
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _tensor(self, x, dtype, what):
        if not (_is_torch(x) and x.is_cuda):
            raise ValueError(f"plan execution takes CUDA tensors ({what})")
        t, _, _, _ = _prep(x, dtype)
        return t

    def ms2dirty(self, vis, dirty=None, accumulate=False):
        """Images of all jobs: list of (npix_x, npix_y) tensors."""
        v = self._tensor(vis, self.vis_dtype, "vis")
        if tuple(v.shape) != (self.nrows, self.nchan):
            raise ValueError("vis must be nrows x nchan")
        tdt = torch.float64 if self.dirty_dtype == np.float64 else torch.float32
        if dirty is None:
            dirty = [torch.zeros((j["npix_x"], j["npix_y"]), dtype=tdt, device=v.device)
                     for j in self.jobs]
        elif _is_torch(dirty):
            dirty = [dirty]
        outs = [self._tensor(d, self.dirty_dtype, "dirty") for d in dirty]
        if any(o is not d for o, d in zip(outs, dirty)):
            raise ValueError("dirty images must be contiguous tensors of the plan's dirty dtype")
        ptrs = (ctypes.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        self.ctx._bind_stream(v)
        L.check(L.lib().wsg_plan_ms2dirty(self._h, v.data_ptr(), ptrs, int(bool(accumulate))))
        self._keep = (v, outs)
        return outs

    def dirty2ms(self, dirty, vis=None):
        """Sum over jobs of the predicted visibilities (nrows x nchan tensor)."""
        if _is_torch(dirty):
            dirty = [dirty]
        ins = [self._tensor(d, self.dirty_dtype, "dirty") for d in dirty]
        if len(ins) != len(self.jobs):
            raise ValueError("one image per job is required")
        tdt = torch.complex128 if self.vis_dtype == np.complex128 else torch.complex64
        if vis is None:
            vis = torch.empty((self.nrows, self.nchan), dtype=tdt, device=ins[0].device)
        out = self._tensor(vis, self.vis_dtype, "vis")
        if out is not vis:
            raise ValueError("vis must be a contiguous tensor of the plan's vis dtype")
        ptrs = (ctypes.c_void_p * len(ins))(*[d.data_ptr() for d in ins])
        self.ctx._bind_stream(out)
        L.check(L.lib().wsg_plan_dirty2ms(self._h, ptrs, out.data_ptr()))
        self._keep = (ins, out)
        return out

    def stats(self, job=0):
        s = L.WsgStats()
        L.check(L.lib().wsg_plan_get_stats(self._h, int(job), ctypes.byref(s)))
        return s.as_dict()


def data_extent(uvw, freq):
    """(wmin, wmax, umax, vmax) in wavelengths over all rows and channels:
    the extent a Stream is planned for."""
    uvw = np.asarray(uvw, dtype=np.float64)
    f = np.asarray(freq, dtype=np.float64) / 299792458.0
    au = np.abs(uvw)
    return (float(au[:, 2].min() * f.min()), float(au[:, 2].max() * f.max()),
            float(au[:, 0].max() * f.max()), float(au[:, 1].max() * f.max()))


class Stream:
    """Streaming gridding into a resident grid (``wsg_stream_create``): the
    grid is planned once for the declared extent (see ``data_extent``), each
    ``add`` sorts and spreads one chunk of rows while the next chunk's copy
    is in flight, and ``finish`` transforms once.  ``predict_begin`` /
    ``predict`` run the transpose.  Chunks may be numpy arrays, page-locked
    torch CPU tensors or CUDA tensors."""

    def __init__(self, freq, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, extent, nvis=0,
                 do_wgridding=True, negate_v=False, divide_by_n=True, sigma_min=1.1,
                 sigma_max=2.6, center_x=0.0, center_y=0.0, precision="mixed",
                 vis_dtype=np.complex64, dirty_dtype=None, wgt_dtype=np.float32, context=None,
                 device=-1):
        self.ctx = context if context is not None else Context(device)
        self._own_ctx = context is None
        self.nchan = int(np.shape(freq)[0])
        self.npix = (int(npix_x), int(npix_y))
        self.vis_dtype = np.dtype(vis_dtype)
        self.wgt_dtype = np.dtype(wgt_dtype)
        pr = _precision(precision)
        self.dirty_dtype = np.dtype(dirty_dtype) if dirty_dtype is not None else (
            np.dtype(np.float64) if pr == L.WSG_PREC_FP64 else np.dtype(np.float32))
        keep = []
        dummy = np.zeros((1, 3))
        a = self.ctx._args(dummy, freq, 1, self.nchan, None, None, npix_x, npix_y, pixsize_x,
                           pixsize_y, epsilon, do_wgridding, negate_v, divide_by_n, sigma_min,
                           sigma_max, center_x, center_y, precision, _NP_C[self.vis_dtype],
                           _NP_F[self.dirty_dtype], keep)
        a.wgt_type = _NP_F[self.wgt_dtype]
        wmin, wmax, umax, vmax = extent
        h = ctypes.c_void_p()
        L.check(L.lib().wsg_stream_create(self.ctx._h, ctypes.byref(a), float(wmin), float(wmax),
                                          float(umax), float(vmax), int(nvis), ctypes.byref(h)))
        self._h = h
        self._inflight = []

    def close(self):
        if getattr(self, "_h", None):
            L.lib().wsg_stream_destroy(self._h)
            self._h = None
        if getattr(self, "_own_ctx", False) and self.ctx is not None:
            self.ctx.close()
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _hold(self, objs):
        # inputs of the last two chunks may still be copied from
        self._inflight = (self._inflight + [objs])[-2:]

    def add(self, uvw, vis, wgt=None, mask=None):
        u, up, _, _ = _prep(uvw, np.float64)
        v, vp, _, _ = _prep(vis, self.vis_dtype)
        w, wp, _, _ = _prep(wgt, self.wgt_dtype)
        m, mp, _, _ = _prep(mask, np.uint8)
        nrows = int(u.shape[0])
        if tuple(v.shape) != (nrows, self.nchan):
            raise ValueError("vis must be nrows x nchan")
        self.ctx._bind_stream(u, v, w, m)
        L.check(L.lib().wsg_stream_add(self._h, nrows, up, vp, wp, mp))
        self._hold((u, v, w, m))

    def finish(self, dirty=None, accumulate=False):
        if dirty is None:
            dirty = np.zeros(self.npix, dtype=self.dirty_dtype)
        d, dp, ddt, _ = _prep(dirty)
        if ddt != self.dirty_dtype or (d is not dirty and not _is_torch(dirty)):
            raise ValueError("dirty must be a contiguous array of the stream's dirty dtype")
        self.ctx._bind_stream(d)
        L.check(L.lib().wsg_stream_finish(self._h, dp, int(bool(accumulate))))
        self._inflight = []
        return d

    def predict_begin(self, dirty):
        d, dp, _, _ = _prep(dirty, self.dirty_dtype)
        self.ctx._bind_stream(d)
        L.check(L.lib().wsg_stream_predict_begin(self._h, dp))
        self._model = d

    def predict(self, uvw, vis=None, wgt=None, mask=None):
        u, up, _, ucuda = _prep(uvw, np.float64)
        nrows = int(u.shape[0])
        if vis is None:
            if ucuda:
                tdt = torch.complex128 if self.vis_dtype == np.complex128 else torch.complex64
                vis = torch.zeros((nrows, self.nchan), dtype=tdt, device=u.device)
            else:
                vis = np.zeros((nrows, self.nchan), dtype=self.vis_dtype)
        v, vp, _, _ = _prep(vis, self.vis_dtype)
        w, wp, _, _ = _prep(wgt, self.wgt_dtype)
        m, mp, _, _ = _prep(mask, np.uint8)
        self.ctx._bind_stream(u, v, w, m)
        L.check(L.lib().wsg_stream_predict(self._h, nrows, up, vp, wp, mp))
        self._hold((u, w, m))
        return v

    def stats(self):
        s = L.WsgStats()
        L.check(L.lib().wsg_stream_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

    def set_imaging_weights(self, weights):
        """Fold a finished ``ImageWeights`` into every later ``add``: each
        visibility is gridded with weight x the imaging weight of its uv cell,
        looked up on the device (None turns it off)."""
        L.check(L.lib().wsg_stream_set_imaging_weights(self._h, weights._h if weights else None))
        self._imaging_weights = weights


class ImageWeights:
    """WSClean's ImageWeights on the GPU (``wsg_weights_*``): ``grid`` the
    visibility weights of any number of chunks, ``finish`` into natural,
    uniform or Briggs weights, ``apply`` to get each visibility's weight
    times its imaging weight (what MSGridderBase multiplies into the data)."""

    NATURAL, UNIFORM, BRIGGS = L.WSG_WEIGHT_NATURAL, L.WSG_WEIGHT_UNIFORM, L.WSG_WEIGHT_BRIGGS

    def __init__(self, mode, robust, width, height, pixel_scale_x, pixel_scale_y,
                 weights_as_taper=False, super_weight=1.0, context=None, device=-1):
        if isinstance(mode, str):
            mode = {"natural": self.NATURAL, "uniform": self.UNIFORM, "briggs": self.BRIGGS}[mode]
        self.ctx = context if context is not None else Context(device)
        self._own_ctx = context is None
        h = ctypes.c_void_p()
        L.check(L.lib().wsg_weights_create(self.ctx._h, int(mode), float(robust), int(width),
                                           int(height), float(pixel_scale_x),
                                           float(pixel_scale_y), int(bool(weights_as_taper)),
                                           float(super_weight), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            L.lib().wsg_weights_destroy(self._h)
            self._h = None
        if getattr(self, "_own_ctx", False) and self.ctx is not None:
            self.ctx.close()
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def grid(self, uvw, freq, weights=None, npol=1):
        u, up, _, _ = _prep(uvw, np.float64)
        f, fp, _, _ = _prep(freq, np.float64)
        w, wp, _, _ = _prep(weights, np.float32)
        self.ctx._bind_stream(u, w)
        L.check(L.lib().wsg_weights_grid(self._h, int(u.shape[0]), int(f.shape[0]), int(npol),
                                         up, fp, wp))

    def finish(self):
        L.check(L.lib().wsg_weights_finish(self._h))

    def apply(self, uvw, freq, weights=None, npol=1, out=None):
        u, up, _, ucuda = _prep(uvw, np.float64)
        f, fp, _, _ = _prep(freq, np.float64)
        w, wp, _, _ = _prep(weights, np.float32)
        shape = (int(u.shape[0]), int(f.shape[0])) + ((int(npol),) if npol > 1 else ())
        if out is None:
            out = (torch.zeros(shape, dtype=torch.float32, device=u.device) if ucuda
                   else np.zeros(shape, dtype=np.float32))
        o, op, _, _ = _prep(out, np.float32)
        self.ctx._bind_stream(u, w, o)
        L.check(L.lib().wsg_weights_apply(self._h, shape[0], shape[1], int(npol), up, fp, wp, op))
        return o

    def grid_array(self):
        """(grid as a (height/2, width) array indexed [y, x], total weight)."""
        wd, ht, tot = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_double()
        L.check(L.lib().wsg_weights_get(self._h, None, ctypes.byref(wd), ctypes.byref(ht),
                                        ctypes.byref(tot)))
        g = np.zeros((ht.value // 2, wd.value))
        L.check(L.lib().wsg_weights_get(self._h, g.ctypes.data, None, None, None))
        return g, tot.value
