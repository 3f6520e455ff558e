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

    def _bind_stream(self, *tensors):
        """Run the call on torch's current stream of the tensors' device when
        any operand is a CUDA tensor, so that it is ordered after the torch
        work that produced its inputs (the context's own stream otherwise)."""
        dev = next((t.device for t in tensors if _is_torch(t) and t.is_cuda), None)
        s = torch.cuda.current_stream(dev).cuda_stream if dev is not None else None
        L.check(L.lib().wsg_ctx_set_stream(self._h, s))

    def stats(self):
        s = L.WsgStats()
        L.check(L.lib().wsg_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

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
                 precision="mixed", dirty=None, accumulate=False, dirty_dtype=None):
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
        L.check(L.lib().wsg_ms2dirty(self._h, ctypes.byref(a), vp, dp, int(bool(accumulate))))
        return d

    def dirty2ms(self, uvw, freq, dirty, pixsize_x, pixsize_y, epsilon, do_wgridding=True,
                 wgt=None, mask=None, negate_v=False, divide_by_n=True, sigma_min=1.1,
                 sigma_max=2.6, center_x=0.0, center_y=0.0, precision="mixed",
                 vis=None, vis_dtype=np.complex64):
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
        L.check(L.lib().wsg_dirty2ms(self._h, ctypes.byref(a), dp, vp))
        return v


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
