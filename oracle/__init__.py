"""Test infrastructure only: the CPU checkers for the w-gridding path.

Nothing in the product imports this package.  Only tests/, the smoke() check
and bench.py's CPU-baseline / reference arm use it, and only as the checker or
the timed CPU baseline.

* ``ref_ms2dirty`` / ``ref_dirty2ms``: the reference's own vendored ducc0
  w-gridder (external/wgridder/ducc0/wgridder/wgridder.h:1696-1729, and the
  tuned variants :1781-1877), compiled in place from the reference sources by
  oracle/Makefile into oracle/_ref/ and called through ref_shim.cpp with
  WSClean's argument pattern (wgridder/wgriddinggridder_simple.cpp:56-58).
* ``dft_ms2dirty`` / ``dft_dirty2ms``: the FP64 direct Fourier transform
  (oracle/dft.c), WSClean's DirectMSGridder semantics in ducc0's convention.
* ``parse_report``: the grid parameters from ducc0's verbosity-1 report.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ref_lib = None
_dft_lib = None


def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def ref_isa():
    """The ISA level of the compiled reference that fits this host CPU."""
    fl = _cpu_flags()
    if {"avx512f", "avx512bw", "avx512dq", "avx512vl"} <= fl:
        return "v4"
    return "v3"


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", f"libducc_ref_{ref_isa()}.so"))


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        path = os.path.join(HERE, "_ref", f"libducc_ref_{ref_isa()}.so")
        if not os.path.exists(path):
            raise RuntimeError(f"compiled reference missing: {path} (run make -C oracle ref)")
        lib = ctypes.CDLL(path)
        sz, dbl, i32, vp = ctypes.c_size_t, ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        args = [i32, i32, i32, sz, sz, vp, vp, vp, vp, vp, sz, sz, dbl, dbl, dbl,
                i32, sz, vp, sz, i32, i32, dbl, dbl, dbl, dbl, ctypes.c_char_p, sz]
        for name in ("ducc_ref_ms2dirty", "ducc_ref_dirty2ms"):
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = i32
        lib.ducc_ref_last_error.restype = ctypes.c_char_p
        _ref_lib = lib
    return _ref_lib


def dft_lib():
    global _dft_lib
    if _dft_lib is None:
        path = os.path.join(HERE, "_build", "libwsg_dft.so")
        if not os.path.exists(path):
            raise RuntimeError(f"DFT oracle missing: {path} (run make -C oracle dft)")
        lib = ctypes.CDLL(path)
        sz, dbl, i32, vp = ctypes.c_size_t, ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        lib.wsg_dft_ms2dirty.argtypes = [sz, sz, vp, vp, vp, vp, vp, sz, sz, dbl, dbl,
                                         i32, i32, dbl, dbl, sz, vp, vp]
        lib.wsg_dft_dirty2ms.argtypes = [sz, sz, vp, vp, vp, vp, vp, sz, sz, dbl, dbl,
                                         i32, i32, dbl, dbl, sz, vp, vp]
        _dft_lib = lib
    return _dft_lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _prep_common(uvw, freq, wgt, mask, nrows, nchan, wdtype):
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    freq = np.ascontiguousarray(freq, dtype=np.float64)
    if wgt is not None:
        wgt = np.ascontiguousarray(wgt, dtype=wdtype).reshape(nrows, nchan)
    if mask is not None:
        mask = np.ascontiguousarray(mask, dtype=np.uint8).reshape(nrows, nchan)
    return uvw, freq, wgt, mask


_GRID_RE = re.compile(r"grid=\((\d+)x(\d+)(?:x(\d+))?\), supp=(\d+)")


def parse_report(text):
    """ducc0's verbosity-1 report -> list of dicts {nu, nv, nplanes, supp}."""
    out = []
    for m in _GRID_RE.finditer(text):
        out.append(dict(nu=int(m.group(1)), nv=int(m.group(2)),
                        nplanes=int(m.group(3) or 0), supp=int(m.group(4))))
    return out


def ref_ms2dirty(uvw, freq, vis, npix_x, npix_y, pixsize_x, pixsize_y, epsilon,
                 do_wgridding=True, nthreads=0, wgt=None, mask=None, prec="double",
                 negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0,
                 center_x=0.0, center_y=0.0, tuning=False, verbosity=0,
                 return_report=False):
    """ducc0 ms2dirty through the compiled reference.  Defaults follow WSClean
    (wgriddinggridder_simple.cpp:56-58: negate_v, no divide_by_n, sigma
    1.1..2.0).  vis complex64 -> Tms=float; complex128 requires prec='double'."""
    vis = np.ascontiguousarray(vis)
    nrows, nchan = vis.shape
    vis_double = vis.dtype == np.complex128
    pd = 1 if prec == "double" else 0
    uvw, freq, wgt, mask = _prep_common(uvw, freq, wgt, mask, nrows, nchan,
                                        np.float64 if vis_double else np.float32)
    dirty = np.zeros((npix_x, npix_y), dtype=np.float64 if pd else np.float32)
    rep = ctypes.create_string_buffer(1 << 16) if (verbosity or return_report) else None
    rc = ref_lib().ducc_ref_ms2dirty(
        pd, int(vis_double), int(tuning), nrows, nchan, _ptr(uvw), _ptr(freq),
        _ptr(vis), _ptr(wgt), _ptr(mask), npix_x, npix_y, pixsize_x, pixsize_y,
        epsilon, int(do_wgridding), nthreads or os.cpu_count(), _ptr(dirty),
        max(verbosity, 1 if return_report else 0), int(negate_v), int(divide_by_n),
        sigma_min, sigma_max, center_x, center_y, rep, (1 << 16) if rep else 0)
    if rc:
        raise RuntimeError(ref_lib().ducc_ref_last_error().decode())
    if return_report:
        return dirty, rep.value.decode()
    return dirty


def ref_dirty2ms(uvw, freq, dirty, pixsize_x, pixsize_y, epsilon, do_wgridding=True,
                 nthreads=0, wgt=None, mask=None, prec="double", vis_dtype=np.complex64,
                 negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0,
                 center_x=0.0, center_y=0.0, tuning=False, verbosity=0,
                 return_report=False):
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    freq = np.ascontiguousarray(freq, dtype=np.float64)
    nrows, nchan = uvw.shape[0], freq.shape[0]
    vis_double = np.dtype(vis_dtype) == np.complex128
    pd = 1 if prec == "double" else 0
    dirty = np.ascontiguousarray(dirty, dtype=np.float64 if pd else np.float32)
    npix_x, npix_y = dirty.shape
    uvw, freq, wgt, mask = _prep_common(uvw, freq, wgt, mask, nrows, nchan,
                                        np.float64 if vis_double else np.float32)
    vis = np.zeros((nrows, nchan), dtype=vis_dtype)
    rep = ctypes.create_string_buffer(1 << 16) if (verbosity or return_report) else None
    rc = ref_lib().ducc_ref_dirty2ms(
        pd, int(vis_double), int(tuning), nrows, nchan, _ptr(uvw), _ptr(freq),
        _ptr(dirty), _ptr(wgt), _ptr(mask), npix_x, npix_y, pixsize_x, pixsize_y,
        epsilon, int(do_wgridding), nthreads or os.cpu_count(), _ptr(vis),
        max(verbosity, 1 if return_report else 0), int(negate_v), int(divide_by_n),
        sigma_min, sigma_max, center_x, center_y, rep, (1 << 16) if rep else 0)
    if rc:
        raise RuntimeError(ref_lib().ducc_ref_last_error().decode())
    if return_report:
        return vis, rep.value.decode()
    return vis


def dft_ms2dirty(uvw, freq, vis, npix_x, npix_y, pixsize_x, pixsize_y, wgt=None,
                 mask=None, negate_v=True, divide_by_n=False, center_x=0.0,
                 center_y=0.0, pixels=None):
    """FP64 DFT image (or the listed flat pixel indices i*ny+j)."""
    vis = np.ascontiguousarray(vis, dtype=np.complex128)
    nrows, nchan = vis.shape
    uvw, freq, wgt, mask = _prep_common(uvw, freq, wgt, mask, nrows, nchan, np.float64)
    if pixels is not None:
        pixels = np.ascontiguousarray(pixels, dtype=np.int64)
        out = np.zeros(len(pixels))
    else:
        out = np.zeros((npix_x, npix_y))
    dft_lib().wsg_dft_ms2dirty(nrows, nchan, _ptr(uvw), _ptr(freq), _ptr(vis),
                               _ptr(wgt), _ptr(mask), npix_x, npix_y, pixsize_x,
                               pixsize_y, int(negate_v), int(divide_by_n), center_x,
                               center_y, 0 if pixels is None else len(pixels),
                               _ptr(pixels), _ptr(out))
    return out


def dft_dirty2ms(uvw, freq, dirty, pixsize_x, pixsize_y, wgt=None, mask=None,
                 negate_v=True, divide_by_n=False, center_x=0.0, center_y=0.0,
                 select=None):
    """FP64 DFT visibilities (or the listed flat visibility indices)."""
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    freq = np.ascontiguousarray(freq, dtype=np.float64)
    nrows, nchan = uvw.shape[0], freq.shape[0]
    dirty = np.ascontiguousarray(dirty, dtype=np.float64)
    nx, ny = dirty.shape
    uvw, freq, wgt, mask = _prep_common(uvw, freq, wgt, mask, nrows, nchan, np.float64)
    if select is not None:
        select = np.ascontiguousarray(select, dtype=np.int64)
        out = np.zeros(len(select), dtype=np.complex128)
    else:
        out = np.zeros((nrows, nchan), dtype=np.complex128)
    dft_lib().wsg_dft_dirty2ms(nrows, nchan, _ptr(uvw), _ptr(freq), _ptr(dirty),
                               _ptr(wgt), _ptr(mask), nx, ny, pixsize_x, pixsize_y,
                               int(negate_v), int(divide_by_n), center_x, center_y,
                               0 if select is None else len(select), _ptr(select),
                               _ptr(out))
    return out


def rel_rms(a, b):
    """Relative RMS error of a against b (the truth)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))
