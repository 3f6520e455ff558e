"""The allocation-free gridding entry point, through the C ABI.

wsg_ms2dirty_noalloc serves callers that cannot allocate device memory while
they grid (a CUDA graph being recorded, a device pool owned by another
framework): it takes all scratch from a static device array.  Its image must
agree with the regular wsg_ms2dirty on the same inputs within the mixed-
precision tolerance (relative RMS 1e-5), on consecutive calls that share the
array.  This file is collected last so that a stop at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(torch, dev):
    rng = np.random.default_rng(8)
    nrow, nchan, nx, ny = 5000, 2, 128, 96
    px = np.deg2rad(20 / 3600)
    uvw = torch.as_tensor(rng.uniform(-1, 1, (nrow, 3)) * np.array([900.0, 900.0, 300.0]), device=dev)
    freq = torch.as_tensor(np.array([1.40e8, 1.45e8]), device=dev)
    vis = torch.as_tensor((rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan)))
                          .astype(np.complex64), device=dev)
    return nrow, nchan, nx, ny, px, uvw, freq, vis


def _args(L, lib, nrow, nchan, nx, ny, px, uvw, freq):
    a = L.WsgArgs()
    lib.wsg_args_init(ctypes.byref(a))
    a.nrows, a.nchan = nrow, nchan
    a.uvw, a.freq = uvw.data_ptr(), freq.data_ptr()
    a.npix_x, a.npix_y = nx, ny
    a.pixsize_x = a.pixsize_y = px
    a.epsilon = 1e-5
    a.negate_v, a.divide_by_n = 1, 0
    a.sigma_min, a.sigma_max = 1.1, 2.0
    a.center_x, a.center_y = 2 * px, -px
    a.precision = L.WSG_PREC_MIXED
    a.vis_type, a.dirty_type = L.WSG_C64, L.WSG_F64
    return a


def test_noalloc_matches_ms2dirty_on_consecutive_calls():
    import torch
    from wsclean_b200 import _lib as L
    lib = L.lib()
    dev = torch.device("cuda", 0)
    nrow, nchan, nx, ny, px, uvw, freq, vis = _problem(torch, dev)
    a = _args(L, lib, nrow, nchan, nx, ny, px, uvw, freq)
    ctx = ctypes.c_void_p()
    L.check(lib.wsg_ctx_create(0, ctypes.byref(ctx)))
    ref = torch.zeros((nx, ny), dtype=torch.float64, device=dev)
    L.check(lib.wsg_ms2dirty(ctx, ctypes.byref(a), vis.data_ptr(), ref.data_ptr(), 0))
    L.check(lib.wsg_ctx_destroy(ctx))
    for _ in range(2):
        out = torch.full((nx, ny), float("nan"), dtype=torch.float64, device=dev)
        L.check(lib.wsg_ms2dirty_noalloc(ctypes.byref(a), vis.data_ptr(), out.data_ptr(), None))
        torch.cuda.synchronize(dev)
        err = ((out - ref).norm() / ref.norm()).item()
        assert err < 1e-5, err


def test_noalloc_rejects_host_memory_and_oversize():
    import torch
    from wsclean_b200 import _lib as L
    lib = L.lib()
    dev = torch.device("cuda", 0)
    nrow, nchan, nx, ny, px, uvw, freq, vis = _problem(torch, dev)
    a = _args(L, lib, nrow, nchan, nx, ny, px, uvw, freq)
    host_out = np.zeros((nx, ny))
    rc = lib.wsg_ms2dirty_noalloc(ctypes.byref(a), vis.data_ptr(), host_out.ctypes.data, None)
    assert rc == L.WSG_ERR_INVALID and b"device" in lib.wsg_last_error()
    a.npix_x = a.npix_y = 8192   # the FP64 image alone exceeds the scratch array
    big = torch.zeros((8192, 8192), dtype=torch.float64, device=dev)
    rc = lib.wsg_ms2dirty_noalloc(ctypes.byref(a), vis.data_ptr(), big.data_ptr(), None)
    assert rc == L.WSG_ERR_INVALID and b"scratch" in lib.wsg_last_error()
