"""The allocation-free gridding entry point, through the C ABI.

wsg_ms2dirty_noalloc serves callers that cannot allocate device memory while
they grid -- a plugin in a host application that reserved the whole device for
its own memory pool, or a service held to a device-memory budget fixed at
start-up: it takes all scratch from a static device array.  Its image must
agree with the regular wsg_ms2dirty on the same inputs within the mixed-
precision tolerance (relative RMS 1e-5), on consecutive calls that share the
array, and with the FP64 direct Fourier transform (the oracle) within the
same tolerance.  Cases: a small image in one pass of w planes; a 2048^2 image
whose planes go through the array one pass at a time (the band cleared and
the image accumulated across passes); weights, a mask and an FP32 image.
This file is collected last so that a stop at the first failure has already
run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _problem(torch, dev, nrow=5000, wscale=300.0, seed=8):
    rng = np.random.default_rng(seed)
    nchan = 2
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([900.0, 900.0, wscale])
    freq = np.array([1.40e8, 1.45e8])
    vis = (rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))).astype(np.complex64)
    d = dict(uvw=torch.as_tensor(uvw, device=dev), freq=torch.as_tensor(freq, device=dev),
             vis=torch.as_tensor(vis, device=dev))
    return uvw, freq, vis, d, rng


def _args(L, lib, d, nx, ny, px, dirty_type=None):
    a = L.WsgArgs()
    lib.wsg_args_init(ctypes.byref(a))
    a.nrows, a.nchan = d["vis"].shape
    a.uvw, a.freq = d["uvw"].data_ptr(), d["freq"].data_ptr()
    a.npix_x, a.npix_y = nx, ny
    a.pixsize_x = a.pixsize_y = px
    a.epsilon = 1e-5
    a.negate_v, a.divide_by_n = 1, 0
    a.sigma_min, a.sigma_max = 1.1, 2.0
    a.center_x, a.center_y = 2 * px, -px
    a.precision = L.WSG_PREC_MIXED
    a.vis_type = L.WSG_C64
    a.dirty_type = L.WSG_F64 if dirty_type is None else dirty_type
    return a


def _regular(torch, L, lib, a, d, nx, ny, dtype):
    """wsg_ms2dirty on a fresh context (the allocating entry point)."""
    ctx = ctypes.c_void_p()
    L.check(lib.wsg_ctx_create(0, ctypes.byref(ctx)))
    ref = torch.zeros((nx, ny), dtype=dtype, device=d["vis"].device)
    try:
        L.check(lib.wsg_ms2dirty(ctx, ctypes.byref(a), d["vis"].data_ptr(), ref.data_ptr(), 0))
    finally:
        L.check(lib.wsg_ctx_destroy(ctx))
    return ref


def _noalloc_twice(torch, L, lib, a, d, nx, ny, dtype, ref):
    """Two consecutive calls (the second sees the first one's leftovers in
    the shared array), each within TOL of the regular entry point."""
    outs = []
    for _ in range(2):
        out = torch.full((nx, ny), float("nan"), dtype=dtype, device=d["vis"].device)
        L.check(lib.wsg_ms2dirty_noalloc(ctypes.byref(a), d["vis"].data_ptr(), out.data_ptr(), None))
        torch.cuda.synchronize()
        err = ((out.double() - ref.double()).norm() / ref.double().norm()).item()
        assert err < TOL, err
        outs.append(out)
    return outs


def test_noalloc_matches_ms2dirty_and_dft_on_consecutive_calls():
    import torch
    from wsclean_b200 import _lib as L
    lib = L.lib()
    dev = torch.device("cuda", 0)
    nx, ny, px = 128, 96, np.deg2rad(20 / 3600)
    uvw, freq, vis, d, _ = _problem(torch, dev)
    a = _args(L, lib, d, nx, ny, px)
    ref = _regular(torch, L, lib, a, d, nx, ny, torch.float64)
    out = _noalloc_twice(torch, L, lib, a, d, nx, ny, torch.float64, ref)[-1]
    dft = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, px, negate_v=True, divide_by_n=False,
                         center_x=2 * px, center_y=-px)
    assert O.rel_rms(out.cpu().numpy(), dft) < TOL


def test_noalloc_plane_passes_through_the_array():
    """A 2048^2 image: the FP64 image and one w plane of the band grid and of
    the transformed columns use most of the 96 MiB, so the w planes go
    through the array in several passes."""
    import torch
    from wsclean_b200 import _lib as L
    lib = L.lib()
    dev = torch.device("cuda", 0)
    nx = ny = 2048
    px = np.deg2rad(20 / 3600)
    uvw, freq, vis, d, rng = _problem(torch, dev, nrow=6000, wscale=600.0, seed=9)
    a = _args(L, lib, d, nx, ny, px)
    st = L.WsgStats()
    # the regular planner's plane count (the allocation-free grid is similar)
    lam = uvw[:, :, None] * (freq / 299792458.0)[None, None, :]   # rows x (u, v, w) x channels
    aw = np.abs(lam[:, 2])
    L.check(lib.wsg_plan_grid(ctypes.byref(a), vis.size, float(aw.min()), float(aw.max()),
                              float(np.abs(lam[:, 0]).max()), float(np.abs(lam[:, 1]).max()),
                              ctypes.byref(st)))
    assert st.nplanes >= 4, st.nplanes   # more planes than one pass of the array holds
    ref = _regular(torch, L, lib, a, d, nx, ny, torch.float64)
    out = _noalloc_twice(torch, L, lib, a, d, nx, ny, torch.float64, ref)[-1]
    pix = rng.integers(0, nx * ny, 64)
    dft = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, px, negate_v=True, divide_by_n=False,
                         center_x=2 * px, center_y=-px, pixels=pix)
    assert O.rel_rms(out.cpu().numpy().ravel()[pix], dft) < TOL


def test_noalloc_weights_mask_and_f32_image():
    import torch
    from wsclean_b200 import _lib as L
    lib = L.lib()
    dev = torch.device("cuda", 0)
    nx, ny, px = 128, 96, np.deg2rad(20 / 3600)
    uvw, freq, vis, d, rng = _problem(torch, dev, seed=10)
    wgt = rng.uniform(0.5, 2.0, vis.shape).astype(np.float32)
    mask = (rng.uniform(size=vis.shape) > 0.2).astype(np.uint8)
    d_wgt, d_mask = torch.as_tensor(wgt, device=dev), torch.as_tensor(mask, device=dev)
    a = _args(L, lib, d, nx, ny, px, dirty_type=L.WSG_F32)
    a.wgt, a.wgt_type, a.mask = d_wgt.data_ptr(), L.WSG_F32, d_mask.data_ptr()
    ref = _regular(torch, L, lib, a, d, nx, ny, torch.float32)
    out = _noalloc_twice(torch, L, lib, a, d, nx, ny, torch.float32, ref)[-1]
    dft = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, px, wgt=wgt, mask=mask, negate_v=True,
                         divide_by_n=False, center_x=2 * px, center_y=-px)
    assert O.rel_rms(out.double().cpu().numpy(), dft) < TOL


def test_noalloc_rejects_host_memory_and_oversize():
    import torch
    from wsclean_b200 import _lib as L
    lib = L.lib()
    dev = torch.device("cuda", 0)
    nx, ny, px = 128, 96, np.deg2rad(20 / 3600)
    _, _, _, d, _ = _problem(torch, dev)
    a = _args(L, lib, d, nx, ny, px)
    host_out = np.zeros((nx, ny))
    rc = lib.wsg_ms2dirty_noalloc(ctypes.byref(a), d["vis"].data_ptr(), host_out.ctypes.data, None)
    assert rc == L.WSG_ERR_INVALID and b"device" in lib.wsg_last_error()
    a.npix_x = a.npix_y = 8192   # the FP64 image alone exceeds the scratch array
    big = torch.zeros((8192, 8192), dtype=torch.float64, device=dev)
    rc = lib.wsg_ms2dirty_noalloc(ctypes.byref(a), d["vis"].data_ptr(), big.data_ptr(), None)
    assert rc == L.WSG_ERR_INVALID and b"scratch" in lib.wsg_last_error()
