"""The tuned schedule's subdivision, on the CPU.

wsg_tuning_choice restates the reference's rule for ms2dirty_tuning /
dirty2ms_tuning (get_tuning_parameters, wgridder.cc:144-278): from the 50-bin
|w| histogram of the masked-in visibilities it picks no subdivision, facets,
or a |w| cut with facets above it.  Here the same histogram is formed in
numpy (get_winfo, wgridder.cc:28-89) and the choice is compared with the one
the compiled reference prints in its verbosity report for the same data.
"""
import ctypes
import re

import numpy as np
import pytest

import oracle as O

C = 299792458.0


def _whist(uvw, freq, mask=None):
    aw = np.abs(uvw[:, 2:3] * (freq[None, :] / C))
    if mask is not None:
        aw = aw[mask.astype(bool)]
    aw = aw.ravel()
    wmin, wmax = aw.min(), aw.max()
    xdw = 50 / (wmax - wmin)
    b = np.minimum(((aw - wmin) * xdw).astype(np.uint64), 49)
    return wmin, wmax, np.bincount(b.astype(np.int64), minlength=50).astype(np.uint64)


def _ours(uvw, freq, nx, ny, px, eps, mask=None, center=(0.0, 0.0)):
    from wsclean_b200 import _lib as L
    lib = L.lib()
    a = L.WsgArgs()
    lib.wsg_args_init(ctypes.byref(a))
    a.nrows, a.nchan = uvw.shape[0], len(freq)
    a.npix_x, a.npix_y = nx, ny
    a.pixsize_x = a.pixsize_y = px
    a.epsilon = eps
    a.do_wgridding = 1
    a.center_x, a.center_y = center
    wmin, wmax, hist = _whist(uvw, freq, mask)
    h = (ctypes.c_uint64 * 50)(*[int(x) for x in hist])
    nfx, nfy, icut = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.check(lib.wsg_tuning_choice(ctypes.byref(a), uvw.shape[0] * len(freq), wmin, wmax, h,
                                  ctypes.byref(nfx), ctypes.byref(nfy), ctypes.byref(icut)))
    if nfx.value == 0:
        return "no subdivision"
    if icut.value == 0:
        return f"{nfx.value}x{nfy.value} facets"
    return f"w={wmin + icut.value * (wmax - wmin) / 50:.6g} {nfx.value}x{nfy.value} facets"


def _reference(report):
    m = re.search(r"subdividing w range at w=(\S+), subdividing high w part into (\d+)x(\d+)", report)
    if m:
        return f"w={float(m.group(1)):.6g} {m.group(2)}x{m.group(3)} facets"
    m = re.search(r"subdividing into (\d+)x(\d+) facets", report)
    if m:
        return f"{m.group(1)}x{m.group(2)} facets"
    assert "no subdivision" in report, report
    return "no subdivision"


def _data(nrow, wmax_m, power, seed, nchan=1):
    rng = np.random.default_rng(seed)
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([3000.0, 3000.0, 1.0])
    uvw[:, 2] = np.sign(uvw[:, 2]) * wmax_m * np.abs(uvw[:, 2]) ** power
    freq = np.linspace(1.4e8, 1.5e8, nchan)
    vis = (rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))).astype(np.complex64)
    return uvw, freq, vis, rng


# (rows, image, pixel arcsec, max |w| m, |w| distribution power, epsilon, channels)
CASES = [
    (20000, 1024, 60.0, 3000.0, 1.0, 1e-5, 1),   # facets only
    (30000, 1024, 60.0, 5000.0, 6.0, 1e-5, 2),   # w cut, facets above it
    (30000, 1000, 60.0, 5000.0, 4.0, 1e-4, 1),   # another cut and facet count
    (50000, 512, 10.0, 3000.0, 1.0, 1e-5, 1),    # narrow field: no subdivision
    (4000, 400, 60.0, 5000.0, 1.0, 1e-5, 1),     # below 500 pixels: no subdivision
]


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference missing")
@pytest.mark.parametrize("nrow,nx,pxas,wmax,power,eps,nchan", CASES)
def test_tuning_choice_matches_reference(nrow, nx, pxas, wmax, power, eps, nchan):
    uvw, freq, vis, _ = _data(nrow, wmax, power, seed=nrow + nx, nchan=nchan)
    px = np.deg2rad(pxas / 3600)
    _, rep = O.ref_ms2dirty(uvw, freq, vis, nx, nx, px, px, eps, prec="float", tuning=True,
                            return_report=True)
    assert _ours(uvw, freq, nx, nx, px, eps) == _reference(rep)


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference missing")
def test_tuning_choice_with_mask_and_shift():
    """The histogram counts masked-in visibilities only, and the field
    centre moves the n-1 range that decides the facet split."""
    uvw, freq, vis, rng = _data(30000, 5000.0, 6.0, seed=7)
    mask = (rng.uniform(size=vis.shape) > 0.3).astype(np.uint8)
    px = np.deg2rad(60 / 3600)
    center = (40 * px, -25 * px)
    _, rep = O.ref_ms2dirty(uvw, freq, vis, 1024, 1024, px, px, 1e-5, prec="float", mask=mask,
                            tuning=True, center_x=center[0], center_y=center[1],
                            return_report=True)
    assert _ours(uvw, freq, 1024, 1024, px, 1e-5, mask=mask, center=center) == _reference(rep)


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference missing")
def test_reference_tuned_facets_mirror_with_negate_v():
    """A property of the reference that the tuned schedule here does not
    copy: its faceting (get_facet_data, wgridder.cc:92-108) moves each
    facet's centre_y the same way whether or not v is negated, so with
    negate_v -- WSClean's call, wgriddinggridder_simple.cpp:59-63 -- the
    facets of a subdivided image land mirrored along y.  Without negate_v its
    tuned image matches its plain one and the DFT; with it, it does not."""
    uvw, freq, vis, rng = _data(20000, 3000.0, 1.0, seed=21)
    px = np.deg2rad(60 / 3600)
    pix = rng.integers(0, 1024 * 1024, 16)
    err = {}
    for nv in (False, True):
        kw = dict(negate_v=nv, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
        dt, rep = O.ref_ms2dirty(uvw, freq, vis, 1024, 1024, px, px, 1e-5, prec="float",
                                 tuning=True, return_report=True, **kw)
        assert _reference(rep) != "no subdivision"
        dft = O.dft_ms2dirty(uvw, freq, vis, 1024, 1024, px, px, pixels=pix, negate_v=nv,
                             divide_by_n=False)
        err[nv] = O.rel_rms(dt.ravel()[pix], dft)
    assert err[False] < 1e-5
    assert err[True] > 0.1
