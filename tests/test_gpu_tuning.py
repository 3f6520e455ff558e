"""The tuned schedule (wsg_ms2dirty_tuning / wsg_dirty2ms_tuning) on the GPU,
on wide fields where the reference's tuned calls (ducc0 ms2dirty_tuning /
dirty2ms_tuning, wgridder.h:1781-1877, through the compiled reference)
subdivide: a |w| cut with facets above it, facets only, and odd image sizes.
The subdivision reported by wsg_get_tuning must be the one the reference
prints; the results must agree with the FP64 DFT and the plain operators
within epsilon, and -- without negate_v, where the reference's faceting is
right -- with the reference's tuned results.  (With negate_v, WSClean's call,
the reference's facets come out mirrored along y: tests/test_tuning.py.)
The drop-in gridder made with tuning on runs the same schedule."""
import re

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
C = 299792458.0


def _data(nrow, wmax_m, power, seed, nchan):
    rng = np.random.default_rng(seed)
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([3000.0, 3000.0, 1.0])
    uvw[:, 2] = np.sign(uvw[:, 2]) * wmax_m * np.abs(uvw[:, 2]) ** power
    freq = np.linspace(1.4e8, 1.5e8, nchan)
    vis = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    return uvw, freq, vis, rng


def _ref_split(report):
    m = re.search(r"subdividing w range at w=(\S+), subdividing high w part into (\d+)x(\d+)", report)
    if m:
        return int(m.group(2)), int(m.group(3)), float(m.group(1))
    m = re.search(r"subdividing into (\d+)x(\d+) facets", report)
    if m:
        return int(m.group(1)), int(m.group(2)), None
    return 0, 0, None


# (precision, epsilon, tolerance against the reference's tuned result,
#  (rows, channels, image x, image y, max |w| m, |w| distribution power)):
# per form a |w| cut with facets above it, facets only, and odd sizes (the
# FP64 cost model subdivides only with fewer visibilities).  Images are not
# square with a central phase centre unless the choice is symmetric: there
# nfx x nfy and nfy x nfx cost the same up to rounding, and which one wins
# depends on how the compiler contracts the reference's arithmetic.
CASES = [
    ("mixed", 1e-5, 2e-5, (30000, 2, 1024, 1024, 5000.0, 6.0)),
    ("mixed", 1e-5, 2e-5, (20000, 1, 1024, 960, 3000.0, 1.0)),
    ("mixed", 1e-5, 2e-5, (30000, 2, 1023, 1001, 5000.0, 6.0)),
    ("fp64", 1e-12, 1e-11, (6000, 2, 1024, 1024, 8000.0, 8.0)),
    ("fp64", 1e-12, 1e-11, (3000, 1, 1024, 960, 3000.0, 1.0)),
    ("fp64", 1e-12, 1e-11, (4000, 1, 1023, 1001, 5000.0, 6.0)),
]


@pytest.fixture(scope="module")
def ctx():
    from wsclean_b200.gridder import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("prec,eps,tol,geom", CASES)
def test_tuned_matches_reference_and_dft(ctx, prec, eps, tol, geom):
    """With negate_v off, the tuned calls agree with the reference's tuned
    calls; with negate_v on (WSClean's call), where the reference mirrors its
    facets along y, they agree with the plain operator and the DFT.  Both
    ways the subdivision is the reference's and the results match the FP64
    DFT; odd sizes put pixel (i, j) at (i - n/2) pixels from the centre in
    both directions."""
    nrow, nchan, nx, ny, wmax, power = geom
    uvw, freq, vis, rng = _data(nrow, wmax, power, seed=nrow + nx + ny, nchan=nchan)
    px = np.deg2rad(60 / 3600)
    cdt = np.complex64 if prec == "mixed" else np.complex128
    fdt = np.float32 if prec == "mixed" else np.float64
    vis = vis.astype(cdt)
    rp = "float" if prec == "mixed" else "double"
    even = nx % 2 == 0 and ny % 2 == 0
    tol_dft = 1e-5 if prec == "mixed" else 1e-11
    kw0 = dict(KW, negate_v=False)
    dref, rep = O.ref_ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, prec=rp, tuning=True,
                               return_report=True, **kw0)
    rfx, rfy, rcut = _ref_split(rep)
    assert rfx > 0, rep   # the geometry is one where the reference subdivides
    model = np.zeros((nx, ny))
    model[rng.integers(0, nx, 40), rng.integers(0, ny, 40)] = rng.uniform(0.1, 3, 40)
    pix = rng.integers(0, nx * ny, 32)
    sel = rng.choice(vis.size, min(4000, vis.size), replace=False)
    for negate_v in (False, True):
        kw = dict(KW, negate_v=negate_v)
        d = ctx.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, precision=prec,
                         dirty_dtype=np.float64, tuning=True, **kw)
        t = ctx.last_tuning()
        assert (t["nfx"], t["nfy"]) == (rfx, rfy)   # the rule ignores negate_v
        if rcut is None:
            assert t["icut"] == 0
        else:
            assert t["icut"] > 0 and abs(t["wcut"] - rcut) <= 1e-5 * rcut
        dft = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, px, pixels=pix, negate_v=negate_v,
                             divide_by_n=False)
        assert O.rel_rms(d.ravel()[pix], dft) < tol_dft, negate_v
        if not negate_v:
            assert O.rel_rms(d, dref.astype(np.float64)) < tol
        if even:
            dp = ctx.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, precision=prec,
                              dirty_dtype=np.float64, **kw)
            assert O.rel_rms(d, dp) < tol
        v = ctx.dirty2ms(uvw, freq, model.astype(fdt), px, px, eps, precision=prec,
                         vis_dtype=np.complex128, tuning=True, **kw)
        assert (ctx.last_tuning()["nfx"], ctx.last_tuning()["nfy"]) == (rfx, rfy)
        vdft = O.dft_dirty2ms(uvw, freq, model, px, px, negate_v=negate_v, divide_by_n=False,
                              select=sel)
        assert O.rel_rms(v.ravel()[sel], vdft) < tol_dft, negate_v
        if not negate_v and even:
            vr = O.ref_dirty2ms(uvw, freq, model.astype(fdt), px, px, eps, prec=rp, tuning=True,
                                vis_dtype=cdt, **kw0)
            assert O.rel_rms(v, vr.astype(np.complex128)) < tol


def test_tuned_pair_is_adjoint_on_odd_sizes(ctx):
    """<y, A x> = <A^H y, x> for the tuned pair on an odd image with negate_v."""
    uvw, freq, vis, rng = _data(4000, 5000.0, 6.0, seed=5, nchan=1)
    nx, ny = 1023, 1001
    px = np.deg2rad(60 / 3600)
    x = rng.normal(size=(nx, ny))
    y = vis
    Ax = ctx.dirty2ms(uvw, freq, x, px, px, 1e-12, precision="fp64", vis_dtype=np.complex128,
                      tuning=True, **KW)
    assert ctx.last_tuning()["nfx"] > 0
    Aty = ctx.ms2dirty(uvw, freq, y, nx, ny, px, px, 1e-12, precision="fp64",
                       dirty_dtype=np.float64, tuning=True, **KW)
    a = np.vdot(y.ravel(), Ax.ravel()).real
    b = np.vdot(Aty.ravel(), x.ravel()).real
    assert abs(a - b) / (np.linalg.norm(y) * np.linalg.norm(Ax)) < 1e-12


def test_tuned_accumulate_weights_and_device_inputs(ctx):
    """accumulate adds to the caller's image; weights and a mask restrict
    the parts; torch device tensors are used in place."""
    uvw, freq, vis, rng = _data(30000, 5000.0, 6.0, seed=11, nchan=2)
    nx = ny = 1024
    px = np.deg2rad(60 / 3600)
    vis = vis.astype(np.complex64)
    wgt = rng.uniform(0.5, 2, vis.shape).astype(np.float32)
    mask = (rng.uniform(size=vis.shape) > 0.2).astype(np.uint8)
    # (WSClean's arguments, negate_v: the plain reference operator is the check)
    dref = O.ref_ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-5, prec="float", wgt=wgt, mask=mask,
                          **KW)
    dev = torch.device("cuda", 0)
    base = torch.ones((nx, ny), dtype=torch.float64, device=dev)
    out = base.clone()
    ctx.ms2dirty(torch.as_tensor(uvw, device=dev), torch.as_tensor(freq, device=dev),
                 torch.as_tensor(vis, device=dev), nx, ny, px, px, 1e-5,
                 wgt=torch.as_tensor(wgt, device=dev), mask=torch.as_tensor(mask, device=dev),
                 dirty=out, accumulate=True, tuning=True, **KW)
    assert ctx.last_tuning()["nfx"] > 0
    assert O.rel_rms((out - base).cpu().numpy(), dref.astype(np.float64)) < 2e-5


def test_dropin_gridder_with_tuning():
    """WGriddingGridder_Simple(..., tuning=true) runs the tuned schedule in
    AddInversionData and PredictVisibilities (wgriddinggridder_simple.cpp:59-63,
    :109-113)."""
    from wsclean_b200.gridder import WGriddingGridder
    uvw, freq, vis, rng = _data(30000, 5000.0, 6.0, seed=12, nchan=2)
    vis = vis.astype(np.complex64)
    n = 1024
    px = np.deg2rad(60 / 3600)
    g = WGriddingGridder(n, n, n, n, px, px, 0.0, 0.0, 4, 1e-4, 0, True, "mixed")
    g.InitializeInversion()
    g.AddInversionData(uvw, freq, vis)
    t = g.last_tuning()
    assert t["nfx"] > 0
    img = g.RealImage()
    # WSClean's arguments (negate_v): the plain reference operator is the
    # check (the reference's own tuned result mirrors its facets here)
    dref = O.ref_ms2dirty(uvw, freq, vis, n, n, px, px, 1e-4, prec="float", **KW)
    assert O.rel_rms(img.T.astype(np.float64), dref.astype(np.float64)) < 2e-4
    model = np.zeros((n, n), np.float32)
    model[rng.integers(0, n, 30), rng.integers(0, n, 30)] = 1.0
    g.InitializePrediction(model)
    v = g.PredictVisibilities(uvw, freq)
    assert g.last_tuning()["nfx"] > 0
    vref = O.ref_dirty2ms(uvw, freq, model.T.copy(), px, px, 1e-4, prec="float", **KW)
    assert O.rel_rms(v, vref) < 2e-4
    g.close()
