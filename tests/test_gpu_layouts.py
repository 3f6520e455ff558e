"""Awkward image geometries for the u transform's segmented rows: widths that
are not multiples of 32, unequal sides, and u bands narrow enough that the
transform of an image column runs as several twisted passes (nu = K M with
K > 1, so each row holds K segments); and long rows whose transform length
M is 4096 or 8192.  Both precisions, both directions, against the FP64 DFT,
plus the adjoint identity."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
C = 299792458.0
# (nx, ny): odd multiples of 2, one side far from a multiple of 32
CASES = [(1000, 1002), (1234, 778), (258, 1030), (998, 64)]
TOL = {"mixed": (1e-5, 1e-5), "fp64": (1e-12, 1e-11)}  # (epsilon, tolerance vs DFT)


@pytest.fixture(scope="module")
def ctx():
    from wsclean_b200.gridder import Context
    c = Context(0)
    yield c
    c.close()


def _problem(nx, ny, seed, frac=0.12):
    rng = np.random.default_rng(seed)
    nrow, nchan = 4000, 2
    px = np.deg2rad(10 / 3600)
    freq = np.array([1.40e8, 1.45e8])
    # |u|, |v| up to 0.12 / px wavelengths: the data fill about a quarter of
    # the grid along u, so the pruned u transform needs K > 1 passes
    umax = frac / px * C / freq.max()
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([umax, umax, 0.2 * umax])
    vis = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    return rng, uvw, freq, vis, px


def _check(ctx, prec, nx, ny, rng, uvw, freq, vis, px, kw):
    """ms2dirty and dirty2ms against the DFT, and their adjoint identity;
    returns the grid statistics of the ms2dirty call."""
    eps, tol = TOL[prec]
    d = ctx.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, precision=prec,
                     dirty_dtype=np.float64, **kw)
    st = ctx.stats()
    pix = np.concatenate([rng.integers(0, nx * ny, 48), [0, ny - 1, (nx - 1) * ny, nx * ny - 1]])
    dft = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, px, negate_v=True, divide_by_n=False,
                         pixels=pix)
    assert O.rel_rms(d.ravel()[pix], dft) < tol
    # prediction of a sparse model, including the image's corner pixels
    model = np.zeros((nx, ny))
    model[rng.integers(0, nx, 30), rng.integers(0, ny, 30)] = rng.uniform(0.5, 2, 30)
    model[0, 0] = model[nx - 1, ny - 1] = model[0, ny - 1] = model[nx - 1, 0] = 1.0
    fdt = np.float32 if prec == "mixed" else np.float64
    v = ctx.dirty2ms(uvw, freq, model.astype(fdt), px, px, eps, precision=prec,
                     vis_dtype=np.complex128, **kw)
    sel = rng.choice(v.size, 3000, replace=False)
    vdft = O.dft_dirty2ms(uvw, freq, model, px, px, negate_v=True, divide_by_n=False, select=sel)
    assert O.rel_rms(v.ravel()[sel], vdft) < tol
    # <y, A x> = <A^H y, x> with A = dirty2ms
    x = rng.normal(size=(nx, ny))
    ax = ctx.dirty2ms(uvw, freq, x.astype(fdt), px, px, eps, precision=prec,
                      vis_dtype=np.complex128, **kw)
    aty = ctx.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, precision=prec,
                       dirty_dtype=np.float64, **kw)
    a = np.vdot(vis.astype(np.complex128).ravel(), ax.ravel()).real
    b = np.vdot(aty.ravel(), x.ravel()).real
    assert abs(a - b) / (np.linalg.norm(vis) * np.linalg.norm(ax)) < (1e-6 if prec == "mixed" else 1e-12)
    return st


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("nx,ny", CASES)
def test_segmented_rows_match_dft_and_adjoint(ctx, prec, nx, ny):
    rng, uvw, freq, vis, px = _problem(nx, ny, nx * 7 + ny)
    vis = vis.astype(np.complex64 if prec == "mixed" else np.complex128)
    st = _check(ctx, prec, nx, ny, rng, uvw, freq, vis, px, KW)
    assert 2 * st["band_rows"] <= st["nu"]  # a pruned band: K = nu / M >= 2


# Long image rows whose u transform is 4096 or 8192 points long: one CTA then
# holds one column's transform (in single precision two adjacent columns
# share a CTA; an FP64 8192-point transform reads its last stage's twiddles
# from global memory).  (nx, ny, max |u| px, nu, transform length M)
WIDE = [(2000, 64, 0.45, 4096, 4096), (4000, 64, 0.2, 8192, 4096),
        (4200, 32, 0.45, 8192, 8192), (6000, 32, 0.2, 16384, 8192)]


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("nx,ny,frac,nu,m", WIDE)
def test_long_transforms_match_dft_and_adjoint(ctx, prec, nx, ny, frac, nu, m):
    rng, uvw, freq, vis, px = _problem(nx, ny, nx + ny, frac)
    vis = vis.astype(np.complex64 if prec == "mixed" else np.complex128)
    st = _check(ctx, prec, nx, ny, rng, uvw, freq, vis, px, dict(KW, sigma_min=1.5))
    # M: the band rounded up to a power of two; K = nu / M passes
    assert st["nu"] == nu
    assert 1 << int(np.ceil(np.log2(st["band_rows"]))) == m


# Occupied u bands wider than the longest pruned column transform (8192
# points): the grid keeps every u row (nu of any 2,3,5,7-smooth length) and
# the u transform runs over whole grid columns; once with all w planes in
# one pass, once five planes a pass.
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("max_planes", [0, 5])
def test_bands_wider_than_the_pruned_transform(ctx, monkeypatch, prec, max_planes):
    nx, ny, frac = 6000, 32, 0.45
    if max_planes:
        monkeypatch.setenv("WSG_MAX_PLANES", str(max_planes))
    rng, uvw, freq, vis, px = _problem(nx, ny, 77 + max_planes, frac)
    vis = vis.astype(np.complex64 if prec == "mixed" else np.complex128)
    st = _check(ctx, prec, nx, ny, rng, uvw, freq, vis, px, dict(KW, sigma_min=1.5))
    assert st["band_rows"] == st["nu"] > 8192
    if max_planes:
        assert st["plane_batch"] <= max_planes < st["nplanes"]
