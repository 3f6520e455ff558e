"""Seeded synthetic observations with the shapes of the benchmark configurations.

No measurement set is available, so every input is generated: antenna
layouts, Earth-rotation uvw tracks, point-source skies with a power-law flux
distribution, and their FP64 visibilities.  Conventions follow the w-gridder
(v negated at the gridder call, u,v,w in metres, frequencies in Hz).

Observatory latitude: -26.7 deg.  Rows are time-major (all baselines of one
timestep, then the next), as a measurement set stores them.
"""
from __future__ import annotations

import math

import numpy as np

C_LIGHT = 299792458.0
LATITUDE = np.deg2rad(-26.7)
ARCSEC = np.pi / (180 * 3600)


def antenna_layout(n, radius_m, rng, log_radial=False, r_min=50.0):
    """East/north positions of n antennas in a disk (uniform in area) or with
    log-uniform radii between r_min and radius_m."""
    if log_radial:
        r = r_min * (radius_m / r_min) ** rng.uniform(0, 1, n)
    else:
        r = radius_m * np.sqrt(rng.uniform(0, 1, n))
    phi = rng.uniform(0, 2 * np.pi, n)
    return np.stack([r * np.cos(phi), r * np.sin(phi), np.zeros(n)], axis=1)


def baselines(n):
    i, j = np.triu_indices(n, k=1)
    return i, j


def earth_rotation_uvw(enu, hour_angles, dec, lat=LATITUDE):
    """uvw (metres) for all i<j baselines and hour angles, time-major rows."""
    e, nn, up = enu[:, 0], enu[:, 1], enu[:, 2]
    # local ENU -> equatorial XYZ
    X = -np.sin(lat) * nn + np.cos(lat) * up
    Y = e
    Z = np.cos(lat) * nn + np.sin(lat) * up
    i, j = baselines(len(enu))
    bx, by, bz = X[j] - X[i], Y[j] - Y[i], Z[j] - Z[i]
    H = np.asarray(hour_angles)[:, None]
    sd, cd = np.sin(dec), np.cos(dec)
    u = np.sin(H) * bx + np.cos(H) * by
    v = -sd * np.cos(H) * bx + sd * np.sin(H) * by + cd * bz
    w = cd * np.cos(H) * bx - cd * np.sin(H) * by + sd * bz
    return np.stack([u.ravel(), v.ravel(), w.ravel()], axis=1)


def scale_w(uvw, frac):
    """Rescale w so that max|w| = frac * max|(u,v)| (the stated wide-field
    w range of the configurations)."""
    uvmax = np.max(np.hypot(uvw[:, 0], uvw[:, 1]))
    wmax = np.max(np.abs(uvw[:, 2]))
    out = uvw.copy()
    if wmax > 0:
        out[:, 2] *= frac * uvmax / wmax
    return out


def power_law_flux(n, rng, index=-1.6, smin=0.01, smax=10.0):
    """Inverse-CDF draws from dN/dS ~ S^index on [smin, smax]."""
    a = index + 1.0
    u = rng.uniform(0, 1, n)
    return (smin ** a + u * (smax ** a - smin ** a)) ** (1.0 / a)


def point_sky(n, npix_x, npix_y, rng, margin=0.1):
    """n point sources at pixel centres away from the edges: (ix, iy, flux)."""
    lo_x, hi_x = int(margin * npix_x), int((1 - margin) * npix_x)
    lo_y, hi_y = int(margin * npix_y), int((1 - margin) * npix_y)
    ix = rng.integers(lo_x, hi_x, n)
    iy = rng.integers(lo_y, hi_y, n)
    return ix, iy, power_law_flux(n, rng)


def sky_image(npix_x, npix_y, ix, iy, flux):
    img = np.zeros((npix_x, npix_y))
    np.add.at(img, (ix, iy), flux)
    return img


def pixel_lm(ix, iy, npix_x, npix_y, px, py, center_x=0.0, center_y=0.0, negate_v=True):
    """(l, m') of pixels in the gridder's convention: l = cx + (i - nx/2) px,
    m' = my + (j - ny/2) py with my = -cy when v is negated."""
    ms = -center_y if negate_v else center_y
    return center_x + (ix - npix_x / 2) * px, ms + (iy - npix_y / 2) * py


def predict_vis(uvw, freq, npix_x, npix_y, px, py, ix, iy, flux, negate_v=True,
                center_x=0.0, center_y=0.0, chunk=1 << 18, device=None):
    """FP64 visibilities of point sources at pixels (ix, iy): the exact
    transform that dirty2ms approximates.  Uses torch on `device` if given."""
    l, m = pixel_lm(np.asarray(ix, float), np.asarray(iy, float), npix_x, npix_y, px, py,
                    center_x, center_y, negate_v)
    nm1 = -(l * l + m * m) / (np.sqrt(1 - l * l - m * m) + 1)
    vfac = -1.0 if negate_v else 1.0
    nrows, nchan = uvw.shape[0], len(freq)
    if device is not None:
        import torch
        dev = torch.device(device)
        U = torch.as_tensor(uvw, dtype=torch.float64, device=dev)
        L = torch.as_tensor(np.stack([l, vfac * m, -nm1]), dtype=torch.float64, device=dev)
        Fl = torch.as_tensor(flux, dtype=torch.float64, device=dev)
        out = torch.empty((nrows, nchan), dtype=torch.complex128, device=dev)
        for c, f in enumerate(freq):
            for r0 in range(0, nrows, chunk):
                ph = (U[r0:r0 + chunk] * (f / C_LIGHT)) @ L
                ph = ph - torch.round(ph)
                out[r0:r0 + chunk, c] = torch.exp(-2j * math.pi * ph) @ Fl.to(torch.complex128)
        return out.cpu().numpy()
    out = np.empty((nrows, nchan), dtype=np.complex128)
    Lm = np.stack([l, vfac * m, -nm1])
    for c, f in enumerate(freq):
        for r0 in range(0, nrows, chunk):
            ph = (uvw[r0:r0 + chunk] * (f / C_LIGHT)) @ Lm
            ph -= np.round(ph)
            out[r0:r0 + chunk, c] = np.exp(-2j * np.pi * ph) @ flux
    return out


def observation(nant, radius_m, hours, cadence_s, dec_deg, freq, seed, wfrac=None,
                log_radial=False, ntimes=None):
    rng = np.random.default_rng(seed)
    enu = antenna_layout(nant, radius_m, rng, log_radial=log_radial)
    nt = ntimes if ntimes is not None else int(round(hours * 3600 / cadence_s))
    ha = np.linspace(-0.5, 0.5, nt) * (nt * cadence_s / 3600.0) * (2 * np.pi / 24.0)
    uvw = earth_rotation_uvw(enu, ha, np.deg2rad(dec_deg))
    if wfrac is not None:
        uvw = scale_w(uvw, wfrac)
    return uvw, np.asarray(freq, dtype=np.float64), rng


# The benchmark configurations (seeds 1..5).  `scale` < 1 shrinks the number
# of timesteps (and the image) for quick tests while keeping the geometry.
def config2(scale=1.0, npix=4096, pixsize_arcsec=5.0):
    """128 antennas within 6 km, 8 s cadence, 1 channel at 150 MHz, |w| up to
    30% of max|uv|; 997 timesteps give the stated ~8.1M visibilities."""
    nt = max(2, int(round(997 * scale)))
    uvw, freq, rng = observation(128, 6000.0, None, 8.0, -30.0, [150e6], seed=2, wfrac=0.3,
                                 ntimes=nt)
    return dict(uvw=uvw, freq=freq, rng=rng, npix_x=npix, npix_y=npix,
                pixsize=pixsize_arcsec * ARCSEC, nsrc=200)


def config1(scale=1.0, npix=1024):
    """64 antennas within 3 km, 1 h at 10 s, 4 channels 150-151.5 MHz."""
    nt = max(2, int(round(360 * scale)))
    uvw, freq, rng = observation(64, 3000.0, None, 10.0, -30.0,
                                 np.linspace(150e6, 151.5e6, 4), seed=1, ntimes=nt)
    return dict(uvw=uvw, freq=freq, rng=rng, npix_x=npix, npix_y=npix,
                pixsize=10.0 * ARCSEC, nsrc=20)


def config3(scale=1.0, npix=2048, pixsize_arcsec=8.0):
    """The config-2 array and sky imaged at 2048^2 and 8" pixels (the
    chi^2-gradient configuration); Briggs weights come from briggs_weights."""
    return config2(scale=scale, npix=npix, pixsize_arcsec=pixsize_arcsec)


def config4(scale=1.0):
    """96 antennas within 10 km, 1 h at 10 s (360 timesteps), 64 channels at
    120-180 MHz, dec -30 deg; a 4096^2 field of 10" pixels cut into the 16
    facets of facets4().  Each of the 8 output channels covers 8 input
    channels."""
    nt = max(2, int(round(360 * scale)))
    freq = 120e6 + (np.arange(64) + 0.5) * (60e6 / 64)
    uvw, freq, rng = observation(96, 10000.0, None, 10.0, -30.0, freq, seed=4, ntimes=nt)
    return dict(uvw=uvw, freq=freq, rng=rng, npix_x=4096, npix_y=4096,
                pixsize=10.0 * ARCSEC, nsrc=200, out_channels=8)


def facets4(npix=4096, nfacets=16, seed=4, min_box=512, max_box=2048):
    """Seeded Voronoi facets of an npix^2 field: for each site, the bounding
    box of its Voronoi cell (on a coarse raster), its sides clamped to
    [min_box, max_box] and made even.  Returns a list of dicts with the box
    size (nx, ny) and its centre offset from the field centre in pixels
    (dx, dy): the facet's phase centre is l = dx * pixsize, m = dy * pixsize."""
    rng = np.random.default_rng(seed)
    sites = rng.uniform(0, npix, (nfacets, 2))
    step = 16
    g = (np.arange(0, npix, step) + step / 2)
    X, Y = np.meshgrid(g, g, indexing="ij")
    d2 = (X[..., None] - sites[:, 0]) ** 2 + (Y[..., None] - sites[:, 1]) ** 2
    owner = np.argmin(d2, axis=-1)
    out = []
    for f in range(nfacets):
        xs, ys = X[owner == f], Y[owner == f]
        x0, x1 = xs.min() - step / 2, xs.max() + step / 2
        y0, y1 = ys.min() - step / 2, ys.max() + step / 2
        nx = int(np.clip(x1 - x0, min_box, max_box)) // 2 * 2
        ny = int(np.clip(y1 - y0, min_box, max_box)) // 2 * 2
        cx, cy = 0.5 * (x0 + x1), 0.5 * (y0 + y1)
        out.append(dict(nx=nx, ny=ny, dx=cx - npix / 2, dy=cy - npix / 2))
    return out


def config5(scale=1.0):
    """256 antennas with log-radial radii out to 20 km, 1000 timesteps at 8 s,
    16 channels at 140-190 MHz, dec -30 deg, |w| up to 40% of max|uv|;
    8192^2 at 2" (about 522M visibilities at scale 1)."""
    nt = max(2, int(round(1000 * scale)))
    freq = np.linspace(140e6, 190e6, 16)
    uvw, freq, rng = observation(256, 20000.0, None, 8.0, -30.0, freq, seed=5, wfrac=0.4,
                                 log_radial=True, ntimes=nt)
    return dict(uvw=uvw, freq=freq, rng=rng, npix_x=8192, npix_y=8192,
                pixsize=2.0 * ARCSEC, nsrc=2000, ngauss=5)


def gaussian_blobs(npix_x, npix_y, n, rng, sigma_px=(2.0, 8.0), flux=(0.5, 5.0)):
    """n seeded Gaussian extended sources as a pixel image (each truncated
    at 4 sigma)."""
    img = np.zeros((npix_x, npix_y))
    for _ in range(n):
        s = rng.uniform(*sigma_px)
        cx = rng.uniform(0.2, 0.8) * npix_x
        cy = rng.uniform(0.2, 0.8) * npix_y
        h = int(np.ceil(4 * s))
        ix = np.arange(int(cx) - h, int(cx) + h + 1)
        iy = np.arange(int(cy) - h, int(cy) + h + 1)
        g = np.exp(-0.5 * (((ix[:, None] - cx) ** 2 + (iy[None, :] - cy) ** 2) / s ** 2))
        img[np.ix_(ix, iy)] += rng.uniform(*flux) * g / g.sum()
    return img


def briggs_weights(uvw, freq, nx, ny, px, py, robust=0.0, noise_weights=None):
    """Briggs imaging weights with WSClean's ImageWeights semantics
    (structures/imageweights.cpp:113-143, cell lookup imageweights.h:73-80):
    the weights are summed on a half-plane (v >= 0) grid of nx x ny/2 cells of
    1/(n*pixelscale) wavelengths, and each visibility gets
    1 / (1 + W_cell * s^2) with s^2 = (5*10^-robust)^2 / (sum W^2 / sum W)."""
    nrows, nchan = uvw.shape[0], len(freq)
    w = np.ones((nrows, nchan)) if noise_weights is None else np.asarray(noise_weights, float)
    u = uvw[:, 0:1] * (np.asarray(freq)[None, :] / C_LIGHT)
    v = uvw[:, 1:2] * (np.asarray(freq)[None, :] / C_LIGHT)
    flip = v < 0
    u = np.where(flip, -u, u)
    v = np.where(flip, -v, v)
    x = np.floor(u * nx * px + nx // 2).astype(np.int64)
    y = np.floor(v * ny * py).astype(np.int64)
    ok = (x >= 0) & (x < nx) & (y < ny // 2)
    grid = np.zeros(nx * (ny // 2))
    np.add.at(grid, (x[ok] + y[ok] * nx), w[ok])
    total = w[ok].sum()
    avg = np.sum(grid * grid) / total
    s2 = (5.0 * np.exp(-np.log(10.0) * robust)) ** 2 / avg
    cell = np.where(ok, grid[np.where(ok, x + y * nx, 0)], 0.0)
    return np.where(ok, 1.0 / (1.0 + cell * s2), 0.0)
