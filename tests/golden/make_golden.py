"""Generates the golden fixtures in this directory by running the reference's
own w-gridder (ducc0 as vendored by WSClean, compiled from the reference
sources by oracle/Makefile into oracle/_ref) on small seeded inputs with
WSClean's argument pattern (wgridder/wgriddinggridder_simple.cpp:56-58,
106-108), together with the FP64 direct Fourier transform of the same inputs.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

CASES = [
    # name, seed, nrow, nchan, npix, fov pixel arcsec, center shift (pixels), eps, prec
    ("small_f32", 1, 2000, 2, 64, 30.0, (0, 0), 1e-5, "float"),
    ("small_f64", 2, 2000, 2, 64, 30.0, (0, 0), 1e-12, "double"),
    ("shift_f32", 3, 1500, 3, 48, 40.0, (3, -5), 1e-5, "float"),
    ("shift_f64", 4, 1500, 3, 48, 40.0, (-2, 4), 1e-12, "double"),
    ("rect_f64", 5, 1200, 1, 0, 25.0, (1, 2), 1e-9, "double"),
]


def make(name, seed, nrow, nchan, npix, pixas, shift, eps, prec):
    rng = np.random.default_rng(seed)
    nx, ny = (npix, npix) if npix else (56, 40)
    px = np.deg2rad(pixas / 3600)
    py = px * (1.25 if not npix else 1.0)
    freq = np.linspace(1.4e8, 1.6e8, nchan) if nchan > 1 else np.array([1.5e8])
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([700.0, 700.0, 250.0])
    vis = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    wgt = rng.uniform(0.5, 2.0, (nrow, nchan))
    mask = (rng.uniform(size=(nrow, nchan)) > 0.05).astype(np.uint8)
    cx, cy = shift[0] * px, shift[1] * py
    vdt = np.complex64 if prec == "float" else np.complex128
    wdt = np.float32 if prec == "float" else np.float64
    vis = vis.astype(vdt)
    wgt = wgt.astype(wdt)
    kw = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0,
              center_x=cx, center_y=cy, nthreads=4)
    dirty_ref = O.ref_ms2dirty(uvw, freq, vis, nx, ny, px, py, eps, wgt=wgt, mask=mask,
                               prec=prec, **kw)
    dirty_dft = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, py, wgt=wgt, mask=mask,
                               negate_v=True, divide_by_n=False, center_x=cx, center_y=cy)
    model = np.zeros((nx, ny))
    k = rng.integers(0, nx * ny, 15)
    model.ravel()[k] = rng.normal(size=15)
    vis_ref = O.ref_dirty2ms(uvw, freq, model, px, py, eps, wgt=wgt, mask=mask, prec=prec,
                             vis_dtype=vdt, **kw)
    vis_dft = O.dft_dirty2ms(uvw, freq, model, px, py, wgt=wgt, mask=mask, negate_v=True,
                             divide_by_n=False, center_x=cx, center_y=cy)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), uvw=uvw, freq=freq, vis=vis, wgt=wgt,
                        mask=mask, npix=np.array([nx, ny]), pixsize=np.array([px, py]),
                        center=np.array([cx, cy]), eps=np.array(eps), prec=np.array(prec),
                        dirty_ref=dirty_ref, dirty_dft=dirty_dft, model=model,
                        vis_ref=vis_ref, vis_dft=vis_dft)
    print(name, "ref vs dft:", O.rel_rms(dirty_ref, dirty_dft), O.rel_rms(vis_ref, vis_dft))


if __name__ == "__main__":
    for c in CASES:
        make(*c)
