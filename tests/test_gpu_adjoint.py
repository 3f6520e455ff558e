"""Adjointness of the pair: <y, A x> = <A^H y, x> (real inner product), with
the mismatch normalised by |y| |A x|; target <= 1e-6 for mixed precision."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)


@pytest.mark.parametrize("prec,eps,tol", [("mixed", 1e-5, 1e-6), ("fp64", 1e-12, 1e-12)])
@pytest.mark.parametrize("shift", [0.0, 3.0])
def test_dot_product(prec, eps, tol, shift):
    from wsclean_b200 import gridder as G
    rng = np.random.default_rng(4)
    nrow, nchan, nx, ny = 4000, 3, 96, 80
    px = np.deg2rad(25 / 3600)
    freq = np.linspace(1.3e8, 1.6e8, nchan)
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([900.0, 900.0, 400.0])
    wgt = rng.uniform(0.5, 2, (nrow, nchan))
    x = rng.normal(size=(nx, ny))
    y = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    cx, cy = shift * px, -shift * px
    Ax = G.dirty2ms(uvw, freq, x, px, px, eps, wgt=wgt, precision=prec, center_x=cx,
                    center_y=cy, vis_dtype=np.complex128, **KW)
    Aty = G.ms2dirty(uvw, freq, y, nx, ny, px, px, eps, wgt=wgt, precision=prec, center_x=cx,
                     center_y=cy, dirty_dtype=np.float64, **KW)
    a = np.vdot(y, Ax).real
    b = np.vdot(Aty, x).real
    assert abs(a - b) / (np.linalg.norm(y) * np.linalg.norm(Ax)) < tol
