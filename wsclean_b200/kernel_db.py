"""Generator for the exponential-of-semicircle (ES) kernel table.

The w-gridder spreads each visibility with a separable kernel
phi(t) = exp(beta*W*((1-t^2)^e0 - 1)), |t| <= 1, spanning W grid cells per
axis (the two-parameter ES family ducc0 uses, external/wgridder/ducc0/math/
gridding_kernel.cc:1538-1543).  The reference ships a fixed table of
(W, oversampling, epsilon, beta, e0) rows (gridding_kernel.cc:78-1536); this
module derives this project's own table from first principles instead:

* For a support W and oversampling factor sigma = (grid size)/(image size),
  the gridded, FFT-ed and corrected image at frequency k (cycles per grid
  cell, |k| <= 1/(2 sigma)) carries the aliases Phi(k+m), m != 0, where Phi
  is the kernel's Fourier transform in cell units.  The 1-D error estimate is

      err1d(W, sigma; beta, e0) = max_{0<=k<=1/(2 sigma)}
                                  sqrt(sum_{m != 0} Phi(k+m)^2) / Phi(k)

  (the root-sum-square of the aliased power relative to the kept power; the
  aliases add with effectively random phases over many visibilities).
* beta and e0 are chosen per (W, sigma) by minimising log(err1d) with
  Nelder-Mead, starting from the classic ES value beta=2.3, e0=0.5.
* The error estimate for an n-dimensional gridding (2 for u,v; 3 when
  w-gridding adds the w axis with the same oversampling) is n * err1d.

Running ``python -m wsclean_b200.kernel_db`` rewrites
``wsclean_b200/csrc/es_kernel_db.inc``, the table compiled into libwsg.
"""
from __future__ import annotations

import os
import sys

import numpy as np

W_RANGE = range(4, 17)
SIGMA_GRID = [round(1.15 + 0.05 * i, 2) for i in range(28)]  # 1.15 .. 2.50
N_ALIAS = 12      # aliases m = -N..N (further aliases change err1d by < 1e-3 relative)
N_K = 32          # image-side sample points in [0, 1/(2 sigma)]
N_PANEL = 128     # composite Gauss-Legendre on [0, 1]: panels x nodes per panel.
N_NODE = 16       # (one global rule stalls near 1e-12: phi has a branch point at |t|=1)


def es_kernel(t, W, beta, e0):
    """phi(t) for |t|<=1 (0 outside), beta in per-cell units as in the table."""
    t = np.asarray(t, dtype=np.float64)
    s = np.clip((1.0 - t) * (1.0 + t), 0.0, None)
    return np.where(np.abs(t) <= 1.0, np.exp(beta * W * (s ** e0 - 1.0)), 0.0)


class _Transform:
    """Phi(nu) = (W/2) * int_{-1}^{1} phi(t) cos(pi W nu t) dt on a fixed nu set."""

    def __init__(self, W, nu):
        x, g = np.polynomial.legendre.leggauss(N_NODE)
        edges = np.linspace(0.0, 1.0, N_PANEL + 1)
        h = np.diff(edges)
        t = (edges[:-1, None] + 0.5 * h[:, None] * (x[None, :] + 1.0)).ravel()
        gw = (0.5 * h[:, None] * g[None, :]).ravel()
        self.t = t
        # even integrand: int_{-1}^{1} = 2 int_0^1
        self.mat = (W * gw)[None, :] * np.cos(np.pi * W * np.outer(nu, t))
        self.W = W

    def __call__(self, beta, e0):
        return self.mat @ es_kernel(self.t, self.W, beta, e0)


def _alias_transform(W, sigma):
    k = np.linspace(0.0, 0.5 / sigma, N_K)
    m = np.arange(-N_ALIAS, N_ALIAS + 1)
    return _Transform(W, (k[:, None] + m[None, :]).ravel()), len(k), len(m)


def err1d(W, sigma, beta, e0, tr=None):
    tr, nk, nm = tr if tr is not None else _alias_transform(W, sigma)
    phi = tr(beta, e0).reshape(nk, nm)
    main = phi[:, N_ALIAS]
    alias = np.delete(phi, N_ALIAS, axis=1)
    if np.any(main <= 0):
        return 1.0
    return float(np.max(np.sqrt(np.sum(alias ** 2, axis=1)) / main))


def fit(W, sigma, start=(2.3, 0.5)):
    from scipy.optimize import minimize

    tr = _alias_transform(W, sigma)

    def obj(p):
        beta, e0 = p
        if beta <= 0.5 or not (0.2 < e0 < 1.0):
            return 10.0
        return np.log(err1d(W, sigma, beta, e0, tr))

    best = None
    for s in (start, (2.3, 0.5)):
        r = minimize(obj, s, method="Nelder-Mead",
                     options=dict(xatol=1e-6, fatol=1e-6, maxiter=600))
        if best is None or r.fun < best.fun:
            best = r
    beta, e0 = best.x
    return float(beta), float(e0), float(np.exp(best.fun))


def build_table(verbose=True):
    rows = []
    for W in W_RANGE:
        start = (2.3, 0.5)
        for sigma in SIGMA_GRID:
            beta, e0, e = fit(W, sigma, start)
            start = (beta, e0)
            rows.append((W, sigma, e, beta, e0))
            if verbose:
                print(f"W={W:2d} sigma={sigma:.2f} err1d={e:.3e} beta={beta:.6f} e0={e0:.6f}",
                      file=sys.stderr)
    return rows


def write_inc(rows, path):
    lines = [
        "// Generated by wsclean_b200/kernel_db.py -- do not edit.",
        "// Rows: {W, sigma, err1d, beta, e0}; phi(t) = exp(beta*W*((1-t^2)^e0 - 1)).",
        "// err1d is the 1-D aliasing error estimate; n-D gridding uses n*err1d.",
    ]
    for W, s, e, b, e0 in rows:
        lines.append(f"{{{W}, {s:.2f}, {e:.8e}, {b:.17g}, {e0:.17g}}},")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    rows = build_table()
    write_inc(rows, os.path.join(here, "csrc", "es_kernel_db.inc"))


if __name__ == "__main__":
    main()
