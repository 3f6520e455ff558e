"""Test infrastructure only: a numpy restatement of WSClean's ImageWeights,
the checker for the GPU imaging weights (wsg_weights_*).

Follows structures/imageweights.h:36-100 (Grid, uvToXY, isWithinLimits,
sampleGridValue), structures/imageweights.cpp:36-47 (grid size),
:78-111 (gridding loop, weightsAsTaper, v < 0 flip) and :113-143
(FinishGridding), with u = uInM / lambda and lambda = c / f as aocommon's
BandData::ChannelWavelength computes it (aocommon is an un-vendored
submodule of the reference).  Sums run in the reference's order (rows,
channels, polarisations) so that the grid and total are the reference's
doubles.  No reference test holds golden values for this class, and its
sources need aocommon to compile: parity for this row rests on this
restatement."""
from __future__ import annotations

import numpy as np

C_LIGHT = 299792458.0


class ImageWeights:
    NATURAL, UNIFORM, BRIGGS = 0, 1, 2

    def __init__(self, mode, robust, width, height, psx, psy, weights_as_taper=False,
                 super_weight=1.0):
        self.mode, self.robust = mode, robust
        self.W = int(round(width / super_weight))
        self.H = int(round(height / super_weight))
        self.W += self.W % 2
        self.H += self.H % 2
        self.psx, self.psy = psx, psy
        self.taper = weights_as_taper
        self.grid = np.zeros(self.W * (self.H // 2))
        self.total = 0.0

    def _cells(self, uvw, freq):
        lam = C_LIGHT / np.asarray(freq, dtype=np.float64)
        u = uvw[:, 0:1] / lam[None, :]
        v = uvw[:, 1:2] / lam[None, :]
        flip = v < 0.0
        u = np.where(flip, -u, u)
        v = np.where(flip, -v, v)
        x = np.floor(u * float(self.W) * self.psx + float(self.W // 2)).astype(np.int64)
        y = np.floor(v * float(self.H) * self.psy).astype(np.int64)
        ok = (x >= 0) & (x < self.W) & (y < self.H // 2)
        return x, y, ok

    def grid_weights(self, uvw, freq, weights=None, npol=1):
        nrows, nchan = uvw.shape[0], len(freq)
        w = (np.ones((nrows, nchan, npol), np.float32) if weights is None
             else np.asarray(weights, np.float32).reshape(nrows, nchan, npol))
        if self.taper:
            w = np.where(w != 0, np.float32(1), w)
        x, y, ok = self._cells(uvw, freq)
        idx = np.broadcast_to((x + y * self.W)[..., None], w.shape)
        okk = np.broadcast_to(ok[..., None], w.shape)
        vals = w[okk].astype(np.float64)
        np.add.at(self.grid, idx[okk], vals)
        if vals.size:
            self.total = float(np.cumsum(np.concatenate([[self.total], vals]))[-1])

    def finish(self):
        g = self.grid
        if self.mode == self.BRIGGS:
            avg = float(np.cumsum(g * g)[-1]) / self.total
            num = 5.0 * np.exp(-np.log(10.0) * self.robust)
            self.grid = 1.0 / (1.0 + g * (num * num / avg))
        elif self.mode == self.UNIFORM:
            self.grid = np.where(g != 0.0, 1.0 / np.where(g != 0.0, g, 1.0), 0.0)
        else:
            self.grid = np.where(g != 0.0, 1.0, g)

    def apply(self, uvw, freq, weights=None, npol=1):
        nrows, nchan = uvw.shape[0], len(freq)
        x, y, ok = self._cells(uvw, freq)
        iw = np.where(ok, self.grid[np.where(ok, x + y * self.W, 0)], 0.0)
        w = (np.ones((nrows, nchan, npol), np.float32) if weights is None
             else np.asarray(weights, np.float32).reshape(nrows, nchan, npol))
        return (w.astype(np.float64) * iw[..., None]).astype(np.float32)
