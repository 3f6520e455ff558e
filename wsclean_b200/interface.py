"""Operator interface over the GPU gridder, in the shape of WSClean's Python
interface (interface/pywsclean.py:28-187: Operator with data_size,
image_size, forward = prediction, backward = imaging) but wired straight to
libwsg's C ABI instead of round-tripping through a measurement set and full
wsclean runs.  Also the differentiable pair for gradient-based imaging:

* ``DirtyToVis``: y = A x (dirty2ms, prediction) with backward
  grad_x = Re(A^H grad_y) = ms2dirty(grad_y) -- exact, because the two
  operators are implemented as exact adjoints;
* ``VisToDirty``: x = Re(A^H y) (ms2dirty) with backward A grad_x
  (dirty2ms).

With a weighted chi^2 = sum_k w_k |V_k - (A x)_k|^2 the gradient with respect
to the model image is -2 ms2dirty(w * (V - A x)): one gridding call on the
weighted residuals.
"""
from __future__ import annotations

import numpy as np
import torch

from . import gridder as G


class ImagingParameters:
    """Image geometry and accuracy (the pywsclean ImagingParameters fields
    that apply to the operator), plus the in-memory data the operator maps
    from and to: uvw (nrows x 3, metres), freq (Hz) and optional weights."""

    def __init__(self, uvw, freq, imageWidth=512, imageHeight=512, pixelScaleX=1e-5,
                 pixelScaleY=None, epsilon=1e-5, precision="mixed", weights=None,
                 center_x=0.0, center_y=0.0, device=0):
        self.uvw = uvw
        self.freq = freq
        self.imageWidth = imageWidth
        self.imageHeight = imageHeight
        self.pixelScaleX = pixelScaleX
        self.pixelScaleY = pixelScaleX if pixelScaleY is None else pixelScaleY
        self.epsilon = epsilon
        self.precision = precision
        self.weights = weights
        self.center_x = center_x
        self.center_y = center_y
        self.device = device


def _kw(p):
    # WSClean's call pattern (wgridder/wgriddinggridder_simple.cpp:56-58)
    return dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0,
                center_x=p.center_x, center_y=p.center_y, precision=p.precision)


class Operator:
    """forward(dataOut, dataIn): image (float64, width*height, index
    i*height + j for x-major pixel (i, j)) -> visibilities (complex128,
    nrows*nchan); backward(dataOut, dataIn): visibilities -> image.  Usable as
    a context manager like the reference's Operator."""

    def __init__(self, parameters):
        self._p = parameters
        self._ctx = None

    def __enter__(self):
        self._ctx = G.Context(self._p.device)
        return self

    def __exit__(self, *exc):
        if self._ctx is not None:
            self._ctx.close()
            self._ctx = None

    def _check_open(self, what):
        if self._ctx is None:
            raise RuntimeError(f'Operator.{what}() was called outside "with" block')

    def data_size(self):
        return int(self._p.uvw.shape[0]) * int(len(self._p.freq))

    def image_size(self):
        return self._p.imageWidth * self._p.imageHeight

    def forward(self, dataOut, dataIn):
        self._check_open("forward")
        if np.shape(dataOut)[0] != self.data_size():
            raise RuntimeError("Size of output argument does not match the number of visibilities")
        if np.shape(dataIn)[0] != self.image_size():
            raise RuntimeError("Size of input argument does not match the image size")
        if dataOut.dtype.name != "complex128" or dataIn.dtype.name != "float64":
            raise RuntimeError("forward() takes complex128 output and float64 input")
        p = self._p
        img = np.ascontiguousarray(dataIn).reshape(p.imageWidth, p.imageHeight)
        v = self._ctx.dirty2ms(p.uvw, p.freq, img, p.pixelScaleX, p.pixelScaleY, p.epsilon,
                               wgt=p.weights, vis_dtype=np.complex128, **_kw(p))
        dataOut[:] = np.asarray(v).ravel()

    def backward(self, dataOut, dataIn):
        self._check_open("backward")
        if np.shape(dataOut)[0] != self.image_size():
            raise RuntimeError("Size of output argument does not match the image size")
        if np.shape(dataIn)[0] != self.data_size():
            raise RuntimeError("Size of input argument does not match the number of visibilities")
        if dataOut.dtype.name != "float64" or dataIn.dtype.name != "complex128":
            raise RuntimeError("backward() takes float64 output and complex128 input")
        p = self._p
        vis = np.ascontiguousarray(dataIn).reshape(self._p.uvw.shape[0], len(p.freq))
        d = self._ctx.ms2dirty(p.uvw, p.freq, vis, p.imageWidth, p.imageHeight, p.pixelScaleX,
                               p.pixelScaleY, p.epsilon, wgt=p.weights, dirty_dtype=np.float64,
                               **_kw(p))
        dataOut[:] = np.asarray(d).ravel()


class DirtyToVis(torch.autograd.Function):
    """y = A x: model image (real, nx x ny) -> visibilities (complex)."""

    @staticmethod
    def forward(ctx, image, op):
        ctx.op = op
        p = op._p
        return op._ctx.dirty2ms(p.uvw, p.freq, image.detach().contiguous(), p.pixelScaleX,
                                p.pixelScaleY, p.epsilon, wgt=p.weights,
                                vis_dtype=np.complex128, **_kw(p))

    @staticmethod
    def backward(ctx, grad_vis):
        # for real x and complex y = A x, dL/dx = Re(A^H g) with g torch's
        # complex gradient of y; ms2dirty computes exactly Re(A^H g)
        op = ctx.op
        p = op._p
        g = op._ctx.ms2dirty(p.uvw, p.freq, grad_vis.contiguous(), p.imageWidth, p.imageHeight,
                             p.pixelScaleX, p.pixelScaleY, p.epsilon, wgt=p.weights,
                             dirty_dtype=np.float64, **_kw(p))
        return g, None


class VisToDirty(torch.autograd.Function):
    """x = Re(A^H y): visibilities -> dirty image (the adjoint)."""

    @staticmethod
    def forward(ctx, vis, op):
        ctx.op = op
        p = op._p
        return op._ctx.ms2dirty(p.uvw, p.freq, vis.detach().contiguous(), p.imageWidth,
                                p.imageHeight, p.pixelScaleX, p.pixelScaleY, p.epsilon,
                                wgt=p.weights, dirty_dtype=np.float64, **_kw(p))

    @staticmethod
    def backward(ctx, grad_img):
        op = ctx.op
        p = op._p
        v = op._ctx.dirty2ms(p.uvw, p.freq, grad_img.contiguous(), p.pixelScaleX, p.pixelScaleY,
                             p.epsilon, wgt=p.weights, vis_dtype=np.complex128, **_kw(p))
        return v, None


def chi2(op, image, vis, noise_weights):
    """sum_k w_k |V_k - (A x)_k|^2 as a differentiable torch scalar."""
    model = DirtyToVis.apply(image, op)
    r = vis - model
    return torch.sum(noise_weights * (r.real ** 2 + r.imag ** 2))
