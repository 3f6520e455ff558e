"""ctypes binding of libwsg.so (the C ABI declared in include/wsg.h).

The shared library is built in-tree (wsclean_b200/libwsg.so) by
``wsclean_b200.build.build()``.  Loading fails loudly when it is missing: there
is no CPU fallback for the gridder.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwsg.so")

WSG_OK, WSG_ERR_INVALID, WSG_ERR_CUDA, WSG_ERR_NOMEM, WSG_ERR_CUFFT, WSG_ERR_STATE = 0, 1, 2, 3, 4, 5
WSG_ERR_INTERNAL = 7
WSG_PREC_MIXED, WSG_PREC_FP64 = 0, 1
WSG_C64, WSG_C128 = 0, 1
WSG_WEIGHT_NATURAL, WSG_WEIGHT_UNIFORM, WSG_WEIGHT_BRIGGS = 0, 1, 2
WSG_F32, WSG_F64 = 0, 1

# Every symbol include/wsg.h declares (checked by the CPU test suite).
EXPORTED = [
    "wsg_ctx_create", "wsg_ctx_destroy", "wsg_ctx_set_stream", "wsg_ctx_release_buffers",
    "wsg_args_init", "wsg_ms2dirty", "wsg_dirty2ms",
    "wsg_gridder_create", "wsg_gridder_destroy", "wsg_gridder_memory_usage",
    "wsg_gridder_initialize_inversion", "wsg_gridder_add_inversion_data",
    "wsg_gridder_finalize_image", "wsg_gridder_real_image",
    "wsg_gridder_initialize_prediction", "wsg_gridder_predict_visibilities",
    "wsg_gridder_ctx", "wsg_get_stats", "wsg_last_error", "wsg_abi_version",
    "wsg_plan_grid", "wsg_ms2dirty_noalloc",
    "wsg_plan_create", "wsg_plan_destroy", "wsg_plan_ms2dirty", "wsg_plan_dirty2ms",
    "wsg_plan_get_stats", "wsg_ctx_synchronize",
    "wsg_stream_create", "wsg_stream_destroy", "wsg_stream_add", "wsg_stream_finish",
    "wsg_stream_predict_begin", "wsg_stream_predict", "wsg_stream_get_stats",
    "wsg_weights_create", "wsg_weights_destroy", "wsg_weights_grid", "wsg_weights_finish",
    "wsg_weights_apply", "wsg_weights_get", "wsg_autotune", "wsg_ctx_set_async",
    "wsg_ms2dirty_tuning", "wsg_dirty2ms_tuning", "wsg_get_tuning", "wsg_tuning_choice",
    "wsg_stream_set_imaging_weights",
]

c_size_t, c_double, c_int, c_void_p = ctypes.c_size_t, ctypes.c_double, ctypes.c_int, ctypes.c_void_p


class WsgArgs(ctypes.Structure):
    _fields_ = [
        ("nrows", c_size_t), ("nchan", c_size_t),
        ("uvw", c_void_p), ("freq", c_void_p),
        ("wgt", c_void_p), ("wgt_type", c_int),
        ("mask", c_void_p),
        ("npix_x", c_size_t), ("npix_y", c_size_t),
        ("pixsize_x", c_double), ("pixsize_y", c_double),
        ("epsilon", c_double),
        ("do_wgridding", c_int), ("negate_v", c_int), ("divide_by_n", c_int),
        ("sigma_min", c_double), ("sigma_max", c_double),
        ("center_x", c_double), ("center_y", c_double),
        ("precision", c_int), ("vis_type", c_int), ("dirty_type", c_int),
    ]


class WsgGridderParams(ctypes.Structure):
    _fields_ = [
        ("width", c_size_t), ("height", c_size_t),
        ("width_t", c_size_t), ("height_t", c_size_t),
        ("pixel_size_x", c_double), ("pixel_size_y", c_double),
        ("l_shift", c_double), ("m_shift", c_double),
        ("nthreads", c_size_t), ("epsilon", c_double),
        ("verbosity", c_size_t), ("tuning", c_int),
        ("precision", c_int), ("device", c_int),
    ]


class WsgJob(ctypes.Structure):
    _fields_ = [
        ("npix_x", c_size_t), ("npix_y", c_size_t),
        ("center_x", c_double), ("center_y", c_double),
        ("chan_begin", c_size_t), ("chan_end", c_size_t),
    ]


class WsgStats(ctypes.Structure):
    _fields_ = [
        ("nrows", c_size_t), ("nchan", c_size_t), ("nvis", c_size_t),
        ("nu", c_size_t), ("nv", c_size_t), ("nplanes", c_size_t), ("supp", c_size_t),
        ("plane_batch", c_size_t), ("band_rows", c_size_t), ("degree", c_size_t),
        ("sigma", c_double), ("beta", c_double), ("e0", c_double), ("kernel_err", c_double),
        ("wmin", c_double), ("wmax", c_double), ("dw", c_double), ("nshift", c_double),
        ("ms_prep", c_double), ("ms_sort", c_double), ("ms_grid", c_double),
        ("ms_fft", c_double), ("ms_screen", c_double), ("ms_total", c_double),
        ("device_bytes", c_size_t),
        ("gridding", c_int), ("precision", c_int),
        ("kernel_launches", c_size_t),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


class WsgError(RuntimeError):
    """A libwsg call failed; .code is the WSG_ERR_* status."""

    def __init__(self, code, msg):
        super().__init__(f"libwsg error {code}: {msg}")
        self.code = code


class InvalidArgument(WsgError, ValueError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "(there is no CPU fallback for the gridder)")
        L = ctypes.CDLL(LIB_PATH)
        vp = c_void_p
        P = ctypes.POINTER
        L.wsg_ctx_create.argtypes = [c_int, P(vp)]
        L.wsg_ctx_destroy.argtypes = [vp]
        L.wsg_ctx_set_stream.argtypes = [vp, vp]
        L.wsg_ctx_release_buffers.argtypes = [vp]
        L.wsg_args_init.argtypes = [P(WsgArgs)]
        L.wsg_args_init.restype = None
        L.wsg_ms2dirty.argtypes = [vp, P(WsgArgs), vp, vp, c_int]
        L.wsg_dirty2ms.argtypes = [vp, P(WsgArgs), vp, vp]
        L.wsg_gridder_create.argtypes = [P(WsgGridderParams), P(vp)]
        L.wsg_gridder_destroy.argtypes = [vp]
        L.wsg_gridder_memory_usage.argtypes = [vp, P(c_size_t), P(c_size_t)]
        L.wsg_gridder_initialize_inversion.argtypes = [vp]
        L.wsg_gridder_add_inversion_data.argtypes = [vp, c_size_t, c_size_t, vp, vp, vp]
        L.wsg_gridder_finalize_image.argtypes = [vp, c_double]
        L.wsg_gridder_real_image.argtypes = [vp, vp]
        L.wsg_gridder_initialize_prediction.argtypes = [vp, vp]
        L.wsg_gridder_predict_visibilities.argtypes = [vp, c_size_t, c_size_t, vp, vp, vp]
        L.wsg_gridder_ctx.argtypes = [vp]
        L.wsg_gridder_ctx.restype = vp
        L.wsg_get_stats.argtypes = [vp, P(WsgStats)]
        L.wsg_ms2dirty_noalloc.argtypes = [P(WsgArgs), vp, vp, vp]
        L.wsg_plan_grid.argtypes = [P(WsgArgs), c_size_t, c_double, c_double, c_double,
                                    c_double, P(WsgStats)]
        L.wsg_plan_create.argtypes = [vp, P(WsgArgs), P(WsgJob), c_size_t, P(vp)]
        L.wsg_plan_destroy.argtypes = [vp]
        L.wsg_plan_ms2dirty.argtypes = [vp, vp, P(vp), c_int]
        L.wsg_plan_dirty2ms.argtypes = [vp, P(vp), vp]
        L.wsg_plan_get_stats.argtypes = [vp, c_size_t, P(WsgStats)]
        L.wsg_ctx_synchronize.argtypes = [vp]
        L.wsg_stream_create.argtypes = [vp, P(WsgArgs), c_double, c_double, c_double, c_double,
                                        c_size_t, P(vp)]
        L.wsg_stream_destroy.argtypes = [vp]
        L.wsg_stream_add.argtypes = [vp, c_size_t, vp, vp, vp, vp]
        L.wsg_stream_finish.argtypes = [vp, vp, c_int]
        L.wsg_stream_predict_begin.argtypes = [vp, vp]
        L.wsg_stream_predict.argtypes = [vp, c_size_t, vp, vp, vp, vp]
        L.wsg_stream_get_stats.argtypes = [vp, P(WsgStats)]
        L.wsg_stream_set_imaging_weights.argtypes = [vp, vp]
        L.wsg_weights_create.argtypes = [vp, c_int, c_double, c_size_t, c_size_t, c_double,
                                         c_double, c_int, c_double, P(vp)]
        L.wsg_weights_destroy.argtypes = [vp]
        L.wsg_weights_grid.argtypes = [vp, c_size_t, c_size_t, c_size_t, vp, vp, vp]
        L.wsg_weights_finish.argtypes = [vp]
        L.wsg_weights_apply.argtypes = [vp, c_size_t, c_size_t, c_size_t, vp, vp, vp, vp]
        L.wsg_weights_get.argtypes = [vp, vp, P(c_size_t), P(c_size_t), P(c_double)]
        L.wsg_autotune.argtypes = [vp, P(WsgArgs), vp, c_int, P(WsgStats)]
        L.wsg_ctx_set_async.argtypes = [vp, c_int]
        L.wsg_ms2dirty_tuning.argtypes = [vp, P(WsgArgs), vp, vp, c_int]
        L.wsg_dirty2ms_tuning.argtypes = [vp, P(WsgArgs), vp, vp]
        L.wsg_get_tuning.argtypes = [vp, P(c_int), P(c_int), P(c_int), P(c_double)]
        L.wsg_tuning_choice.argtypes = [P(WsgArgs), c_size_t, c_double, c_double,
                                        P(ctypes.c_uint64), P(c_int), P(c_int), P(c_int)]
        L.wsg_last_error.restype = ctypes.c_char_p
        L.wsg_abi_version.restype = c_int
        for name in EXPORTED:
            fn = getattr(L, name)
            if name not in ("wsg_args_init", "wsg_last_error", "wsg_gridder_ctx"):
                if fn.restype is None or fn.restype is ctypes.c_int:
                    fn.restype = c_int
        _lib = L
    return _lib


def check(rc):
    if rc != WSG_OK:
        msg = lib().wsg_last_error().decode(errors="replace")
        if rc == WSG_ERR_INVALID:
            raise InvalidArgument(rc, msg)
        raise WsgError(rc, msg)
