"""ctypes binding of libstrata_cuda (include/strata_cuda.h).

The library is built in-tree (strata_b200/libstrata_cuda.so) by
strata_b200/build.py. Loading fails loudly when it is missing: the device
backend has no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstrata_cuda.so")

OK, EINVAL, ECUDA, ENOMEM, ECANCELED, ETIMEDOUT, EIO, ENOTSUP = 0, -1, -2, -3, -4, -5, -6, -8

OP_GRADIENT, OP_SLOPE, OP_ASPECT, OP_HILLSHADE, OP_CURVATURE, OP_RUGGEDNESS = 1, 2, 3, 4, 5, 6
OP_CORRELATE, OP_SEPARABLE, OP_MEAN, OP_MIN, OP_MAX, OP_LOOKUP, OP_RECLASS = 7, 8, 9, 10, 11, 12, 13
OP_HEATLOAD, OP_ORIENTATION, OP_STEP = 14, 15, 16
# vec.Op (internal/vec/chain.go:24-38), strata_stage.kind of an OP_STEP stage
(VEC_ADD, VEC_SUB, VEC_MUL, VEC_DIV, VEC_MIN, VEC_MAX, VEC_ADD_SCALAR, VEC_MUL_SCALAR, VEC_AFFINE, VEC_SUB_DIV,
 VEC_CLAMP, VEC_ABS, VEC_SQRT) = range(13)
MAX_STEPS = 16
MAX_INPUTS = 4
STAGE_ROTATE180 = 1
STAGE_FIT = 2
EXEC_ASYNC = 1
MAX_RADIUS = 8
MAX_KNOTS = 64
MAX_NOALLOC_BATCH = 64

c_i32, c_i64, c_f32, c_f64, c_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_void_p


class Raster(ctypes.Structure):
    _fields_ = [("data", c_p), ("width", c_i64), ("height", c_i64), ("stride", c_i64),
                ("valid", c_p), ("valid_offset", c_i64), ("on_device", c_i32), ("reserved", c_i32)]


class Stage(ctypes.Structure):
    _fields_ = [("op", ctypes.c_uint32), ("radius", c_i32), ("kind", c_i32), ("flags", c_i32),
                ("k", c_f32 * 16), ("table", c_p * 4), ("table_len", c_i32 * 4), ("input", c_i32),
                ("reserved", c_i32)]


class ExecOpts(ctypes.Structure):
    _fields_ = [("tile_width", c_i64), ("tile_height", c_i64), ("workers", c_i32), ("flags", c_i32),
                ("stream", c_p), ("cancel", ctypes.POINTER(c_i32))]


class Stats(ctypes.Structure):
    _fields_ = [("cells", c_i64), ("ideal", c_i64), ("tiles", c_i64), ("bands", c_i64),
                ("source_read", c_i64), ("sink_written", c_i64), ("kernel_read", c_i64),
                ("kernel_written", c_i64)]


READ_FN = ctypes.CFUNCTYPE(ctypes.c_int, c_p, ctypes.POINTER(Raster), c_i64, c_i64)
WRITE_FN = ctypes.CFUNCTYPE(ctypes.c_int, c_p, ctypes.POINTER(Raster), c_i64, c_i64)


class Strip(ctypes.Structure):
    _fields_ = [("height", c_i64), ("src_row", c_i64), ("dst_row", c_i64)]


class RawFile(ctypes.Structure):
    _fields_ = [("fd", c_i32), ("has_fill", c_i32), ("fill", c_f32), ("reserved", c_i32), ("width", c_i64),
                ("height", c_i64), ("offset", c_i64)]


class Source(ctypes.Structure):
    _fields_ = [("width", c_i64), ("height", c_i64), ("masked", c_i32), ("reserved", c_i32),
                ("user", c_p), ("read", READ_FN)]


class Sink(ctypes.Structure):
    _fields_ = [("width", c_i64), ("height", c_i64), ("masked", c_i32), ("reserved", c_i32),
                ("user", c_p), ("write", WRITE_FN)]


class BatchItem(ctypes.Structure):
    _fields_ = [("stages", ctypes.POINTER(Stage)), ("nstages", c_i32), ("tile_width", c_i32),
                ("tile_height", c_i32), ("reserved", c_i32), ("src", Raster), ("dst", Raster * 2)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("budget_bytes", c_i64), ("streams", c_i32), ("max_batch", c_i32), ("band", c_i32),
                ("reserved", c_i32)]


class ServerResult(ctypes.Structure):
    _fields_ = [("status", c_i32), ("nout", c_i32), ("out", Raster * 2), ("t_submit_ns", c_i64),
                ("t_start_ns", c_i64), ("t_done_ns", c_i64)]


# The same layouts as numpy dtypes, for filling and reading many at once
# (pointers as unsigned 64-bit integers).
RASTER_DTYPE = np.dtype([("data", "<u8"), ("width", "<i8"), ("height", "<i8"), ("stride", "<i8"), ("valid", "<u8"),
                         ("valid_offset", "<i8"), ("on_device", "<i4"), ("reserved", "<i4")])
SERVER_RESULT_DTYPE = np.dtype([("status", "<i4"), ("nout", "<i4"), ("out", RASTER_DTYPE, (2,)),
                                ("t_submit_ns", "<i8"), ("t_start_ns", "<i8"), ("t_done_ns", "<i8")])
SERVER_REQUEST_DTYPE = np.dtype([("stages", "<u8"), ("nstages", "<i4"), ("reserved", "<i4"), ("x", "<i8"),
                                 ("y", "<i8"), ("w", "<i8"), ("h", "<i8")])


class ServerRequest(ctypes.Structure):
    _fields_ = [("stages", ctypes.POINTER(Stage)), ("nstages", c_i32), ("reserved", c_i32), ("x", c_i64),
                ("y", c_i64), ("w", c_i64), ("h", c_i64)]


assert RASTER_DTYPE.itemsize == ctypes.sizeof(Raster)
assert SERVER_RESULT_DTYPE.itemsize == ctypes.sizeof(ServerResult)
assert SERVER_REQUEST_DTYPE.itemsize == ctypes.sizeof(ServerRequest)


class GradientOptions(ctypes.Structure):
    _fields_ = [("cell_size", c_f64), ("cell_size_y", c_f64), ("z_factor", c_f64),
                ("fit_radius", c_i32), ("reserved", c_i32)]


class SlopeOptions(ctypes.Structure):
    _fields_ = [("cell_size", c_f64), ("cell_size_y", c_f64), ("z_factor", c_f64),
                ("fit_radius", c_i32), ("units", c_i32)]


class AspectOptions(ctypes.Structure):
    _fields_ = [("cell_size", c_f64), ("cell_size_y", c_f64), ("z_factor", c_f64),
                ("fit_radius", c_i32), ("zero_for_flat", c_i32), ("trigonometric", c_i32), ("reserved", c_i32)]


class HillshadeOptions(ctypes.Structure):
    _fields_ = [("cell_size", c_f64), ("cell_size_y", c_f64), ("z_factor", c_f64),
                ("fit_radius", c_i32), ("reserved", c_i32), ("azimuth", c_f64), ("altitude", c_f64)]


class CurvatureOptions(ctypes.Structure):
    _fields_ = [("cell_size", c_f64), ("cell_size_y", c_f64), ("z_factor", c_f64),
                ("fit_radius", c_i32), ("type", c_i32)]


class HeatLoadOptions(ctypes.Structure):
    _fields_ = [("cell_size", c_f64), ("cell_size_y", c_f64), ("z_factor", c_f64),
                ("fit_radius", c_i32), ("equation", c_i32), ("latitude", c_f64),
                ("radiation", c_i32), ("linear", c_i32), ("terms", c_f64 * 8)]


class OrientationOptions(ctypes.Structure):
    _fields_ = [("cell_size", c_f64), ("cell_size_y", c_f64), ("z_factor", c_f64),
                ("fit_radius", c_i32), ("component", c_i32), ("unweighted", c_i32), ("reserved", c_i32)]


class RuggednessOptions(ctypes.Structure):
    _fields_ = [("type", c_i32), ("radius", c_i32)]


class WeightsOptions(ctypes.Structure):
    _fields_ = [("radius", c_i32), ("nweights", c_i32), ("weights", c_p)]


class SeparableOptions(ctypes.Structure):
    _fields_ = [("radius", c_i32), ("nrow", c_i32), ("row", c_p), ("ncol", c_i32), ("reserved", c_i32),
                ("col", c_p)]


class BoxOptions(ctypes.Structure):
    _fields_ = [("radius", c_i32)]


# (name, restype, argtypes) of every entry point include/strata_cuda.h declares.
SIGNATURES = [
    ("strata_abi_version", ctypes.c_int, []),
    ("strata_last_error", ctypes.c_char_p, []),
    ("strata_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(c_p)]),
    ("strata_ctx_destroy", None, [c_p]),
    ("strata_ctx_device", ctypes.c_int, [c_p]),
    ("strata_ctx_synchronize", ctypes.c_int, [c_p]),
    ("strata_alloc", ctypes.c_int, [c_p, ctypes.c_size_t, ctypes.POINTER(c_p)]),
    ("strata_free", ctypes.c_int, [c_p, c_p]),
    ("strata_upload", ctypes.c_int, [c_p, c_p, c_p, ctypes.c_size_t]),
    ("strata_download", ctypes.c_int, [c_p, c_p, c_p, ctypes.c_size_t]),
    ("strata_process", ctypes.c_int, [c_p, ctypes.POINTER(Stage), ctypes.c_int, ctypes.POINTER(Raster),
                                      ctypes.c_int, ctypes.POINTER(Raster), ctypes.c_int,
                                      ctypes.POINTER(ExecOpts), ctypes.POINTER(Stats)]),
    ("strata_process_features", ctypes.c_int, [c_p, ctypes.POINTER(Stage), ctypes.POINTER(c_i32), ctypes.c_int,
                                               ctypes.POINTER(Raster), ctypes.POINTER(Raster), ctypes.c_int,
                                               ctypes.POINTER(ExecOpts), ctypes.POINTER(Stats)]),
    ("strata_process_strip", ctypes.c_int, [c_p, ctypes.POINTER(Stage), ctypes.c_int, ctypes.POINTER(Raster),
                                             ctypes.POINTER(Raster), ctypes.c_int, ctypes.POINTER(Strip),
                                             ctypes.POINTER(ExecOpts), ctypes.POINTER(Stats)]),
    ("strata_process_multi", ctypes.c_int, [ctypes.POINTER(c_p), ctypes.c_int, ctypes.POINTER(Stage), ctypes.c_int,
                                             ctypes.POINTER(Raster), ctypes.c_int, ctypes.POINTER(Raster), ctypes.c_int,
                                             ctypes.POINTER(ExecOpts), ctypes.POINTER(Stats)]),
    ("strata_process_raw", ctypes.c_int, [c_p, ctypes.POINTER(Stage), ctypes.c_int, ctypes.POINTER(RawFile),
                                           ctypes.c_int, ctypes.POINTER(RawFile), ctypes.c_int,
                                           ctypes.POINTER(ExecOpts), ctypes.POINTER(Stats)]),
    ("strata_process_chunked", ctypes.c_int, [c_p, ctypes.POINTER(Stage), ctypes.c_int, ctypes.POINTER(Source),
                                              ctypes.c_int, ctypes.POINTER(Sink), ctypes.c_int,
                                              ctypes.POINTER(ExecOpts), ctypes.POINTER(Stats)]),
    ("strata_batch_create", ctypes.c_int, [c_p, ctypes.POINTER(BatchItem), ctypes.c_int, ctypes.POINTER(c_p)]),
    ("strata_batch_run", ctypes.c_int, [c_p, c_p, ctypes.c_int]),
    ("strata_batch_info", ctypes.c_int, [c_p, ctypes.POINTER(Stats), ctypes.POINTER(ctypes.c_int)]),
    ("strata_batch_destroy", None, [c_p]),
    ("strata_batch_run_noalloc", ctypes.c_int, [c_p, ctypes.POINTER(BatchItem), ctypes.c_int, c_p, ctypes.c_int]),
    ("strata_server_create", ctypes.c_int, [c_p, ctypes.POINTER(Raster), ctypes.POINTER(ServerOpts),
                                            ctypes.POINTER(c_p)]),
    ("strata_server_submit", ctypes.c_int, [c_p, ctypes.POINTER(Stage), ctypes.c_int, c_i64, c_i64, c_i64, c_i64,
                                            ctypes.POINTER(ctypes.c_uint64)]),
    ("strata_server_wait", ctypes.c_int, [c_p, ctypes.c_uint64, c_i64, ctypes.POINTER(ServerResult)]),
    ("strata_server_release", ctypes.c_int, [c_p, ctypes.c_uint64]),
    ("strata_server_submit_many", ctypes.c_int, [c_p, ctypes.POINTER(ServerRequest), ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_uint64)]),
    ("strata_server_wait_many", ctypes.c_int, [c_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int, c_i64,
                                               ctypes.POINTER(ServerResult)]),
    ("strata_server_release_many", ctypes.c_int, [c_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]),
    ("strata_server_stats", ctypes.c_int, [c_p, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                                           ctypes.POINTER(c_i64)]),
    ("strata_server_destroy", None, [c_p]),
    ("strata_stage_gradient", ctypes.c_int, [ctypes.POINTER(GradientOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_slope", ctypes.c_int, [ctypes.POINTER(SlopeOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_aspect", ctypes.c_int, [ctypes.POINTER(AspectOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_hillshade", ctypes.c_int, [ctypes.POINTER(HillshadeOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_curvature", ctypes.c_int, [ctypes.POINTER(CurvatureOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_ruggedness", ctypes.c_int, [ctypes.POINTER(RuggednessOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_correlate", ctypes.c_int, [ctypes.POINTER(WeightsOptions), ctypes.c_int, ctypes.POINTER(Stage)]),
    ("strata_stage_separable", ctypes.c_int, [ctypes.POINTER(SeparableOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_box", ctypes.c_int, [ctypes.POINTER(BoxOptions), ctypes.c_uint32, ctypes.POINTER(Stage)]),
    ("strata_stage_lookup", ctypes.c_int, [c_p, c_p, c_i32, ctypes.POINTER(Stage)]),
    ("strata_stage_reclass", ctypes.c_int, [c_p, c_i32, c_p, c_i32, ctypes.POINTER(Stage)]),
    ("strata_stage_heatload", ctypes.c_int, [ctypes.POINTER(HeatLoadOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_orientation", ctypes.c_int, [ctypes.POINTER(OrientationOptions), ctypes.POINTER(Stage)]),
    ("strata_stage_step", ctypes.c_int, [c_i32, c_i32, c_f32, c_f32, ctypes.POINTER(Stage)]),
    ("strata_stage_rescale", ctypes.c_int, [c_f32, c_f32, ctypes.POINTER(Stage)]),
    ("strata_stage_rescale_range", ctypes.c_int, [c_f32, c_f32, c_f32, c_f32, ctypes.POINTER(Stage)]),
    ("strata_focal_gaussian", ctypes.c_int, [c_i32, c_f64, ctypes.POINTER(c_f32)]),
]

_lib = None
_lock = threading.Lock()


def lib():
    """The loaded library; raises if libstrata_cuda.so has not been built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(
                        f"libstrata_cuda.so is not built ({LIB_PATH}); run python -m strata_b200.build")
                L = ctypes.CDLL(LIB_PATH)
                for name, res, args in SIGNATURES:
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


def last_error() -> str:
    return lib().strata_last_error().decode("utf-8", "replace")


def check(rc: int) -> None:
    """Raises the Python form of a status code: StrataPanic for EINVAL,
    NotSupported for ENOTSUP, RuntimeError for device failures. ECANCELED
    and EIO are returned as errors by the Tiled/Chunked functions instead."""
    from .raster import NotSupported, StrataPanic

    if rc == OK:
        return
    msg = last_error()
    if rc == EINVAL:
        raise StrataPanic(msg)
    if rc == ENOTSUP:
        raise NotSupported(msg)
    raise RuntimeError(f"strata_cuda error {rc}: {msg}")
