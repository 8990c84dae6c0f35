"""ctypes binding of the C ABI declared in include/rawengine_b200.h.

The shared library is built in tree (librawops_b200/_lib/librawengine_b200.so,
see build.py).  There is no fallback: if the library is missing, importing the
render API raises, and on a machine without a GPU every device entry point
reports RE_CUDA_ERROR.
"""
from __future__ import annotations

import ctypes as C
import os

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "librawengine_b200.so")

RE_OK, RE_INVALID_ARGUMENT, RE_OUT_OF_RANGE, RE_DOMAIN_ERROR = 0, 1, 2, 3
RE_LENGTH_ERROR, RE_OVERFLOW_ERROR, RE_CANCELLED, RE_CUDA_ERROR, RE_TIMEOUT = 4, 5, 6, 7, 8

STAGE_GAIN3, STAGE_SCALE, STAGE_MATRIX, STAGE_TONE, STAGE_CLIP, STAGE_SRGB, STAGE_CURVES = range(1, 8)
MAX_STAGES = 16

# Every exported symbol of include/rawengine_b200.h (checked by the CPU tests).
EXPORTS = [
    "re_last_error", "re_version", "re_device_count",
    "re_image_create", "re_image_wrap_device", "re_image_destroy", "re_image_metadata",
    "re_raw_metadata_normalize", "re_site_index", "re_cfa_color",
    "re_request_bounds", "re_raw_input_region", "re_mip_native_region", "re_plan_tiles",
    "re_camera_to_working_matrix", "re_working_to_srgb_matrix", "re_working_to_working_matrix",
    "re_exposure_multiplier", "re_curve_set_create", "re_curve_set_destroy",
    "re_render_raw", "re_render_raw_async", "re_menon_directions", "re_render_scratch_bytes", "re_status_from_device",
    "re_release_scratch",
    "re_render_tiles", "re_render_raster", "re_guided_filter", "re_guided_filter_async", "re_guided_filter_scratch_bytes", "re_local_statistics", "re_local_statistics_f64", "re_cubic_resize", "re_rotate",
    "re_cubic_axis", "re_rotation_coefficients", "re_cubic_resize_window", "re_rotate_window",
    "re_rotation_support",
    "re_render_raw_reduced_noalloc", "re_render_raw_reduced_noalloc_max_native_pixels",
    "re_batch_create", "re_batch_destroy", "re_batch_plan", "re_batch_launch", "re_batch_launch_per_request",
    "re_batch_status",
    "re_batch_info_get", "re_batch_autotune",
    "re_diff_bilinear_forward", "re_diff_bilinear_backward", "re_diff_point_forward", "re_diff_point_backward",
    "re_diff_point_grad_count", "re_diff_detail_forward", "re_diff_detail_backward",
    "re_histogram_reset", "re_histogram_rgb", "re_histogram_extremum",
    "re_sharpen_window", "re_clarity_window", "re_texture_window", "re_convolution_window",
    "re_fingerprint_raw", "re_fingerprint_raster", "re_image_create_fingerprinted",
    "re_diff_menon_forward", "re_diff_menon_backward",
]


class ReError(RuntimeError):
    """Raised for a non-zero re_status; `kind` names the reference exception."""
    KINDS = {1: "invalid_argument", 2: "out_of_range", 3: "domain_error", 4: "length_error",
             5: "overflow_error", 6: "cancelled", 7: "cuda_error", 8: "timeout"}

    def __init__(self, code: int, message: str):
        super().__init__(f"{self.KINDS.get(code, code)}: {message}")
        self.code = code
        self.kind = self.KINDS.get(code, str(code))


class Rect(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32)]

    def tuple(self):
        return (self.x, self.y, self.width, self.height)


class RawMetadata(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("row_stride_samples", C.c_uint32),
                ("pattern", C.c_uint32), ("cfa_phase_x", C.c_uint32), ("cfa_phase_y", C.c_uint32),
                ("active_area", Rect), ("black_levels", C.c_uint16 * 4),
                ("white_levels", C.c_uint16 * 4)]


class Stage(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("arg", C.c_uint32), ("f", C.c_float * 12)]


class RenderDesc(C.Structure):
    _fields_ = [("demosaic", C.c_uint32), ("anchor", C.c_int32), ("count", C.c_uint32),
                ("stages", Stage * MAX_STAGES), ("curves", C.c_void_p * 4)]


class RenderStats(C.Structure):
    _fields_ = [("pixels", C.c_uint64), ("native_pixels", C.c_uint64), ("menon_decisions", C.c_uint64),
                ("menon_near_ties", C.c_uint64), ("launches", C.c_uint32), ("device_ms", C.c_float)]


class BatchItem(C.Structure):
    _fields_ = [("image", C.c_void_p), ("desc", C.POINTER(RenderDesc)), ("viewport", Rect), ("mip", C.c_uint32),
                ("quality", C.c_uint32), ("out", C.c_void_p), ("out_row_stride", C.c_size_t),
                ("geometry", C.c_uint32), ("canvas_width", C.c_uint32), ("canvas_height", C.c_uint32),
                ("angle_degrees", C.c_double), ("post", C.POINTER(RenderDesc))]


class BatchOptions(C.Structure):
    _fields_ = [("dispatch", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("order", C.c_uint32),
                ("use_graph", C.c_uint32)]


class BatchInfo(C.Structure):
    _fields_ = [("requests", C.c_uint32), ("reduced_requests", C.c_uint32), ("tasks", C.c_uint32),
                ("tiles", C.c_uint32),
                ("reduce_blocks", C.c_uint32), ("grid", C.c_uint32), ("native_pixels", C.c_uint64),
                ("output_pixels", C.c_uint64), ("raw_bytes", C.c_uint64), ("output_bytes", C.c_uint64),
                ("options", BatchOptions), ("geometry_requests", C.c_uint32)]


class DiffPointParams(C.Structure):
    _fields_ = [("scalars", C.c_void_p), ("knots", C.c_uint32), ("kx", C.c_void_p), ("ky", C.c_void_p),
                ("c0", C.c_void_p), ("c1", C.c_void_p)]


TILE_CALLBACK = C.CFUNCTYPE(C.c_int, C.POINTER(Rect), C.POINTER(C.c_float), C.c_void_p)

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError(f"{_LIB_PATH} is missing: run `python -m librawops_b200.build`")
        L = C.CDLL(_LIB_PATH)
        vp, u32, f32p, f64p = C.c_void_p, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_double)
        sz = C.c_size_t
        L.re_last_error.restype = C.c_char_p
        L.re_image_create.argtypes = [C.POINTER(RawMetadata), C.POINTER(C.c_uint16), sz, C.POINTER(vp)]
        L.re_image_wrap_device.argtypes = [C.POINTER(RawMetadata), vp, sz, C.POINTER(vp)]
        L.re_image_destroy.argtypes = [vp]
        L.re_image_metadata.argtypes = [vp, C.POINTER(RawMetadata)]
        L.re_raw_metadata_normalize.argtypes = [C.POINTER(RawMetadata), sz]
        L.re_site_index.argtypes = [C.POINTER(RawMetadata), u32, u32]
        L.re_cfa_color.argtypes = [C.POINTER(RawMetadata), u32, u32]
        L.re_request_bounds.argtypes = [Rect, u32, u32, C.POINTER(Rect)]
        L.re_raw_input_region.argtypes = [C.POINTER(RawMetadata), u32, Rect, C.POINTER(Rect)]
        L.re_mip_native_region.argtypes = [Rect, u32, Rect, C.POINTER(Rect)]
        L.re_plan_tiles.argtypes = [Rect, u32, C.POINTER(Rect), sz, C.POINTER(sz)]
        L.re_camera_to_working_matrix.argtypes = [f64p, u32, f32p]
        L.re_working_to_srgb_matrix.argtypes = [u32, f32p]
        L.re_working_to_working_matrix.argtypes = [u32, u32, f32p]
        L.re_exposure_multiplier.argtypes = [C.c_float, f32p]
        L.re_curve_set_create.argtypes = [u32, C.POINTER(C.c_uint32), f64p, C.POINTER(vp)]
        L.re_curve_set_destroy.argtypes = [vp]
        L.re_render_raw.argtypes = [vp, C.POINTER(RenderDesc), Rect, u32, u32, vp, sz, C.c_int, vp,
                                    C.POINTER(RenderStats)]
        L.re_render_raw_async.argtypes = [vp, C.POINTER(RenderDesc), Rect, u32, u32, vp, sz, vp, vp, vp]
        L.re_menon_directions.argtypes = [vp, u32, Rect, vp, C.POINTER(C.c_uint64), vp]
        L.re_render_scratch_bytes.argtypes = [vp, C.POINTER(RenderDesc), Rect, u32]
        L.re_render_scratch_bytes.restype = sz
        L.re_status_from_device.argtypes = [u32]
        L.re_release_scratch.argtypes = []
        L.re_render_tiles.argtypes = [vp, C.POINTER(RenderDesc), Rect, u32, u32, u32, TILE_CALLBACK, vp, vp]
        L.re_render_raster.argtypes = [vp, sz, u32, u32, C.POINTER(RenderDesc), Rect, u32, u32, vp, sz, vp]
        L.re_guided_filter.argtypes = [vp, sz, vp, sz, u32, u32, u32, C.c_double, u32, vp]
        L.re_guided_filter_async.argtypes = [vp, sz, vp, sz, u32, u32, u32, C.c_double, u32, vp, vp, vp]
        L.re_guided_filter_scratch_bytes.argtypes = [u32, u32, u32]
        L.re_guided_filter_scratch_bytes.restype = sz
        L.re_local_statistics.argtypes = [vp, sz, u32, u32, u32, vp, vp, vp, vp]
        L.re_local_statistics_f64.argtypes = [vp, sz, u32, u32, u32, vp, vp, vp, vp]
        L.re_cubic_resize.argtypes = [vp, sz, u32, u32, u32, u32, Rect, u32, vp, sz, vp]
        L.re_rotate.argtypes = [vp, sz, u32, u32, C.c_double, Rect, u32, vp, sz, vp]
        L.re_cubic_axis.argtypes = [u32, u32, u32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), f64p,
                                    C.POINTER(C.c_uint32)]
        L.re_rotation_coefficients.argtypes = [C.c_double, f64p, f64p]
        L.re_cubic_resize_window.argtypes = [vp, sz, Rect, u32, u32, u32, u32, Rect, u32, vp, sz, vp]
        L.re_rotate_window.argtypes = [vp, sz, Rect, u32, u32, C.c_double, Rect, u32, vp, sz, vp]
        L.re_rotation_support.argtypes = [u32, u32, C.c_double, Rect, C.POINTER(Rect)]
        L.re_render_raw_reduced_noalloc.argtypes = [vp, C.POINTER(RenderDesc), Rect, u32, vp, sz, vp]
        L.re_render_raw_reduced_noalloc_max_native_pixels.restype = sz
        L.re_batch_create.argtypes = [C.POINTER(vp)]
        L.re_batch_destroy.argtypes = [vp]
        L.re_batch_plan.argtypes = [vp, C.POINTER(BatchItem), sz, C.POINTER(BatchOptions)]
        L.re_batch_launch.argtypes = [vp, vp]
        L.re_batch_launch_per_request.argtypes = [vp, vp]
        L.re_batch_status.argtypes = [vp, vp]
        L.re_batch_info_get.argtypes = [vp, C.POINTER(BatchInfo)]
        L.re_batch_autotune.argtypes = [vp, u32, vp, C.POINTER(BatchOptions)]
        L.re_diff_bilinear_forward.argtypes = [vp, sz, u32, u32, u32, vp, vp]
        L.re_diff_bilinear_backward.argtypes = [vp, u32, u32, u32, vp, sz, vp]
        L.re_diff_point_forward.argtypes = [vp, sz, C.POINTER(DiffPointParams), vp, vp]
        L.re_diff_point_backward.argtypes = [vp, vp, sz, C.POINTER(DiffPointParams), vp, vp, vp]
        L.re_diff_point_grad_count.argtypes = [u32]
        L.re_diff_point_grad_count.restype = sz
        L.re_diff_detail_forward.argtypes = [vp, u32, u32, u32, C.c_double, vp, u32, vp, vp]
        L.re_diff_detail_backward.argtypes = [vp, vp, u32, u32, u32, C.c_double, vp, u32, vp, vp, vp, vp]
        L.re_histogram_reset.argtypes = [u32, vp, vp, vp, vp]
        L.re_histogram_rgb.argtypes = [vp, sz, u32, u32, u32, C.c_uint64, u32, C.c_double, C.c_double, vp, vp, vp,
                                       vp]
        L.re_histogram_extremum.argtypes = [C.c_uint64, C.c_int, C.POINTER(C.c_float)]
        L.re_histogram_extremum.restype = C.c_int
        L.re_diff_menon_forward.argtypes = [vp, sz, u32, u32, u32, vp, vp, vp]
        L.re_diff_menon_backward.argtypes = [vp, u32, u32, u32, vp, vp, sz, vp]
        L.re_fingerprint_raw.argtypes = [C.POINTER(RawMetadata), vp, sz, vp]
        L.re_fingerprint_raster.argtypes = [u32, u32, sz, u32, vp, vp]
        L.re_image_create_fingerprinted.argtypes = [C.POINTER(RawMetadata), vp, sz, C.POINTER(vp), vp]
        L.re_sharpen_window.argtypes = [vp, sz, Rect, Rect, Rect, C.c_double, u32, vp, sz, vp]
        L.re_clarity_window.argtypes = [vp, sz, Rect, Rect, Rect, C.c_double, u32, u32, vp, sz, vp]
        L.re_texture_window.argtypes = [vp, sz, Rect, Rect, Rect, C.c_double, u32, u32, vp, sz, vp]
        L.re_convolution_window.argtypes = [vp, sz, Rect, Rect, Rect, u32, u32, f64p, vp, sz, vp]
        _lib = L
    return _lib


def check(status: int) -> None:
    if status:
        raise ReError(status, lib().re_last_error().decode(errors="replace"))


def library_path() -> str:
    return _LIB_PATH
