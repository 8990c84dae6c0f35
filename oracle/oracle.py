"""Python handle on the oracle -- TEST INFRASTRUCTURE ONLY.

Two checkers live here, both CPU-only:

* ``Oracle``    -- ctypes over ``oracle/liboracle.so``, the C restatement of the
  reference algorithms (``oracle/rawengine_oracle.c``, each function citing the
  reference file:line it follows).  ``render_raw``/``render_raster`` compose
  those primitives into the reference's node chains exactly as the reference's
  pull graph does (RawEngine.cpp:1384-1447 for the renderer, the per-node
  ``render_level`` methods for each stage, the CameraToWorking mip anchor of
  RawEngine.cpp:580-601).
* ``Reference`` -- ctypes over ``oracle/_ref/librefshim.so``: the UNMODIFIED
  reference library compiled from its own sources by ``oracle/Makefile``.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  The product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Op codes shared by the shim (ref_shim.cpp) and the chain composer below.
OP_WB = 1
OP_EXPOSURE = 2
OP_CAMERA_TO_WORKING = 3
OP_WORKING_TO_SRGB = 4
OP_TONE = 5
OP_OUTPUT_CLIP = 6
OP_SRGB_ENCODE = 7
OP_DISPLAY_TAG = 8
OP_CURVES_EXT = 9
OP_GUIDED_FILTER = 10
OP_CUBIC_RESIZE = 11
OP_ROTATE = 12
OP_WORKING_SPACE_CONVERT = 13
OP_SHARPEN = 14          # amount, radius (reference library only)
OP_CLARITY = 15          # amount, radius
OP_TEXTURE = 16          # amount, scale
OP_CONVOLUTION = 17      # width, height, coefficients (row-major)

ERRORS = {1: "invalid_argument", 2: "out_of_range", 3: "domain_error", 4: "length_error",
          5: "overflow_error", 6: "cancelled", 9: "logic_error", 10: "runtime_error"}


class OracleError(RuntimeError):
    def __init__(self, code: int, message: str = ""):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code
        self.kind = ERRORS.get(code, str(code))


class Rect(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32)]

    def tuple(self):
        return (self.x, self.y, self.width, self.height)


class RawMeta(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("row_stride_samples", C.c_uint32),
                ("pattern", C.c_uint32), ("cfa_phase_x", C.c_uint32), ("cfa_phase_y", C.c_uint32),
                ("active_area", Rect), ("black_levels", C.c_uint16 * 4),
                ("white_levels", C.c_uint16 * 4)]


class Curves(C.Structure):
    _fields_ = [("interpolation", C.c_int), ("count", C.c_uint32 * 4),
                ("knots", (C.c_double * 512) * 4), ("slopes", (C.c_double * 256) * 4),
                ("controls", ((C.c_double * 2) * 256) * 4), ("identity", C.c_int * 4)]


class Rotation(C.Structure):
    _fields_ = [("cx", C.c_double), ("cy", C.c_double), ("cosine", C.c_double),
                ("sine", C.c_double), ("width", C.c_uint32), ("height", C.c_uint32)]


def _rect(r) -> Rect:
    return Rect(*[int(v) for v in r])


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


@dataclass
class RawSpec:
    """Reference RawMetadata (RawEngine.hpp:57-65) plus its uint16 samples."""
    width: int
    height: int
    samples: np.ndarray
    row_stride: int = 0
    pattern: int = 0
    phase_x: int = 0
    phase_y: int = 0
    active: tuple = (0, 0, 0, 0)
    black: tuple = (0, 0, 0, 0)
    white: tuple = (65535, 65535, 65535, 65535)

    def meta_words(self) -> np.ndarray:
        return np.array([self.width, self.height, self.row_stride, self.pattern, self.phase_x,
                         self.phase_y, *self.active], dtype=np.uint32)

    def level_words(self) -> np.ndarray:
        return np.array([*self.black, *self.white], dtype=np.uint16)

    def struct(self) -> RawMeta:
        return RawMeta(self.width, self.height, self.row_stride, self.pattern, self.phase_x,
                       self.phase_y, _rect(self.active), (C.c_uint16 * 4)(*self.black),
                       (C.c_uint16 * 4)(*self.white))


@dataclass
class Op:
    """One node of a chain: code + flat parameter list (layout as in ref_shim.cpp)."""
    code: int
    params: list = field(default_factory=list)


def curves_params(interpolation: int, master, red=None, green=None, blue=None) -> list:
    ident = [(0.0, 0.0), (1.0, 1.0)]
    out = [float(interpolation)]
    for curve in (master, red or ident, green or ident, blue or ident):
        out.append(float(len(curve)))
        for x, y in curve:
            out += [float(x), float(y)]
    return out


def flatten_ops(ops):
    codes = np.array([o.code for o in ops], dtype=np.int32)
    params = np.array([float(p) for o in ops for p in o.params] or [0.0], dtype=np.float64)
    return codes, params


# --------------------------------------------------------------------------- oracle

class Oracle:
    """The C restatement (liboracle.so)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        f32p, u16p, u8p = C.POINTER(C.c_float), C.POINTER(C.c_uint16), C.POINTER(C.c_uint8)
        f64p, u32p = C.POINTER(C.c_double), C.POINTER(C.c_uint32)
        L.or_raw_normalize.argtypes = [C.POINTER(RawMeta), C.c_size_t]
        L.or_bilinear.argtypes = [C.POINTER(RawMeta), u16p, Rect, f32p]
        L.or_menon.argtypes = [C.POINTER(RawMeta), u16p, Rect, f32p, u8p]
        L.or_raw_input_region.argtypes = [C.POINTER(RawMeta), C.c_int, Rect, C.POINTER(Rect)]
        L.or_site_index.argtypes = [C.POINTER(RawMeta), C.c_uint32, C.c_uint32]
        L.or_cfa_color.argtypes = [C.POINTER(RawMeta), C.c_uint32, C.c_uint32]
        L.or_sample.argtypes = [C.POINTER(RawMeta), u16p, C.c_uint32, C.c_uint32]
        L.or_sample.restype = C.c_float
        L.or_white_balance.argtypes = [f32p, C.c_size_t, C.c_float, C.c_float, C.c_float]
        L.or_exposure_multiplier.argtypes = [C.c_float]
        L.or_exposure_multiplier.restype = C.c_float
        L.or_scale.argtypes = [f32p, C.c_size_t, C.c_float]
        L.or_camera_to_working_matrix.argtypes = [f64p, C.c_int, f32p]
        L.or_working_to_srgb_matrix.argtypes = [C.c_int, f32p]
        L.or_working_to_working_matrix.argtypes = [C.c_int, C.c_int, f32p]
        L.or_matrix3.argtypes = [f32p, C.c_size_t, f32p]
        L.or_tone_curve.argtypes = [f32p, C.c_size_t, C.c_float, C.c_float]
        L.or_output_clip.argtypes = [f32p, C.c_size_t]
        L.or_srgb_encode.argtypes = [f32p, C.c_size_t]
        L.or_curves_prepare.argtypes = [C.POINTER(Curves)]
        L.or_curves_apply.argtypes = [C.POINTER(Curves), f32p, C.c_size_t]
        L.or_curve_map.argtypes = [C.POINTER(Curves), C.c_uint, C.c_double]
        L.or_curve_map.restype = C.c_double
        L.or_request_bounds.argtypes = [Rect, C.c_uint32, C.c_uint32, C.POINTER(Rect)]
        L.or_mip_native_region.argtypes = [Rect, C.c_uint32, Rect, C.POINTER(Rect)]
        L.or_mip_reduce.argtypes = [f32p, Rect, C.c_uint32, Rect, f32p]
        L.or_guided_filter.argtypes = [f32p, Rect, Rect, Rect, C.c_uint32, C.c_double, C.c_int, f32p]
        L.or_guided_filter_region.argtypes = [Rect, Rect, C.c_uint32, C.POINTER(Rect)]
        L.or_local_statistics.argtypes = [f32p, Rect, Rect, Rect, C.c_uint32, f64p, f64p, u32p]
        L.or_local_statistics_region.argtypes = [Rect, Rect, C.c_uint32, C.POINTER(Rect)]
        L.or_cubic_axis.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p, u32p, f64p]
        L.or_cubic_support.argtypes = [C.c_uint32] * 4 + [Rect, C.POINTER(Rect)]
        L.or_cubic_resize.argtypes = [f32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, Rect, f32p]
        L.or_rotation_prepare.argtypes = [C.c_double, C.c_uint32, C.c_uint32, C.POINTER(Rotation)]
        L.or_rotate_support.argtypes = [C.POINTER(Rotation), Rect, C.POINTER(Rect)]
        L.or_rotate.argtypes = [C.POINTER(Rotation), f32p, Rect, f32p]
        L.or_plan_tiles.argtypes = [Rect, C.c_uint32, C.POINTER(Rect), C.c_size_t]
        L.or_plan_tiles.restype = C.c_size_t

    @staticmethod
    def _check(st):
        if st:
            raise OracleError(st, "oracle")

    # --- metadata / sources
    def normalized(self, raw: RawSpec) -> RawMeta:
        m = raw.struct()
        self._check(self.lib.or_raw_normalize(C.byref(m), int(raw.samples.size)))
        return m

    def demosaic(self, raw: RawSpec, rect, menon: bool, directions: bool = False):
        m = self.normalized(raw)
        s = np.ascontiguousarray(raw.samples, dtype=np.uint16)
        r = _rect(rect)
        out = np.zeros((r.height, r.width, 3), np.float32)
        if menon:
            d = np.zeros((r.height, r.width), np.uint8)
            self._check(self.lib.or_menon(C.byref(m), _ptr(s, C.c_uint16), r, _ptr(out, C.c_float),
                                          _ptr(d, C.c_uint8)))
            return (out, d) if directions else out
        self._check(self.lib.or_bilinear(C.byref(m), _ptr(s, C.c_uint16), r, _ptr(out, C.c_float)))
        return out

    def raw_input_region(self, raw: RawSpec, menon: bool, output):
        m = self.normalized(raw)
        region = Rect()
        self._check(self.lib.or_raw_input_region(C.byref(m), int(menon), _rect(output), C.byref(region)))
        return region.tuple()

    # --- matrices
    def camera_to_working(self, camera_to_xyz, target: int = 0) -> np.ndarray:
        out = np.zeros(9, np.float32)
        cam = np.ascontiguousarray(camera_to_xyz, np.float64).reshape(9)
        self._check(self.lib.or_camera_to_working_matrix(_ptr(cam, C.c_double), target, _ptr(out, C.c_float)))
        return out

    def working_to_srgb(self, source: int = 0) -> np.ndarray:
        out = np.zeros(9, np.float32)
        self._check(self.lib.or_working_to_srgb_matrix(source, _ptr(out, C.c_float)))
        return out

    def working_to_working(self, source: int, target: int) -> np.ndarray:
        out = np.zeros(9, np.float32)
        self._check(self.lib.or_working_to_working_matrix(source, target, _ptr(out, C.c_float)))
        return out

    # --- point stages (in place on a float32 array)
    def white_balance(self, rgb, r, g, b):
        self.lib.or_white_balance(_ptr(rgb, C.c_float), rgb.size // 3, r, g, b)

    def scale(self, rgb, multiplier):
        self.lib.or_scale(_ptr(rgb, C.c_float), rgb.size, multiplier)

    def exposure_multiplier(self, stops) -> float:
        return float(self.lib.or_exposure_multiplier(stops))

    def matrix3(self, rgb, m):
        m = _f32(m)
        self.lib.or_matrix3(_ptr(rgb, C.c_float), rgb.size // 3, _ptr(m, C.c_float))

    def tone_curve(self, rgb, shoulder, gamma):
        self.lib.or_tone_curve(_ptr(rgb, C.c_float), rgb.size, shoulder, gamma)

    def output_clip(self, rgb):
        self._check(self.lib.or_output_clip(_ptr(rgb, C.c_float), rgb.size))

    def srgb_encode(self, rgb):
        self._check(self.lib.or_srgb_encode(_ptr(rgb, C.c_float), rgb.size))

    def curves(self, params) -> Curves:
        c = Curves()
        it = iter(params)
        c.interpolation = int(next(it))
        for k in range(4):
            n = int(next(it))
            c.count[k] = n
            for i in range(n):
                c.knots[k][2 * i] = next(it)
                c.knots[k][2 * i + 1] = next(it)
        self._check(self.lib.or_curves_prepare(C.byref(c)))
        return c

    def curves_apply(self, c: Curves, rgb):
        self._check(self.lib.or_curves_apply(C.byref(c), _ptr(rgb, C.c_float), rgb.size))

    # --- levels
    def request_bounds(self, source, mip, quality):
        out = Rect()
        self._check(self.lib.or_request_bounds(_rect(source), mip, quality, C.byref(out)))
        return out.tuple()

    def mip_native_region(self, area, mip, output):
        out = Rect()
        self._check(self.lib.or_mip_native_region(_rect(area), mip, _rect(output), C.byref(out)))
        return out.tuple()

    def mip_reduce(self, native, mapped, mip, output):
        native = _f32(native)
        o = _rect(output)
        out = np.zeros((o.height, o.width, 3), np.float32)
        self.lib.or_mip_reduce(_ptr(native, C.c_float), _rect(mapped), mip, o, _ptr(out, C.c_float))
        return out

    # --- spatial
    def guided_filter_region(self, output, image, radius):
        out = Rect()
        self._check(self.lib.or_guided_filter_region(_rect(output), _rect(image), radius, C.byref(out)))
        return out.tuple()

    def guided_filter(self, tile, needed, output, image, radius, eps, prophoto=True):
        tile = _f32(tile)
        o = _rect(output)
        out = np.zeros((o.height, o.width, 3), np.float32)
        self._check(self.lib.or_guided_filter(_ptr(tile, C.c_float), _rect(needed), o, _rect(image),
                                              radius, eps, int(prophoto), _ptr(out, C.c_float)))
        return out

    def local_statistics(self, tile, needed, output, image, radius):
        tile = _f32(tile)
        o = _rect(output)
        mean = np.zeros((o.height, o.width, 3), np.float64)
        var = np.zeros_like(mean)
        cnt = np.zeros((o.height, o.width, 3), np.uint32)
        self._check(self.lib.or_local_statistics(_ptr(tile, C.c_float), _rect(needed), o, _rect(image),
                                                 radius, _ptr(mean, C.c_double), _ptr(var, C.c_double),
                                                 _ptr(cnt, C.c_uint32)))
        return mean, var, cnt

    # --- geometry
    def cubic_axis(self, n_in, n_out, index):
        idx = np.zeros(18, np.uint32)
        w = np.zeros(18, np.float64)
        center = C.c_uint32()
        n = self.lib.or_cubic_axis(n_in, n_out, index, C.byref(center), _ptr(idx, C.c_uint32),
                                   _ptr(w, C.c_double))
        if n < 0:
            raise OracleError(-n, "cubic axis")
        return center.value, idx[:n].copy(), w[:n].copy()

    def cubic_support(self, in_w, in_h, out_w, out_h, output):
        out = Rect()
        self._check(self.lib.or_cubic_support(in_w, in_h, out_w, out_h, _rect(output), C.byref(out)))
        return out.tuple()

    def cubic_resize(self, src, out_w, out_h, output):
        src = _f32(src)
        h, w = src.shape[:2]
        o = _rect(output)
        out = np.zeros((o.height, o.width, 3), np.float32)
        self._check(self.lib.or_cubic_resize(_ptr(src, C.c_float), w, h, out_w, out_h, o,
                                             _ptr(out, C.c_float)))
        return out

    def rotation(self, angle, width, height) -> Rotation:
        r = Rotation()
        self._check(self.lib.or_rotation_prepare(angle, width, height, C.byref(r)))
        return r

    def rotate_support(self, rot: Rotation, output):
        out = Rect()
        self._check(self.lib.or_rotate_support(C.byref(rot), _rect(output), C.byref(out)))
        return out.tuple()

    def rotate(self, rot: Rotation, src, output):
        src = _f32(src)
        o = _rect(output)
        out = np.zeros((o.height, o.width, 3), np.float32)
        self._check(self.lib.or_rotate(C.byref(rot), _ptr(src, C.c_float), o, _ptr(out, C.c_float)))
        return out

    def plan_tiles(self, viewport, tile):
        n = self.lib.or_plan_tiles(_rect(viewport), tile, None, 0)
        arr = (Rect * max(n, 1))()
        self.lib.or_plan_tiles(_rect(viewport), tile, arr, n)
        return [arr[i].tuple() for i in range(n)]

    # --- chains ------------------------------------------------------------
    def render_raw(self, raw: RawSpec, menon: bool, ops, viewport, mip: int = 0, quality: int = 1):
        """A RAW node chain rendered through the reference renderer's rules.

        Supports the chain shapes the reference's ImageGraph/ExecutableEditGraph
        build on this path: source -> camera-linear point ops -> optional
        CameraToWorking (the only mip anchor on a RAW chain, RawEngine.cpp:550-601)
        -> scene/display point ops.  Per-pixel results do not depend on the
        render tile size, so the whole viewport is evaluated at once.
        """
        m = self.normalized(raw)
        area = m.active_area.tuple()
        anchor = next((i for i, o in enumerate(ops) if o.code == OP_CAMERA_TO_WORKING), None)
        if mip:
            if anchor is None:
                raise OracleError(1, "RAW chain without camera anchor has no reduced levels")
            reduced = self.request_bounds(area, mip, quality)
            self._inside(reduced, viewport)
            native_rect = self.mip_native_region(area, mip, viewport)
            native = self.demosaic(raw, native_rect, menon)
            self._apply_points(native, ops[:anchor + 1])
            out = self.mip_reduce(native, native_rect, mip, viewport)
            self._apply_points(out, ops[anchor + 1:])
            return out
        self._inside(area, viewport)
        out = self.demosaic(raw, viewport, menon)
        self._apply_points(out, ops)
        return out

    @staticmethod
    def _inside(area, r):
        if (r[0] < area[0] or r[1] < area[1] or r[0] + r[2] > area[0] + area[2]
                or r[1] + r[3] > area[1] + area[3]):
            raise OracleError(2, "viewport outside bounds")

    def _apply_points(self, rgb, ops):
        space = 0
        for o in ops:
            p = o.params
            if o.code == OP_WB:
                self.white_balance(rgb, *p[:3])
            elif o.code == OP_EXPOSURE:
                self.scale(rgb, self.exposure_multiplier(p[0]))
            elif o.code == OP_CAMERA_TO_WORKING:
                space = int(p[9])
                self.matrix3(rgb, self.camera_to_working(p[:9], space))
            elif o.code == OP_WORKING_TO_SRGB:
                self.matrix3(rgb, self.working_to_srgb(space))
            elif o.code == OP_WORKING_SPACE_CONVERT:
                if int(p[0]) != space:
                    self.matrix3(rgb, self.working_to_working(space, int(p[0])))
                space = int(p[0])
            elif o.code == OP_TONE:
                self.tone_curve(rgb, p[0], p[1])
            elif o.code == OP_OUTPUT_CLIP:
                self.output_clip(rgb)
            elif o.code == OP_SRGB_ENCODE:
                self.srgb_encode(rgb)
            elif o.code == OP_DISPLAY_TAG:
                pass
            elif o.code == OP_CURVES_EXT:
                self.curves_apply(self.curves(p), rgb)
            else:
                raise OracleError(1, f"op {o.code} is not a point stage")


# ------------------------------------------------------------------------ reference

def histogram_rgb(rgb, bins=256, lower=0.0, upper=1.0, tile=0):
    """NumPy restatement of histogram_rgb (ImageAnalysis.cpp:9-69) over an
    (h, w, 3) float32 image rendered as one viewport in tiles of `tile` (0: one
    tile).  Bins: min(bins - 1, uint32((double(s) - lower) / span * bins)) in
    binary64; extrema over finite samples, the first in tile traversal order
    among equal values (which decides between +0 and -0)."""
    rgb = np.asarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    t = tile or max(h, w)
    order = []
    for y0 in range(0, h, t):
        for x0 in range(0, w, t):
            order.append(rgb[y0:y0 + t, x0:x0 + t].reshape(-1, 3))
    flat = np.concatenate(order) if order else np.zeros((0, 3), np.float32)
    span = upper - lower
    out = []
    for c in range(3):
        v = flat[:, c]
        fin = np.isfinite(v)
        d = v[fin].astype(np.float64)
        under, over = d < lower, d > upper
        mid = d[~under & ~over]
        idx = np.minimum(bins - 1, ((mid - lower) / span * bins).astype(np.uint64))
        counts = np.bincount(idx.astype(np.int64), minlength=bins).astype(np.uint64)
        fv = v[fin]
        mn = mx = None
        if fv.size:
            mn = float(fv[int(np.argmax(fv == fv.min()))])
            mx = float(fv[int(np.argmax(fv == fv.max()))])
        out.append(dict(counts=counts, underflow=int(under.sum()), overflow=int(over.sum()),
                        nonfinite=int((~fin).sum()), minimum=mn, maximum=mx))
    return out


class Reference:
    """The unmodified reference library (oracle/_ref), through ref_shim.cpp."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "_ref", "librefshim.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        L = self.lib = C.CDLL(path)
        u32p, u16p, i32p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint16), C.POINTER(C.c_int32)
        f64p, f32p = C.POINTER(C.c_double), C.POINTER(C.c_float)
        L.refshim_last_error.restype = C.c_char_p
        L.refshim_render_raw.argtypes = [u32p, u16p, u16p, C.c_size_t, C.c_int, i32p, C.c_int, f64p,
                                         u32p, C.c_uint32, C.c_uint32, C.c_uint32, f32p, u32p]
        L.refshim_render_raw_scheduled.argtypes = [u32p, u16p, u16p, C.c_size_t, C.c_int, i32p, C.c_int,
                                                   f64p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, f32p,
                                                   C.c_uint32]
        L.refshim_render_raster.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, f32p,
                                            C.c_size_t, i32p, C.c_int, f64p, u32p, C.c_uint32,
                                            C.c_uint32, C.c_uint32, f32p, u32p]
        L.refshim_raw_input_region.argtypes = [u32p, u16p, u16p, C.c_size_t, C.c_int, i32p, C.c_int,
                                               f64p, u32p, C.c_uint32, C.c_uint32, u32p]
        L.refshim_raster_input_region.argtypes = [C.c_uint32, C.c_uint32, C.c_int, i32p, C.c_int, f64p,
                                                  u32p, C.c_uint32, C.c_uint32, u32p]
        L.refshim_session_create.restype = C.c_void_p
        L.refshim_session_create.argtypes = [u32p, u16p, u16p, C.c_size_t, C.c_int, i32p, C.c_int, f64p,
                                             C.c_uint32]
        L.refshim_session_render.argtypes = [C.c_void_p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, f32p]
        L.refshim_session_destroy.argtypes = [C.c_void_p]
        L.refshim_local_statistics.argtypes = [f32p, u32p, u32p, u32p, C.c_uint32, C.c_int, f64p, f64p,
                                               u32p]
        L.refshim_guided_filter.argtypes = [f32p, u32p, u32p, u32p, C.c_uint32, C.c_double, C.c_int,
                                            f32p]
        L.refshim_fingerprint_raw.argtypes = [u32p, u16p, u16p, C.c_size_t, C.POINTER(C.c_uint8)]
        L.refshim_fingerprint_raster.argtypes = [C.c_uint32, C.c_uint32, C.c_int, f32p, C.c_size_t,
                                                 C.POINTER(C.c_uint8)]
        L.refshim_stencil_raster.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.c_int, f32p, C.c_size_t, f64p, u32p,
                                             C.c_uint32, C.c_uint32, C.c_uint32, f32p]
        L.refshim_histogram_raster.argtypes = [C.c_uint32, C.c_uint32, C.c_int, f32p, C.c_size_t, i32p, C.c_int,
                                               f64p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                               C.c_double, C.c_double, C.POINTER(C.c_uint64),
                                               C.POINTER(C.c_uint64), f32p, C.POINTER(C.c_uint8)]

    def _check(self, st):
        if st:
            raise OracleError(st, self.lib.refshim_last_error().decode())

    @staticmethod
    def _u32(v):
        return np.ascontiguousarray(v, dtype=np.uint32)

    def render_raw(self, raw: RawSpec, menon: bool, ops, viewport, tile=256, mip=0, quality=1,
                   scheduled_workers: int = 0):
        codes, params = flatten_ops(ops)
        vp = self._u32(viewport)
        out = np.zeros((int(vp[3]), int(vp[2]), 3), np.float32)
        s = np.ascontiguousarray(raw.samples, dtype=np.uint16)
        args = (_ptr(raw.meta_words(), C.c_uint32), _ptr(raw.level_words(), C.c_uint16),
                _ptr(s, C.c_uint16), s.size, int(menon), _ptr(codes, C.c_int32), len(ops),
                _ptr(params, C.c_double), _ptr(vp, C.c_uint32), tile, mip, quality,
                _ptr(out, C.c_float))
        if scheduled_workers:
            self._check(self.lib.refshim_render_raw_scheduled(*args, scheduled_workers))
        else:
            self._check(self.lib.refshim_render_raw(*args, None))
        return out

    def session(self, raw: RawSpec, menon: bool, ops, workers: int) -> "RefSession":
        """A reference render session (RawImage, node chain and TileScheduler
        built once); its render() only submits the tiles and waits."""
        return RefSession(self, raw, menon, ops, workers)

    def raw_bounds(self, raw: RawSpec, menon: bool, ops):
        codes, params = flatten_ops(ops)
        b = np.zeros(4, np.uint32)
        s = np.ascontiguousarray(raw.samples, dtype=np.uint16)
        self._check(self.lib.refshim_render_raw(
            _ptr(raw.meta_words(), C.c_uint32), _ptr(raw.level_words(), C.c_uint16),
            _ptr(s, C.c_uint16), s.size, int(menon), _ptr(codes, C.c_int32), len(ops),
            _ptr(params, C.c_double), _ptr(self._u32([0, 0, 0, 0]), C.c_uint32), 256, 0, 1, None,
            _ptr(b, C.c_uint32)))
        return tuple(int(v) for v in b)

    def render_raster(self, pixels, ops, viewport, tile=256, mip=0, quality=1, space=0, stride=0):
        pixels = _f32(pixels)
        h, w = pixels.shape[:2]
        if stride:
            w = int(pixels.shape[1]) if not stride else w
        codes, params = flatten_ops(ops)
        vp = self._u32(viewport)
        out = np.zeros((int(vp[3]), int(vp[2]), 3), np.float32)
        b = np.zeros(4, np.uint32)
        self._check(self.lib.refshim_render_raster(
            w, h, 0, space, _ptr(pixels, C.c_float), pixels.size, _ptr(codes, C.c_int32), len(ops),
            _ptr(params, C.c_double), _ptr(vp, C.c_uint32), tile, mip, quality,
            _ptr(out, C.c_float), _ptr(b, C.c_uint32)))
        return out

    def raw_input_region(self, raw: RawSpec, menon: bool, ops, output, mip=0, quality=1):
        codes, params = flatten_ops(ops)
        region = np.zeros(4, np.uint32)
        s = np.ascontiguousarray(raw.samples, dtype=np.uint16)
        self._check(self.lib.refshim_raw_input_region(
            _ptr(raw.meta_words(), C.c_uint32), _ptr(raw.level_words(), C.c_uint16),
            _ptr(s, C.c_uint16), s.size, int(menon), _ptr(codes, C.c_int32), len(ops),
            _ptr(params, C.c_double), _ptr(self._u32(output), C.c_uint32), mip, quality,
            _ptr(region, C.c_uint32)))
        return tuple(int(v) for v in region)

    def raster_input_region(self, width, height, ops, output, mip=0, quality=1, space=0):
        codes, params = flatten_ops(ops)
        region = np.zeros(4, np.uint32)
        self._check(self.lib.refshim_raster_input_region(
            width, height, space, _ptr(codes, C.c_int32), len(ops), _ptr(params, C.c_double),
            _ptr(self._u32(output), C.c_uint32), mip, quality, _ptr(region, C.c_uint32)))
        return tuple(int(v) for v in region)

    def local_statistics(self, tile, needed, output, image, radius, space=0):
        tile = _f32(tile)
        o = self._u32(output)
        mean = np.zeros((int(o[3]), int(o[2]), 3), np.float64)
        var = np.zeros_like(mean)
        cnt = np.zeros(mean.shape, np.uint32)
        self._check(self.lib.refshim_local_statistics(
            _ptr(tile, C.c_float), _ptr(self._u32(needed), C.c_uint32), _ptr(o, C.c_uint32),
            _ptr(self._u32(image), C.c_uint32), radius, space, _ptr(mean, C.c_double),
            _ptr(var, C.c_double), _ptr(cnt, C.c_uint32)))
        return mean, var, cnt

    def guided_filter(self, tile, needed, output, image, radius, eps, space=0):
        tile = _f32(tile)
        o = self._u32(output)
        out = np.zeros((int(o[3]), int(o[2]), 3), np.float32)
        self._check(self.lib.refshim_guided_filter(
            _ptr(tile, C.c_float), _ptr(self._u32(needed), C.c_uint32), _ptr(o, C.c_uint32),
            _ptr(self._u32(image), C.c_uint32), radius, eps, space, _ptr(out, C.c_float)))
        return out


    def fingerprint_raw(self, raw: RawSpec) -> bytes:
        d = np.zeros(32, np.uint8)
        s = np.ascontiguousarray(raw.samples, dtype=np.uint16)
        self._check(self.lib.refshim_fingerprint_raw(_ptr(raw.meta_words(), C.c_uint32),
                                                     _ptr(raw.level_words(), C.c_uint16), _ptr(s, C.c_uint16),
                                                     s.size, _ptr(d, C.c_uint8)))
        return d.tobytes()

    def fingerprint_raster(self, pixels, space=0) -> bytes:
        pixels = _f32(pixels)
        h, w = pixels.shape[:2]
        d = np.zeros(32, np.uint8)
        self._check(self.lib.refshim_fingerprint_raster(w, h, space, _ptr(pixels, C.c_float), pixels.size,
                                                        _ptr(d, C.c_uint8)))
        return d.tobytes()

    STENCILS = {"sharpen": 0, "clarity": 1, "texture": 2, "convolution": 3}

    def stencil(self, kind, pixels, viewport, amount=0.0, radius=1, kernel=None, tile=256, mip=0, quality=1,
                space=0):
        """SharpenNode / ClarityNode / TextureNode (radius = scale) /
        ConvolutionNode over a raster source, rendered through render_image."""
        pixels = _f32(pixels)
        h, w = pixels.shape[:2]
        if kind == "convolution":
            k = np.asarray(kernel, np.float64)
            params = np.concatenate([[k.shape[1], k.shape[0]], k.reshape(-1)])
        else:
            params = np.array([amount, radius], np.float64)
        params = np.ascontiguousarray(params, np.float64)
        vp = self._u32(viewport)
        out = np.zeros((int(vp[3]), int(vp[2]), 3), np.float32)
        self._check(self.lib.refshim_stencil_raster(
            self.STENCILS[kind], w, h, space, _ptr(pixels, C.c_float), pixels.size, _ptr(params, C.c_double),
            _ptr(vp, C.c_uint32), tile, mip, quality, _ptr(out, C.c_float)))
        return out

    def histogram(self, pixels, viewport, bins=256, lower=0.0, upper=1.0, ops=(), tile=256, mip=0, quality=1,
                  space=0):
        """histogram_rgb of a raster-source chain (finite pixels only: the
        reference's raster source rejects non-finite input).  Returns per
        channel the same dict layout as librawops_b200.render.histogram_rgb."""
        pixels = _f32(pixels)
        h, w = pixels.shape[:2]
        codes, params = flatten_ops(ops)
        counts = np.zeros(3 * bins, np.uint64)
        tallies = np.zeros(9, np.uint64)
        extrema = np.zeros(6, np.float32)
        present = np.zeros(6, np.uint8)
        self._check(self.lib.refshim_histogram_raster(
            w, h, space, _ptr(pixels, C.c_float), pixels.size, _ptr(codes, C.c_int32), len(ops),
            _ptr(params, C.c_double), _ptr(self._u32(viewport), C.c_uint32), tile, mip, quality, bins, lower, upper,
            _ptr(counts, C.c_uint64), _ptr(tallies, C.c_uint64), _ptr(extrema, C.c_float),
            _ptr(present, C.c_uint8)))
        counts = counts.reshape(3, bins)
        return [dict(counts=counts[c], underflow=int(tallies[c]), overflow=int(tallies[3 + c]),
                     nonfinite=int(tallies[6 + c]), minimum=float(extrema[c]) if present[c] else None,
                     maximum=float(extrema[3 + c]) if present[3 + c] else None) for c in range(3)]


class RefSession:
    """refshim_session_*: setup outside the timed calls."""

    def __init__(self, ref: Reference, raw: RawSpec, menon: bool, ops, workers: int):
        codes, params = flatten_ops(ops)
        self.ref = ref
        self.samples = np.ascontiguousarray(raw.samples, dtype=np.uint16)
        self.handle = ref.lib.refshim_session_create(
            _ptr(raw.meta_words(), C.c_uint32), _ptr(raw.level_words(), C.c_uint16),
            _ptr(self.samples, C.c_uint16), self.samples.size, int(menon), _ptr(codes, C.c_int32), len(ops),
            _ptr(params, C.c_double), workers)
        if not self.handle:
            raise OracleError(10, ref.lib.refshim_last_error().decode())

    def render(self, viewport, tile=256, mip=0, quality=1, out=None):
        vp = Reference._u32(viewport)
        if out is None:
            out = np.zeros((int(vp[3]), int(vp[2]), 3), np.float32)
        self.ref._check(self.ref.lib.refshim_session_render(self.handle, _ptr(vp, C.c_uint32), tile, mip, quality,
                                                            _ptr(out, C.c_float)))
        return out

    def close(self):
        if self.handle:
            self.ref.lib.refshim_session_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


def reference_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "librefshim.so"))
