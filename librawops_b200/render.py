"""Python surface of the B200 render path, over the C ABI (include/rawengine_b200.h).

This is the thin binding tests and benchmarks use.  The reference's own
surface for this path is its C++ API (RawImage, ImageGraph, Renderer, node
classes, TileScheduler); the drop-in C++ mirror lives in include/rawengine/.
Here a render chain is a `Pipeline`: the demosaic policy plus the ordered point
stages of the reference nodes it replaces, compiled into one fused launch.

Device buffers are torch CUDA tensors (PyTorch is only the allocator/stream
plumbing); host buffers are NumPy arrays.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _capi
from ._capi import (MAX_STAGES, Rect, RawMetadata, RenderDesc, RenderStats, ReError, Stage, check,
                    lib)

BILINEAR, MENON, MENON_FAST = 0, 1, 2   # MENON: binary64, bit-exact; MENON_FAST: binary32, exact directions
PROPHOTO, REC2020 = 0, 1
FINAL, PREVIEW = 1, 0


def _rect(r) -> Rect:
    return Rect(*[int(v) for v in r])


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        return None
    return int(getattr(stream, "cuda_stream", stream))


@dataclass
class Metadata:
    """RawMetadata (RawEngine.hpp:57-65)."""
    width: int
    height: int
    row_stride_samples: int = 0
    pattern: int = 0                       # 0 RGGB, 1 BGGR, 2 GRBG, 3 GBRG
    cfa_phase_x: int = 0
    cfa_phase_y: int = 0
    active_area: tuple = (0, 0, 0, 0)
    black_levels: tuple = (0, 0, 0, 0)
    white_levels: tuple = (65535, 65535, 65535, 65535)

    def struct(self) -> RawMetadata:
        return RawMetadata(self.width, self.height, self.row_stride_samples, self.pattern,
                           self.cfa_phase_x, self.cfa_phase_y, _rect(self.active_area),
                           (C.c_uint16 * 4)(*self.black_levels), (C.c_uint16 * 4)(*self.white_levels))

    @staticmethod
    def from_struct(m: RawMetadata) -> "Metadata":
        return Metadata(m.width, m.height, m.row_stride_samples, m.pattern, m.cfa_phase_x,
                        m.cfa_phase_y, m.active_area.tuple(), tuple(m.black_levels),
                        tuple(m.white_levels))


def normalize_metadata(meta: Metadata, count: int) -> Metadata:
    """RawImage's metadata validation/normalization (RawEngine.cpp:223-250)."""
    m = meta.struct()
    check(lib().re_raw_metadata_normalize(C.byref(m), count))
    return Metadata.from_struct(m)


class Image:
    """A device-resident RAW source (RawImage).  `samples` is a host uint16
    array (uploaded) or a CUDA uint16 tensor (wrapped; kept alive here)."""

    def __init__(self, meta: Metadata, samples):
        m = meta.struct()
        handle = C.c_void_p()
        self._keep = None
        if hasattr(samples, "is_cuda") and samples.is_cuda:
            self._keep = samples
            check(lib().re_image_wrap_device(C.byref(m), C.c_void_p(samples.data_ptr()),
                                             samples.numel(), C.byref(handle)))
        else:
            arr = np.ascontiguousarray(samples, dtype=np.uint16).reshape(-1)
            check(lib().re_image_create(C.byref(m), arr.ctypes.data_as(C.POINTER(C.c_uint16)),
                                        arr.size, C.byref(handle)))
        self.handle = handle
        self.metadata = Metadata.from_struct(m)

    @classmethod
    def ingest(cls, meta: Metadata, samples):
        """A host plane uploaded while its canonical fingerprint is computed
        (re_image_create_fingerprinted): returns (image, 32-byte digest)."""
        m = meta.struct()
        handle = C.c_void_p()
        digest = (C.c_uint8 * 32)()
        arr = np.ascontiguousarray(samples, dtype=np.uint16).reshape(-1)
        check(lib().re_image_create_fingerprinted(C.byref(m), arr.ctypes.data, arr.size, C.byref(handle), digest))
        img = cls.__new__(cls)
        img._keep = None
        img.handle = handle
        img.metadata = Metadata.from_struct(m)
        return img, bytes(digest)

    @property
    def active_area(self):
        return self.metadata.active_area

    def close(self):
        if self.handle:
            lib().re_image_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CurveSet:
    """ExtendedCurvesSettings (ToneOps.hpp:19-25) uploaded for the device."""

    def __init__(self, master, red=None, green=None, blue=None, cubic: bool = True):
        ident = [(0.0, 0.0), (1.0, 1.0)]
        curves = [master, red or ident, green or ident, blue or ident]
        counts = (C.c_uint32 * 4)(*[len(c) for c in curves])
        flat = np.array([v for c in curves for p in c for v in p], np.float64)
        h = C.c_void_p()
        check(lib().re_curve_set_create(int(cubic), counts, flat.ctypes.data_as(C.POINTER(C.c_double)),
                                        C.byref(h)))
        self.handle = h

    def __del__(self):
        try:
            if self.handle:
                lib().re_curve_set_destroy(self.handle)
        except Exception:
            pass


def camera_to_working_matrix(camera_to_xyz_d50, target: int = PROPHOTO) -> np.ndarray:
    out = np.zeros(9, np.float32)
    cam = np.ascontiguousarray(camera_to_xyz_d50, np.float64).reshape(9)
    check(lib().re_camera_to_working_matrix(cam.ctypes.data_as(C.POINTER(C.c_double)), target,
                                            out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def working_to_srgb_matrix(source: int = PROPHOTO) -> np.ndarray:
    out = np.zeros(9, np.float32)
    check(lib().re_working_to_srgb_matrix(source, out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def working_to_working_matrix(source: int, target: int) -> np.ndarray:
    out = np.zeros(9, np.float32)
    check(lib().re_working_to_working_matrix(source, target, out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def exposure_multiplier(stops: float) -> float:
    out = C.c_float()
    check(lib().re_exposure_multiplier(C.c_float(stops), C.byref(out)))
    return out.value


@dataclass
class Pipeline:
    """Demosaic policy + ordered point stages of a RAW render chain."""
    demosaic: int = BILINEAR
    stages: list = field(default_factory=list)
    anchor: int = -1
    curves: list = field(default_factory=list)
    space: int = PROPHOTO

    def _add(self, kind, f=(), arg=0):
        if len(self.stages) >= MAX_STAGES:
            raise ReError(_capi.RE_LENGTH_ERROR, "too many fused stages")
        self.stages.append((kind, arg, tuple(float(v) for v in f)))
        return self

    # WhiteBalanceNode (RawEngine.cpp:408-431)
    def white_balance(self, r, g, b):
        for v in (r, g, b):
            if not np.isfinite(v) or v <= 0 or v > 65536:
                raise ReError(1, "white balance gains must be finite and in (0, 65536]")
        return self._add(_capi.STAGE_GAIN3, (np.float32(r), np.float32(g), np.float32(b)))

    # ExposureNode (RawEngine.cpp:465-500)
    def exposure(self, stops):
        return self._add(_capi.STAGE_SCALE, (exposure_multiplier(stops),))

    # CameraToWorkingNode (RawEngine.cpp:502-601); the mip anchor of a RAW chain.
    def camera_to_working(self, camera_to_xyz_d50, target: int = PROPHOTO, anchor: bool = True):
        self.space = target
        self._add(_capi.STAGE_MATRIX, camera_to_working_matrix(camera_to_xyz_d50, target))
        if anchor:
            self.anchor = len(self.stages) - 1
        return self

    def matrix(self, m):
        return self._add(_capi.STAGE_MATRIX, np.asarray(m, np.float32).reshape(9))

    # WorkingToSrgbNode (RawEngine.cpp:658-703)
    def working_to_srgb(self):
        return self._add(_capi.STAGE_MATRIX, working_to_srgb_matrix(self.space))

    # WorkingSpaceConvertNode (RawEngine.cpp:603-656)
    def working_space_convert(self, target):
        if target != self.space:
            self._add(_capi.STAGE_MATRIX, working_to_working_matrix(self.space, target))
        self.space = target
        return self

    # ToneCurveNode (RawEngine.cpp:705-758)
    def tone_curve(self, shoulder=0.25, gamma=1.0):
        inv = np.float32(1.0) / np.float32(gamma)
        if not (np.isfinite(shoulder) and shoulder > 0 and np.isfinite(gamma) and gamma > 0
                and np.isfinite(inv)):
            raise ReError(1, "tone shoulder and gamma must be finite and positive")
        return self._add(_capi.STAGE_TONE, (np.float32(shoulder), inv))

    # ExtendedCurvesNode (ToneOps.cpp:795-844)
    def extended_curves(self, curve_set: CurveSet):
        idx = len(self.curves)
        if idx >= 4:
            raise ReError(1, "at most four curve stages per chain")
        self.curves.append(curve_set)
        return self._add(_capi.STAGE_CURVES, (), idx)

    # OutputClipNode (RawEngine.cpp:1215-1233)
    def output_clip(self):
        return self._add(_capi.STAGE_CLIP)

    # SrgbEncodeNode (RawEngine.cpp:1235-1277)
    def srgb_encode(self):
        return self._add(_capi.STAGE_SRGB)

    def desc(self) -> RenderDesc:
        d = RenderDesc()
        d.demosaic = self.demosaic
        d.anchor = self.anchor
        d.count = len(self.stages)
        for i, (kind, arg, f) in enumerate(self.stages):
            d.stages[i].kind = kind
            d.stages[i].arg = arg
            for j, v in enumerate(f):
                d.stages[i].f[j] = v
        for i, cs in enumerate(self.curves):
            d.curves[i] = cs.handle
        return d


def request_bounds(source, mip=0, quality=FINAL):
    out = Rect()
    check(lib().re_request_bounds(_rect(source), mip, quality, C.byref(out)))
    return out.tuple()


def raw_input_region(meta: Metadata, demosaic: int, output):
    out = Rect()
    m = meta.struct()
    check(lib().re_raw_input_region(C.byref(m), demosaic, _rect(output), C.byref(out)))
    return out.tuple()


def mip_native_region(native_bounds, mip, output):
    out = Rect()
    check(lib().re_mip_native_region(_rect(native_bounds), mip, _rect(output), C.byref(out)))
    return out.tuple()


def plan_tiles(viewport, tile_size):
    n = C.c_size_t()
    check(lib().re_plan_tiles(_rect(viewport), tile_size, None, 0, C.byref(n)))
    arr = (Rect * max(n.value, 1))()
    check(lib().re_plan_tiles(_rect(viewport), tile_size, arr, n.value, C.byref(n)))
    return [arr[i].tuple() for i in range(n.value)]


def render(image: Image, pipe: Pipeline, viewport, mip: int = 0, quality: int = FINAL, out=None,
           stream=None, stats: bool = False):
    """Renderer::render_image of a RAW chain.  Returns float32 (h, w, 3): a NumPy
    array by default, or fills `out` (a CUDA float tensor of shape (h, w, 3) or a
    NumPy array) in place."""
    vp = _rect(viewport)
    d = pipe.desc()
    st = RenderStats()
    if out is None:
        out = np.empty((vp.height, vp.width, 3), np.float32)
    on_device = hasattr(out, "is_cuda") and out.is_cuda
    ptr = out.data_ptr() if on_device else out.ctypes.data
    stride = (out.stride(0) if on_device else out.strides[0] // 4)
    check(lib().re_render_raw(image.handle, C.byref(d), vp, mip, quality, C.c_void_p(ptr), stride,
                              int(on_device), C.c_void_p(_stream_ptr(stream)),
                              C.byref(st) if stats else None))
    if stats:
        return out, {"pixels": st.pixels, "native_pixels": st.native_pixels,
                     "menon_decisions": st.menon_decisions, "menon_ties": st.menon_near_ties,
                     "launches": st.launches, "device_ms": st.device_ms}
    return out


def render_async(image: Image, pipe: Pipeline, viewport, out, device_status, mip=0, quality=FINAL,
                 scratch=None, stream=None):
    """Enqueue-only render into a CUDA tensor; guards land in `device_status`
    (a CUDA int32 tensor holding one zeroed word)."""
    vp = _rect(viewport)
    d = pipe.desc()
    check(lib().re_render_raw_async(image.handle, C.byref(d), vp, mip, quality,
                                    C.c_void_p(out.data_ptr()), out.stride(0),
                                    C.c_void_p(device_status.data_ptr()),
                                    C.c_void_p(scratch.data_ptr() if scratch is not None else None),
                                    C.c_void_p(_stream_ptr(stream))))


def menon_directions(image: Image, viewport, demosaic: int = MENON, out=None, stream=None):
    """Menon direction map of a viewport (CUDA uint8, 1 = horizontal; green
    sites 1) and the number of near-tie decisions (re_menon_directions)."""
    import torch
    vp = _rect(viewport)
    if out is None:
        out = torch.empty((vp.height, vp.width), dtype=torch.uint8, device="cuda")
    ties = C.c_uint64()
    check(lib().re_menon_directions(image.handle, demosaic, vp, C.c_void_p(out.data_ptr()), C.byref(ties),
                                    C.c_void_p(_stream_ptr(stream))))
    return out, ties.value


def scratch_bytes(image: Image, pipe: Pipeline, viewport, mip: int) -> int:
    d = pipe.desc()
    return int(lib().re_render_scratch_bytes(image.handle, C.byref(d), _rect(viewport), mip))


def status_from_device(word: int) -> None:
    check(lib().re_status_from_device(int(word) & 0xFFFFFFFF))


def render_tiles(image: Image, pipe: Pipeline, viewport, tile_size: int, callback, mip=0,
                 quality=FINAL, stream=None):
    """Renderer::render_tiles: `callback(bounds, rgb)` per tile in the
    reference's row-major order; a truthy return cancels (RE_CANCELLED)."""
    d = pipe.desc()
    errors = []

    def _cb(rect_p, rgb_p, _user):
        r = rect_p.contents.tuple()
        arr = np.ctypeslib.as_array(rgb_p, shape=(r[3], r[2], 3)).copy()
        try:
            return 1 if callback(r, arr) else 0
        except Exception as e:  # propagate after the C call returns
            errors.append(e)
            return 1

    cb = _capi.TILE_CALLBACK(_cb)
    status = lib().re_render_tiles(image.handle, C.byref(d), _rect(viewport), tile_size, mip, quality, cb,
                                   None, C.c_void_p(_stream_ptr(stream)))
    if errors:
        raise errors[0]
    check(status)


# ------------------------------------------------------------------ batches

def synthetic_samples(img, device="cuda"):
    """Device-synthesized sensor codes for a workloads.MixedImage."""
    from . import synthetic
    return synthetic.bayer_device(img.width, img.height, seed=img.seed, pattern=img.pattern, phase=img.phase,
                                  stride=img.stride, black=img.black, white=img.white, device=device)


@dataclass
class Geometry:
    """A cubic resize (kind "cubic", canvas (w, h)) or rotation (kind
    "rotate", angle in degrees) between a RAW chain and later point stages
    (`post`, a Pipeline of point stages or None), for batch requests."""
    kind: str
    canvas: tuple = (0, 0)
    angle: float = 0.0
    post: Optional["Pipeline"] = None


class Batch:
    """Many render requests drained by one persistent kernel (re_batch_*).

    requests: (image, pipeline, viewport, mip, quality, out[, geometry]) with
    `out` a CUDA float32 tensor of shape (h, w, 3) (row stride from the
    tensor).  With a Geometry, `pipeline` renders the RAW source at native
    resolution (the geometry's input), the geometry maps it to its canvas at
    level `mip`, then geometry.post runs; viewport is in canvas level
    coordinates.  The batch keeps references to the images, pipelines'
    descriptions and outputs it was planned with."""

    def __init__(self):
        h = C.c_void_p()
        check(lib().re_batch_create(C.byref(h)))
        self.handle = h.value
        self._keep = []

    def plan(self, requests, dispatch=None, ctas_per_sm=4, order=1, use_graph=True):
        items = (_capi.BatchItem * max(len(requests), 1))()
        descs = []
        cache = {}
        def desc_of(pipe):
            if id(pipe) not in cache:
                cache[id(pipe)] = pipe.desc()
                descs.append(cache[id(pipe)])
            return C.pointer(cache[id(pipe)])

        for i, req in enumerate(requests):
            image, pipe, viewport, mip, quality, out = req[:6]
            geo = req[6] if len(req) > 6 else None
            items[i].image = image.handle
            items[i].desc = desc_of(pipe)
            if geo is not None:
                items[i].geometry = {"cubic": 1, "rotate": 2}[geo.kind]
                items[i].canvas_width, items[i].canvas_height = (int(v) for v in geo.canvas)
                items[i].angle_degrees = float(geo.angle)
                if geo.post is not None:
                    items[i].post = desc_of(geo.post)
            items[i].viewport = _rect(viewport)
            items[i].mip = mip
            items[i].quality = quality
            items[i].out = out.data_ptr()
            items[i].out_row_stride = out.stride(0)
        opt = None
        if dispatch is not None:
            opt = _capi.BatchOptions(dispatch, ctas_per_sm, order, int(use_graph))
        check(lib().re_batch_plan(self.handle, items, len(requests), C.byref(opt) if opt is not None else None))
        self._keep = [requests, descs, items]
        return self

    def launch(self, stream=None):
        check(lib().re_batch_launch(self.handle, C.c_void_p(_stream_ptr(stream))))

    def launch_per_request(self, stream=None):
        """The planned requests as one single-request launch sequence each."""
        check(lib().re_batch_launch_per_request(self.handle, C.c_void_p(_stream_ptr(stream))))

    def status(self, stream=None):
        check(lib().re_batch_status(self.handle, C.c_void_p(_stream_ptr(stream))))

    def info(self) -> dict:
        i = _capi.BatchInfo()
        check(lib().re_batch_info_get(self.handle, C.byref(i)))
        o = i.options
        return {"requests": i.requests, "reduced_requests": i.reduced_requests, "tasks": i.tasks, "tiles": i.tiles,
                "reduce_blocks": i.reduce_blocks, "grid": i.grid, "native_pixels": i.native_pixels,
                "output_pixels": i.output_pixels, "raw_bytes": i.raw_bytes, "output_bytes": i.output_bytes,
                "geometry_requests": i.geometry_requests,
                "options": {"dispatch": o.dispatch, "ctas_per_sm": o.ctas_per_sm, "order": o.order,
                            "use_graph": o.use_graph}}

    def autotune(self, reps: int = 5, stream=None) -> dict:
        best = _capi.BatchOptions()
        check(lib().re_batch_autotune(self.handle, reps, C.c_void_p(_stream_ptr(stream)), C.byref(best)))
        return {"dispatch": best.dispatch, "ctas_per_sm": best.ctas_per_sm, "order": best.order,
                "use_graph": best.use_graph}

    def close(self):
        if getattr(self, "handle", None):
            lib().re_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ spatial / geometry

def _dev(t):
    return C.c_void_p(t.data_ptr())


def guided_filter(rgb, radius: int, epsilon: float, working_space: int = PROPHOTO, out=None, stream=None):
    """working_y_guided_filter_rgb over a whole CUDA float tensor (h, w, 3)."""
    h, w = int(rgb.shape[0]), int(rgb.shape[1])
    if out is None:
        out = rgb.new_empty(rgb.shape)
    check(lib().re_guided_filter(_dev(rgb), rgb.stride(0), _dev(out), out.stride(0), w, h, radius,
                                 float(epsilon), working_space, C.c_void_p(_stream_ptr(stream))))
    return out


def local_statistics(rgb, radius: int, with_count: bool = False, stream=None):
    """local_statistics_rgb over a whole CUDA float tensor: (mean, variance[, count])."""
    import torch
    h, w = int(rgb.shape[0]), int(rgb.shape[1])
    mean = rgb.new_empty(rgb.shape)
    var = rgb.new_empty(rgb.shape)
    cnt = torch.empty(rgb.shape, dtype=torch.int32, device=rgb.device) if with_count else None
    check(lib().re_local_statistics(_dev(rgb), rgb.stride(0), w, h, radius, _dev(mean), _dev(var),
                                    _dev(cnt) if cnt is not None else None,
                                    C.c_void_p(_stream_ptr(stream))))
    return (mean, var, cnt) if with_count else (mean, var)


def histogram_rgb(rgb, bins: int = 256, lower: float = 0.0, upper: float = 1.0, tile_size: int = 0, stream=None):
    """histogram_rgb of a CUDA float tensor (h, w, 3) rendered as one viewport
    whose tiles are tile_size (0: one tile), the order that decides between
    equal extrema.  Returns per channel a dict with counts (numpy uint64),
    underflow, overflow, nonfinite, minimum and maximum (None when absent)."""
    import torch
    h, w = int(rgb.shape[0]), int(rgb.shape[1])
    dev = rgb.device
    counts = torch.empty(3 * bins, dtype=torch.int64, device=dev)
    tallies = torch.empty(9, dtype=torch.int64, device=dev)
    extrema = torch.empty(6, dtype=torch.int64, device=dev)
    s = C.c_void_p(_stream_ptr(stream))
    check(lib().re_histogram_reset(bins, _dev(counts), _dev(tallies), _dev(extrema), s))
    check(lib().re_histogram_rgb(_dev(rgb), rgb.stride(0), w, h, tile_size, 0, bins, float(lower), float(upper),
                                 _dev(counts), _dev(tallies), _dev(extrema), s))
    counts = counts.cpu().numpy().view(np.uint64).reshape(3, bins)
    tallies = tallies.cpu().numpy().view(np.uint64)
    keys = extrema.cpu().numpy().view(np.uint64)
    out = []
    for c in range(3):
        ext = []
        for k, is_max in ((keys[c], 0), (keys[3 + c], 1)):
            v = C.c_float()
            ext.append(v.value if lib().re_histogram_extremum(int(k), is_max, C.byref(v)) else None)
        out.append(dict(counts=counts[c], underflow=int(tallies[c]), overflow=int(tallies[3 + c]),
                        nonfinite=int(tallies[6 + c]), minimum=ext[0], maximum=ext[1]))
    return out


def stencil(kind: str, rgb, window, image, output, amount: float = 0.0, radius: int = 1,
            working_space: int = PROPHOTO, kernel=None, stream=None):
    """SharpenNode / ClarityNode / TextureNode / ConvolutionNode::render_level
    on a CUDA float tensor holding the image rectangle `window`: returns the
    output rectangle.  `radius` is the scale for "texture"; "convolution"
    takes `kernel`, a 2-D array of odd sizes (flipped when applied)."""
    o = _rect(output)
    out = rgb.new_empty((o.height, o.width, 3))
    args = (_dev(rgb), rgb.stride(0), _rect(window), _rect(image), o)
    tail = (_dev(out), out.stride(0), C.c_void_p(_stream_ptr(stream)))
    L = lib()
    if kind == "sharpen":
        check(L.re_sharpen_window(*args, float(amount), radius, *tail))
    elif kind == "clarity":
        check(L.re_clarity_window(*args, float(amount), radius, working_space, *tail))
    elif kind == "texture":
        check(L.re_texture_window(*args, float(amount), radius, working_space, *tail))
    elif kind == "convolution":
        k = np.ascontiguousarray(kernel, dtype=np.float64)
        check(L.re_convolution_window(*args, k.shape[1], k.shape[0], k.ctypes.data_as(C.POINTER(C.c_double)),
                                      *tail))
    else:
        raise ValueError(f"unknown stencil {kind}")
    return out


def render_raster(rgb, pipe: "Pipeline", viewport=None, mip: int = 0, quality: int = FINAL, stream=None):
    """RasterSourceNode over a CUDA float tensor (h, w, 3) followed by the
    point stages of `pipe` (re_render_raster)."""
    h, w = int(rgb.shape[0]), int(rgb.shape[1])
    viewport = viewport or (0, 0, *request_bounds((0, 0, w, h), mip, quality)[2:])
    o = _rect(viewport)
    out = rgb.new_empty((o.height, o.width, 3))
    d = pipe.desc()
    check(lib().re_render_raster(_dev(rgb), rgb.stride(0), w, h, C.byref(d), o, mip, quality, _dev(out),
                                 out.stride(0), C.c_void_p(_stream_ptr(stream))))
    return out


def cubic_resize(rgb, out_w: int, out_h: int, output=None, mip: int = 0, stream=None):
    h, w = int(rgb.shape[0]), int(rgb.shape[1])
    output = output or (0, 0, *request_bounds((0, 0, out_w, out_h), mip, PREVIEW if mip else FINAL)[2:])
    o = _rect(output)
    out = rgb.new_empty((o.height, o.width, 3))
    check(lib().re_cubic_resize(_dev(rgb), rgb.stride(0), w, h, out_w, out_h, o, mip, _dev(out),
                                out.stride(0), C.c_void_p(_stream_ptr(stream))))
    return out


def rotate(rgb, angle_degrees: float, output=None, mip: int = 0, stream=None):
    h, w = int(rgb.shape[0]), int(rgb.shape[1])
    output = output or (0, 0, *request_bounds((0, 0, w, h), mip, PREVIEW if mip else FINAL)[2:])
    o = _rect(output)
    out = rgb.new_empty((o.height, o.width, 3))
    check(lib().re_rotate(_dev(rgb), rgb.stride(0), w, h, float(angle_degrees), o, mip, _dev(out),
                          out.stride(0), C.c_void_p(_stream_ptr(stream))))
    return out


def cubic_axis(n_in: int, n_out: int, index: int):
    center = C.c_uint32()
    idx = (C.c_uint32 * 18)()
    wts = (C.c_double * 18)()
    n = C.c_uint32()
    check(lib().re_cubic_axis(n_in, n_out, index, C.byref(center), idx, wts, C.byref(n)))
    return center.value, np.array(idx[:n.value], np.uint32), np.array(wts[:n.value], np.float64)


def rotation_coefficients(angle: float):
    c, s = C.c_double(), C.c_double()
    check(lib().re_rotation_coefficients(angle, C.byref(c), C.byref(s)))
    return c.value, s.value
