"""The allocation-free reduced render (re_render_raw_reduced_noalloc).

Callers that cannot allocate device memory while rendering -- plug-ins whose
device memory is budgeted up front, real-time preview threads -- use this
entry point; its native-resolution scratch lives in a fixed device array
instead of a per-call allocation.  Its output must equal the allocating entry
point's (re_render_raw with device output) on the same inputs, on two calls in
a row (the shared array keeps the previous call's contents, which must not
leak into the next result).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal
from librawops_b200 import _capi, render, workloads

pytestmark = pytest.mark.gpu


def _noalloc(img, pipe, viewport, mip, out):
    d = pipe.desc()
    ptr, stride = (None, 0) if out is None else (C.c_void_p(out.data_ptr()), out.stride(0))
    _capi.check(_capi.lib().re_render_raw_reduced_noalloc(
        img.handle, C.byref(d), _capi.Rect(*viewport), mip, ptr, stride, None))


def test_noalloc_reduced_render_matches_allocating_render():
    import torch
    w = workloads.menon_24mp(width=1040, height=720, stride=1048, active=(8, 4, 1024, 708))
    meta = render.Metadata(w.width, w.height, w.stride, w.pattern, *w.phase, w.active, w.black, (w.white,) * 4)
    img = render.Image(meta, w.samples())
    pipe = render.Pipeline(demosaic=render.MENON).white_balance(*w.wb).exposure(0.25)
    pipe.camera_to_working(w.camera_to_xyz, 0)
    pipe.extended_curves(render.CurveSet(w.curve)).working_to_srgb().srgb_encode()
    limit = int(_capi.lib().re_render_raw_reduced_noalloc_max_native_pixels())
    assert limit == 1 << 20
    for mip, viewport in ((1, (0, 0, 512, 354)), (2, (13, 7, 200, 150))):
        want = torch.empty((viewport[3], viewport[2], 3), dtype=torch.float32, device="cuda")
        render.render(img, pipe, viewport, mip=mip, quality=render.PREVIEW, out=want)
        for _ in range(2):
            got = torch.full_like(want, float("nan"))
            _noalloc(img, pipe, viewport, mip, got)
            torch.cuda.synchronize()
            assert bits_equal(got.cpu().numpy(), want.cpu().numpy()), (mip, viewport)
    # a footprint beyond the fixed scratch is refused with a clear error
    big = render.Image(render.Metadata(2400, 1600, 0, 0, 0, 0, (0, 0, 2400, 1600), (512,) * 4, (16383,) * 4),
                       np.full((1600, 2400), 2000, np.uint16))
    out = torch.empty((800, 1200, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(_capi.ReError) as e:
        _noalloc(big, pipe, (0, 0, 1200, 800), 1, out)
    assert e.value.kind == "length_error" and "exceeds" in str(e.value)
    # an empty viewport renders nothing and, like re_render_raw, needs no output buffer
    _noalloc(img, pipe, (0, 0, 0, 0), 1, None)
