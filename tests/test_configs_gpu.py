"""Parity of every benchmark configuration at its stated size, on a B200.

* bilinear 1024x768 RGGB (black 512, white 16383, WB (2.0, 1.0, 1.6), a
  camera->ProPhoto matrix with unit row sums, tile 256, float32 linear output
  of the CameraToWorking node): bit for bit against the unmodified reference
  library (oracle/_ref) rendering the same request through
  Renderer::render_image.
* Menon 24 MP -> sRGB (6016x4016 BGGR, stride 6080, active (16,8,6000,4000)):
  the WHOLE frame against the reference library rendering it through its own
  TileScheduler (tile 512, one worker per host core), within 1e-5 and one
  16-bit code; the whole direction map against the C restatement under both
  Menon policies; exact ties and binary32 rechecks counted.
* Guided filter on the 6000x4000 raster at r 8 (eps 1e-3, 1e-2) against the
  reference library on an interior 1024x1024 window and an image-corner
  window, and at r 32 against the O(r^2) restatement on a 512x512 interior
  window, where every window is a full 65x65 interior window; local
  statistics at r 16 against the restatement on an interior window and at r 8
  against the reference.

The GPU computes each operator over the whole image; windows of its output
are compared with the checker's output for that window (each checker reads
the window plus its halo, which makes the comparison exact).
"""
import os

import numpy as np
import pytest

from conftest import bits_equal, within_tolerance
from librawops_b200 import render, synthetic, workloads
from oracle.oracle import (OP_CAMERA_TO_WORKING, OP_CURVES_EXT, OP_DISPLAY_TAG, OP_SRGB_ENCODE, OP_WB,
                           OP_WORKING_TO_SRGB, Op, RawSpec, curves_params)

pytestmark = pytest.mark.gpu


def _raw_spec(w, samples):
    return RawSpec(w.width, w.height, samples.reshape(-1), w.stride, w.pattern, *w.phase, w.active, w.black,
                   (w.white,) * 4)


def _image(w, samples):
    meta = render.Metadata(w.width, w.height, w.stride, w.pattern, *w.phase, w.active, w.black, (w.white,) * 4)
    return render.Image(meta, samples)


def test_bilinear_1024x768_bit_exact_against_reference(reference):
    w = workloads.bilinear_1mp()
    samples = w.samples()
    img = _image(w, samples)
    got = render.render(img, workloads.pipeline_for(w), w.active)
    ops = [Op(OP_WB, list(w.wb)), Op(OP_CAMERA_TO_WORKING, list(w.camera_to_xyz.reshape(9)) + [0])]
    want = reference.render_raw(_raw_spec(w, samples), False, ops, w.active, tile=w.tile)
    assert bits_equal(got, want)
    # the reference's per-tile loop (tile 256) assembles the same frame
    tiled = np.zeros_like(got)

    def cb(r, rgb):
        tiled[r[1]:r[1] + r[3], r[0]:r[0] + r[2]] = rgb
    render.render_tiles(img, workloads.pipeline_for(w), w.active, w.tile, cb)
    assert bits_equal(tiled, want)


@pytest.fixture(scope="module")
def menon_frame():
    w = workloads.menon_24mp()
    samples = w.samples()
    return w, samples, _image(w, samples)


def test_menon_24mp_whole_frame_against_reference(menon_frame, reference):
    w, samples, img = menon_frame
    got = render.render(img, workloads.pipeline_for(w), w.active)
    ops = [Op(OP_WB, list(w.wb)), Op(OP_CAMERA_TO_WORKING, list(w.camera_to_xyz.reshape(9)) + [0]),
           Op(OP_CURVES_EXT, curves_params(1, w.curve)), Op(OP_WORKING_TO_SRGB), Op(OP_DISPLAY_TAG),
           Op(OP_SRGB_ENCODE)]
    want = reference.render_raw(_raw_spec(w, samples), True, ops, w.active, tile=w.tile,
                                scheduled_workers=os.cpu_count() or 1)
    assert got.shape == want.shape == (w.active[3], w.active[2], 3)
    within_tolerance(got, want)


def test_menon_24mp_direction_map_and_near_ties(menon_frame, oracle):
    """Every direction decision of the frame equals the restatement's, under
    both policies; the binary64 policy's exact ties and the binary32 policy's
    binary64 rechecks are counted."""
    w, samples, img = menon_frame
    _, want = oracle.demosaic(_raw_spec(w, samples), w.active, True, directions=True)
    ties = {}
    for policy in (render.MENON, render.MENON_FAST):
        got, n = render.menon_directions(img, w.active, policy)
        assert np.array_equal(got.cpu().numpy(), want), policy
        ties[policy] = n
    decisions = w.active[2] * w.active[3] // 2
    assert 0 <= ties[render.MENON] <= ties[render.MENON_FAST] < decisions // 100, ties
    # the render's own counter agrees with the direction map's
    _, stats = render.render(img, workloads.pipeline_for(w), w.active, stats=True)
    assert stats["menon_decisions"] == decisions


@pytest.fixture(scope="module")
def raster_frame():
    import torch
    rgb = synthetic.raster(6000, 4000, seed=3)
    return rgb, torch.from_numpy(rgb).cuda()


def _window(rgb, output, halo):
    """The checker's input: the output window grown by `halo`, clipped to the image."""
    h, w = rgb.shape[:2]
    x0, y0 = max(0, output[0] - halo), max(0, output[1] - halo)
    x1, y1 = min(w, output[0] + output[2] + halo), min(h, output[1] + output[3] + halo)
    needed = (x0, y0, x1 - x0, y1 - y0)
    return np.ascontiguousarray(rgb[y0:y1, x0:x1]), needed


def _crop(a, r):
    return a[r[1]:r[1] + r[3], r[0]:r[0] + r[2]]


@pytest.mark.parametrize("eps", [1e-3, 1e-2])
def test_guided_filter_r8_24mp_against_reference(raster_frame, reference, eps):
    rgb, dev = raster_frame
    image = (0, 0, 6000, 4000)
    got = render.guided_filter(dev, 8, eps).cpu().numpy()
    for out in [(2488, 1488, 1024, 1024), (0, 0, 256, 192), (6000 - 200, 4000 - 160, 200, 160)]:
        tile, needed = _window(rgb, out, 16)
        want = reference.guided_filter(tile, needed, out, image, 8, eps)
        within_tolerance(_crop(got, out), want, lsb16=False)


@pytest.mark.parametrize("eps", [1e-3, 1e-2])
def test_guided_filter_r32_24mp_against_restatement(raster_frame, oracle, eps):
    rgb, dev = raster_frame
    image = (0, 0, 6000, 4000)
    got = render.guided_filter(dev, 32, eps).cpu().numpy()
    for out in [(3000, 2000, 512, 512), (0, 3872, 160, 128)]:
        tile, needed = _window(rgb, out, 64)
        want = oracle.guided_filter(tile, needed, out, image, 32, eps)
        within_tolerance(_crop(got, out), want, lsb16=False)


def _ls_close(got, want):
    got = np.asarray(got, np.float64)
    fin = np.isfinite(want)
    assert np.array_equal(np.isfinite(got), fin)
    err = np.abs(got[fin] - want[fin]) / np.maximum(1.0, np.abs(want[fin]))
    assert err.max(initial=0) <= 2e-7, err.max()


def test_local_statistics_24mp(raster_frame, oracle, reference):
    rgb, dev = raster_frame
    image = (0, 0, 6000, 4000)
    for radius, checker in ((16, oracle), (8, reference)):
        mean, var, cnt = render.local_statistics(dev, radius, with_count=True)
        mean, var, cnt = mean.cpu().numpy(), var.cpu().numpy(), cnt.cpu().numpy()
        for out in [(2400, 1400, 1024, 1024), (6000 - 300, 0, 300, 200)]:
            tile, needed = _window(rgb, out, radius)
            want_m, want_v, want_n = checker.local_statistics(tile, needed, out, image, radius)
            _ls_close(_crop(mean, out), want_m)
            _ls_close(_crop(var, out), want_v)
            assert np.array_equal(_crop(cnt, out).astype(np.uint32), want_n)
