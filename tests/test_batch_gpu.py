"""The batched render (re_batch_*): many requests, one persistent kernel.

A batch mixes images (all Bayer patterns, both CFA phases, padded strides,
inset active areas), demosaic policies, recipes (with and without extended
curves), mip 0 Final and mip 1/2 Preview, and tiles with edge remainders, as
TileScheduler and Renderer::render_tiles issue them (TileScheduler.cpp:19-304,
RawEngine.cpp:1390-1412).  Every request's pixels must equal the single-request
render (re_render_raw, itself pinned to the oracle) bit for bit, under every
dispatch choice the autotuner can make and in the per-request launch form.
"""
import numpy as np
import pytest

from conftest import bits_equal
from librawops_b200 import render, workloads
from librawops_b200._capi import ReError

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _small_batch(seed=11):
    rng = np.random.default_rng(seed)
    sizes = [(300, 200), (257, 181), (160, 96), (411, 233), (96, 64), (333, 250)]
    images, recipes = [], []
    for i, (w, h) in enumerate(sizes):
        stride = w + 16 * (i % 3)
        inset = (i % 2) * 5
        images.append(workloads.MixedImage(w, h, stride, i % 4, (i % 2, (i // 2) % 2),
                                           (inset, inset // 2 + 1, w - 2 * inset, h - inset - 1),
                                           tuple(int(v) for v in rng.integers(500, 530, 4)),
                                           int(rng.integers(15800, 16384)), (i // 2) % 2, 70 + i))
        cam = workloads.CALIBRATION_24MP * (1.0 + rng.uniform(-0.05, 0.05, (3, 3)))
        wb = (float(rng.uniform(1.5, 2.2)), 1.0, float(rng.uniform(1.2, 1.8)))
        if i % 3 == 0:
            knots = [(0.0, 0.0), (0.2, 0.3), (0.5, 0.62), (0.9, 0.95), (1.5, 1.2)]
            recipes.append(workloads.MixedRecipe(wb, float(rng.uniform(-1, 1)), cam, None, knots))
        else:
            recipes.append(workloads.MixedRecipe(wb, float(rng.uniform(-1, 1)), cam,
                                                 (float(rng.uniform(0.15, 0.4)), float(rng.uniform(1.0, 2.4))),
                                                 None))
    tiles = []
    for i, img in enumerate(images):
        ax, ay, aw, ah = img.active
        for mip, quality in ((0, 1), (1, 0), (2, 0)):
            s = 1 << mip
            lw, lh = (aw, ah) if mip == 0 else (-(-aw // s), -(-ah // s))
            ox0, oy0 = (ax, ay) if mip == 0 else (0, 0)
            vw, vh = max(1, int(lw * 0.7)), max(1, int(lh * 0.6))
            vx, vy = ox0 + (lw - vw) // 3, oy0 + (lh - vh) // 2
            t = [37, 64, 100][(i + mip) % 3]
            for y in range(vy, vy + vh, t):
                for x in range(vx, vx + vw, t):
                    tiles.append(workloads.MixedTile(i, i, (x, y, min(t, vx + vw - x), min(t, vy + vh - y)),
                                                     mip, quality))
    return images, recipes, tiles


def _device_images(images):
    out = []
    for img in images:
        samples = render.synthetic_samples(img)
        meta = render.Metadata(img.width, img.height, img.stride, img.pattern, img.phase[0], img.phase[1],
                               img.active, img.black, (img.white,) * 4)
        out.append(render.Image(meta, samples))
    return out


def _requests(imgs, pipes, tiles):
    outs = [torch.full((t.viewport[3], t.viewport[2], 3), float("nan"), device="cuda") for t in tiles]
    reqs = [(imgs[t.image], pipes[t.recipe], t.viewport, t.mip, t.quality, o) for t, o in zip(tiles, outs)]
    return reqs, outs


def test_batch_equals_single_requests():
    images, recipes, tiles = _small_batch()
    imgs = _device_images(images)
    pipes = [workloads.mixed_pipeline(im, r) for im, r in zip(images, recipes)]
    want = [render.render(imgs[t.image], pipes[t.recipe], t.viewport, t.mip, t.quality) for t in tiles]
    reqs, outs = _requests(imgs, pipes, tiles)
    batch = render.Batch()
    combos = [(d, c, o, g) for d in (0, 1, 2) for c in ((1, 4) if d != 1 else (4,)) for o in (0, 1) for g in (0, 1)]
    for d, c, o, g in combos:
        for out in outs:
            out.fill_(float("nan"))
        batch.plan(reqs, dispatch=d, ctas_per_sm=c, order=o, use_graph=bool(g))
        batch.launch()
        batch.status()
        for k, (out, w) in enumerate(zip(outs, want)):
            assert bits_equal(out.cpu().numpy(), w), (d, c, o, g, k, tiles[k])
    info = batch.info()
    assert info["requests"] == len(tiles)
    assert info["reduced_requests"] == sum(1 for t in tiles if t.mip)
    assert info["output_pixels"] == sum(t.viewport[2] * t.viewport[3] for t in tiles)
    for out in outs:
        out.fill_(float("nan"))
    batch.launch_per_request()
    batch.status()
    for out, w in zip(outs, want):
        assert bits_equal(out.cpu().numpy(), w)
    best = batch.autotune(reps=2)
    assert best["dispatch"] in (0, 1, 2) and 1 <= best["ctas_per_sm"] <= 4
    for out in outs:
        out.fill_(float("nan"))
    batch.launch()
    batch.status()
    for out, w in zip(outs, want):
        assert bits_equal(out.cpu().numpy(), w)
    # a plan without options takes the tuned choice for this shape
    batch.plan(reqs)
    assert batch.info()["options"] == best
    batch.close()


def test_batch_validates_like_single_requests():
    images, recipes, tiles = _small_batch()
    imgs = _device_images(images[:1])
    pipes = [workloads.mixed_pipeline(images[0], recipes[0])]
    out = torch.zeros((8, 8, 3), device="cuda")
    batch = render.Batch()
    ax, ay, aw, ah = images[0].active
    with pytest.raises(ReError) as e:
        batch.plan([(imgs[0], pipes[0], (ax + aw - 4, ay, 8, 8), 0, 1, out)])
    assert e.value.kind == "out_of_range"
    with pytest.raises(ReError) as e:
        batch.plan([(imgs[0], pipes[0], (0, 0, 8, 8), 1, 1, out)])   # mip 1 Final
    assert e.value.kind == "invalid_argument"
    legacy = render.Pipeline(demosaic=0)
    legacy.white_balance(2.0, 1.0, 1.5)
    with pytest.raises(ReError) as e:
        batch.plan([(imgs[0], legacy, (0, 0, 8, 8), 1, 0, out)])      # no mip anchor
    assert e.value.kind == "invalid_argument"
    batch.plan([])
    batch.launch()
    batch.status()
    batch.close()


def test_mixed_batch_shape():
    images, recipes, tiles = workloads.mixed_batch()
    assert len(images) == 16 and 2900 <= len(tiles) <= 3300
    assert {t.mip for t in tiles} == {0, 1, 2}
    assert {im.pattern for im in images} == {0, 1, 2, 3}


def test_batch_splits_into_launch_groups():
    """More distinct programs than one launch group holds (24): the batch is
    split into groups launched back to back, with identical results."""
    images, recipes, _ = _small_batch(seed=5)
    imgs = _device_images(images)
    rng = np.random.default_rng(3)
    pipes, tiles = [], []
    for k in range(30):
        i = k % len(images)
        r = recipes[i]
        wb = (r.wb[0] * float(rng.uniform(0.9, 1.1)), 1.0, r.wb[2])
        pipes.append(workloads.mixed_pipeline(images[i], workloads.MixedRecipe(wb, r.stops, r.camera_to_xyz,
                                                                                r.tone, r.curve)))
        ax, ay, aw, ah = images[i].active
        mip = k % 3
        if mip == 0:
            vp = (ax + k % 7, ay + k % 5, min(40, aw - k % 7), min(30, ah - k % 5))
        else:
            vp = (k % 4, k % 3, 20, 12)
        tiles.append(workloads.MixedTile(i, k, vp, mip, 1 if mip == 0 else 0))
    want = [render.render(imgs[t.image], pipes[t.recipe], t.viewport, t.mip, t.quality) for t in tiles]
    reqs, outs = _requests(imgs, pipes, tiles)
    batch = render.Batch()
    for d in (0, 1, 2):
        for out in outs:
            out.fill_(float("nan"))
        batch.plan(reqs, dispatch=d, ctas_per_sm=2, order=0, use_graph=True)
        batch.launch()
        batch.status()
        for k, (out, w) in enumerate(zip(outs, want)):
            assert bits_equal(out.cpu().numpy(), w), (d, k)
    batch.close()


def test_batch_mixes_menon_policies():
    """Requests of both Menon policies (binary64 and binary32) in one batch run
    in separate launch groups and equal their single renders bit for bit."""
    images, recipes, tiles = _small_batch(seed=8)
    imgs = _device_images(images)
    pipes = []
    for im, r in zip(images, recipes):
        pipes.append(workloads.mixed_pipeline(im, r))
        fast = workloads.mixed_pipeline(im, r)
        fast.demosaic = render.MENON_FAST if fast.demosaic else 0
        pipes.append(fast)
    tiles = [workloads.MixedTile(t.image, 2 * t.recipe + (k % 2), t.viewport, t.mip, t.quality)
             for k, t in enumerate(tiles)]
    want = [render.render(imgs[t.image], pipes[t.recipe], t.viewport, t.mip, t.quality) for t in tiles]
    reqs, outs = _requests(imgs, pipes, tiles)
    batch = render.Batch()
    for d in (0, 1, 2):
        for out in outs:
            out.fill_(float("nan"))
        batch.plan(reqs, dispatch=d, ctas_per_sm=4, order=1, use_graph=True)
        batch.launch()
        batch.status()
        for k, (out, w) in enumerate(zip(outs, want)):
            assert bits_equal(out.cpu().numpy(), w), (d, k)
    batch.close()


def test_batch_merges_tiles_of_one_render():
    """Tiles of one viewport written into one frame (the reference renderer's
    render_image) merge into one render per viewport; the frame equals the
    single render under every dispatch choice."""
    images, recipes, _ = _small_batch(seed=13)
    imgs = _device_images(images)
    pipes = [workloads.mixed_pipeline(im, r) for im, r in zip(images, recipes)]
    frames, reqs, wants = [], [], []
    for i, img in enumerate(images):
        ax, ay, aw, ah = img.active
        for mip, quality in ((0, 1), (1, 0)):
            s = 1 << mip
            lw, lh = (aw, ah) if mip == 0 else (-(-aw // s), -(-ah // s))
            ox0, oy0 = (ax, ay) if mip == 0 else (0, 0)
            vp = (ox0 + 3, oy0 + 2, lw - 5, lh - 4)
            frame = torch.full((vp[3], vp[2], 3), float("nan"), device="cuda")
            frames.append(frame)
            wants.append(render.render(imgs[i], pipes[i], vp, mip, quality))
            t = 41
            for y in range(vp[1], vp[1] + vp[3], t):
                for x in range(vp[0], vp[0] + vp[2], t):
                    w_, h_ = min(t, vp[0] + vp[2] - x), min(t, vp[1] + vp[3] - y)
                    part = frame[y - vp[1]:y - vp[1] + h_, x - vp[0]:x - vp[0] + w_]
                    reqs.append((imgs[i], pipes[i], (x, y, w_, h_), mip, quality, part))
    batch = render.Batch()
    for d in (0, 1, 2, 3):
        for f in frames:
            f.fill_(float("nan"))
        batch.plan(reqs, dispatch=d, ctas_per_sm=4, order=1, use_graph=bool(d % 2))
        info = batch.info()
        assert info["requests"] == len(reqs) and info["tasks"] == len(frames), info
        batch.launch()
        batch.status()
        for f, w in zip(frames, wants):
            assert bits_equal(f.cpu().numpy(), w), d
    for f in frames:
        f.fill_(float("nan"))
    batch.launch_per_request()
    batch.status()
    for f, w in zip(frames, wants):
        assert bits_equal(f.cpu().numpy(), w)
    batch.close()


def test_batch_keeps_row_tiles_apart_when_the_stride_is_too_small():
    """One-row tiles whose outputs lie back to back in one buffer, each with
    its own narrow row stride (a scheduler's packed output block): the
    planner must not merge them into a render wider than that stride."""
    images, recipes, _ = _small_batch(seed=17)
    imgs = _device_images(images)
    pipes = [workloads.mixed_pipeline(im, r) for im, r in zip(images, recipes)]
    img, pipe = imgs[0], pipes[0]
    ax, ay, aw, ah = images[0].active
    width = 8
    vps = [(ax + 16 + k * width, ay + 9, width, 1) for k in range(6)]
    arena = torch.full((len(vps) * width * 3,), float("nan"), device="cuda")
    outs = [arena[k * width * 3:(k + 1) * width * 3].view(1, width, 3) for k in range(len(vps))]
    batch = render.Batch().plan([(img, pipe, vp, 0, 1, o) for vp, o in zip(vps, outs)])
    batch.launch()
    batch.status()
    for vp, o in zip(vps, outs):
        assert bits_equal(o.cpu().numpy(), render.render(img, pipe, vp))
    batch.close()


# ------------------------------------------------------------- geometry requests

def _geometry_tiles(images):
    """Cubic resizes (enlarge and shrink, up to fourfold) and rotations
    (including the exact quarter turns and +-45 degrees) of every image, at mip
    0 Final and mip 1/2 Preview, viewports tiled with edge remainders."""
    tiles = []
    angles = [-45.0, -13.7, 0.0, 27.5, 45.0, 90.0]
    for i, img in enumerate(images):
        ax, ay, aw, ah = img.active
        canvases = [workloads.long_edge_canvas(aw, ah, 2 * max(aw, ah) // 3), (aw // 4 + 1, ah // 3 + 1),
                    (aw + 37, ah + 11)]
        for k, (mip, quality) in enumerate(((0, 1), (1, 0), (2, 0))):
            for geometry, canvas, angle in ((1, canvases[(i + k) % 3], 0.0), (2, (aw, ah), angles[(i + k) % 6])):
                cw, ch = canvas
                s = 1 << mip
                lw, lh = (cw, ch) if mip == 0 else (-(-cw // s), -(-ch // s))
                vw, vh = max(1, int(lw * 0.8)), max(1, int(lh * 0.7))
                vx, vy = (lw - vw) // 4, (lh - vh) // 2
                t = [41, 64][(i + k) % 2]
                for y in range(vy, vy + vh, t):
                    for x in range(vx, vx + vw, t):
                        tiles.append(workloads.MixedTile(i, i, (x, y, min(t, vx + vw - x), min(t, vy + vh - y)),
                                                         mip, quality, geometry, canvas, angle))
    return tiles


def _geometry_single(img, image, recipe, tile):
    """One geometry request composed of single-request calls over the whole
    image: the RAW chain over the active area, the geometry over all of it at
    the request's level, then the later stages on the result."""
    pre, post = workloads.mixed_geometry_pipelines(image, recipe)
    ax, ay, aw, ah = image.active
    working = render.render(img, pre, image.active, out=torch.empty((ah, aw, 3), device="cuda"))
    if tile.geometry == 1:
        out = render.cubic_resize(working, *tile.canvas, output=tile.viewport, mip=tile.mip)
    else:
        out = render.rotate(working, tile.angle, output=tile.viewport, mip=tile.mip)
    return render.render_raster(out, post)


def test_batch_geometry_requests_equal_composed_single_renders():
    images, recipes, _ = _small_batch()
    imgs = _device_images(images)
    tiles = _geometry_tiles(images)
    plain = _small_batch()[2][::5]
    want = [_geometry_single(imgs[t.image], images[t.image], recipes[t.recipe], t).cpu().numpy() for t in tiles]
    want += [render.render(imgs[t.image], workloads.mixed_pipeline(images[t.image], recipes[t.recipe]), t.viewport,
                           t.mip, t.quality) for t in plain]
    tiles = tiles + plain
    outs = [torch.full((t.viewport[3], t.viewport[2], 3), float("nan"), device="cuda") for t in tiles]
    reqs = workloads.mixed_requests(render, imgs, images, recipes, tiles, outs)
    batch = render.Batch()
    for d, g in ((2, 1), (0, 0), (1, 1), (3, 1)):
        for o in outs:
            o.fill_(float("nan"))
        batch.plan(reqs, dispatch=d, use_graph=bool(g))
        batch.launch()
        batch.status()
        for k, (o, w) in enumerate(zip(outs, want)):
            assert bits_equal(o.cpu().numpy(), w), (d, k, tiles[k])
    info = batch.info()
    n_geo = sum(1 for t in tiles if t.geometry)
    assert info["geometry_requests"] == n_geo and info["requests"] == len(tiles)
    assert info["output_pixels"] == sum(t.viewport[2] * t.viewport[3] for t in tiles)
    for o in outs:
        o.fill_(float("nan"))
    batch.launch_per_request()
    batch.status()
    for k, (o, w) in enumerate(zip(outs, want)):
        assert bits_equal(o.cpu().numpy(), w), ("per request", k, tiles[k])
    batch.close()


def test_batch_geometry_matches_reference(reference):
    """Cubic resize and rotation requests of the batch against the reference
    library's CubicResizeNode / RotateNode over its own RAW chain: bit for bit
    for the working image, within the render tolerance after sRGB encoding."""
    from conftest import within_tolerance
    from oracle.oracle import (OP_CAMERA_TO_WORKING, OP_CUBIC_RESIZE, OP_EXPOSURE, OP_ROTATE, OP_SRGB_ENCODE,
                               OP_TONE, OP_WB, OP_WORKING_TO_SRGB, Op, RawSpec)
    images, recipes, _ = _small_batch()
    imgs = _device_images(images)
    cases = []
    for i in (1, 2, 4, 5):            # tone-curve recipes, bilinear and Menon, inset active areas
        im, r = images[i], recipes[i]
        ax, ay, aw, ah = im.active
        for geometry, canvas, angle in ((1, (aw * 3 // 2, ah * 2 // 3), 0.0), (2, (aw, ah), 33.0 - 11 * i)):
            for mip, quality in ((0, 1), (1, 0)):
                s = 1 << mip
                lw, lh = (canvas[0], canvas[1]) if mip == 0 else (-(-canvas[0] // s), -(-canvas[1] // s))
                vp = (lw // 5, lh // 4, lw // 2, lh // 2)
                for srgb in (False, True):
                    cases.append((i, workloads.MixedTile(i, i, vp, mip, quality, geometry, canvas, angle), srgb))
    reqs, wants = [], []
    for i, t, srgb in cases:
        im, r = images[i], recipes[i]
        pre, post = workloads.mixed_geometry_pipelines(im, r)
        if not srgb:
            post = None
        out = torch.full((t.viewport[3], t.viewport[2], 3), float("nan"), device="cuda")
        geo = render.Geometry("cubic" if t.geometry == 1 else "rotate", t.canvas, t.angle, post)
        reqs.append((imgs[i], pre, t.viewport, t.mip, t.quality, out, geo))
        spec = RawSpec(im.width, im.height, render.synthetic_samples(im).cpu().numpy().reshape(-1), im.stride,
                       im.pattern, *im.phase, im.active, im.black, (im.white,) * 4)
        ops = [Op(OP_WB, list(r.wb)), Op(OP_EXPOSURE, [r.stops]),
               Op(OP_CAMERA_TO_WORKING, list(np.asarray(r.camera_to_xyz).reshape(9)) + [0])]
        ops.append(Op(OP_CUBIC_RESIZE, list(t.canvas)) if t.geometry == 1 else Op(OP_ROTATE, [t.angle]))
        if srgb:
            ops += [Op(OP_WORKING_TO_SRGB), Op(OP_TONE, list(r.tone)), Op(OP_SRGB_ENCODE)]
        wants.append((reference.render_raw(spec, bool(im.demosaic), ops, t.viewport, tile=64, mip=t.mip,
                                           quality=t.quality), srgb))
    batch = render.Batch().plan(reqs)
    batch.launch()
    batch.status()
    for k, (req, (want, srgb)) in enumerate(zip(reqs, wants)):
        got = req[5].cpu().numpy()
        if srgb:
            within_tolerance(got, want)
        else:
            assert bits_equal(got, want), (k, cases[k])
    batch.close()
