"""The benchmark workloads of the render path, with their exact recipes.

* ``bilinear_1mp``  -- 1024x768 RGGB, 14-bit, phase 0, black 512, white 16383;
  WB (2.0, 1.0, 1.6) and a fixed camera->ProPhoto matrix whose rows sum to one;
  float32 linear ProPhoto output (the CameraToWorking node), tile 256, mip 0.
* ``menon_24mp``    -- 6016x4016 BGGR, stride 6080, active (16,8,6000,4000),
  black (510,512,511,513), white 15800; Menon, WB (1.9,1.0,1.5), a 3x3
  calibration matrix, a 16-knot monotone tone curve, working->sRGB, clip and
  sRGB encode; tiles 512.
* ``raster_24mp``   -- 6000x4000 float32 ProPhoto raster for the guided filter
  (r 8/32, eps 1e-3/1e-2) and box local statistics (r 16).
* ``mixed_batch``   -- 16 RAWs (4x 1920x1080, 6x 4000x3000, 4x 6000x4000,
  2x 8256x5504; all patterns, both phases, padded strides, inset active areas),
  half Menon and half bilinear, each with its own recipe (WB, exposure in
  [-1, 1] EV, a perturbed calibration matrix, a tone curve or a random monotone
  extended curve, sRGB output); render requests over random viewports at mip 0
  Final and mip 1/2 Preview, split into the reference renderer's tiles of 128,
  256, 512 or 1024 with edge remainders -- about 3,000 tiles.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import synthetic

# ProPhoto RGB -> XYZ(D50) (ROMM primaries, D50 white), the standard matrix.
PROPHOTO_TO_XYZ = np.array([[0.7976749, 0.1351917, 0.0313534],
                            [0.2880402, 0.7118741, 0.0000857],
                            [0.0000000, 0.0000000, 0.8252100]], np.float64)
# Camera -> ProPhoto with unit row sums (white maps to white).
CAMERA_TO_PROPHOTO = np.array([[1.60, -0.40, -0.20],
                               [-0.20, 1.45, -0.25],
                               [0.05, -0.55, 1.50]], np.float64)
# A calibrated camera -> XYZ(D50) matrix of plausible magnitude for the 24 MP case.
CALIBRATION_24MP = np.array([[0.6722, 0.2175, 0.0746],
                             [0.2598, 0.8467, -0.1065],
                             [0.0310, -0.1628, 0.9568]], np.float64)


def tone_knots_16():
    """16-knot monotone tone curve over [0, 1.5] (shape-preserving cubic)."""
    x = np.concatenate([[0.0], np.geomspace(0.004, 1.5, 15)])
    y = (x / (x + 0.18)) * (1.5 + 0.18) / 1.5
    y = np.maximum.accumulate(np.round(y, 6))
    return [(float(a), float(b)) for a, b in zip(x, y)]


@dataclass
class RawWorkload:
    name: str
    width: int
    height: int
    stride: int
    pattern: int
    phase: tuple
    active: tuple
    black: tuple
    white: int
    demosaic: int
    wb: tuple
    camera_to_xyz: np.ndarray
    tile: int
    curve: list | None
    srgb: bool
    chirp: bool
    lines: bool
    seed: int

    @property
    def pixels(self) -> int:
        return self.active[2] * self.active[3]

    def samples(self) -> np.ndarray:
        return synthetic.bayer(self.width, self.height, seed=self.seed, pattern=self.pattern,
                               phase=self.phase, stride=self.stride, active=self.active,
                               black=self.black, white=self.white, chirp=self.chirp,
                               lines=self.lines)


def bilinear_1mp(width=1024, height=768, seed=1) -> RawWorkload:
    return RawWorkload("bilinear_linear_prophoto_1024x768", width, height, width, 0, (0, 0),
                       (0, 0, width, height), (512, 512, 512, 512), 16383, 0, (2.0, 1.0, 1.6),
                       PROPHOTO_TO_XYZ @ CAMERA_TO_PROPHOTO, 256, None, False, False, False, seed)


def menon_24mp(seed=2, width=6016, height=4016, stride=6080, active=(16, 8, 6000, 4000)) -> RawWorkload:
    return RawWorkload("menon_srgb_24mp_6000x4000", width, height, stride, 1, (0, 0), active,
                       (510, 512, 511, 513), 15800, 1, (1.9, 1.0, 1.5), CALIBRATION_24MP, 512,
                       tone_knots_16(), True, True, True, seed)


def pipeline_for(w: RawWorkload):
    """The fused render chain of a workload (see module docstring)."""
    from .render import CurveSet, Pipeline
    p = Pipeline(demosaic=w.demosaic)
    p.white_balance(*w.wb)
    p.camera_to_working(w.camera_to_xyz, 0)
    if w.curve is not None:
        p.extended_curves(CurveSet(w.curve, cubic=True))
    if w.srgb:
        p.working_to_srgb()
        p.srgb_encode()
    return p


# ------------------------------------------------------------------ mixed batch

@dataclass
class MixedImage:
    width: int
    height: int
    stride: int
    pattern: int
    phase: tuple
    active: tuple
    black: tuple
    white: int
    demosaic: int
    seed: int


@dataclass
class MixedRecipe:
    wb: tuple
    stops: float
    camera_to_xyz: np.ndarray
    tone: tuple | None          # (shoulder, gamma) of the ToneCurve chain
    curve: list | None          # extended-curve knots of the curves chain


@dataclass
class MixedTile:
    image: int
    recipe: int
    viewport: tuple
    mip: int
    quality: int
    geometry: int = 0           # 0 none, 1 cubic resize to `canvas`, 2 rotation by `angle`
    canvas: tuple = (0, 0)      # geometry canvas at mip 0 (the active area's extent for a rotation)
    angle: float = 0.0


MIXED_SIZES = [(1920, 1080)] * 4 + [(4000, 3000)] * 6 + [(6000, 4000)] * 4 + [(8256, 5504)] * 2


def mixed_batch(seed: int = 4, target_tiles: int = 3000, geometry_share: float = 0.2):
    """Images, recipes (one per image) and the tile list of the mixed batch.
    A share of the viewports (geometry_share) is rendered through a cubic
    resize to a 2048 long edge or a rotation by a uniform angle in [-45, 45]
    degrees placed after the camera-to-working stage."""
    rng = np.random.default_rng(seed)
    images, recipes = [], []
    for i, (w, h) in enumerate(MIXED_SIZES):
        stride = w + 64 * (i % 3)
        inset = (i % 2) * 8
        active = (inset, inset // 2, w - 2 * inset, h - inset)
        black = tuple(int(v) for v in rng.integers(500, 530, 4))
        images.append(MixedImage(w, h, stride, i % 4, ((i // 4) % 2, (i // 2) % 2), active, black,
                                 int(rng.integers(15800, 16384)), i % 2, seed * 100 + i))
        cam = CALIBRATION_24MP * (1.0 + rng.uniform(-0.05, 0.05, (3, 3)))
        wb = (float(rng.uniform(1.5, 2.2)), 1.0, float(rng.uniform(1.2, 1.8)))
        if i % 3 == 0:
            n = int(rng.integers(4, 17))
            xs = np.concatenate([[0.0], np.sort(rng.uniform(0.01, 1.4, n - 2)), [1.5]])
            xs = np.maximum.accumulate(xs + np.arange(n) * 1e-3)
            ys = np.maximum.accumulate(np.sort(rng.uniform(0, 1.2, n)))
            ys = ys + np.arange(n) * 1e-3
            recipes.append(MixedRecipe(wb, float(rng.uniform(-1, 1)), cam, None,
                                       [(float(a), float(b)) for a, b in zip(xs, ys)]))
        else:
            recipes.append(MixedRecipe(wb, float(rng.uniform(-1, 1)), cam,
                                       (float(rng.uniform(0.15, 0.4)), float(rng.uniform(1.0, 2.4))), None))
    tiles = []
    while len(tiles) < target_tiles:
        i = int(rng.integers(0, len(images)))
        img = images[i]
        level = rng.choice(3, p=[0.5, 0.3, 0.2])
        mip, quality = (0, 1) if level == 0 else (int(level), 0)
        ax, ay, aw, ah = img.active
        geometry, canvas, angle = 0, (aw, ah), 0.0
        if geometry_share and rng.uniform() < geometry_share:
            # cubic resize to a 2048 long edge where the reference accepts it
            # (at most a fourfold shrink per axis), else a rotation
            geometry = 1 if max(aw, ah) <= 4 * 2048 and rng.uniform() < 0.5 else 2
            if geometry == 1:
                canvas = long_edge_canvas(aw, ah, 2048)
            else:
                angle = float(rng.uniform(-45.0, 45.0))
        cw, ch = canvas
        s = 1 << mip
        lw, lh = (cw, ch) if mip == 0 else (-(-cw // s), -(-ch // s))
        ox0, oy0 = (ax, ay) if mip == 0 and not geometry else (0, 0)
        vw = max(1, int(lw * rng.uniform(0.05, 0.35)))
        vh = max(1, int(lh * rng.uniform(0.05, 0.35)))
        vx = ox0 + int(rng.integers(0, lw - vw + 1))
        vy = oy0 + int(rng.integers(0, lh - vh + 1))
        t = int(rng.choice([128, 256, 512, 1024]))
        for y in range(vy, vy + vh, t):
            for x in range(vx, vx + vw, t):
                tiles.append(MixedTile(i, i, (x, y, min(t, vx + vw - x), min(t, vy + vh - y)), mip, quality,
                                       geometry, canvas if geometry else (0, 0), angle))
    return images, recipes, tiles


def long_edge_canvas(width: int, height: int, edge: int):
    """The canvas of a resize whose long edge is `edge`, aspect kept (rounded)."""
    if width >= height:
        return edge, max(1, int(round(height * edge / width)))
    return max(1, int(round(width * edge / height))), edge


def mixed_pipeline(image: MixedImage, recipe: MixedRecipe):
    """The render chain of one mixed-batch recipe (CameraToWorking is the mip anchor)."""
    from .render import CurveSet, Pipeline
    p = Pipeline(demosaic=image.demosaic)
    p.white_balance(*recipe.wb)
    if recipe.curve is None:
        p.exposure(recipe.stops)
        p.camera_to_working(recipe.camera_to_xyz, 0)
        p.working_to_srgb()
        p.tone_curve(*recipe.tone)
        p.srgb_encode()
    else:
        p.camera_to_working(recipe.camera_to_xyz, 0)
        p.exposure(recipe.stops)
        p.extended_curves(CurveSet(recipe.curve, cubic=True))
        p.working_to_srgb()
        p.srgb_encode()
    return p


def mixed_geometry_pipelines(image: MixedImage, recipe: MixedRecipe):
    """A mixed-batch recipe split around a geometry stage: (pre, post), the
    RAW source's stages through CameraToWorking (scene-linear ProPhoto, the
    geometry's input) and the point stages after the geometry."""
    from .render import CurveSet, Pipeline
    pre = Pipeline(demosaic=image.demosaic)
    pre.white_balance(*recipe.wb)
    post = Pipeline()
    if recipe.curve is None:
        pre.exposure(recipe.stops)
        pre.camera_to_working(recipe.camera_to_xyz, 0)
        post.working_to_srgb()
        post.tone_curve(*recipe.tone)
        post.srgb_encode()
    else:
        pre.camera_to_working(recipe.camera_to_xyz, 0)
        post.exposure(recipe.stops)
        post.extended_curves(CurveSet(recipe.curve, cubic=True))
        post.working_to_srgb()
        post.srgb_encode()
    return pre, post


def mixed_requests(render, imgs, images, recipes, tiles, outs):
    """Batch request tuples of the mixed batch (render.Batch.plan), geometry
    tiles included; one pipeline (or pipeline pair) per recipe."""
    plain, split = {}, {}
    reqs = []
    for t, o in zip(tiles, outs):
        if not t.geometry:
            if t.recipe not in plain:
                plain[t.recipe] = mixed_pipeline(images[t.image], recipes[t.recipe])
            reqs.append((imgs[t.image], plain[t.recipe], t.viewport, t.mip, t.quality, o))
            continue
        if t.recipe not in split:
            split[t.recipe] = mixed_geometry_pipelines(images[t.image], recipes[t.recipe])
        pre, post = split[t.recipe]
        geo = render.Geometry("cubic" if t.geometry == 1 else "rotate", t.canvas, t.angle, post)
        reqs.append((imgs[t.image], pre, t.viewport, t.mip, t.quality, o, geo))
    return reqs


def write_scheduler_spec(path: str, images, recipes, tiles) -> None:
    """The mixed batch as the text spec read by the C++ scheduler driver
    (tests/cpp/scheduler_driver.cpp): image, recipe and tile lines (a tile's
    geometry, canvas and angle last).  A recipe
    without a tone curve (the extended-curve recipes) gets the default tone
    shoulder 0.25 and gamma 1 in the C++ chain."""
    with open(path, "w") as f:
        for im in images:
            f.write("image %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d\n" % (
                im.width, im.height, im.stride, im.pattern, im.phase[0], im.phase[1], *im.active, *im.black,
                im.white, im.demosaic, im.seed))
        for r in recipes:
            shoulder, gamma = r.tone if r.tone is not None else (0.25, 1.0)
            knots = r.curve or []
            f.write("recipe %r %r %r %r %s %r %r %d %s\n" % (
                r.wb[0], r.wb[1], r.wb[2], r.stops, " ".join(repr(float(v)) for v in np.asarray(r.camera_to_xyz).reshape(9)),
                shoulder, gamma, len(knots), " ".join("%r %r" % (x, y) for x, y in knots)))
        for t in tiles:
            f.write("tile %d %d %d %d %d %d %d %d %d %d %d %r\n" % (t.image, t.recipe, *t.viewport, t.mip, t.quality,
                                                                   t.geometry, *t.canvas, float(t.angle)))
