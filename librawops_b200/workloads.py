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
