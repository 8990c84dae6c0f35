"""Seeded synthetic scenes standing in for camera RAWs (no dataset is used).

Bayer scenes: a linear gradient, 32 Gaussian colour blobs (sigma 10-120 px,
radiance 0-0.9) and 8 hard-edged rectangles, optionally a 512x512 zone-plate
chirp and 1-px diagonal line pairs (which stress Menon's directional
decisions), mosaicked through the CFA, then Poisson-Gaussian noise (gain
0.5 DN/e-, read sigma 3 DN) above the black level, clipped to 14 bits.

Raster scenes (for the guided filter / local statistics): lognormal luminance
(mu -1.5, sigma 1.2) with random straight edges, 2% slightly negative samples
(down to -0.01), 0.5% highlights up to 4.0, chroma of random hue with
saturation in [0, 0.6].
"""
from __future__ import annotations

import numpy as np

PATTERN_COLORS = [(0, 1, 1, 2), (2, 1, 1, 0), (1, 0, 2, 1), (1, 2, 0, 1)]


def _blobs_and_rects(rng, w, h, img):
    yy = np.arange(h, dtype=np.float32)[:, None]
    xx = np.arange(w, dtype=np.float32)[None, :]
    for _ in range(32):
        sigma = rng.uniform(10, 120)
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        colour = rng.uniform(0, 0.9, 3).astype(np.float32)
        x0, x1 = int(max(0, cx - 3 * sigma)), int(min(w, cx + 3 * sigma + 1))
        y0, y1 = int(max(0, cy - 3 * sigma)), int(min(h, cy + 3 * sigma + 1))
        if x1 <= x0 or y1 <= y0:
            continue
        g = np.exp(-(((xx[:, x0:x1] - cx) ** 2) + ((yy[y0:y1] - cy) ** 2)) / (2 * sigma * sigma))
        img[y0:y1, x0:x1] += g[..., None].astype(np.float32) * colour
    for _ in range(8):
        rw, rh = rng.integers(max(2, w // 20), max(3, w // 4)), rng.integers(max(2, h // 20), max(3, h // 4))
        x0, y0 = rng.integers(0, max(1, w - rw)), rng.integers(0, max(1, h - rh))
        img[y0:y0 + rh, x0:x0 + rw] = rng.uniform(0, 0.9, 3).astype(np.float32)


def radiance(width: int, height: int, seed: int, chirp: bool = False, lines: bool = False) -> np.ndarray:
    """Scene-linear RGB radiance (height, width, 3) float32, mostly in [0, 1]."""
    rng = np.random.default_rng(seed)
    img = np.empty((height, width, 3), np.float32)
    gx = np.linspace(0.05, 0.6, width, dtype=np.float32)[None, :]
    gy = np.linspace(0.0, 0.3, height, dtype=np.float32)[:, None]
    img[..., 0] = gx + 0.5 * gy
    img[..., 1] = 0.8 * gx + gy
    img[..., 2] = 0.4 * gx + 0.3 * gy + 0.1
    _blobs_and_rects(rng, width, height, img)
    if chirp:
        n = min(512, width, height)
        x0, y0 = (width - n) // 3, (height - n) // 3
        ys, xs = np.mgrid[0:n, 0:n].astype(np.float32) - n / 2
        zone = 0.45 + 0.4 * np.cos(np.pi * (xs * xs + ys * ys) / n)
        img[y0:y0 + n, x0:x0 + n] = zone[..., None]
    if lines:
        n = min(256, width // 2, height // 2)
        x0, y0 = (2 * width) // 3 - n // 2, (2 * height) // 3 - n // 2
        x0, y0 = max(0, min(x0, width - n)), max(0, min(y0, height - n))
        ys, xs = np.mgrid[0:n, 0:n]
        stripes = (((xs + ys) // 1) % 4 < 2).astype(np.float32)
        img[y0:y0 + n, x0:x0 + n] = (0.1 + 0.7 * stripes)[..., None]
    return img


def bayer(width: int, height: int, *, seed: int, pattern: int = 0, phase=(0, 0), stride: int = 0,
          active=None, black=(512, 512, 512, 512), white=16383, chirp=False, lines=False,
          gain_dn_per_e=0.5, read_sigma_dn=3.0, bits=14) -> np.ndarray:
    """uint16 sensor samples, shape (height, stride) (stride defaults to width)."""
    stride = stride or width
    ax, ay, aw, ah = active if active else (0, 0, width, height)
    rng = np.random.default_rng(seed + 7919)
    scene = radiance(width, height, seed, chirp, lines)
    site = (((np.arange(height)[:, None] & 1) + phase[1]) & 1) * 2 + \
           (((np.arange(width)[None, :] & 1) + phase[0]) & 1)
    colours = np.array(PATTERN_COLORS[pattern])[site]
    mosaic = np.take_along_axis(scene, colours[..., None], axis=2)[..., 0]
    black_site = np.array(black, np.float32)[site]
    span = np.float32(white) - black_site
    signal_dn = np.clip(mosaic, 0, None) * span
    electrons = rng.poisson(signal_dn / gain_dn_per_e).astype(np.float32)
    dn = electrons * gain_dn_per_e + rng.normal(0, read_sigma_dn, signal_dn.shape).astype(np.float32)
    dn += black_site
    samples = np.clip(np.rint(dn), 0, (1 << bits) - 1).astype(np.uint16)
    out = np.zeros((height, stride), np.uint16)
    out[:, :width] = samples
    # outside the active area the sensor holds optical-black-like codes
    mask = np.ones((height, width), bool)
    mask[ay:ay + ah, ax:ax + aw] = False
    out[:, :width][mask] = np.array(black, np.uint16)[site][mask]
    return out


def raster(width: int, height: int, seed: int) -> np.ndarray:
    """Scene-linear ProPhoto RGB (height, width, 3) float32 for spatial stages."""
    rng = np.random.default_rng(seed)
    lum = np.exp(rng.normal(-1.5, 1.2, (height, width)).astype(np.float32) * 0.35 - 1.0)
    # smooth the noise field a little so that edges dominate texture
    base = np.exp(np.float32(-1.5)) * np.ones((height, width), np.float32)
    for _ in range(24):
        nx, ny = rng.normal(size=2)
        c = rng.uniform(-1, 1) * (width + height) / 4
        side = (np.arange(width)[None, :] - width / 2) * nx + (np.arange(height)[:, None] - height / 2) * ny > c
        base = np.where(side, base * np.float32(np.exp(rng.normal(0, 0.6))), base)
    lum = np.clip(base * lum * 2.0, 0, 4.0).astype(np.float32)
    hue = rng.uniform(0, 2 * np.pi, 64)
    sat = rng.uniform(0, 0.6, 64)
    region = (np.arange(height)[:, None] * 8 // height) * 8 + (np.arange(width)[None, :] * 8 // width)
    h, s = hue[region], sat[region]
    rgb = np.empty((height, width, 3), np.float32)
    for k in range(3):
        rgb[..., k] = lum * (1 + s * np.cos(h - k * 2 * np.pi / 3)).astype(np.float32)
    flat = rgb.reshape(-1)
    n = flat.size
    neg = rng.choice(n, n // 50, replace=False)
    flat[neg] = -rng.uniform(0, 0.01, neg.size).astype(np.float32)
    hi = rng.choice(n, n // 200, replace=False)
    flat[hi] = rng.uniform(1.0, 4.0, hi.size).astype(np.float32)
    return rgb


def bayer_device(width: int, height: int, *, seed: int, pattern: int = 0, phase=(0, 0), stride: int = 0,
                 black=(512, 512, 512, 512), white=16383, device="cuda"):
    """A CUDA int16 tensor (height, stride) of 14-bit sensor codes (all below
    2^15, so the int16 bits are the uint16 codes), synthesized on the device for
    large batches: a smooth colour field with edges plus Gaussian read noise.
    Content is seeded and deterministic on one device."""
    import torch
    stride = stride or width
    g = torch.Generator(device=device).manual_seed(seed)
    y = torch.arange(height, device=device, dtype=torch.float32)[:, None]
    x = torch.arange(stride, device=device, dtype=torch.float32)[None, :]
    f1, f2, f3 = 17.0 + seed % 11, 29.0 + seed % 7, 211.0 + seed % 97
    base = 0.30 + 0.22 * torch.sin(x / f1 + seed) * torch.cos(y / f2) + 0.18 * (x / stride) + \
        0.15 * torch.sign(torch.sin((x + 0.6 * y) / f3))
    site = ((((y.long() & 1) + phase[1]) & 1) * 2 + (((x.long() & 1) + phase[0]) & 1))
    colours = torch.tensor(PATTERN_COLORS[pattern], device=device)[site]
    gain = torch.tensor([0.85, 1.0, 0.7], device=device)[colours]
    lv = torch.tensor(black, device=device, dtype=torch.float32)[site]
    signal = base.clamp(0.0, 1.3) * gain * (float(white) - lv) + lv
    noise = torch.randn(signal.shape, generator=g, device=device) * 6.0
    return (signal + noise).round().clamp(0, 16383 + 900).to(torch.int16)
