"""Regenerates the committed golden fixtures under tests/golden/ (run in a
checkout that has the reference at $REF -- by default a directory named
"reference" beside this checkout -- and the reference library built by
`make -C oracle ref`).

* menon_native_base_v1.npz -- the reference's own frozen Menon vectors
  (tests/reference/raw/menon_native_base_v1.bin, format documented in its
  .index.json and read by tests/raw_menon_native_tests.cpp:40-61), repacked.
* reference_renders.npz    -- outputs of the unmodified reference library
  (oracle/_ref) on small seeded synthetic inputs: RAW chains (bilinear and
  Menon, linear and sRGB, mip 0/1/2), guided filter, local statistics, cubic
  resize and rotate.  Inputs are stored beside the outputs.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import (OP_CAMERA_TO_WORKING, OP_CUBIC_RESIZE, OP_CURVES_EXT,  # noqa: E402
                           OP_DISPLAY_TAG, OP_EXPOSURE, OP_GUIDED_FILTER, OP_OUTPUT_CLIP, OP_ROTATE,
                           OP_SRGB_ENCODE, OP_TONE, OP_WB, OP_WORKING_TO_SRGB, Op, RawSpec, Reference,
                           curves_params)
from librawops_b200 import synthetic, workloads  # noqa: E402

REF = os.environ.get("REF", os.path.join(os.path.dirname(ROOT), "reference"))


def menon_fixtures():
    path = os.path.join(REF, "tests", "reference", "raw", "menon_native_base_v1.bin")
    data = open(path, "rb").read()
    assert data[:8] == b"LRMENON1"
    off = 8
    (count,) = struct.unpack_from("<I", data, off)
    off += 4
    metas, levels, samples, expected, offsets, eoffsets = [], [], [], [], [0], [0]
    for _ in range(count):
        w = struct.unpack_from("<10I", data, off); off += 40
        lv = struct.unpack_from("<8H", data, off); off += 16
        (n,) = struct.unpack_from("<I", data, off); off += 4
        s = np.frombuffer(data, np.uint16, n, off); off += 2 * n
        k = w[8] * w[9] * 3
        e = np.frombuffer(data, np.float32, k, off); off += 4 * k
        metas.append(w); levels.append(lv); samples.append(s); expected.append(e)
        offsets.append(offsets[-1] + n); eoffsets.append(eoffsets[-1] + k)
    assert off == len(data)
    np.savez_compressed(os.path.join(HERE, "menon_native_base_v1.npz"),
                        meta=np.array(metas, np.uint32), levels=np.array(levels, np.uint16),
                        samples=np.concatenate(samples), sample_offsets=np.array(offsets, np.int64),
                        expected=np.concatenate(expected), expected_offsets=np.array(eoffsets, np.int64))
    print("menon fixtures:", count)


def raw_chains():
    """Small seeded RAW cases rendered by the reference library."""
    ref = Reference()
    out = {}
    cases = [
        # name, (w, h, stride, pattern, phase, active, black, white), menon, chain kind
        ("bl_rggb", (96, 64, 100, 0, (0, 0), (2, 2, 90, 60), (512, 512, 512, 512), 16383), False, "linear"),
        ("bl_gbrg", (77, 51, 80, 3, (1, 0), (3, 1, 71, 49), (500, 510, 490, 505), 15000), False, "legacy"),
        ("mn_bggr", (96, 64, 104, 1, (0, 0), (4, 2, 88, 58), (510, 512, 511, 513), 15800), True, "srgb_curve"),
        ("mn_grbg", (71, 45, 71, 2, (0, 1), (1, 3, 69, 41), (256, 260, 250, 255), 4095), True, "srgb_curve"),
        ("mn_rggb_prev", (96, 64, 96, 0, (1, 1), (0, 0, 96, 64), (512, 512, 512, 512), 16383), True, "preview"),
    ]
    for i, (name, (w, h, stride, pat, ph, act, black, white), menon, kind) in enumerate(cases):
        s = synthetic.bayer(w, h, seed=100 + i, pattern=pat, phase=ph, stride=stride, active=act,
                            black=black, white=white, chirp=True, lines=True).reshape(-1)
        raw = RawSpec(w, h, s, stride, pat, ph[0], ph[1], act, black, (white,) * 4)
        cam = list((workloads.PROPHOTO_TO_XYZ @ workloads.CAMERA_TO_PROPHOTO).reshape(9)) + [0]
        curve = curves_params(1, workloads.tone_knots_16())
        if kind == "linear":
            ops = [Op(OP_WB, [2.0, 1.0, 1.6]), Op(OP_EXPOSURE, [0.5]), Op(OP_CAMERA_TO_WORKING, cam)]
        elif kind == "legacy":
            ops = [Op(OP_WB, [1.5, 1.0, 1.2]), Op(OP_EXPOSURE, [-0.25]), Op(OP_CAMERA_TO_WORKING, cam),
                   Op(OP_TONE, [0.25, 1.0]), Op(OP_OUTPUT_CLIP)]
        elif kind == "srgb_curve":
            ops = [Op(OP_WB, [1.9, 1.0, 1.5]), Op(OP_CAMERA_TO_WORKING, cam), Op(OP_CURVES_EXT, curve),
                   Op(OP_WORKING_TO_SRGB), Op(OP_DISPLAY_TAG), Op(OP_SRGB_ENCODE)]
        else:
            ops = [Op(OP_WB, [1.9, 1.0, 1.5]), Op(OP_EXPOSURE, [0.3]), Op(OP_CAMERA_TO_WORKING, cam),
                   Op(OP_WORKING_TO_SRGB), Op(OP_TONE, [0.25, 2.2]), Op(OP_SRGB_ENCODE)]
        out[f"{name}/samples"] = s
        out[f"{name}/meta"] = np.array([w, h, stride, pat, ph[0], ph[1], *act], np.uint32)
        out[f"{name}/levels"] = np.array([*black, *(white,) * 4], np.uint16)
        out[f"{name}/ops"] = np.array([o.code for o in ops], np.int32)
        out[f"{name}/params"] = np.array([p for o in ops for p in o.params] or [0.0], np.float64)
        mips = [0, 1, 2] if kind == "preview" else [0]
        for mip in mips:
            if mip == 0:
                vp = act
            else:
                sc = 1 << mip
                vp = (0, 0, (act[2] + sc - 1) // sc, (act[3] + sc - 1) // sc)
            out[f"{name}/mip{mip}/viewport"] = np.array(vp, np.uint32)
            out[f"{name}/mip{mip}/rgb"] = ref.render_raw(raw, menon, ops, vp, tile=37, mip=mip,
                                                         quality=0 if mip else 1)
    return out


def spatial_geometry(out):
    ref = Reference()
    img = synthetic.raster(61, 43, seed=7)
    out["raster/rgb"] = img
    for r in (1, 3, 8):
        for eps in (1e-3, 1e-2, 1.0):
            out[f"gf/r{r}_e{eps:g}"] = ref.render_raster(img, [Op(OP_GUIDED_FILTER, [r, eps])],
                                                        (0, 0, 61, 43), tile=16)
    full = (0, 0, 61, 43)
    for r in (0, 1, 3, 8):
        mean, var, cnt = ref.local_statistics(img, full, full, full, r)
        out[f"ls/r{r}/mean"], out[f"ls/r{r}/var"], out[f"ls/r{r}/count"] = mean, var, cnt
    for (w, h) in ((80, 50), (61, 43), (20, 15), (16, 11), (128, 90)):
        out[f"cubic/{w}x{h}"] = ref.render_raster(img, [Op(OP_CUBIC_RESIZE, [w, h])], (0, 0, w, h), tile=32)
        for mip in (1, 2):
            sc = 1 << mip
            vp = (0, 0, (w + sc - 1) // sc, (h + sc - 1) // sc)
            out[f"cubic/{w}x{h}/mip{mip}"] = ref.render_raster(
                img, [Op(OP_CUBIC_RESIZE, [w, h])], vp, tile=32, mip=mip, quality=0)
    for angle in (0.0, 90.0, -90.0, 180.0, 33.3, -45.0, 12.5):
        out[f"rotate/{angle:g}"] = ref.render_raster(img, [Op(OP_ROTATE, [angle])], full, tile=40)
        for mip in (1, 2):
            sc = 1 << mip
            vp = (0, 0, (61 + sc - 1) // sc, (43 + sc - 1) // sc)
            out[f"rotate/{angle:g}/mip{mip}"] = ref.render_raster(
                img, [Op(OP_ROTATE, [angle])], vp, tile=40, mip=mip, quality=0)
    return out


if __name__ == "__main__":
    menon_fixtures()
    out = raw_chains()
    out = spatial_geometry(out)
    np.savez_compressed(os.path.join(HERE, "reference_renders.npz"), **out)
    print("reference renders:", len(out), "arrays")
