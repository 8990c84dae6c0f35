"""The C ABI library without a GPU: it loads, exports every symbol the header
declares, and its host-side planning (the reference's integer rules and colour
maths) equals the oracle's bit for bit.  No device entry point is called."""
import os
import re

import numpy as np
import pytest

from librawops_b200 import _capi, render
from librawops_b200._capi import ReError
from oracle.oracle import RawSpec

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "rawengine_b200.h")


def test_library_exports_every_declared_symbol():
    text = open(HEADER).read()
    declared = set(re.findall(r"RE_API\s+[\w\s\*]+?\b(re_\w+)\s*\(", text))
    assert declared == set(_capi.EXPORTS)
    lib = _capi.lib()
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing


def test_request_bounds_matches_oracle(oracle):
    for src in [(0, 0, 1, 1), (16, 8, 6000, 4000), (3, 5, 7, 9), (0, 0, 5, 1)]:
        for mip in range(4):
            for q in (0, 1, 2):
                try:
                    want = oracle.request_bounds(src, mip, q)
                except Exception as e:
                    with pytest.raises(ReError) as got:
                        render.request_bounds(src, mip, q)
                    assert got.value.kind == e.kind
                    continue
                assert render.request_bounds(src, mip, q) == want


def test_halo_mip_and_tile_planning_match_oracle(oracle):
    rng = np.random.default_rng(3)
    for _ in range(200):
        w, h = int(rng.integers(1, 60)), int(rng.integers(1, 60))
        ax, ay = int(rng.integers(0, w)), int(rng.integers(0, h))
        aw, ah = int(rng.integers(1, w - ax + 1)), int(rng.integers(1, h - ay + 1))
        raw = RawSpec(w, h, np.zeros(w * h, np.uint16), 0, 0, 0, 0, (ax, ay, aw, ah), (0,) * 4, (9,) * 4)
        meta = render.Metadata(w, h, 0, 0, 0, 0, (ax, ay, aw, ah), (0,) * 4, (9,) * 4)
        ox, oy = ax + int(rng.integers(0, aw)), ay + int(rng.integers(0, ah))
        out = (ox, oy, int(rng.integers(1, ax + aw - ox + 1)), int(rng.integers(1, ay + ah - oy + 1)))
        for d in (0, 1):
            assert render.raw_input_region(meta, d, out) == oracle.raw_input_region(raw, d, out)
        for mip in (1, 2):
            sc = 1 << mip
            red = (0, 0, (aw + sc - 1) // sc, (ah + sc - 1) // sc)
            rx, ry = int(rng.integers(0, red[2])), int(rng.integers(0, red[3]))
            vp = (rx, ry, int(rng.integers(1, red[2] - rx + 1)), int(rng.integers(1, red[3] - ry + 1)))
            assert render.mip_native_region((ax, ay, aw, ah), mip, vp) == \
                oracle.mip_native_region((ax, ay, aw, ah), mip, vp)
        tile = int(rng.integers(1, 70))
        assert render.plan_tiles(out, tile) == oracle.plan_tiles(out, tile)
    with pytest.raises(ReError) as e:
        render.raw_input_region(render.Metadata(10, 10, 0, 0, 0, 0, (0, 0, 10, 10)), 1, (5, 5, 6, 1))
    assert e.value.kind == "out_of_range"


def test_colour_matrices_match_oracle(oracle):
    rng = np.random.default_rng(4)
    for _ in range(50):
        cam = rng.normal(0, 0.3, (3, 3)) + np.eye(3)
        for t in (0, 1):
            assert np.array_equal(render.camera_to_working_matrix(cam, t), oracle.camera_to_working(cam, t))
    for s in (0, 1):
        assert np.array_equal(render.working_to_srgb_matrix(s), oracle.working_to_srgb(s))
        for t in (0, 1):
            assert np.array_equal(render.working_to_working_matrix(s, t), oracle.working_to_working(s, t))
    with pytest.raises(ReError) as e:
        render.camera_to_working_matrix(np.zeros((3, 3)))
    assert e.value.kind == "invalid_argument"
    for stops in (-32, -1.5, 0, 0.25, 1, 32):
        assert render.exposure_multiplier(stops) == oracle.exposure_multiplier(stops)
    for bad in (-33, 33, float("nan")):
        with pytest.raises(ReError):
            render.exposure_multiplier(bad)


def test_metadata_normalization_matches_reference_rules(oracle):
    ok = render.normalize_metadata(render.Metadata(6, 4, 0, 1, 1, 0), 24)
    assert ok.row_stride_samples == 6 and ok.active_area == (0, 0, 6, 4)
    bad = [
        (render.Metadata(0, 4), 0),                                   # empty
        (render.Metadata(6, 4, 5), 20),                               # stride < width
        (render.Metadata(6, 4, 0, 4), 24),                            # pattern
        (render.Metadata(6, 4, 0, 0, 2), 24),                         # phase
        (render.Metadata(6, 4, 0, 0, 0, 0, (2, 0, 5, 4)), 24),        # active outside
        (render.Metadata(6, 4, 0, 0, 0, 0, (0, 0, 0, 0), (9, 0, 0, 0), (9, 1, 1, 1)), 24),  # white<=black
        (render.Metadata(6, 4), 23),                                  # count
    ]
    for meta, count in bad:
        with pytest.raises(ReError) as e:
            render.normalize_metadata(meta, count)
        assert e.value.kind == "invalid_argument"
        raw = RawSpec(meta.width, meta.height, np.zeros(count, np.uint16), meta.row_stride_samples,
                      meta.pattern, meta.cfa_phase_x, meta.cfa_phase_y, meta.active_area,
                      meta.black_levels, meta.white_levels)
        with pytest.raises(Exception):
            oracle.normalized(raw)


def test_site_and_colour_lookup_match_oracle(oracle):
    lib = _capi.lib()
    for pattern in range(4):
        for px in (0, 1):
            for py in (0, 1):
                meta = render.Metadata(8, 8, 0, pattern, px, py)
                m = render.normalize_metadata(meta, 64).struct()
                raw = RawSpec(8, 8, np.zeros(64, np.uint16), 0, pattern, px, py)
                om = oracle.normalized(raw)
                for y in range(4):
                    for x in range(4):
                        assert lib.re_site_index(m, x, y) == oracle.lib.or_site_index(om, x, y)
                        assert lib.re_cfa_color(m, x, y) == oracle.lib.or_cfa_color(om, x, y)
