"""Pins the oracle before it is trusted as the checker (CPU only).

* Against the reference's own frozen Menon vectors (93 fixtures, every
  pattern/phase/origin, block-crossing 269x263 case; the reference checks them
  bit-exactly in tests/raw_menon_native_tests.cpp:40-102).
* Against outputs of the unmodified reference library (oracle/_ref) on seeded
  inputs (tests/golden/reference_renders.npz, made by make_golden.py), and
  live against the reference library when it is present.
* Against the reference tests' known answers (sRGB encode, curve truth,
  guided-filter rational impulse, local-statistics closed forms).
"""
import numpy as np
import pytest

from conftest import bits_equal
from oracle.oracle import (OP_CAMERA_TO_WORKING, OP_CURVES_EXT, OP_EXPOSURE, OP_WB, Op, Oracle,
                           OracleError, RawSpec, curves_params)


def _raw(meta, levels, samples):
    w = meta
    return RawSpec(w[0], w[1], np.asarray(samples, np.uint16), w[2], w[3], w[4], w[5],
                   tuple(w[6:10]), tuple(levels[:4]), tuple(levels[4:]))


def test_menon_oracle_matches_frozen_fixtures(oracle, menon_fixtures):
    assert len(menon_fixtures) == 93
    channels = 0
    for i, (meta, levels, samples, expected) in enumerate(menon_fixtures):
        raw = _raw(meta, levels, samples)
        area = meta[6:10]
        exp = expected.reshape(area[3], area[2], 3)
        assert bits_equal(oracle.demosaic(raw, area, True), exp), f"fixture {i}"
        roi = (area[0] + area[2] // 3, area[1] + area[3] // 3, max(1, area[2] // 3), max(1, area[3] // 3))
        crop = exp[roi[1] - area[1]:roi[1] - area[1] + roi[3], roi[0] - area[0]:roi[0] - area[0] + roi[2]]
        assert bits_equal(oracle.demosaic(raw, roi, True), crop), f"fixture {i} roi"
        # padding and inactive photosites cannot affect reconstruction
        padded = np.array(samples, np.uint16).reshape(meta[1], meta[2])
        mask = np.ones_like(padded, bool)
        mask[area[1]:area[1] + area[3], area[0]:area[0] + area[2]] = False
        padded[mask] = 0
        assert bits_equal(oracle.demosaic(_raw(meta, levels, padded.reshape(-1)), area, True), exp)
        channels += exp.size
    assert channels == 352221


def test_reference_library_matches_frozen_fixtures(reference, menon_fixtures):
    for i, (meta, levels, samples, expected) in enumerate(menon_fixtures[:40]):
        area = meta[6:10]
        got = reference.render_raw(_raw(meta, levels, samples), True, [], area, tile=37)
        assert bits_equal(got, expected.reshape(area[3], area[2], 3)), f"fixture {i}"


def _golden_case(goldens, name):
    meta = [int(v) for v in goldens[f"{name}/meta"]]
    levels = [int(v) for v in goldens[f"{name}/levels"]]
    raw = _raw(meta, levels, goldens[f"{name}/samples"])
    codes = goldens[f"{name}/ops"]
    params = list(goldens[f"{name}/params"])
    from oracle import oracle as O
    counts = {O.OP_WB: 3, O.OP_EXPOSURE: 1, O.OP_CAMERA_TO_WORKING: 10, O.OP_WORKING_TO_SRGB: 0,
              O.OP_TONE: 2, O.OP_OUTPUT_CLIP: 0, O.OP_SRGB_ENCODE: 0, O.OP_DISPLAY_TAG: 0}
    ops, k = [], 0
    for c in codes:
        c = int(c)
        if c == O.OP_CURVES_EXT:
            n0 = 1
            j = k + 1
            for _ in range(4):
                n = int(params[j]); j += 1 + 2 * n
            n0 = j - k
        else:
            n0 = counts[c]
        ops.append(Op(c, params[k:k + n0]))
        k += n0
    return raw, ops


@pytest.mark.parametrize("name,menon", [("bl_rggb", False), ("bl_gbrg", False), ("mn_bggr", True),
                                        ("mn_grbg", True), ("mn_rggb_prev", True)])
def test_oracle_chains_match_reference_renders(oracle, goldens, name, menon):
    raw, ops = _golden_case(goldens, name)
    for mip in (0, 1, 2):
        key = f"{name}/mip{mip}/rgb"
        if key not in goldens:
            continue
        vp = tuple(int(v) for v in goldens[f"{name}/mip{mip}/viewport"])
        got = oracle.render_raw(raw, menon, ops, vp, mip=mip, quality=0 if mip else 1)
        assert bits_equal(got, goldens[key]), f"{name} mip {mip}"


def test_oracle_random_bilinear_chains_match_reference(oracle, reference):
    rng = np.random.default_rng(5)
    for trial in range(12):
        w, h = int(rng.integers(2, 40)), int(rng.integers(2, 30))
        stride = w + int(rng.integers(0, 5))
        ax, ay = int(rng.integers(0, 3)), int(rng.integers(0, 3))
        aw, ah = max(1, w - ax - int(rng.integers(0, 3))), max(1, h - ay - int(rng.integers(0, 3)))
        black = tuple(int(v) for v in rng.integers(0, 2000, 4))
        white = tuple(b + int(rng.integers(1, 20000)) for b in black)
        s = rng.integers(0, 65536, stride * h).astype(np.uint16)
        raw = RawSpec(w, h, s, stride, int(rng.integers(0, 4)), int(rng.integers(0, 2)),
                      int(rng.integers(0, 2)), (ax, ay, aw, ah), black, white)
        cam = list(rng.normal(0, 0.2, 9) + np.eye(3).reshape(9)) + [int(rng.integers(0, 2))]
        ops = [Op(OP_WB, list(rng.uniform(0.5, 3, 3))), Op(OP_EXPOSURE, [float(rng.uniform(-2, 2))]),
               Op(OP_CAMERA_TO_WORKING, cam)]
        menon = bool(trial % 2)
        vp = (ax, ay, aw, ah)
        want = reference.render_raw(raw, menon, ops, vp, tile=int(rng.integers(1, 40)))
        assert bits_equal(oracle.render_raw(raw, menon, ops, vp), want), trial


def test_srgb_encode_known_answers(oracle):
    # tests/core_tests.cpp:457-470 known answers (2e-6 relative there)
    v = np.array([0.0031308, 0.18, 1.2, -1.0], np.float32)
    oracle.srgb_encode(v)
    assert abs(v[0] - 0.04045) < 2e-6 and abs(v[1] - 0.461356) < 2e-6
    assert abs(v[2] - 1.0) < 2e-6 and v[3] == 0.0
    bad = np.array([np.nan, 0, 0], np.float32)
    with pytest.raises(OracleError) as e:
        oracle.srgb_encode(bad)
    assert e.value.kind == "domain_error"


def test_curves_truth(oracle):
    # tests/curves_levels_tests.cpp:14-20: master then channel, one float cast
    c = oracle.curves(curves_params(1, [(0, 0), (.5, .25), (1, 1)], [(0, 0), (.5, .75), (1, 1)],
                                    [(0, 0), (.5, .75), (1, 1)], [(0, 0), (.5, .75), (1, 1)]))
    v = np.array([.25, .25, .25, .5029296875, .5029296875, .5029296875], np.float32)
    oracle.curves_apply(c, v)
    assert v[0] == np.float32(.2109375) and v[3] == np.float32(.4401211142539978)
    flat = oracle.curves(curves_params(1, [(0, 0), (1, 1), (2, 1), (3, 2)]))
    v = np.array([1.25, 1.5, 1.75], np.float32)
    oracle.curves_apply(flat, v)
    assert list(v) == [1, 1, 1]


def test_guided_filter_rational_impulse(oracle):
    # tests/guided_filter_tests.cpp:40-49: exact neutral impulse at r=1, eps=1
    img = np.zeros((1, 5, 3), np.float32)
    img[0, 2] = 1
    full = (0, 0, 5, 1)
    for prophoto in (True, False):
        out = oracle.guided_filter(img, full, full, full, 1, 1.0, prophoto)
        want = np.array([3 / 22, 2 / 11, 5 / 11, 2 / 11, 3 / 22], np.float32)
        for c in range(3):
            assert np.array_equal(out[0, :, c], want)


def test_guided_filter_constants_exact(oracle):
    # tests/guided_filter_tests.cpp:63-67: constants/extremes/signed zero exact
    m = np.finfo(np.float32).max
    for vals in ([-0.0, 0.0, -0.0], [m, m, m], [-m, m, -m], [1e-45, 1e-45, 1e-45], [-.5, .25, 2]):
        img = np.array(vals, np.float32).reshape(1, 1, 3)
        for r in (0, 1, 8):
            for eps in (2.0 ** -24, 65536.0):
                out = oracle.guided_filter(img, (0, 0, 1, 1), (0, 0, 1, 1), (0, 0, 1, 1), r, eps)
                assert bits_equal(out, img)


def test_local_statistics_closed_forms(oracle):
    # tests/spatial_ops_tests.cpp:49-70: affine ramp mean, population variance (n^2-1)/12
    w = 17
    ramp = np.zeros((1, w, 3), np.float32)
    ramp[0, :, 0] = np.arange(w)
    ramp[0, :, 1] = 3 * np.arange(w) + 1
    ramp[0, :, 2] = 1e20 + 0 * np.arange(w)
    full = (0, 0, w, 1)
    for r in (1, 3, 8):
        mean, var, cnt = oracle.local_statistics(ramp, full, full, full, r)
        x = 8
        n = 2 * r + 1
        assert cnt[0, x, 0] == n and mean[0, x, 0] == 8.0
        assert abs(var[0, x, 0] - (n * n - 1) / 12) < 1e-12
        assert var[0, x, 2] == 0.0 and mean[0, x, 2] == np.float32(1e20)


@pytest.mark.parametrize("kind", ["gf", "ls", "cubic", "rotate"])
def test_oracle_spatial_geometry_match_reference_renders(oracle, goldens, kind):
    img = goldens["raster/rgb"]
    h, w = img.shape[:2]
    full = (0, 0, w, h)
    if kind == "gf":
        for r in (1, 3, 8):
            for eps in (1e-3, 1e-2, 1.0):
                got = oracle.guided_filter(img, full, full, full, r, eps)
                assert bits_equal(got, goldens[f"gf/r{r}_e{eps:g}"]), (r, eps)
    elif kind == "ls":
        for r in (0, 1, 3, 8):
            mean, var, cnt = oracle.local_statistics(img, full, full, full, r)
            assert np.array_equal(mean, goldens[f"ls/r{r}/mean"])
            assert np.array_equal(var, goldens[f"ls/r{r}/var"])
            assert np.array_equal(cnt, goldens[f"ls/r{r}/count"])
    elif kind == "cubic":
        for (ow, oh) in ((80, 50), (61, 43), (20, 15), (16, 11), (128, 90)):
            got = oracle.cubic_resize(img, ow, oh, (0, 0, ow, oh))
            assert bits_equal(got, goldens[f"cubic/{ow}x{oh}"]), (ow, oh)
            for mip in (1, 2):
                sc = 1 << mip
                vp = (0, 0, (ow + sc - 1) // sc, (oh + sc - 1) // sc)
                native = oracle.mip_native_region((0, 0, ow, oh), mip, vp)
                full_native = oracle.cubic_resize(img, ow, oh, native)
                got = oracle.mip_reduce(full_native, native, mip, vp)
                assert bits_equal(got, goldens[f"cubic/{ow}x{oh}/mip{mip}"]), (ow, oh, mip)
    else:
        for angle in (0.0, 90.0, -90.0, 180.0, 33.3, -45.0, 12.5):
            rot = oracle.rotation(angle, w, h)
            assert bits_equal(oracle.rotate(rot, img, full), goldens[f"rotate/{angle:g}"]), angle
            for mip in (1, 2):
                sc = 1 << mip
                vp = (0, 0, (w + sc - 1) // sc, (h + sc - 1) // sc)
                native = oracle.mip_native_region(full, mip, vp)
                nat = oracle.rotate(rot, img, native)
                got = oracle.mip_reduce(nat, native, mip, vp)
                assert bits_equal(got, goldens[f"rotate/{angle:g}/mip{mip}"]), (angle, mip)


def test_plan_and_halo_match_reference(oracle, reference):
    rng = np.random.default_rng(9)
    for _ in range(30):
        w, h = int(rng.integers(1, 50)), int(rng.integers(1, 50))
        s = np.zeros(w * h, np.uint16)
        ax, ay = int(rng.integers(0, w)), int(rng.integers(0, h))
        aw, ah = int(rng.integers(1, w - ax + 1)), int(rng.integers(1, h - ay + 1))
        raw = RawSpec(w, h, s, 0, 0, 0, 0, (ax, ay, aw, ah), (0,) * 4, (1000,) * 4)
        ox, oy = ax + int(rng.integers(0, aw)), ay + int(rng.integers(0, ah))
        out = (ox, oy, int(rng.integers(1, ax + aw - ox + 1)), int(rng.integers(1, ay + ah - oy + 1)))
        for menon in (False, True):
            assert oracle.raw_input_region(raw, menon, out) == reference.raw_input_region(raw, menon, [], out)
    vp = (3, 5, 517, 301)
    tiles = oracle.plan_tiles(vp, 128)
    assert tiles[0] == (3, 5, 128, 128) and tiles[-1] == (3 + 512, 5 + 256, 5, 45)
    assert len(tiles) == 5 * 3


def _probe_pattern(bounds, viewport):
    """The reference's analysis probe (image_analysis_tests.cpp:20-41):
    R = (x % 9) / 4 - 0.5, G = (y % 9) / 4 - 0.5, B = NaN over the viewport."""
    x0, y0, w, h = viewport
    y, x = np.mgrid[y0:y0 + h, x0:x0 + w]
    return np.stack([(x % 9) * 0.25 - 0.5, (y % 9) * 0.25 - 0.5, np.full(x.shape, np.nan)], -1).astype(np.float32)


def test_histogram_restatement_known_answers():
    """The discrete truths of image_analysis_tests.cpp:44-103, restated."""
    from oracle.oracle import histogram_rgb
    vp = (9, 7, 19, 13)
    img = _probe_pattern(None, vp)
    for tile in (1, 3, 4, 7, 256):
        h = histogram_rgb(img, 4, 0.0, 1.0, tile)
        for c in range(2):
            expected, below, above = np.zeros(4, np.uint64), 0, 0
            for y in range(7, 20):
                for x in range(9, 28):
                    site = (x if c == 0 else y) % 9
                    if site < 2:
                        below += 1
                    elif site > 6:
                        above += 1
                    else:
                        expected[3 if site == 6 else site - 2] += 1
            assert np.array_equal(h[c]["counts"], expected)
            assert (h[c]["underflow"], h[c]["overflow"], h[c]["nonfinite"]) == (below, above, 0)
            assert (h[c]["minimum"], h[c]["maximum"]) == (-0.5, 1.5)
        assert h[2]["nonfinite"] == 247 and h[2]["minimum"] is None and h[2]["maximum"] is None
    inf = np.float32(np.inf)
    vals = np.array([[[-inf, 0, -2], [inf, 1, 2], [np.nan, 0.5, 0]]], np.float32)
    h = histogram_rgb(vals, 1, 0.0, 1.0)
    assert h[0]["nonfinite"] == 3 and h[0]["minimum"] is None
    assert h[1]["counts"][0] == 3 and h[2]["underflow"] == 1 and h[2]["overflow"] == 1
    assert histogram_rgb(vals, 65536, -1e300, 1e300)[1]["counts"][32768] == 3
    h = histogram_rgb(vals, 2, 0.0, 5e-324)
    assert h[1]["counts"][0] == 1 and h[1]["overflow"] == 2


@pytest.mark.parametrize("bins,lower,upper,tile", [(4, 0.0, 1.0, 7), (256, -0.5, 1.5, 16), (5000, 0.2, 0.3, 8),
                                                   (65536, -1e300, 1e300, 256), (1, 0.0, 1.0, 5)])
def test_histogram_restatement_matches_reference(reference, bins, lower, upper, tile):
    """Finite images (the reference's raster source rejects others), including
    +0 / -0 ties at the minimum of a channel."""
    from oracle.oracle import histogram_rgb
    rng = np.random.default_rng(bins)
    img = rng.normal(0.5, 0.6, (37, 53, 3)).astype(np.float32)
    img[..., 2] = np.abs(img[..., 2])
    img[1, 40, 2] = -0.0          # first in row order, in a later tile ...
    img[3, 2, 2] = 0.0            # ... than this +0 when tiles are narrower than 40
    img[20, 50, 2] = -0.0
    want = reference.histogram(img, (0, 0, 53, 37), bins, lower, upper, tile=tile)
    got = histogram_rgb(img, bins, lower, upper, tile)
    for c in range(3):
        for k in ("underflow", "overflow", "nonfinite"):
            assert got[c][k] == want[c][k], (c, k)
        assert np.array_equal(got[c]["counts"], want[c]["counts"]), c
        for k in ("minimum", "maximum"):
            assert np.float32(got[c][k]).tobytes() == np.float32(want[c][k]).tobytes(), (c, k)
