"""Parity of the CUDA RAW render path, through the C ABI, on a B200.

Integer/index work and the Menon/bilinear demosaic (with WB, exposure and the
3x3 matrices) must be bit-exact against the reference; stages that call powf or
evaluate curves in float32 must stay within 1e-5 max-abs of full scale and one
16-bit code.  Checkers: the reference's frozen Menon vectors, outputs of the
reference library (committed goldens and oracle/_ref live), and the C oracle.
"""
import numpy as np
import pytest

from conftest import ABS_TOL, bits_equal, within_tolerance
from librawops_b200 import render, workloads
from librawops_b200._capi import ReError
from oracle.oracle import RawSpec

pytestmark = pytest.mark.gpu


def _meta(m, lv):
    return render.Metadata(m[0], m[1], m[2], m[3], m[4], m[5], tuple(m[6:10]), tuple(lv[:4]), tuple(lv[4:]))


def test_menon_frozen_fixtures_bit_exact(menon_fixtures):
    """The binary64 policy against the reference's frozen vectors, bit for bit."""
    pipe = render.Pipeline(demosaic=render.MENON)
    for i, (m, lv, samples, expected) in enumerate(menon_fixtures):
        img = render.Image(_meta(m, lv), samples)
        area = m[6:10]
        exp = expected.reshape(area[3], area[2], 3)
        assert bits_equal(render.render(img, pipe, area), exp), f"fixture {i}"
        roi = (area[0] + area[2] // 3, area[1] + area[3] // 3, max(1, area[2] // 3), max(1, area[3] // 3))
        crop = exp[roi[1] - area[1]:roi[1] - area[1] + roi[3], roi[0] - area[0]:roi[0] - area[0] + roi[2]]
        assert bits_equal(render.render(img, pipe, roi), crop), f"fixture {i} roi"
        # reference render_tiles with tile 3 (37 for the block-crossing case)
        tile = 37 if i == 92 else 3
        assembled = np.zeros_like(exp)

        def cb(r, rgb):
            assembled[r[1] - area[1]:r[1] - area[1] + r[3], r[0] - area[0]:r[0] - area[0] + r[2]] = rgb
        render.render_tiles(img, pipe, area, tile, cb)
        assert bits_equal(assembled, exp), f"fixture {i} tiled"
        padded = np.array(samples, np.uint16).reshape(m[1], m[2])
        mask = np.ones_like(padded, bool)
        mask[area[1]:area[1] + area[3], area[0]:area[0] + area[2]] = False
        padded[mask] = 0
        assert bits_equal(render.render(render.Image(_meta(m, lv), padded), pipe, area), exp)


def test_menon_binary32_fixtures(menon_fixtures, oracle):
    """The binary32 policy: every direction decision equals the reference's,
    demosaic outputs within a few ulp of the frozen vectors, and results
    independent of the viewport and tile size bit for bit."""
    pipe = render.Pipeline(demosaic=render.MENON_FAST)
    for i, (m, lv, samples, expected) in enumerate(menon_fixtures):
        img = render.Image(_meta(m, lv), samples)
        area = m[6:10]
        exp = expected.reshape(area[3], area[2], 3)
        full = render.render(img, pipe, area)
        scale = max(1.0, float(np.abs(exp).max()))
        within_tolerance(full / scale, exp / scale, abs_tol=1e-6, lsb16=False)
        if area[2] > 1 and area[3] > 1:
            raw = RawSpec(m[0], m[1], np.asarray(samples, np.uint16), m[2], m[3], m[4], m[5], tuple(area),
                          tuple(lv[:4]), tuple(lv[4:]))
            _, want_dirs = oracle.demosaic(raw, area, True, directions=True)
            for policy in (render.MENON, render.MENON_FAST):
                got_dirs, _ = render.menon_directions(img, area, policy)
                assert np.array_equal(got_dirs.cpu().numpy(), want_dirs), (i, policy)
        roi = (area[0] + area[2] // 3, area[1] + area[3] // 3, max(1, area[2] // 3), max(1, area[3] // 3))
        crop = full[roi[1] - area[1]:roi[1] - area[1] + roi[3], roi[0] - area[0]:roi[0] - area[0] + roi[2]]
        assert bits_equal(render.render(img, pipe, roi), crop), f"fixture {i} roi"
        tile = 37 if i == 92 else 3
        assembled = np.zeros_like(exp)

        def cb(r, rgb):
            assembled[r[1] - area[1]:r[1] - area[1] + r[3], r[0] - area[0]:r[0] - area[0] + r[2]] = rgb
        render.render_tiles(img, pipe, area, tile, cb)
        assert bits_equal(assembled, full), f"fixture {i} tiled"


def _pipeline_from_golden(goldens, name, menon):
    from test_oracle_pin import _golden_case
    from oracle import oracle as O
    raw, ops = _golden_case(goldens, name)
    p = render.Pipeline(demosaic=int(menon))
    for op in ops:
        if op.code == O.OP_WB:
            p.white_balance(*op.params)
        elif op.code == O.OP_EXPOSURE:
            p.exposure(op.params[0])
        elif op.code == O.OP_CAMERA_TO_WORKING:
            p.camera_to_working(np.array(op.params[:9]).reshape(3, 3), int(op.params[9]))
        elif op.code == O.OP_WORKING_TO_SRGB:
            p.working_to_srgb()
        elif op.code == O.OP_TONE:
            p.tone_curve(op.params[0], op.params[1])
        elif op.code == O.OP_OUTPUT_CLIP:
            p.output_clip()
        elif op.code == O.OP_SRGB_ENCODE:
            p.srgb_encode()
        elif op.code == O.OP_CURVES_EXT:
            it = iter(op.params)
            cubic = bool(next(it))
            curves = []
            for _ in range(4):
                n = int(next(it))
                curves.append([(next(it), next(it)) for _ in range(n)])
            p.extended_curves(render.CurveSet(*curves, cubic=cubic))
    meta = render.Metadata(raw.width, raw.height, raw.row_stride, raw.pattern, raw.phase_x, raw.phase_y,
                           raw.active, raw.black, raw.white)
    return render.Image(meta, raw.samples), p, raw, ops


@pytest.mark.parametrize("name,menon,exact", [("bl_rggb", False, True), ("bl_gbrg", False, True),
                                              ("mn_bggr", True, False), ("mn_grbg", True, False),
                                              ("mn_rggb_prev", True, False)])
def test_chains_match_reference_renders(goldens, name, menon, exact):
    img, pipe, raw, ops = _pipeline_from_golden(goldens, name, menon)
    for mip in (0, 1, 2):
        key = f"{name}/mip{mip}/rgb"
        if key not in goldens:
            continue
        vp = tuple(int(v) for v in goldens[f"{name}/mip{mip}/viewport"])
        got = render.render(img, pipe, vp, mip=mip, quality=render.PREVIEW if mip else render.FINAL)
        if exact:
            assert bits_equal(got, goldens[key]), (name, mip)
        else:
            within_tolerance(got, goldens[key])


def test_random_chains_bit_exact_against_oracle(oracle):
    """Demosaic + WB + exposure + matrix are bit-exact for any metadata (Menon in
    its binary64 policy; the binary32 policy within tolerance)."""
    from oracle.oracle import OP_CAMERA_TO_WORKING, OP_EXPOSURE, OP_WB, Op
    rng = np.random.default_rng(11)
    for trial in range(24):
        w, h = int(rng.integers(1, 90)), int(rng.integers(1, 70))
        stride = w + int(rng.integers(0, 9))
        ax, ay = int(rng.integers(0, min(4, w))), int(rng.integers(0, min(4, h)))
        aw, ah = max(1, w - ax - int(rng.integers(0, 4))), max(1, h - ay - int(rng.integers(0, 4)))
        black = tuple(int(v) for v in rng.integers(0, 3000, 4))
        white = tuple(min(65535, b + int(rng.integers(1, 30000))) for b in black)
        s = rng.integers(0, 65536, stride * h).astype(np.uint16)
        pat, px, py = int(rng.integers(0, 4)), int(rng.integers(0, 2)), int(rng.integers(0, 2))
        raw = RawSpec(w, h, s, stride, pat, px, py, (ax, ay, aw, ah), black, white)
        meta = render.Metadata(w, h, stride, pat, px, py, (ax, ay, aw, ah), black, white)
        cam = rng.normal(0, 0.2, (3, 3)) + np.eye(3)
        wb = [float(np.float32(v)) for v in rng.uniform(0.5, 3, 3)]
        stops = float(np.float32(rng.uniform(-2, 2)))
        menon = bool(trial % 2)
        ops = [Op(OP_WB, wb), Op(OP_EXPOSURE, [stops]), Op(OP_CAMERA_TO_WORKING, list(cam.reshape(9)) + [0])]
        pipe = render.Pipeline(demosaic=int(menon)).white_balance(*wb).exposure(stops)
        pipe.camera_to_working(cam, 0)
        img = render.Image(meta, s)
        vx, vy = ax + int(rng.integers(0, aw)), ay + int(rng.integers(0, ah))
        vp = (vx, vy, int(rng.integers(1, ax + aw - vx + 1)), int(rng.integers(1, ay + ah - vy + 1)))
        want = oracle.render_raw(raw, menon, ops, vp)
        assert bits_equal(render.render(img, pipe, vp), want), trial
        if menon:
            fast = render.Pipeline(demosaic=render.MENON_FAST).white_balance(*wb).exposure(stops)
            fast.camera_to_working(cam, 0)
            got = render.render(img, fast, vp)
            scale = max(1.0, float(np.abs(want).max()))
            within_tolerance(got / scale, want / scale, abs_tol=1e-6, lsb16=False)


def test_errors_follow_reference_exceptions():
    w = workloads.bilinear_1mp(64, 48)
    img = render.Image(render.Metadata(64, 48, 0, 0, 0, 0, (0, 0, 64, 48), w.black, (w.white,) * 4),
                       w.samples())
    linear = workloads.pipeline_for(w)
    with pytest.raises(ReError) as e:
        render.render(img, linear, (60, 40, 8, 8))
    assert e.value.kind == "out_of_range"
    plain = render.Pipeline().white_balance(2, 1, 1)
    with pytest.raises(ReError) as e:
        render.render(img, plain, (0, 0, 8, 8), mip=1, quality=render.PREVIEW)
    assert e.value.kind == "invalid_argument"          # no reduction anchor
    with pytest.raises(ReError) as e:
        render.render(img, linear, (0, 0, 8, 8), mip=3, quality=render.PREVIEW)
    assert e.value.kind == "invalid_argument"
    with pytest.raises(ReError) as e:
        render.render(img, linear, (0, 0, 8, 8), mip=1, quality=render.FINAL)
    assert e.value.kind == "invalid_argument"
    # overflow to infinity reaches the sRGB output boundary: domain_error
    hot = render.Pipeline().white_balance(65536, 65536, 65536)
    for _ in range(4):
        hot.exposure(32)
    hot.srgb_encode()
    with pytest.raises(ReError) as e:
        render.render(img, hot, (0, 0, 64, 48))
    assert e.value.kind == "domain_error"
    # the earliest failing stage wins: curves reject non-finite input first
    cs = render.CurveSet([(0, 0), (0.5, 0.3), (1, 1)])
    early = render.Pipeline().white_balance(65536, 65536, 65536)
    for _ in range(4):
        early.exposure(32)
    early.extended_curves(cs).srgb_encode()
    with pytest.raises(ReError) as e:
        render.render(img, early, (0, 0, 64, 48))
    assert e.value.kind == "invalid_argument"


def test_menon_24mp_properties(oracle):
    """Full-size headline frame: tile invariance (bitwise), finite [0,1] output,
    and a 384x256 crop against the oracle within tolerance."""
    w = workloads.menon_24mp()
    samples = w.samples()
    meta = render.Metadata(w.width, w.height, w.stride, w.pattern, *w.phase, w.active, w.black, (w.white,) * 4)
    img = render.Image(meta, samples)
    pipe = workloads.pipeline_for(w)
    full, stats = render.render(img, pipe, w.active, stats=True)
    assert np.isfinite(full).all() and full.min() >= 0 and full.max() <= 1
    ax, ay, aw, ah = w.active
    quads = [(ax, ay, aw // 2, ah // 2), (ax + aw // 2, ay, aw - aw // 2, ah // 2),
             (ax, ay + ah // 2, aw // 2, ah - ah // 2), (ax + aw // 2, ay + ah // 2, aw - aw // 2, ah - ah // 2)]
    for q in quads:
        part = render.render(img, pipe, q)
        assert bits_equal(part, full[q[1] - ay:q[1] - ay + q[3], q[0] - ax:q[0] - ax + q[2]])
    from oracle.oracle import OP_CAMERA_TO_WORKING, OP_CURVES_EXT, OP_SRGB_ENCODE, OP_WB, \
        OP_WORKING_TO_SRGB, Op, curves_params
    raw = RawSpec(w.width, w.height, samples.reshape(-1), w.stride, w.pattern, *w.phase, w.active, w.black,
                  (w.white,) * 4)
    ops = [Op(OP_WB, list(w.wb)), Op(OP_CAMERA_TO_WORKING, list(w.camera_to_xyz.reshape(9)) + [0]),
           Op(OP_CURVES_EXT, curves_params(1, w.curve)), Op(OP_WORKING_TO_SRGB), Op(OP_SRGB_ENCODE)]
    for crop in [(ax, ay, 384, 256), (ax + 2000, ay + 1300, 384, 256), (ax + aw - 384, ay + ah - 256, 384, 256)]:
        want = oracle.render_raw(raw, True, ops, crop)
        got = full[crop[1] - ay:crop[1] - ay + crop[3], crop[0] - ax:crop[0] - ax + crop[2]]
        within_tolerance(got, want)
        _, want_dirs = oracle.demosaic(raw, crop, True, directions=True)
        for policy in (render.MENON, render.MENON_FAST):
            got_dirs, _ = render.menon_directions(img, crop, policy)
            assert np.array_equal(got_dirs.cpu().numpy(), want_dirs), (crop, policy)
    # the binary32 policy: decisions taken by the binary64 recheck, tile invariance
    _, ties = render.menon_directions(img, w.active, render.MENON_FAST)
    assert 0 <= ties < aw * ah // 2
    fast = workloads.pipeline_for(w)
    fast.demosaic = render.MENON_FAST
    whole = render.render(img, fast, w.active)
    for q in quads[:2]:
        part = render.render(img, fast, q)
        assert bits_equal(part, whole[q[1] - ay:q[1] - ay + q[3], q[0] - ax:q[0] - ax + q[2]])
    assert stats["pixels"] == aw * ah and stats["launches"] >= 1


def test_device_output_and_async_status():
    import torch
    w = workloads.bilinear_1mp()
    meta = render.Metadata(w.width, w.height, 0, 0, 0, 0, w.active, w.black, (w.white,) * 4)
    samples = torch.from_numpy(w.samples().reshape(-1).astype(np.int16)).cuda()
    img = render.Image(meta, samples.view(torch.uint16) if hasattr(torch, "uint16") else samples)
    pipe = workloads.pipeline_for(w)
    host = render.render(img, pipe, w.active)
    dev = torch.empty((w.height, w.width, 3), dtype=torch.float32, device="cuda")
    render.render(img, pipe, w.active, out=dev)
    assert bits_equal(dev.cpu().numpy(), host)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    dev2 = torch.empty_like(dev)
    render.render_async(img, pipe, w.active, dev2, status)
    torch.cuda.synchronize()
    render.status_from_device(int(status.item()))
    assert bits_equal(dev2.cpu().numpy(), host)


def test_extended_curves_against_oracle(oracle):
    """Curve evaluation (cell lookup, binary-search fallback, linear and cubic,
    extrapolation on both sides, samples exactly at knots) vs the reference's
    binary64 restatement, through a bilinear chain."""
    from oracle.oracle import OP_CURVES_EXT, Op, curves_params
    rng = np.random.default_rng(21)
    w, h = 96, 64
    s = rng.integers(300, 16000, w * h).astype(np.uint16)
    raw = RawSpec(w, h, s, 0, 0, 0, 0, (0, 0, w, h), (512,) * 4, (16383,) * 4)
    meta = render.Metadata(w, h, 0, 0, 0, 0, (0, 0, w, h), (512,) * 4, (16383,) * 4)
    img = render.Image(meta, s)
    cases = []
    for n in (2, 3, 5, 16, 40):
        xs = np.sort(rng.uniform(0.05, 0.9, n))
        ys = np.cumsum(rng.uniform(0.0, 0.3, n))
        cases.append([(float(a), float(b)) for a, b in zip(xs, ys)])
    tiny = [(0.0, 0.0), (1e-4, 0.3), (0.5, 0.6), (1.0, 1.0)]        # forces the search fallback
    cases.append(tiny)
    exact = [(0.25, 0.3), (0.5, 0.5), (0.75, 0.9)]                   # knots that are floats
    cases.append(exact)
    for knots in cases:
        for cubic in (True, False):
            chans = [knots, None, [(0.0, 0.0), (0.5, 0.7), (1.5, 1.6)], None]
            pipe = render.Pipeline().extended_curves(render.CurveSet(*chans, cubic=cubic))
            ops = [Op(OP_CURVES_EXT, curves_params(int(cubic), *chans))]
            got = render.render(img, pipe, (0, 0, w, h))
            want = oracle.render_raw(raw, False, ops, (0, 0, w, h))
            within_tolerance(got, want, lsb16=False)
