"""Guided filter, local statistics, cubic resize and rotate on the GPU against
the reference library's renders (committed goldens) and the C oracle.

Cubic resize and rotate are bit-exact restatements.  The guided filter uses
the box-filter form (tolerance 1e-5 absolute); local statistics use shifted
binary64 sums (float32 outputs within float32 rounding of the reference's
binary64 values; counts exact)."""
import numpy as np
import pytest

from conftest import bits_equal, within_tolerance
from librawops_b200 import render, synthetic
from librawops_b200._capi import ReError

pytestmark = pytest.mark.gpu


def _cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def test_cubic_resize_matches_reference(goldens, oracle):
    img = goldens["raster/rgb"]
    t = _cuda(img)
    for (w, h) in ((80, 50), (61, 43), (20, 15), (16, 11), (128, 90)):
        got = render.cubic_resize(t, w, h).cpu().numpy()
        assert bits_equal(got, goldens[f"cubic/{w}x{h}"]), (w, h)
        for mip in (1, 2):
            sc = 1 << mip
            vp = (0, 0, (w + sc - 1) // sc, (h + sc - 1) // sc)
            got = render.cubic_resize(t, w, h, output=vp, mip=mip).cpu().numpy()
            assert bits_equal(got, goldens[f"cubic/{w}x{h}/mip{mip}"]), (w, h, mip)
    rng = np.random.default_rng(3)
    for _ in range(6):
        ih, iw = int(rng.integers(4, 70)), int(rng.integers(4, 70))
        src = rng.normal(0.3, 0.5, (ih, iw, 3)).astype(np.float32)
        ow, oh = int(rng.integers((iw + 3) // 4, 2 * iw)), int(rng.integers((ih + 3) // 4, 2 * ih))
        ox, oy = int(rng.integers(0, ow)), int(rng.integers(0, oh))
        out = (ox, oy, int(rng.integers(1, ow - ox + 1)), int(rng.integers(1, oh - oy + 1)))
        got = render.cubic_resize(_cuda(src), ow, oh, output=out).cpu().numpy()
        assert bits_equal(got, oracle.cubic_resize(src, ow, oh, out))
    with pytest.raises(ReError) as e:
        render.cubic_resize(_cuda(np.zeros((40, 41, 3))), 10, 10)      # 4.1x shrink
    assert e.value.kind == "invalid_argument"
    bad = np.zeros((8, 8, 3), np.float32)
    bad[3, 3, 1] = np.inf
    with pytest.raises(ReError) as e:
        render.cubic_resize(_cuda(bad), 12, 12)
    assert e.value.kind == "invalid_argument"


def test_rotate_matches_reference(goldens, oracle):
    img = goldens["raster/rgb"]
    h, w = img.shape[:2]
    t = _cuda(img)
    for angle in (0.0, 90.0, -90.0, 180.0, 33.3, -45.0, 12.5):
        assert bits_equal(render.rotate(t, angle).cpu().numpy(), goldens[f"rotate/{angle:g}"]), angle
        for mip in (1, 2):
            sc = 1 << mip
            vp = (0, 0, (w + sc - 1) // sc, (h + sc - 1) // sc)
            got = render.rotate(t, angle, output=vp, mip=mip).cpu().numpy()
            assert bits_equal(got, goldens[f"rotate/{angle:g}/mip{mip}"]), (angle, mip)
    rng = np.random.default_rng(4)
    for _ in range(6):
        angle = float(rng.uniform(-180, 180))
        src = rng.normal(0.3, 0.5, (37, 53, 3)).astype(np.float32)
        rot = oracle.rotation(angle, 53, 37)
        want = oracle.rotate(rot, src, (5, 3, 40, 30))
        got = render.rotate(_cuda(src), angle, output=(5, 3, 40, 30)).cpu().numpy()
        assert bits_equal(got, want), angle
    assert render.rotation_coefficients(90.0) == (0.0, 1.0)
    with pytest.raises(ReError):
        render.rotate(t, 181.0)


def test_guided_filter_matches_reference(goldens):
    img = goldens["raster/rgb"]
    t = _cuda(img)
    for r in (1, 3, 8):
        for eps in (1e-3, 1e-2, 1.0):
            got = render.guided_filter(t, r, eps).cpu().numpy()
            within_tolerance(got, goldens[f"gf/r{r}_e{eps:g}"], lsb16=False)


def test_guided_filter_known_answers():
    impulse = np.zeros((1, 5, 3), np.float32)
    impulse[0, 2] = 1
    want = np.array([3 / 22, 2 / 11, 5 / 11, 2 / 11, 3 / 22], np.float32)
    for space in (0, 1):
        got = render.guided_filter(_cuda(impulse), 1, 1.0, working_space=space).cpu().numpy()
        for c in range(3):
            assert np.array_equal(got[0, :, c], want)
    m = np.finfo(np.float32).max
    for vals in ([-0.0, 0.0, -0.0], [m, m, m], [-m, m, -m], [1e-45, 1e-45, 1e-45], [-.5, .25, 2]):
        img = np.array(vals, np.float32).reshape(1, 1, 3)
        for r in (0, 1, 8):
            for eps in (2.0 ** -24, 65536.0):
                assert bits_equal(render.guided_filter(_cuda(img), r, eps).cpu().numpy(), img)
    bad = np.zeros((4, 4, 3), np.float32)
    bad[1, 1, 0] = np.nan
    with pytest.raises(ReError) as e:
        render.guided_filter(_cuda(bad), 1, 1e-3)
    assert e.value.kind == "invalid_argument"


@pytest.mark.parametrize("radius", [16, 32])
def test_guided_filter_large_radius_against_oracle(oracle, radius):
    """Radii beyond the reference's 8 (the r 16/32 configurations) against the
    O(r^2) restatement of the reference's arithmetic."""
    img = synthetic.raster(72, 54, seed=21)
    full = (0, 0, 72, 54)
    for eps in (1e-3, 1e-2):
        want = oracle.guided_filter(img, full, full, full, radius, eps)
        got = render.guided_filter(_cuda(img), radius, eps).cpu().numpy()
        within_tolerance(got, want, lsb16=False)


def _ls_close(got, want):
    got = np.asarray(got, np.float64)
    fin = np.isfinite(want)
    assert np.array_equal(np.isfinite(got), fin)
    err = np.abs(got[fin] - want[fin]) / np.maximum(1.0, np.abs(want[fin]))
    assert err.max(initial=0) <= 2e-7, err.max()


def test_local_statistics_match_reference(goldens, oracle):
    img = goldens["raster/rgb"]
    t = _cuda(img)
    for r in (0, 1, 3, 8):
        mean, var, cnt = render.local_statistics(t, r, with_count=True)
        _ls_close(mean.cpu().numpy(), goldens[f"ls/r{r}/mean"])
        _ls_close(var.cpu().numpy(), goldens[f"ls/r{r}/var"])
        assert np.array_equal(cnt.cpu().numpy().astype(np.uint32), goldens[f"ls/r{r}/count"])
    # non-finite samples are excluded; empty windows give NaN
    rng = np.random.default_rng(8)
    x = rng.normal(0, 1, (20, 30, 3)).astype(np.float32)
    x[rng.random((20, 30, 3)) < 0.1] = np.nan
    x[0:3, 0:3, 2] = np.inf
    full = (0, 0, 30, 20)
    for r in (0, 1, 16):
        want_m, want_v, want_n = oracle.local_statistics(x, full, full, full, r)
        m, v, n = render.local_statistics(_cuda(x), r, with_count=True)
        _ls_close(m.cpu().numpy(), want_m)
        _ls_close(v.cpu().numpy(), want_v)
        assert np.array_equal(n.cpu().numpy().astype(np.uint32), want_n)
    # far-from-zero windows keep precision (tests/spatial_ops_tests.cpp high-offset case)
    ramp = np.zeros((1, 17, 3), np.float32)
    ramp[0, :, 0] = 1e20
    ramp[0, :, 1] = np.arange(17) + 1e6
    m, v = render.local_statistics(_cuda(ramp), 8)
    assert float(v[0, 8, 0]) == 0.0 and float(m[0, 8, 0]) == np.float32(1e20)
    assert abs(float(v[0, 8, 1]) - (17 * 17 - 1) / 12) < 1e-3
