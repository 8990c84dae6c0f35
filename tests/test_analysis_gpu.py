"""The device histogram (re_histogram_rgb, csrc/analysis.cu) on a B200.

* Finite images: equal to the unmodified reference library's histogram_rgb
  (counts, tallies, and the extrema bit for bit, +0 / -0 ties included) for
  several bin counts, ranges and tile sizes.
* Non-finite samples (which the reference's raster source refuses) and the
  reference's own known-answer probe: against the NumPy restatement, itself
  pinned to the reference on CPU.
* A 6000x4000 frame with NaN, infinities and signed zeros, bins 256 (shared
  memory counters) and 65536 (global counters), against the restatement.
"""
import numpy as np
import pytest

from oracle.oracle import histogram_rgb as restated

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _same(got, want):
    for c in range(3):
        for k in ("underflow", "overflow", "nonfinite"):
            assert got[c][k] == want[c][k], (c, k, got[c][k], want[c][k])
        assert np.array_equal(got[c]["counts"], want[c]["counts"]), c
        for k in ("minimum", "maximum"):
            if want[c][k] is None:
                assert got[c][k] is None, (c, k)
            else:
                assert np.float32(got[c][k]).tobytes() == np.float32(want[c][k]).tobytes(), (c, k)


def _gpu(img, *args):
    from librawops_b200 import render
    return render.histogram_rgb(torch.from_numpy(np.ascontiguousarray(img)).cuda(), *args)


@pytest.mark.parametrize("bins,lower,upper,tile", [(4, 0.0, 1.0, 7), (256, -0.5, 1.5, 16), (5000, 0.2, 0.3, 8),
                                                   (65536, -1e300, 1e300, 256), (1, 0.0, 1.0, 5),
                                                   (4096, -1.0, 2.0, 3)])
def test_histogram_matches_reference(reference, bins, lower, upper, tile):
    rng = np.random.default_rng(bins)
    img = rng.normal(0.5, 0.6, (37, 53, 3)).astype(np.float32)
    img[..., 2] = np.abs(img[..., 2])
    img[1, 40, 2] = -0.0
    img[3, 2, 2] = 0.0
    img[20, 50, 2] = -0.0
    want = reference.histogram(img, (0, 0, 53, 37), bins, lower, upper, tile=tile)
    _same(_gpu(img, bins, lower, upper, tile), want)


def test_histogram_probe_and_nonfinite_known_answers():
    y, x = np.mgrid[7:20, 9:28]
    img = np.stack([(x % 9) * 0.25 - 0.5, (y % 9) * 0.25 - 0.5, np.full(x.shape, np.nan)], -1).astype(np.float32)
    for tile in (1, 3, 4, 7, 256):
        got = _gpu(img, 4, 0.0, 1.0, tile)
        _same(got, restated(img, 4, 0.0, 1.0, tile))
        assert got[2]["nonfinite"] == 247 and got[2]["minimum"] is None
    inf = np.float32(np.inf)
    vals = np.array([[[-inf, 0, -2], [inf, 1, 2], [np.nan, 0.5, 0]]], np.float32)
    for bins, lo, hi in ((1, 0.0, 1.0), (65536, -1e300, 1e300), (2, 0.0, 5e-324)):
        _same(_gpu(vals, bins, lo, hi), restated(vals, bins, lo, hi))


@pytest.mark.parametrize("bins", [256, 65536])
def test_histogram_24mp_with_nonfinite_and_signed_zeros(bins):
    rng = np.random.default_rng(11)
    img = rng.normal(0.45, 0.5, (4000, 6000, 3)).astype(np.float32)
    img[..., 1] = np.abs(img[..., 1])
    flat = img.reshape(-1)
    for value, n in ((np.nan, 5000), (np.inf, 300), (-np.inf, 300), (-0.0, 40), (0.0, 40)):
        flat[rng.choice(flat.size, n, replace=False)] = value
    img[2000, 5999, 1] = -0.0   # the green minimum: zeros of both signs
    img[0, 5000, 1] = 0.0
    for tile in (512, 0):
        _same(_gpu(img, bins, -0.25, 1.25, tile), restated(img, bins, -0.25, 1.25, tile))


@pytest.mark.parametrize("bins,lower,upper", [(7, -0.3, 1.1), (1000, 0.0, 1.0), (65536, -2.0, 3.0), (3, 0.1, 0.4)])
def test_histogram_bin_edges_exact(bins, lower, upper):
    """Samples on and next to every bin edge (the kernel approximates the
    bin with one product and falls back to the reference's division near an
    edge) land where the reference's expression puts them."""
    span = upper - lower
    k = np.arange(0, bins + 1, max(1, bins // 500), dtype=np.float64)
    edges = (lower + k / bins * span).astype(np.float32)
    near = np.concatenate([edges, np.nextafter(edges, np.float32(np.inf)), np.nextafter(edges, np.float32(-np.inf))])
    rng = np.random.default_rng(bins)
    vals = np.concatenate([near, rng.uniform(lower, upper, 20000).astype(np.float32)])
    n = vals.size - vals.size % 3
    img = vals[:n].reshape(1, -1, 3)
    _same(_gpu(img, bins, lower, upper, 0), restated(img, bins, lower, upper, 0))
