"""The strip-streaming guided filter and local statistics kernels' indexing
(spatial.cu), modelled on the CPU (strip_model.py): in bounds, no read of an
entry the current block did not write, every output written once, and the
results of the oracle -- over several strips and bands, partial last strips
and bands, images narrower and shorter than one strip, and every kernel
configuration (radius up to 32)."""
import numpy as np
import pytest

import strip_model
from conftest import within_tolerance
from librawops_b200 import synthetic

GF_CASES = [  # width, height, radius, NT, R, K
    (600, 150, 3, 256, 4, 8), (250, 70, 8, 256, 4, 8), (40, 30, 2, 256, 4, 8), (7, 5, 1, 256, 4, 8),
    (300, 90, 16, 256, 4, 8), (300, 150, 32, 256, 4, 8), (300, 150, 32, 256, 8, 16), (1, 1, 0, 256, 4, 8)]


@pytest.mark.parametrize("w,h,r,nt,rows,k", GF_CASES)
def test_guided_filter_strip_model(oracle, w, h, r, nt, rows, k):
    img = synthetic.raster(w, h, seed=w + h + r)
    full = (0, 0, w, h)
    for eps, space in ((1e-3, 0), (1e-2, 1)):
        got = strip_model.guided_filter(img, r, eps, space, NT=nt, R=rows, K=k)
        want = oracle.guided_filter(img, full, full, full, r, eps, prophoto=space == 0)
        within_tolerance(got, want, lsb16=False)


@pytest.mark.parametrize("w,h,r", [(600, 140, 4), (90, 40, 16), (300, 120, 32), (3, 2, 1)])
def test_local_statistics_strip_model(oracle, w, h, r):
    rng = np.random.default_rng(w * h)
    img = rng.normal(0.5, 1.0, (h, w, 3)).astype(np.float32)
    img[rng.random((h, w, 3)) < 0.05] = np.nan
    img[0:2, 0:3, 1] = np.inf
    full = (0, 0, w, h)
    mean, var, cnt = strip_model.local_statistics(img, r)
    want_m, want_v, want_n = oracle.local_statistics(img, full, full, full, r)
    assert np.array_equal(cnt, want_n)
    fin = np.isfinite(want_m)
    assert np.array_equal(np.isfinite(mean), fin)
    for got, want in ((mean, want_m), (var, want_v)):
        err = np.abs(got[fin] - want[fin]) / np.maximum(1.0, np.abs(want[fin]))
        assert err.max(initial=0) <= 1e-12, err.max()
