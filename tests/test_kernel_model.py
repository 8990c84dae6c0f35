"""The Menon kernel's shared-memory indexing, modelled on the CPU (see
kernel_model.py), stays in bounds, never reads an unwritten entry and equals
the oracle bit for bit on tiny, mirrored, multiply-folded and partial tiles."""
import numpy as np
import pytest

from conftest import bits_equal
from kernel_model import model_render
from oracle.oracle import RawSpec

CASES = [(2, 2, None), (3, 5, None), (5, 3, None), (2, 9, None), (33, 17, None), (40, 20, (1, 1, 37, 17)),
         (64, 34, None), (37, 19, (2, 1, 33, 17)), (90, 50, (1, 0, 87, 49)),
         (80, 84, (1, 3, 77, 79))]


@pytest.mark.parametrize("w,h,act", CASES)
def test_menon_kernel_model(oracle, w, h, act):
    rng = np.random.default_rng(w * 100 + h)
    for pattern in range(4):
        W, H = w + 5, h + 4
        stride = W + 3
        a = (2, 1, w, h) if act is None else (act[0] + 2, act[1] + 1, act[2], act[3])
        s = rng.integers(0, 16384, stride * H).astype(np.uint16)
        px, py = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        raw = RawSpec(W, H, s, stride, pattern, px, py, a, (500, 510, 490, 505), (15000, 15500, 16000, 16383))
        meta = dict(width=W, height=H, stride=stride, pattern=pattern, phase_x=px, phase_y=py, active=a,
                    black=raw.black, white=raw.white)
        for vp in (a, (a[0] + a[2] // 3, a[1] + a[3] // 3, max(1, a[2] // 3), max(1, a[3] // 3)),
                   (a[0] + a[2] - 1, a[1] + a[3] - 1, 1, 1), (a[0] + 1, a[1] + 1, a[2] - 1, a[3] - 1)):
            assert bits_equal(model_render(meta, s, vp), oracle.demosaic(raw, vp, True)), (pattern, vp)
