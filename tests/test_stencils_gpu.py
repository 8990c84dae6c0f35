"""Sharpen, Clarity, Texture and Convolution (csrc/stencils.cu) on a B200,
bit for bit against the unmodified reference library's nodes
(SpatialOps.cpp:319-701) over the same raster, for both working spaces,
interior, edge and corner viewports, zero amounts and identity kernels; the
device reads either the whole image or exactly the reference's `needed`
region.  Non-finite samples inside the needed region and results beyond
float32 raise the reference's errors; non-finite samples outside it do not.
The C++ nodes (levels, validation) are covered by tests/cpp/api_driver.cpp.
"""
import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

RNG = np.random.default_rng(5)
CASES = [
    ("sharpen", dict(amount=0.7, radius=1)),
    ("sharpen", dict(amount=2.0, radius=3)),
    ("sharpen", dict(amount=0.0, radius=2)),
    ("clarity", dict(amount=0.5, radius=3)),
    ("clarity", dict(amount=-1.0, radius=8)),
    ("clarity", dict(amount=1.0, radius=1)),
    ("texture", dict(amount=0.6, radius=1)),
    ("texture", dict(amount=-0.8, radius=4)),
    ("texture", dict(amount=1.0, radius=2)),
    ("convolution", dict(kernel=RNG.normal(size=(3, 3)))),
    ("convolution", dict(kernel=RNG.normal(size=(5, 7)) / 8)),
    ("convolution", dict(kernel=RNG.normal(size=(17, 17)) / 40)),
    ("convolution", dict(kernel=np.pad([[1.0]], 1))),
    ("sharpen", dict(amount=1.3, radius=2)),
    ("clarity", dict(amount=0.8, radius=5)),
    ("convolution", dict(kernel=RNG.normal(size=(5, 5)) / 5)),
]


def _images():
    h, w = 67, 83
    y, x = np.mgrid[0:h, 0:w]
    smooth = np.stack([0.1 + 0.8 * x / w, 0.2 + 0.6 * y / h, 0.5 + 0.3 * np.sin(x / 6.0) * np.cos(y / 5.0)], -1)
    noisy = smooth + 0.08 * RNG.normal(size=smooth.shape)
    wide = RNG.normal(0.4, 1.5, size=(h, w, 3))      # signed and above one: Y outside (0, 1) too
    return [noisy.astype(np.float32), wide.astype(np.float32)]


IMAGES = _images()
MESSAGES = {"sharpen": "sharpen requires finite complete RGB halo",
            "clarity": "clarity requires finite complete input halo",
            "texture": "texture requires finite complete input halo",
            "convolution": "convolution requires finite input samples"}
VIEWPORTS = [(0, 0, 83, 67), (20, 11, 37, 29), (0, 0, 9, 7), (83 - 13, 67 - 10, 13, 10), (41, 0, 1, 1)]


def _halo(kind, p):
    if kind == "convolution":
        k = np.asarray(p["kernel"])
        ident = k.size and np.array_equal(k.reshape(-1), np.eye(1, k.size, k.size // 2).reshape(-1))
        return (0, 0) if ident else (k.shape[1] // 2, k.shape[0] // 2)
    if p["amount"] == 0:
        return (0, 0)
    return (2 * p["radius"],) * 2 if kind == "texture" else (p["radius"],) * 2


def _needed(vp, hx, hy, w, h):
    x0, y0 = max(0, vp[0] - hx), max(0, vp[1] - hy)
    x1, y1 = min(w, vp[0] + vp[2] + hx), min(h, vp[1] + vp[3] + hy)
    return (x0, y0, x1 - x0, y1 - y0)


@pytest.mark.parametrize("kind,params", CASES, ids=[f"{k}{i}" for i, (k, _) in enumerate(CASES)])
@pytest.mark.parametrize("space", [0, 1])
def test_stencil_bit_exact_against_reference(reference, kind, params, space):
    from librawops_b200 import render
    for img in IMAGES:
        h, w = img.shape[:2]
        whole = torch.from_numpy(img).cuda()
        hx, hy = _halo(kind, params)
        for vp in VIEWPORTS:
            want = reference.stencil(kind, img, vp, space=space, **params)
            got = render.stencil(kind, whole, (0, 0, w, h), (0, 0, w, h), vp, working_space=space, **params)
            assert bits_equal(got.cpu().numpy(), want), (vp, "whole image window")
            nd = _needed(vp, hx, hy, w, h)
            crop = torch.from_numpy(np.ascontiguousarray(img[nd[1]:nd[1] + nd[3], nd[0]:nd[0] + nd[2]])).cuda()
            got = render.stencil(kind, crop, nd, (0, 0, w, h), vp, working_space=space, **params)
            assert bits_equal(got.cpu().numpy(), want), (vp, "needed window")


@pytest.mark.parametrize("kind,params", [CASES[0], CASES[3], CASES[7], CASES[10], CASES[2], CASES[12]])
def test_stencil_nonfinite_inputs(reference, kind, params):
    from librawops_b200 import render
    from librawops_b200._capi import ReError
    img = IMAGES[0].copy()
    h, w = img.shape[:2]
    vp = (30, 20, 10, 8)
    hx, hy = _halo(kind, params)
    nd = _needed(vp, hx, hy, w, h)
    # inside the needed region (its last corner): the reference's message
    bad = img.copy()
    bad[nd[1] + nd[3] - 1, nd[0] + nd[2] - 1, 1] = np.nan
    with pytest.raises(ReError) as e:
        render.stencil(kind, torch.from_numpy(bad).cuda(), (0, 0, w, h), (0, 0, w, h), vp, **params)
    # (the reference's raster source refuses non-finite pixels itself, so the
    # node's message is quoted from SpatialOps.cpp:358, 418, 523, 654)
    assert e.value.kind == "invalid_argument" and str(e.value) == "invalid_argument: " + MESSAGES[kind]
    # just outside it: no error, same pixels as the clean image
    far = img.copy()
    far[nd[1] + nd[3], nd[0] + nd[2], 0] = np.inf
    got = render.stencil(kind, torch.from_numpy(far).cuda(), (0, 0, w, h), (0, 0, w, h), vp, **params)
    assert bits_equal(got.cpu().numpy(), reference.stencil(kind, img, vp, **params))


def test_stencil_results_beyond_float32(reference):
    from librawops_b200 import render
    from librawops_b200._capi import ReError
    from oracle.oracle import OracleError
    img = np.full((9, 9, 3), 0.5, np.float32)
    img[4, 4] = 3.0e38
    img[4, 5] = -3.0e38
    for kind, p in [("sharpen", dict(amount=2.0, radius=1)),
                    ("convolution", dict(kernel=np.array([[0, 0, 0], [0, 2.0, 0], [0, 0, 0]])))]:
        with pytest.raises(OracleError) as want:
            reference.stencil(kind, img, (0, 0, 9, 9), **p)
        with pytest.raises(ReError) as got:
            render.stencil(kind, torch.from_numpy(img).cuda(), (0, 0, 9, 9), (0, 0, 9, 9), (0, 0, 9, 9), **p)
        assert got.value.kind == want.value.kind == "invalid_argument"
        assert str(got.value) == str(want.value), (str(got.value), str(want.value))


@pytest.mark.parametrize("kind,params", [("sharpen", dict(amount=1.0, radius=2)), ("clarity", dict(amount=0.7, radius=8)),
                                         ("texture", dict(amount=0.9, radius=4)),
                                         ("convolution", dict(kernel=np.random.default_rng(9).normal(size=(5, 5)) / 5))])
def test_stencil_600x400_against_reference(reference, kind, params):
    """A frame large enough that most threads of the register-blocked tiles
    (16 x 64 for sharpen, clarity and square convolutions, 32 x 32 for
    texture) take the unclipped path, and partial tiles sit on both edges."""
    from librawops_b200 import render
    rng = np.random.default_rng(21)
    h, w = 400, 600
    y, x = np.mgrid[0:h, 0:w]
    img = np.stack([0.5 + 0.4 * np.sin(x / 17.0), 0.5 + 0.4 * np.cos(y / 11.0), 0.3 + 0.2 * np.sin((x + y) / 7.0)], -1)
    img = (img + 0.05 * rng.normal(size=img.shape)).astype(np.float32)
    vp = (5, 3, w - 11, h - 7)
    want = reference.stencil(kind, img, vp, **params)
    got = render.stencil(kind, torch.from_numpy(img).cuda(), (0, 0, w, h), (0, 0, w, h), vp, **params)
    assert bits_equal(got.cpu().numpy(), want)
