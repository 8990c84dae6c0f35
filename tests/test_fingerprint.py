"""Source fingerprints (csrc/fingerprint.cpp, SourceFingerprint.cpp:65-101).

re_fingerprint_raw / re_fingerprint_raster are host code: on the CPU they are
checked against (a) the reference's byte stream restated here and hashed with
Python's hashlib, and (b) the unmodified reference library's own
fingerprint_raw_source / fingerprint_raster_source on the same sources --
padded strides, inset and defaulted active areas, every pattern and phase,
and signed zeros in rasters.  The overlapped upload
(re_image_create_fingerprinted) needs a GPU: its digest equals the host one
and its image renders exactly like re_image_create's.
"""
import ctypes as C
import hashlib
import struct

import numpy as np
import pytest

from librawops_b200 import _capi, render
from oracle.oracle import RawSpec


def _raw_cases():
    rng = np.random.default_rng(3)
    cases = []
    for i, (w, h, stride, active) in enumerate([(16, 12, 0, (0, 0, 0, 0)), (37, 21, 40, (3, 2, 30, 17)),
                                                  (64, 48, 64, (0, 0, 64, 48)), (9, 7, 13, (1, 1, 7, 5)),
                                                  (300, 211, 320, (8, 3, 280, 200))]):
        st = stride or w
        samples = rng.integers(0, 65536, st * h, dtype=np.uint16)
        black = tuple(int(v) for v in rng.integers(0, 600, 4))
        white = tuple(int(v) for v in rng.integers(15000, 65536, 4))
        cases.append(RawSpec(w, h, samples, stride, i % 4, i % 2, (i // 2) % 2, active, black, white))
    return cases


def _restated_raw(spec: RawSpec) -> bytes:
    """The byte stream of SourceFingerprint.cpp:65-84, hashed with hashlib."""
    w, h = spec.width, spec.height
    stride = spec.row_stride or w
    ax, ay, aw, ah = spec.active if any(spec.active) else (0, 0, w, h)
    m = hashlib.sha256()
    m.update(b"librawops.source.raw.u16.v1\0")
    m.update(struct.pack("<IIBBBIIII", w, h, spec.pattern, spec.phase_x, spec.phase_y, ax, ay, aw, ah))
    m.update(struct.pack("<4H4H", *spec.black, *spec.white))
    plane = np.asarray(spec.samples, np.uint16).reshape(h, stride)
    m.update(np.ascontiguousarray(plane[ay:ay + ah, ax:ax + aw]).astype("<u2").tobytes())
    return m.digest()


def _meta(spec: RawSpec):
    return _capi.RawMetadata(spec.width, spec.height, spec.row_stride, spec.pattern, spec.phase_x, spec.phase_y,
                             _capi.Rect(*spec.active), (C.c_uint16 * 4)(*spec.black), (C.c_uint16 * 4)(*spec.white))


def _ours_raw(spec: RawSpec) -> bytes:
    meta = _meta(spec)
    s = np.ascontiguousarray(spec.samples, np.uint16)
    d = (C.c_uint8 * 32)()
    _capi.check(_capi.lib().re_fingerprint_raw(C.byref(meta), s.ctypes.data, s.size, d))
    return bytes(d)


def test_raw_fingerprint_matches_restatement_and_reference(reference):
    for spec in _raw_cases():
        ours = _ours_raw(spec)
        assert ours == _restated_raw(spec)
        assert ours == reference.fingerprint_raw(spec)


def test_raw_fingerprint_changes_with_any_hashed_field():
    spec = _raw_cases()[1]
    base = _ours_raw(spec)
    s2 = np.array(spec.samples, copy=True)
    s2[spec.active[1] * 40 + spec.active[0]] ^= 1           # first active sample
    assert _ours_raw(RawSpec(**{**spec.__dict__, "samples": s2})) != base
    s3 = np.array(spec.samples, copy=True)
    s3[0] ^= 1                                               # outside the active area: not hashed
    assert _ours_raw(RawSpec(**{**spec.__dict__, "samples": s3})) == base
    assert _ours_raw(RawSpec(**{**spec.__dict__, "pattern": (spec.pattern + 1) % 4})) != base


def test_raster_fingerprint_matches_restatement_and_reference(reference):
    rng = np.random.default_rng(8)
    for w, h, space in [(5, 3, 0), (64, 33, 1), (1, 1, 0)]:
        px = rng.normal(0.4, 1.0, (h, w, 3)).astype(np.float32)
        px.reshape(-1)[0] = -0.0
        d = (C.c_uint8 * 32)()
        _capi.check(_capi.lib().re_fingerprint_raster(w, h, 0, space, px.ctypes.data, d))
        m = hashlib.sha256()
        m.update(b"librawops.source.raster.f32.v1\0")
        m.update(struct.pack("<IIB", w, h, space))
        m.update(px.astype("<f4").tobytes())
        assert bytes(d) == m.digest()
        assert bytes(d) == reference.fingerprint_raster(px, space)


@pytest.mark.gpu
def test_fingerprinted_upload_equals_plain_upload():
    from librawops_b200 import workloads
    w = workloads.menon_24mp()
    samples = w.samples()
    spec = RawSpec(w.width, w.height, samples.reshape(-1), w.stride, w.pattern, *w.phase, w.active, w.black,
                   (w.white,) * 4)
    meta = render.Metadata(w.width, w.height, w.stride, w.pattern, *w.phase, w.active, w.black, (w.white,) * 4)
    img, digest = render.Image.ingest(meta, samples)
    assert digest == _ours_raw(spec) == _restated_raw(spec)
    pipe = workloads.pipeline_for(w)
    vp = (w.active[0] + 1000, w.active[1] + 700, 1500, 900)
    got = render.render(img, pipe, vp)
    want = render.render(render.Image(meta, samples), pipe, vp)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
