import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)
GOLDEN = os.path.join(TESTS, "golden")

# Float tolerance of the render path: 1e-5 max-abs of full scale and at most
# one 16-bit code after encoding.
ABS_TOL = 1e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and runs the CUDA path")


def _ensure_built():
    from librawops_b200 import build
    if build.stale():
        build.build()
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       stdout=subprocess.DEVNULL)


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("reference library (oracle/_ref) not built")
    return Reference()


@pytest.fixture(scope="session")
def menon_fixtures():
    z = np.load(os.path.join(GOLDEN, "menon_native_base_v1.npz"))
    out = []
    so, eo = z["sample_offsets"], z["expected_offsets"]
    for i, (m, lv) in enumerate(zip(z["meta"], z["levels"])):
        out.append((tuple(int(v) for v in m), tuple(int(v) for v in lv),
                    z["samples"][so[i]:so[i + 1]], z["expected"][eo[i]:eo[i + 1]]))
    return out


@pytest.fixture(scope="session")
def goldens():
    return np.load(os.path.join(GOLDEN, "reference_renders.npz"))


def within_tolerance(got, want, abs_tol=ABS_TOL, lsb16=True):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    assert got.shape == want.shape
    diff = np.abs(got - want)
    worst = float(diff.max()) if diff.size else 0.0
    assert worst <= abs_tol, f"max abs diff {worst:.3g} > {abs_tol}"
    if lsb16:
        codes = np.abs(np.rint(np.clip(got, 0, 1) * 65535) - np.rint(np.clip(want, 0, 1) * 65535))
        assert codes.max(initial=0) <= 1, f"16-bit code diff {codes.max()} > 1"
    return worst


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))
