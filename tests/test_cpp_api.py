"""The drop-in C++ surface (include/rawengine/*.hpp) against the oracle.

tests/cpp/api_driver.cpp is compiled against the in-tree library the way a
user of the reference's C++ headers would build: `#include <rawengine/...>`,
link -lrawengine_b200.  Host-only behaviour (constructor validation, regions,
descriptors, scheduler argument checks) runs here without a GPU; the render
scenarios (ImageGraph, Renderer, point/spatial/geometry nodes, foreign nodes,
cancellation, TileScheduler order and supersession) run on the GPU and are
compared with the oracle on the same inputs.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, bits_equal, within_tolerance
from oracle import oracle as O
from oracle.oracle import Op, RawSpec

LIB_DIR = os.path.join(ROOT, "librawops_b200", "_lib")
DRIVER_SRC = os.path.join(ROOT, "tests", "cpp", "api_driver.cpp")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "api_driver")
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           DRIVER_SRC, "-L", LIB_DIR, "-lrawengine_b200", f"-Wl,-rpath,{LIB_DIR}", "-pthread", "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def _run(args, timeout=300):
    p = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    lines = p.stdout.splitlines()
    fails = [ln for ln in lines if ln.startswith("FAIL")]
    assert p.returncode == 0 and not fails, p.stdout[-4000:] + p.stderr[-2000:]
    return lines


# ---------------------------------------------------------------- host only

def test_cpp_validation_and_regions(driver, oracle):
    lines = _run([driver, "validate"])
    checks = [ln for ln in lines if ln.startswith("CHECK")]
    assert len(checks) >= 40
    regions = {ln.split()[1]: tuple(int(v) for v in ln.split()[2:]) for ln in lines if ln.startswith("REGION")}
    area = (4, 2, 32, 26)
    raw = RawSpec(40, 30, np.full(1200, 1000, np.uint16), active=area)
    assert regions["bilinear_input"] == oracle.raw_input_region(raw, False, (4, 2, 5, 5))
    assert regions["menon_input"] == oracle.raw_input_region(raw, True, (10, 9, 7, 6))
    assert regions["menon_input_edge"] == oracle.raw_input_region(raw, True, (33, 25, 3, 3))
    assert regions["ctw_mip1"] == oracle.mip_native_region(area, 1, (3, 2, 6, 5))
    assert regions["ctw_mip2_edge"] == oracle.mip_native_region(area, 2, (6, 4, 2, 3))
    assert regions["gf_region"] == oracle.guided_filter_region((10, 8, 6, 5), area, 3)
    assert regions["gf_region_edge"] == oracle.guided_filter_region((4, 2, 3, 3), area, 2)
    assert regions["gf_node_mip1"] == oracle.guided_filter_region((2, 3, 4, 4), (0, 0, 16, 13), 2)
    ls = oracle.guided_filter_region((10, 8, 6, 5), area, 2)  # 2*2 == the statistics radius 4
    assert regions["ls_region"] == ls

    def offset(r):
        return (r[0] + area[0], r[1] + area[1], r[2], r[3])

    assert regions["cubic_support"] == offset(oracle.cubic_support(32, 26, 20, 17, (3, 4, 6, 5)))
    native = oracle.mip_native_region((0, 0, 20, 17), 1, (1, 2, 4, 3))
    assert regions["cubic_support_mip1"] == offset(oracle.cubic_support(32, 26, 20, 17, native))
    rot = oracle.rotation(23.5, 32, 26)
    assert regions["rotate_support"] == offset(oracle.rotate_support(rot, (5, 6, 7, 4)))
    native = oracle.mip_native_region((0, 0, 32, 26), 2, (1, 1, 3, 2))
    assert regions["rotate_support_mip2"] == offset(oracle.rotate_support(rot, native))


# ---------------------------------------------------------------- on the GPU

CAMERA = [0.62, 0.27, 0.07, 0.26, 0.78, -0.04, 0.03, -0.11, 0.91]
LEGACY = [1.8, 1.0, 1.3, 0.25, 0.3, 1.1]   # gains, stops, shoulder, gamma
SRGB = [2.0, 1.0, 1.5, 0.5, 0.25, 2.2]
CURVE = [(0.0, 0.0), (0.25, 0.35), (0.6, 0.7), (1.0, 1.0)]
PARAMS = {
    "raw_meta": [150, 110, 152, 2, 1, 0, 6, 4, 136, 98, 512, 520, 508, 515, 16000, 16383, 16200, 16100],
    "camera": CAMERA,
    "legacy": LEGACY,
    "srgb": SRGB,
    "srgb_native_vp": [10, 9, 50, 40],
    "gf": [3, 2.0 ** -10],
    "curve_master": [v for p in CURVE for v in p],
    "gf_vp": [20, 15, 60, 50],
    "ls_vp": [8, 6, 70, 55],
    "ls_radius": [3],
    "cubic": [90, 70],
    "cubic_vp": [5, 7, 60, 50],
    "cubic_vp_mip1": [3, 2, 30, 25],
    "rotate_angle": [12.5],
    "rotate_vp": [10, 8, 80, 60],
    "rotate_vp_mip2": [2, 3, 25, 18],
    "raster_meta": [45, 37, 0],
    "raster_recipe": [0.5, 2.2],
    "stencil_vp": [12, 10, 70, 60],
    "sharpen": [1.3, 2],
    "clarity": [0.6, 5],
    "texture": [-0.7, 3],
    "convolution": [5, 3] + [round(0.05 * (i % 7) - 0.1, 3) for i in range(15)],
}


def _inputs(tmp):
    rng = np.random.default_rng(7)
    m = PARAMS["raw_meta"]
    h, stride = m[1], m[2]
    yy, xx = np.mgrid[0:h, 0:stride]
    smooth = 4000 + 3000 * np.sin(xx / 9.0) * np.cos(yy / 7.0) + 20 * xx
    raw = np.clip(smooth + rng.normal(0, 300, smooth.shape), 0, 17000).astype(np.uint16)
    raw[20, 40] = 65535                       # above white
    raw[30, 50] = 0                           # below black
    raster = rng.uniform(0, 1.2, (37, 45, 3)).astype(np.float32)
    raw.tofile(os.path.join(tmp, "raw.u16"))
    raster.tofile(os.path.join(tmp, "raster.f32"))
    with open(os.path.join(tmp, "params.txt"), "w") as f:
        for k, v in PARAMS.items():
            f.write(k + " " + " ".join(repr(float(x)) for x in v) + "\n")
    spec = RawSpec(m[0], m[1], raw.reshape(-1), row_stride=stride, pattern=m[3], phase_x=m[4], phase_y=m[5],
                   active=tuple(m[6:10]), black=tuple(m[10:14]), white=tuple(m[14:18]))
    return spec, raster


def _outputs(tmp, lines):
    out = {}
    for ln in lines:
        if not ln.startswith("OUT"):
            continue
        _, name, x, y, w, h, t = ln.split()
        dt = {"f32": np.float32, "f64": np.float64, "u32": np.uint32}[t]
        a = np.fromfile(os.path.join(tmp, name + ".bin"), dt).reshape(int(h), int(w), 3)
        out[name] = ((int(x), int(y), int(w), int(h)), a)
    return out


@pytest.mark.gpu
def test_cpp_renders_match_oracle(driver, oracle, reference, tmp_path):
    spec, raster = _inputs(str(tmp_path))
    lines = _run([driver, "render", str(tmp_path)])
    assert sum(ln.startswith("CHECK") for ln in lines) >= 30
    got = _outputs(str(tmp_path), lines)
    area = tuple(PARAMS["raw_meta"][6:10])
    g = LEGACY
    legacy_ops = [Op(O.OP_WB, g[:3]), Op(O.OP_EXPOSURE, [g[3]]), Op(O.OP_TONE, g[4:6]), Op(O.OP_OUTPUT_CLIP)]
    rect, a = got["legacy"]
    assert rect == area
    within_tolerance(a, oracle.render_raw(spec, False, legacy_ops, area))

    s = SRGB
    srgb_ops = [Op(O.OP_WB, s[:3]), Op(O.OP_EXPOSURE, [s[3]]), Op(O.OP_CAMERA_TO_WORKING, CAMERA + [0]),
                Op(O.OP_WORKING_TO_SRGB), Op(O.OP_TONE, s[4:6]), Op(O.OP_SRGB_ENCODE)]
    rect, a = got["srgb_mip1"]
    within_tolerance(a, oracle.render_raw(spec, True, srgb_ops, rect, mip=1, quality=0))
    rect, a = got["srgb_native"]
    assert rect == tuple(PARAMS["srgb_native_vp"])
    within_tolerance(a, oracle.render_raw(spec, True, srgb_ops, rect))

    # guided filter (+ curves) over Menon -> WB -> camera-to-ProPhoto
    working = [Op(O.OP_WB, s[:3]), Op(O.OP_CAMERA_TO_WORKING, CAMERA + [0])]
    radius, eps = PARAMS["gf"]
    vp = tuple(PARAMS["gf_vp"])
    needed = oracle.guided_filter_region(vp, area, int(radius))
    tile = oracle.render_raw(spec, True, working, needed)
    gf = oracle.guided_filter(tile, needed, vp, area, int(radius), eps, prophoto=True)
    within_tolerance(got["gf_only"][1], gf, lsb16=False)
    curved = gf.copy()
    oracle.curves_apply(oracle.curves(O.curves_params(1, CURVE)), curved)
    within_tolerance(got["gf_curves"][1], curved, lsb16=False)

    # local statistics, tile by tile through analyze_local_rgb
    lvp = tuple(PARAMS["ls_vp"])
    r = int(PARAMS["ls_radius"][0])
    left, top = max(area[0], lvp[0] - r), max(area[1], lvp[1] - r)
    right = min(area[0] + area[2], lvp[0] + lvp[2] + r)
    bottom = min(area[1] + area[3], lvp[1] + lvp[3] + r)
    lneed = (left, top, right - left, bottom - top)
    ltile = oracle.render_raw(spec, True, working, lneed)
    mean, var, cnt = oracle.local_statistics(ltile, lneed, lvp, area, r)
    assert np.array_equal(got["ls_count"][1], cnt)
    np.testing.assert_allclose(got["ls_mean"][1], mean, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(got["ls_var"][1], var, rtol=1e-6, atol=1e-12)

    # Rec.2020 working image -> cubic resize / rotate
    rec_ops = [Op(O.OP_WB, s[:3]), Op(O.OP_CAMERA_TO_WORKING, CAMERA + [1])]
    src = oracle.render_raw(spec, False, rec_ops, area)
    assert bits_equal(got["rec2020_native"][1], src)
    cw, ch = PARAMS["cubic"]
    rect, a = got["cubic"]
    within_tolerance(a, oracle.cubic_resize(src, int(cw), int(ch), rect), lsb16=False)
    rect, a = got["cubic_mip1"]
    native = oracle.mip_native_region((0, 0, int(cw), int(ch)), 1, rect)
    want = oracle.mip_reduce(oracle.cubic_resize(src, int(cw), int(ch), native), native, 1, rect)
    within_tolerance(a, want, lsb16=False)
    rot = oracle.rotation(PARAMS["rotate_angle"][0], area[2], area[3])
    rect, a = got["rotate"]
    within_tolerance(a, oracle.rotate(rot, src, rect), lsb16=False)
    rect, a = got["rotate_mip2"]
    native = oracle.mip_native_region((0, 0, area[2], area[3]), 2, rect)
    want = oracle.mip_reduce(oracle.rotate(rot, src, native), native, 2, rect)
    within_tolerance(a, want, lsb16=False)

    # stencils over Menon -> WB -> exposure -> camera-to-ProPhoto, against the
    # reference library's nodes over its own render of the same chain
    base = [Op(O.OP_WB, s[:3]), Op(O.OP_EXPOSURE, [s[3]]), Op(O.OP_CAMERA_TO_WORKING, CAMERA + [0])]
    codes = {"sharpen": O.OP_SHARPEN, "clarity": O.OP_CLARITY, "texture": O.OP_TEXTURE,
             "convolution": O.OP_CONVOLUTION}
    for name, code in codes.items():
        ops = base + [Op(code, PARAMS[name])]
        rect, a = got["stencil_" + name]
        assert rect == tuple(PARAMS["stencil_vp"])
        assert bits_equal(a, reference.render_raw(spec, True, ops, rect)), name
        rect, a = got["stencil_" + name + "_mip1"]
        assert bits_equal(a, reference.render_raw(spec, True, ops, rect, mip=1, quality=0)), name

    # raster graph, sRGB preview
    stops, gamma = PARAMS["raster_recipe"]
    rops = [Op(O.OP_EXPOSURE, [stops]), Op(O.OP_WORKING_TO_SRGB), Op(O.OP_TONE, [0.25, gamma]), Op(O.OP_SRGB_ENCODE)]
    rect, a = got["raster_mip2"]
    red = oracle.mip_reduce(raster, (0, 0, 45, 37), 2, rect)
    oracle._apply_points(red, rops)
    within_tolerance(a, red)
    rect, a = got["raster_native"]
    nat = raster.copy()
    oracle._apply_points(nat, rops)
    within_tolerance(a, nat)


# ------------------------------------------------- scheduler over the batch

SCHED_SRC = os.path.join(ROOT, "tests", "cpp", "scheduler_driver.cpp")


@pytest.mark.gpu
def test_scheduler_mixed_batch_equals_direct_renders(tmp_path):
    """TileScheduler drains a mixed batch (RAWs of several sizes, Bayer
    patterns and phases, bilinear and Menon, mip 0/1/2, tiles 128..1024 with
    edge remainders, cubic resizes and rotations between the camera-to-working
    stage and the rest of the recipe) into batched device renders: every host
    and device tile
    equals Renderer::render_image of the same request bit for bit, and the
    waves really went through the batch."""
    import json
    from librawops_b200 import workloads
    exe = str(tmp_path / "scheduler_driver")
    subprocess.run(["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    SCHED_SRC, "-L", LIB_DIR, "-lrawengine_b200", f"-Wl,-rpath,{LIB_DIR}", "-pthread", "-o", exe],
                   check=True)
    images, recipes, tiles = workloads.mixed_batch(seed=11, target_tiles=400)
    spec = str(tmp_path / "spec.txt")
    workloads.write_scheduler_spec(spec, images, recipes, tiles)
    p = subprocess.run([exe, spec, "2"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    out = json.loads(p.stdout.strip().splitlines()[-1])
    assert out["mismatches"] == 0 and out["requests"] == len(tiles), json.dumps(out)
    assert out["batched_requests"] == 2 * len(tiles) and out["node_requests"] == 0, json.dumps(out)
