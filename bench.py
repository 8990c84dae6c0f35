"""Benchmark of the B200 render path (one JSON line on rank 0).

Workload: the 24 MP Menon -> sRGB render (6016x4016 BGGR sensor, stride 6080,
active 6000x4000 at (16,8), per-site black (510,512,511,513), white 15800;
Menon demosaic, WB (1.9,1.0,1.5), 3x3 calibration, 16-knot monotone tone
curve, working->sRGB, clip + sRGB encode; float32 RGB out).  One step renders
the frame as the reference's renderer cuts it -- 96 tile requests of 512 with
edge remainders -- drained by one persistent batched launch.  The same
requests launched one by one (per tile), the whole frame as one launch, and the
mixed batch (16 RAWs, ~3,000 tiles at mip 0/1/2, batched vs per request) are
reported beside it.  Inputs (48.8 MB) and outputs (288 MB) exceed the 126 MB
L2, so no explicit flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torch.distributed.run, one rank per GPU, each rank rendering
its own frame (replicas: the frames are independent, there is no collective on
the data path); value = all ranks' pixels / the max-over-ranks device time.
`--impl reference` times the reference's own CPU implementation (the reference
library built from its sources in oracle/_ref, else the C oracle port) on the
host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpix/s 24MP Menon render, batched vs per-tile, at 1e-5 err; HBM % of peak"
ALGO_BYTES_PER_PX = 14          # 2 B Bayer in + 12 B float32 RGB out per output pixel


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_from_profile():
    """DRAM bytes per launch of the render kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "menon_kernel_24mp_srgb.md")
    try:
        with open(path) as f:
            m = re.search(r"DRAM traffic of one launch \(read \+ write\): (\d+) bytes", f.read())
        return int(m.group(1)) if m else None
    except OSError:
        return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        """Starts sampling and waits for the first sample, so that the tool's
        start-up never overlaps the timed region."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def mark(self):
        self.first = len(self.lines)

    def stop(self):
        self.last = len(self.lines)
        self.__exit__()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, window="timed region"):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sampled = self.lines[getattr(self, "first", 0):getattr(self, "last", len(self.lines)) + 1]
        for line in sampled:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0, "window": window}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "window": window}


class CpuReference:
    """The reference's own CPU implementation of the workload: the reference
    library built from its sources (oracle/_ref), driven through its own
    TileScheduler with one worker per host core.  The RawImage, the node chain
    and the scheduler are built once, outside the timing; a timed render
    submits the frame's render tiles (tile 512: 96 requests for the
    6000x4000 frame), waits for them and assembles the frame -- the work a
    reference caller repeats per frame.  When that library is absent, the C
    oracle port renders the frame on one thread."""

    def __init__(self, workload):
        from oracle.oracle import (OP_CAMERA_TO_WORKING, OP_CURVES_EXT, OP_DISPLAY_TAG, OP_SRGB_ENCODE,
                                   OP_WB, OP_WORKING_TO_SRGB, Op, Oracle, RawSpec, Reference, curves_params,
                                   reference_available)
        w = self.w = workload
        samples = w.samples().reshape(-1)
        self.raw = RawSpec(w.width, w.height, samples, w.stride, w.pattern, *w.phase, w.active, w.black,
                           (w.white,) * 4)
        self.ops = [Op(OP_WB, list(w.wb)), Op(OP_CAMERA_TO_WORKING, list(w.camera_to_xyz.reshape(9)) + [0]),
                    Op(OP_CURVES_EXT, curves_params(1, w.curve)), Op(OP_WORKING_TO_SRGB), Op(OP_DISPLAY_TAG),
                    Op(OP_SRGB_ENCODE)]
        self.cores = os.cpu_count() or 1
        self.out = np.zeros((w.active[3], w.active[2], 3), np.float32)
        if reference_available():
            self.kind, self.threads = "reference", min(self.cores, 64)
            self.session = Reference().session(self.raw, True, self.ops, self.threads)
        else:
            self.kind, self.threads = "port", 1
            self.oracle = Oracle()
            self.ops = [o for o in self.ops if o.code != OP_DISPLAY_TAG]

    def frame_seconds(self):
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.session.render(self.w.active, tile=self.w.tile, out=self.out)
        else:
            self.out = self.oracle.render_raw(self.raw, True, self.ops, self.w.active)
        return time.perf_counter() - t0

    def rate(self, repeats):
        self.frame_seconds()
        times = [self.frame_seconds() for _ in range(repeats)]
        return self.w.pixels / statistics.median(times) / 1e6

    def sample_text(self, repeats, stat="median"):
        ax, ay, aw, ah = self.w.active
        how = (f"its TileScheduler, {self.threads} workers, tile {self.w.tile}" if self.kind == "reference"
               else "the C port, one thread")
        return f"the whole {aw}x{ah} frame through {how}; setup outside the timing; {stat} of {repeats} frames"


def run_reference(args, rank):
    from librawops_b200 import workloads
    if rank != 0:
        return
    ref = CpuReference(workloads.menon_24mp())
    # one step renders the whole frame, as the GPU arm's step does
    for _ in range(args.warmup):
        ref.frame_seconds()
    t = [ref.frame_seconds() for _ in range(args.steps)]
    value = ref.w.pixels * len(t) / sum(t) / 1e6
    line = {"metric": METRIC, "value": round(value, 3), "unit": "Mpix/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(t) / len(t), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": ref.w.name, "tile": ref.w.tile,
                       "frame": f"{ref.w.active[2]}x{ref.w.active[3]} active of {ref.w.width}x{ref.w.height} "
                                f"BGGR stride {ref.w.stride}"},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mpix/s", "cores": ref.threads, "kind": ref.kind,
                             "sample": ref.sample_text(args.steps, "mean")},
            "e2e": {"value": round(value, 3), "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from librawops_b200 import render, workloads

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = workloads.menon_24mp(seed=2 + rank)
    samples_host = w.samples()
    meta = render.Metadata(w.width, w.height, w.stride, w.pattern, *w.phase, w.active, w.black, (w.white,) * 4)
    ax, ay, aw, ah = w.active
    pixels = aw * ah
    samples_dev = torch.from_numpy(samples_host.reshape(-1).view(np.int16)).to(dev)
    img = render.Image(meta, samples_dev)
    pipe = workloads.pipeline_for(w)
    out = torch.empty((ah, aw, 3), dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    # the frame as the reference renders it: tile-size requests in row-major
    # order (RawEngine.cpp:1390-1412), each writing its part of the frame
    tiles = render.plan_tiles(w.active, w.tile)
    requests = [(img, pipe, t, 0, render.FINAL, out[t[1] - ay:t[1] - ay + t[3], t[0] - ax:t[0] - ax + t[2]])
                for t in tiles]
    batch = render.Batch().plan(requests)
    with torch.cuda.stream(stream):
        tuned = batch.autotune(reps=3, stream=stream)

    def step():
        batch.launch(stream=stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    batch.status(stream=stream)

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local_rank).start()
    # The timed region is short (K steps of well under a millisecond), shorter
    # than the sampler's interval.  Untimed steps run for half a second right
    # before it, inside the sampled window, so the clock record covers the GPU
    # under this load: the reported window is that soak plus the timed steps.
    clocks.mark()
    soak_end = time.time() + 0.5
    with torch.cuda.stream(stream):
        while time.time() < soak_end:
            for _ in range(20):
                step()
            torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_begin = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_begin.record(stream)
    for i in range(args.steps):
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    clocks.stop()
    if world > 1:
        dist.barrier()
    total_ms = t_begin.elapsed_time(t_end)
    launch_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    batch.status(stream=stream)

    # the same tile requests launched one by one, and the whole frame as one launch
    def timed(fn, reps):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    reps = max(3, min(args.steps, 50))
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    per_tile_ms = timed(lambda: batch.launch_per_request(stream=stream), reps)
    batch.status(stream=stream)
    whole_ms = timed(lambda: render.render_async(img, pipe, w.active, out, status, stream=stream), reps)
    render.status_from_device(int(status.item()))

    # end-to-end through the public API: each step uploads its Bayer frame from
    # pinned host memory, renders it and reads the RGB back into pinned host
    # memory.  Two slots (stream, device input and output, host output)
    # alternate, so one frame's read-back overlaps the next frame's upload and
    # render -- as a caller rendering a frame sequence would run it.
    pinned_in = torch.from_numpy(samples_host.reshape(-1).view(np.int16)).pin_memory()
    slots = []
    for k in range(2):
        s_dev = samples_dev if k == 0 else torch.empty_like(samples_dev)
        s_img = img if k == 0 else render.Image(meta, s_dev)
        s_out = out if k == 0 else torch.empty_like(out)
        s_stream = stream if k == 0 else torch.cuda.Stream(device=dev)
        s_batch = batch if k == 0 else render.Batch().plan(
            [(s_img, pipe, t, 0, render.FINAL, s_out[t[1] - ay:t[1] - ay + t[3], t[0] - ax:t[0] - ax + t[2]])
             for t in tiles])
        slots.append(dict(dev=s_dev, img=s_img, out=s_out, stream=s_stream, batch=s_batch,
                          host=torch.empty((ah, aw, 3), dtype=torch.float32).pin_memory()))

    def e2e_step(i):
        sl = slots[i % 2]
        with torch.cuda.stream(sl["stream"]):
            sl["dev"].copy_(pinned_in, non_blocking=True)
            sl["batch"].launch(stream=sl["stream"])
            sl["host"].copy_(sl["out"], non_blocking=True)

    e2e_steps = max(4, min(args.steps, 20))
    for i in range(4):
        e2e_step(i)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    e0.record(slots[0]["stream"])
    slots[1]["stream"].wait_event(e0)
    for i in range(e2e_steps):
        e2e_step(i)
    slots[0]["stream"].wait_stream(slots[1]["stream"])
    e1.record(slots[0]["stream"])
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    for sl in slots:
        sl["batch"].status(stream=sl["stream"])

    stats = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(stats, op=dist.ReduceOp.MAX)
    total_ms, e2e_ms = float(stats[0]), float(stats[1])
    if rank != 0:
        return
    # the other workloads and legs: rank 0 only, after the last collective
    mixed = _mixed_batch(render, workloads, torch, dev, stream, reps=max(3, min(args.steps, 20)))
    peak, peak_kind = _peaks()
    configs = _config_legs(render, workloads, torch, dev, stream, peak, reps=max(3, min(args.steps, 10)))
    try:
        scheduler = _scheduler_leg(workloads)
    except Exception as e:   # no host compiler
        scheduler = {"error": str(e)[-300:]}
    differentiable = _differentiable(torch, dev, reps=3)
    directions = _menon_direction_counts(render, img, w)
    ms_per_step = total_ms / args.steps
    value = world * pixels / (ms_per_step * 1e-3) / 1e6
    kernel_ms = statistics.mean(launch_ms)
    achieved = ALGO_BYTES_PER_PX * pixels / (kernel_ms * 1e-3) / 1e9
    peak, peak_kind = _peaks()
    traffic = _traffic_from_profile()
    try:
        ref = CpuReference(w)
        cpu = {"value": round(ref.rate(3), 3), "unit": "Mpix/s", "cores": ref.threads, "kind": ref.kind,
               "sample": ref.sample_text(3)}
    except Exception as e:  # the checker libraries are missing
        cpu = {"value": None, "unit": "Mpix/s", "cores": 0, "kind": "port", "sample": f"unavailable: {e}"}
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w.name, "frame": f"{aw}x{ah} active of {w.width}x{w.height} BGGR stride {w.stride}",
                   "tile": w.tile,
                   "per_launch": f"{len(tiles)} tile requests of {w.tile} (edge remainders) as one batch "
                                 "(CUDA graph): adjacent requests merge into one render, the autotuner picks "
                                 "the tile-queue kernel or a plain launch per merged render",
                   "batch_options": tuned,
                   "l2": "inputs+outputs 337 MB > 126 MB L2 (no flush needed)",
                   "parallelism": f"replicas x{world}"},
        "batched_vs_per_tile": {
            "batched_mpix_s": round(pixels / (ms_per_step * 1e-3) / 1e6, 2),
            "per_tile_mpix_s": round(pixels / (per_tile_ms * 1e-3) / 1e6, 2),
            "speedup": round(per_tile_ms / ms_per_step, 3),
            "single_launch_whole_frame_mpix_s": round(pixels / (whole_ms * 1e-3) / 1e6, 2),
            "mixed_batch": mixed,
            "mixed_batch_through_tile_scheduler": scheduler},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6.65 TB/s", "algorithmic_bytes_per_px": ALGO_BYTES_PER_PX,
                     "kernel": "menon_kernel" if tuned["dispatch"] == 3 else "batch_render_kernel",
                     "kernel_ms": round(kernel_ms, 5)},
        "configs": configs,
        "menon_directions": directions,
        "differentiable": differentiable,
        "cpu_baseline": cpu,
        "e2e": {"value": round(world * pixels / (e2e_ms * 1e-3) / 1e6, 2), "unit": "Mpix/s",
                "h2d_bytes_per_step": int(samples_host.nbytes), "d2h_bytes_per_step": int(pixels * 12)},
        "gpu_launches": args.steps,
        "clocks": clocks.summary("0.5 s of untimed steps immediately before the timed steps, and the timed "
                                 "steps"),
    }
    print(json.dumps(line), flush=True)


def _scheduler_leg(workloads):
    """The mixed batch submitted through the drop-in C++ TileScheduler
    (tests/cpp/scheduler_driver.cpp, compiled against include/ and the
    library): wall time of all requests through Renderer::render_image one at
    a time vs through the scheduler's batched waves, host and device tiles,
    every tile checked bit-equal to the direct render."""
    import tempfile
    lib_dir = os.path.join(ROOT, "librawops_b200", "_lib")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "scheduler_driver")
        subprocess.run(["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "scheduler_driver.cpp"), "-L", lib_dir,
                        "-lrawengine_b200", f"-Wl,-rpath,{lib_dir}", "-pthread", "-o", exe], check=True)
        images, recipes, tiles = workloads.mixed_batch()
        spec = os.path.join(tmp, "spec.txt")
        workloads.write_scheduler_spec(spec, images, recipes, tiles)
        p = subprocess.run([exe, spec, "2"], capture_output=True, text=True, timeout=900)
        if p.returncode != 0:
            return {"error": (p.stdout + p.stderr)[-500:]}
        r = json.loads(p.stdout.strip().splitlines()[-1])
    r["speedup_host_tiles"] = round(r["per_request_s"] / r["scheduler_host_s"], 3)
    r["speedup_device_tiles"] = round(r["per_request_s"] / r["scheduler_device_s"], 3)
    return r


def _per_launch_ms(torch, stream, fn, reps, flush=None):
    """Mean device time of one call of `fn` (CUDA events on `stream` around
    each call), after three untimed calls; `flush` (untimed, between calls)
    evicts L2 when a call's inputs and outputs fit in it."""
    with torch.cuda.stream(stream):
        for _ in range(3):
            fn()
        times = []
        for _ in range(reps):
            if flush is not None:
                flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            times.append((e0, e1))
    torch.cuda.synchronize()
    return statistics.mean(a.elapsed_time(b) for a, b in times)


def _roofline_leg(ms, pixels, bytes_per_px, peak, **extra):
    achieved = bytes_per_px * pixels / (ms * 1e-3) / 1e9
    leg = {"ms": round(ms, 5), "mpix_s": round(pixels / (ms * 1e-3) / 1e6, 1),
           "algorithmic_bytes_per_px": bytes_per_px, "achieved_gb_s": round(achieved, 1),
           "frac": round(achieved / peak, 4)}
    leg.update(extra)
    return leg


def _config_legs(render, workloads, torch, dev, stream, peak, reps):
    """The other configurations, each kernel timed by CUDA events against the
    HBM roofline: the bilinear render to float32 linear ProPhoto (1024x768,
    and a 6000x4000 instance of the same generator and recipe), the guided
    filter on the 6000x4000 raster at r 8/32 x eps 1e-3/1e-2, and box local
    statistics at r 16."""
    from librawops_b200 import synthetic
    legs = {}
    flush_buf = torch.empty(64 << 20, dtype=torch.float32, device=dev)   # 256 MB > L2

    def flush():
        flush_buf.zero_()

    for w in (workloads.bilinear_1mp(), workloads.bilinear_1mp(width=6000, height=4000, seed=5)):
        meta = render.Metadata(w.width, w.height, w.stride, w.pattern, *w.phase, w.active, w.black,
                               (w.white,) * 4)
        img = render.Image(meta, torch.from_numpy(w.samples().reshape(-1).view(np.int16)).to(dev))
        pipe = workloads.pipeline_for(w)
        out = torch.empty((w.active[3], w.active[2], 3), dtype=torch.float32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        small = w.pixels * 14 < (126 << 20)
        ms = _per_launch_ms(torch, stream, lambda: render.render_async(img, pipe, w.active, out, status,
                                                                     stream=stream),
                            reps, flush if small else None)
        render.status_from_device(int(status.item()))
        legs[f"bilinear_linear_prophoto_{w.width}x{w.height}"] = _roofline_leg(
            ms, w.pixels, 14, peak, kernel="bilinear_kernel",
            l2="L2 flushed between launches" if small else "inputs+outputs > L2")
        img.close()
    rgb = torch.from_numpy(synthetic.raster(6000, 4000, seed=3)).to(dev)
    px = 6000 * 4000
    gf_out = torch.empty_like(rgb)
    for radius in (8, 32):
        for eps in (1e-3, 1e-2):
            ms = _per_launch_ms(torch, stream, lambda: render.guided_filter(rgb, radius, eps, out=gf_out,
                                                                          stream=stream), reps)
            legs[f"guided_filter_6000x4000_r{radius}_eps{eps:g}"] = _roofline_leg(ms, px, 24, peak,
                                                                                 kernel="guided filter")
    ms = _per_launch_ms(torch, stream, lambda: render.local_statistics(rgb, 16, stream=stream), reps)
    legs["local_statistics_6000x4000_r16"] = _roofline_leg(ms, px, 36, peak, kernel="local statistics")
    from librawops_b200 import _capi
    import ctypes
    L = _capi.lib()
    counters = torch.empty(3 * 256 + 15, dtype=torch.int64, device=dev)
    cp = [ctypes.c_void_p(counters.data_ptr() + 8 * o) for o in (0, 3 * 256, 3 * 256 + 9)]
    sp = ctypes.c_void_p(stream.cuda_stream)

    def hist():
        _capi.check(L.re_histogram_reset(256, *cp, sp))
        _capi.check(L.re_histogram_rgb(ctypes.c_void_p(rgb.data_ptr()), rgb.stride(0), 6000, 4000, 512, 0, 256,
                                       0.0, 1.0, *cp, sp))
    ms = _per_launch_ms(torch, stream, hist, reps)
    legs["histogram_rgb_6000x4000_256_bins"] = _roofline_leg(
        ms, px, 12, peak, kernel="histogram_kernel", note="counter reset (memsets) and the histogram kernel")
    image = (0, 0, 6000, 4000)
    for name, kw in _STENCIL_CASES.items():
        ms = _per_launch_ms(torch, stream, lambda: render.stencil(name.split("_")[0], rgb, image, image, image,
                                                                   stream=stream, **kw), reps)
        legs[f"{name}_6000x4000"] = _roofline_leg(ms, px, 24, peak, kernel=f"{name.split('_')[0]}_kernel",
                                                   note="synchronous call (status read-back included)")
    return legs


# Stencil settings timed on the 6000x4000 raster (radius is the scale for texture).
_STENCIL_CASES = {"sharpen_r2": dict(amount=1.0, radius=2), "clarity_r8": dict(amount=0.5, radius=8),
                  "texture_s4": dict(amount=0.5, radius=4),
                  "convolution_5x5": dict(kernel=np.full((5, 5), 1.0 / 25))}


def run_case(args):
    """One workload's kernel launched --warmup + --steps times with nothing
    else on the device: the command the ncu summaries in profiles/ name.
    Cases: menon_24mp_srgb, bilinear_6000x4000, gf_r8, gf_r32, ls_r16,
    histogram_24mp, sharpen_r2, clarity_r8, texture_s4, convolution_5x5,
    mixed_batch (the batched persistent render of the mixed workload),
    differentiable (forward and backward of the 8-frame recipe fit)."""
    import torch
    from librawops_b200 import render, synthetic, workloads
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    name = args.case
    if name in ("menon_24mp_srgb", "bilinear_6000x4000"):
        w = workloads.menon_24mp() if name.startswith("menon") else workloads.bilinear_1mp(6000, 4000, seed=5)
        meta = render.Metadata(w.width, w.height, w.stride, w.pattern, *w.phase, w.active, w.black, (w.white,) * 4)
        img = render.Image(meta, torch.from_numpy(w.samples().reshape(-1).view(np.int16)).to(dev))
        pipe = workloads.pipeline_for(w)
        out = torch.empty((w.active[3], w.active[2], 3), dtype=torch.float32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        fn = lambda: render.render_async(img, pipe, w.active, out, status, stream=stream)
    elif name == "differentiable":
        from librawops_b200 import diff
        knots = workloads.tone_knots_16()
        model = diff.RecipeModel((0, 1, 1, 2), [k[0] for k in knots], [k[1] for k in knots], wb=(2.0, 1.0, 1.6),
                                 stops=0.2, matrix=workloads.CAMERA_TO_PROPHOTO, strength=0.5, radius=16, eps=1e-3,
                                 device=dev)
        planes = []
        for i in range(8):
            codes = synthetic.bayer_device(4000, 3000, seed=40 + i, pattern=0, black=(512,) * 4, white=16383,
                                           device=dev)
            planes.append(((codes.float() - 512.0) / (16383.0 - 512.0)).contiguous())
        with torch.no_grad():
            targets = [model(pl) * 1.01 for pl in planes]

        def fn():
            model.zero_grad(set_to_none=True)
            loss = sum(torch.mean((model(pl) - t) ** 2) for pl, t in zip(planes, targets)) / len(planes)
            loss.backward()
    elif name == "mixed_batch":
        images, recipes, tiles = workloads.mixed_batch()
        imgs = []
        for im in images:
            meta = render.Metadata(im.width, im.height, im.stride, im.pattern, im.phase[0], im.phase[1], im.active,
                                   im.black, (im.white,) * 4)
            imgs.append(render.Image(meta, render.synthetic_samples(im, device=dev)))
        outs = [torch.empty((t.viewport[3], t.viewport[2], 3), device=dev) for t in tiles]
        batch = render.Batch().plan(workloads.mixed_requests(render, imgs, images, recipes, tiles, outs))
        fn = lambda: batch.launch(stream=stream)
    else:
        rgb = torch.from_numpy(synthetic.raster(6000, 4000, seed=3)).to(dev)
        out = torch.empty_like(rgb)
        image = (0, 0, 6000, 4000)
        if name in ("gf_r8", "gf_r32"):
            fn = lambda: render.guided_filter(rgb, int(name[4:]), 1e-3, out=out, stream=stream)
        elif name == "ls_r16":
            fn = lambda: render.local_statistics(rgb, 16, stream=stream)
        elif name == "histogram_24mp":
            fn = lambda: render.histogram_rgb(rgb, 256, 0.0, 1.0, 512, stream=stream)
        elif name in _STENCIL_CASES:
            fn = lambda: render.stencil(name.split("_")[0], rgb, image, image, image, stream=stream,
                                        **_STENCIL_CASES[name])
        else:
            raise SystemExit(f"unknown case {name}")
    with torch.cuda.stream(stream):
        for _ in range(args.warmup + args.steps):
            fn()
    torch.cuda.synchronize()
    print(json.dumps({"case": name, "launches": args.warmup + args.steps}))


def _mixed_batch(render, workloads, torch, dev, stream, reps):
    """The mixed batch (16 RAWs, ~3,000 tiles, mip 0/1/2, a fifth of the
    viewports through a cubic resize to a 2048 long edge or a rotation):
    batched persistent launch vs the same requests launched one by one,
    device time per pass."""
    images, recipes, tiles = workloads.mixed_batch()
    imgs = []
    for im in images:
        meta = render.Metadata(im.width, im.height, im.stride, im.pattern, im.phase[0], im.phase[1], im.active,
                               im.black, (im.white,) * 4)
        imgs.append(render.Image(meta, render.synthetic_samples(im, device=dev)))
    sizes = [t.viewport[2] * t.viewport[3] * 3 for t in tiles]
    arena = torch.empty(sum(sizes), dtype=torch.float32, device=dev)
    outs, off = [], 0
    for t, n in zip(tiles, sizes):
        outs.append(arena[off:off + n].view(t.viewport[3], t.viewport[2], 3))
        off += n
    reqs = workloads.mixed_requests(render, imgs, images, recipes, tiles, outs)
    batch = render.Batch().plan(reqs)
    with torch.cuda.stream(stream):
        tuned = batch.autotune(reps=3, stream=stream)

    def timed(fn):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    batched_ms = timed(lambda: batch.launch(stream=stream))
    batch.status(stream=stream)
    per_ms = timed(lambda: batch.launch_per_request(stream=stream))
    batch.status(stream=stream)
    info = batch.info()
    algo = info["raw_bytes"] + info["output_bytes"]
    out_px = info["output_pixels"]
    result = {"requests": info["requests"], "reduced_requests": info["reduced_requests"],
              "geometry_requests": info["geometry_requests"],
              "tiles_queued": info["tiles"], "output_mpix": round(out_px / 1e6, 2),
              "native_mpix": round(info["native_pixels"] / 1e6, 2),
              "batched_ms": round(batched_ms, 4), "per_request_ms": round(per_ms, 4),
              "speedup": round(per_ms / batched_ms, 3),
              "batched_mpix_s": round(out_px / (batched_ms * 1e-3) / 1e6, 1),
              "batched_gb_s": round(algo / (batched_ms * 1e-3) / 1e9, 1), "options": tuned}
    batch.close()
    del arena
    return result


def _menon_direction_counts(render, img, w):
    """Direction decisions of the frame under both Menon policies: the
    binary64 policy's exact ties (v == h, decided horizontal as in the
    reference) and the binary32 policy's decisions inside its proved error
    band, re-decided in binary64; the two maps are equal."""
    a, ties = render.menon_directions(img, w.active, render.MENON)
    b, rechecks = render.menon_directions(img, w.active, render.MENON_FAST)
    aw, ah = w.active[2], w.active[3]
    return {"decisions": aw * ah // 2, "binary64_exact_ties": int(ties), "binary32_rechecked_near_ties": int(rechecks),
            "maps_equal": bool((a == b).all().item())}


def _differentiable(torch, dev, reps):
    """The differentiable render on 8 frames of 4000x3000 RGGB (bilinear, WB,
    exposure, 3x3, 16-knot curve, detail boost r 16 / eps 1e-3 / strength 0.5),
    MSE loss: device time of the forward and of the backward (all adjoints)."""
    from librawops_b200 import diff, synthetic, workloads
    knots = workloads.tone_knots_16()
    model = diff.RecipeModel((0, 1, 1, 2), [k[0] for k in knots], [k[1] for k in knots], wb=(2.0, 1.0, 1.6),
                             stops=0.2, matrix=workloads.CAMERA_TO_PROPHOTO, strength=0.5, radius=16, eps=1e-3,
                             device=dev)
    planes, targets = [], []
    for i in range(8):
        codes = synthetic.bayer_device(4000, 3000, seed=40 + i, pattern=0, black=(512,) * 4, white=16383,
                                       device=dev)
        planes.append(((codes.float() - 512.0) / (16383.0 - 512.0)).contiguous())
    with torch.no_grad():
        for pl in planes:
            targets.append(model(pl) * 1.01)
    fwd, bwd = [], []
    for it in range(reps + 1):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        model.zero_grad(set_to_none=True)
        e0.record()
        loss = sum(torch.mean((model(pl) - t) ** 2) for pl, t in zip(planes, targets)) / len(planes)
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        if it:
            fwd.append(e0.elapsed_time(e1))
            bwd.append(e1.elapsed_time(e2))
    f, b = statistics.median(fwd), statistics.median(bwd)
    px = 8 * 4000 * 3000
    return {"frames": 8, "frame": "4000x3000 RGGB", "chain": "bilinear, WB, exposure, 3x3, 16-knot curve, "
            "detail boost r16 eps1e-3", "forward_ms": round(f, 3), "backward_ms": round(b, 3),
            "backward_over_forward": round(b / f, 3), "forward_mpix_s": round(px / (f * 1e-3) / 1e6, 1),
            "forward_backward_mpix_s": round(px / ((f + b) * 1e-3) / 1e6, 1)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default=None, help="run one workload's kernel only (profiling captures)")
    args = ap.parse_args()
    if args.case:
        run_case(args)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
