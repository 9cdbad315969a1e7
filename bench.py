#!/usr/bin/env python
"""Throughput of the wavefront path tracer on one B200: Mrays/s of closest-hit plus
shadow rays on the incoherent 1,048,576-triangle scene at 1920x1080, depth 6.

A step is one pass of the hot path over one batch: one sample of every pixel of the
1080p frame (camera -> 7 rounds of closest / shade / shadow -> film). `value` is the
rays of all ranks over the slowest rank's device time (CUDA events on the renderer's
stream, inputs resident in HBM); `e2e` is the same metric through the public API
(Renderer.advance + Renderer.read into pinned host memory every step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) each rank renders its own replica (no data exchange: the path
shards by scene) and the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s closest+shadow; batched vs per-scene spp/s at equal RMSE; p50/p99 ms"
WIDTH, HEIGHT, BOUNCES = 1920, 1080, 6
WORKLOAD = ("incoherent traversal: 1,048,576 triangles (512 icospheres of 1,280 and 512 tori of 768, "
            "seeded placement in a 100-unit box), 4 rect + 1 distant light, Lambertian albedo U(0.2,0.9), "
            "1920x1080, one sample per pixel per step (a 16-spp render is 16 steps), depth 6")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--rgb", action="store_true", help="the RGB build instead of the spectral one")
    p.add_argument("--skip-batched", action="store_true", help="leave out the 64-scene batched comparison")
    p.add_argument("--skip-served", action="store_true", help="leave out the served arrival stream")
    p.add_argument("--skip-cornell", action="store_true", help="leave out the glossy Cornell benchmark lines")
    p.add_argument("--skip-refit", action="store_true", help="leave out the moved-geometry refit line")
    p.add_argument("--refit-only", action="store_true", help="only the moved-geometry refit line (for profiling)")
    p.add_argument("--trace-only", action="store_true",
                   help="only the headline renderer's passes (--warmup, then --steps), for profiling; one JSON line")
    p.add_argument("--width", type=int, default=0, help="with --trace-only: the BVH width (2, 4, 8; 0 the default)")
    p.add_argument("--refill", type=int, default=-1,
                   help="with --trace-only: idle lanes at which traversal warps refill (1-32; 0 grid-stride)")
    p.add_argument("--cornell-only", action="store_true",
                   help="only the glossy Cornell benchmark lines (--steps samples each), one JSON line")
    p.add_argument("--served-seconds", type=float, default=60.0,
                   help="length of the served arrival stream (the workload's 60 s by default)")
    return p.parse_args()


class Dist:
    """torch.distributed plumbing for N > 1: barrier, max and sum over ranks (NCCL on GPUs,
    gloo on a host without one). No data crosses ranks: each renders its own replica."""

    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            if torch.cuda.is_available():
                torch.cuda.set_device(self.local)
                backend, self.device = "nccl", f"cuda:{self.local}"
            else:
                backend, self.device = "gloo", "cpu"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.torch, self.dist = torch, dist
            self.pg = True

    def barrier(self):
        if self.pg:
            self.dist.barrier()

    def max(self, value: float) -> float:
        if not self.pg:
            return value
        t = self.torch.tensor([value], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, value: float) -> float:
        if not self.pg:
            return value
        t = self.torch.tensor([value], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


class Clocks:
    """nvidia-smi samples of SM clocks and throttle reasons around the timed region: the
    sampler runs from before the region (`ready` waits for its first sample) to after it
    (`stop` waits for one sample past the end), every 100 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        import threading

        self.lines, self.proc = [], None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line)

    def _wait_for(self, count: int, seconds: float) -> None:
        end = time.perf_counter() + seconds
        while len(self.lines) < count and time.perf_counter() < end and self.proc.poll() is None:
            time.sleep(0.01)

    def ready(self) -> None:
        if self.proc:
            self._wait_for(1, 5.0)
        self.first = len(self.lines)

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self._wait_for(len(self.lines) + 1, 2.0)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        # The sample just before the region, the samples in it and the one just after.
        lines = self.lines[max(0, getattr(self, "first", 1) - 1):]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return json.loads(path.read_text())
    return {}


def build_scene(lr, scenes):
    meshes, mats, lights, cam = scenes.incoherent_scene()
    return lr.compile_scene(meshes, [cam], lights, mats), lights, mats


def settings_for(lr, samples: int, spectral: bool, profile: int = 0, light_tracing: float = 0.0):
    s = lr.RenderSettings.of(WIDTH, HEIGHT, samples)
    s.max_bounces = BOUNCES
    s.spectral = 1 if spectral else 0
    s.light_tracing = light_tracing
    s.profile = profile
    s.c.material = lr.OpenPbr.lambert()
    return s


def config_of(spectral: bool, world: int) -> dict:
    """The workload's description, the same in both arms."""
    return {"workload": WORKLOAD, "triangles": 1 << 20, "width": WIDTH, "height": HEIGHT, "max_bounces": BOUNCES,
            "spectral": spectral, "samples_per_step": 1, "light_tracing": 0.0,
            "l2": "inputs larger than L2: each pass streams ~0.9 GB of path state, ray queues and film",
            "parallelism": f"replicas x{world}"}


def mapped_libraries() -> list[str]:
    """This repository's shared libraries mapped into the process."""
    found = set()
    try:
        for line in open("/proc/self/maps"):
            path = line.split()[-1] if line.strip() else ""
            if path.endswith(".so") and path.startswith(str(ROOT)):
                found.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(found)


class CpuReference:
    """The oracle's f64 path tracer -- the reference's estimator, scene compile and BVH2
    traversal restated on the host -- over strips of pixels of the workload's frame, on
    all host cores. Built from the scene generator's meshes through the oracle alone
    (compile, BVH, camera frame), so the process maps no library of the CUDA path."""

    def __init__(self, spectral: bool, oracle):
        from luce_render_b200 import scenes  # describing the workload maps no library

        meshes, mats, lights, cam = scenes.incoherent_scene()
        self.arrays = oracle.compile_meshes(meshes, len(mats))
        status, frame = oracle.frame_of_camera(list(cam.matrix), cam.projection, cam.focal_length,
                                               cam.horizontal_aperture, cam.f_stop, cam.focus_distance, WIDTH, HEIGHT)
        if status != 0:
            raise RuntimeError("the oracle refused the workload's camera")
        default = oracle.material_standard()
        default.specular_weight = 0.0  # the render's default material: Lambertian, albedo 0.8
        self.job = oracle.RenderJob(self.arrays, lights, [default] + list(mats), frame, BOUNCES, spectral)
        self.cores = os.cpu_count() or 1
        self.pixels = 2048
        self.step = 0
        # The first strip that shades a surface builds the oracle's tables (a one-time
        # cost of seconds): kept out of timing by a strip across the frame's middle.
        self.job.region(1, 0, (HEIGHT // 2) * WIDTH, 2 * WIDTH, self.cores)

    def calibrate(self, seconds_per_step: float) -> None:
        """Sizes a step to about `seconds_per_step` of wall time from a timed strip."""
        largest = WIDTH * HEIGHT // 2
        while True:
            _, secs, _ = self.run(1)
            if secs >= 0.25 * seconds_per_step or self.pixels >= largest:
                break
            self.pixels = min(largest, self.pixels * 4)
        self.pixels = int(min(largest, max(256, self.pixels * seconds_per_step / max(secs, 1e-3))))

    def run(self, steps: int):
        """(Mrays/s, seconds, rays) of `steps` strips, one sample per pixel each."""
        total_rays, seconds = 0, 0.0
        for _ in range(steps):
            first = (self.step * 7919 * 64) % (WIDTH * HEIGHT - self.pixels)
            self.step += 1
            t0 = time.perf_counter()
            _, _, rays = self.job.region(1, 0, first, self.pixels, self.cores)
            seconds += time.perf_counter() - t0
            total_rays += rays[0] + rays[1]
        return total_rays / seconds / 1e6, seconds, total_rays


BATCH_SPP, BATCH_BOUNCES, BATCH_POOL = 32, 6, 1 << 23


def batch_cases(lr, scenes):
    """The 64 scenes of the batched and served workloads with their plan entries."""
    plan = scenes.batch_plan()
    cases = []
    for i, p in enumerate(plan):
        meshes, materials, lights, cam = scenes.scene_of_size(p["triangles"], seed=0xBA7C4 + i)
        cases.append((lr.compile_scene(meshes, [cam], lights, materials), p))
    return cases


def arrival_stream(seconds: float, scenes: int, rate: float = 200.0, seed: int = 0x5E4E):
    """The served workload's requests: (time, "probe", scene, width, height) for 20 %
    (1k..2M pixel rays, log-uniform, 16:9) and (time, "render", scene, spp, 0) for 80 %
    (spp uniform in 16..256), Poisson arrivals at `rate` a second."""
    import numpy as np

    rng = np.random.default_rng(seed)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        if rng.random() < 0.2:
            px = int(round(math.exp(rng.uniform(math.log(1000.0), math.log(2_000_000.0)))))
            w = max(1, int(round(math.sqrt(px * 16.0 / 9.0))))
            arrivals.append((t, "probe", int(rng.integers(scenes)), w, max(1, px // w)))
        else:
            arrivals.append((t, "render", int(rng.integers(scenes)), int(rng.integers(16, 257)), 0))
    return arrivals


def percentiles(values):
    if not values:
        return {"count": 0, "p50_ms": None, "p99_ms": None}
    import numpy as np

    v = np.asarray(values, np.float64) * 1e3
    return {"count": len(values), "p50_ms": float(np.percentile(v, 50)), "p99_ms": float(np.percentile(v, 99)),
            "max_ms": float(v.max())}


def served(lr, scenes, dist, seconds: float):
    """The served workload: a Poisson stream (200 requests/s, seed 0x5E4E) of 80% render
    sessions (a scene of the batched workload at its film size, spp uniform in 16..256,
    depth 6) and 20% probes (1k to 2M pixel rays, log-uniform, through the scene's
    camera) into one Server (150 GB budget, 256 live sessions, pool 2^23). Latency is
    the server's own host clock from submission: probes to their result in pinned host
    memory, sessions to their first image and to completion."""
    import numpy as np

    cases = batch_cases(lr, scenes)
    arrivals = arrival_stream(seconds, len(cases))
    server = lr.Server(lr.ServerSettings.default(budget_bytes=150 * 10**9, capacity=256, pool=1 << 23,
                                                 max_bounces=BATCH_BOUNCES))
    ids = [server.add_scene(sc) for sc, _ in cases]
    for sid in ids:  # the catalog starts resident, as a running service keeps it
        server.preload(sid)
    ring = [(lr.PinnedArray((2_000_000,), np.uint32), lr.PinnedArray((2_000_000,), np.float32)) for _ in range(32)]
    submitted = []
    dist.barrier()
    clocks = Clocks(dist.local)
    clocks.ready()
    start = time.perf_counter()
    for k, (at, kind, scene, a, b) in enumerate(arrivals):
        while time.perf_counter() - start < at:
            time.sleep(min(2e-4, max(0.0, at - (time.perf_counter() - start))))
        sc, p = cases[scene]
        if kind == "probe":
            faces, distances = ring[k % len(ring)]
            frame = lr.ray_frame(sc.camera(), a, b)
            submitted.append(("probe", server.submit_probe(ids[scene], frame, faces.array, distances.array)))
        else:
            s = lr.RenderSettings.of(p["side"], p["side"], a)
            s.spectral = 1 if p["spectral"] else 0
            s.max_bounces = BATCH_BOUNCES
            s.light_tracing = 0.0
            submitted.append(("render", server.submit_render(ids[scene], s)))
    window = time.perf_counter() - start
    stats_window = server.stats()
    clock_record = clocks.stop()
    # Probes still queued finish; sessions are cut at the end of the stream.
    for kind, rid in submitted:
        if kind == "probe":
            try:
                server.wait(rid, 30.0)
            except lr.RenderError:
                pass
    infos = [(kind, server.info(rid)) for kind, rid in submitted]
    failures = {}
    for (kind, rid), (_, info) in zip(submitted, infos):
        if info["state"] == "failed":
            try:
                server.wait(rid, 0.0)
            except lr.RenderError as e:
                key = f"{kind}: {e}"
                failures[key] = failures.get(key, 0) + 1
    server.destroy()
    for f, d in ring:
        f.close()
        d.close()
    for sc, _ in cases:
        sc.close()
    probes = [i for k, i in infos if k == "probe"]
    renders = [i for k, i in infos if k == "render"]
    done_probes = [i["finished"] - i["submitted"] for i in probes if i["state"] == "done"]
    first_images = [i["first"] - i["submitted"] for i in renders if i["first"] >= 0]
    completed = [i["finished"] - i["submitted"] for i in renders if i["state"] == "done"]
    demand = sum(i["pixels"] * i["samples"] for i in renders)
    slowest = sorted((i for i in probes if i["state"] == "done"), key=lambda i: i["finished"] - i["submitted"])[-3:]
    return {
        "workload": ("Poisson arrivals at 200 requests/s (seed 0x5E4E): 80% render sessions of the batched "
                     "workload's scenes at their film sizes, 16..256 spp, depth 6; 20% probes of 1k..2M pixel rays "
                     "(log-uniform); budget 150 GB, 256 live sessions, pool 2^23, LRU eviction of idle scenes"),
        "seconds": window, "requests": len(submitted),
        "probe_latency": percentiles(done_probes),
        "slowest_probes": [{"pixels": i["pixels"], "submitted_s": i["submitted"],
                            "wait_ms": (i["admitted"] - i["submitted"]) * 1e3,
                            "latency_ms": (i["finished"] - i["submitted"]) * 1e3} for i in slowest],
        "session_first_image": percentiles(first_images),
        "session_completion": percentiles(completed),
        "sessions": {"submitted": len(renders), "admitted": sum(1 for i in renders if i["admitted"] >= 0),
                     "first_image": len(first_images), "done": len(completed)},
        "probes": {"submitted": len(probes), "done": len(done_probes)},
        "render_msamples_s": stats_window["pixel_samples"] / window / 1e6,
        "probe_mrays_s": stats_window["probe_rays"] / window / 1e6,
        "demand_msamples_s": demand / window / 1e6,
        "failures": failures,
        "uploads": stats_window["uploads"], "evictions": stats_window["evictions"],
        "tunings": stats_window.get("tunings", 0),
        "render_thread": {k: stats_window[k] for k in ("passes", "seconds_advance", "seconds_wait",
                                                       "seconds_progress", "seconds_admit", "seconds_tune")},
        "clocks": clock_record,
        "queued_at_end": stats_window["queued"], "live_at_end": stats_window["live"],
        "timing": "host steady clock of the server, from submission; the stream is cut at its end",
    }


def batched(lr, scenes, ctx, dist):
    """The batched workload: 64 scenes of the incoherent generator (triangles log-normal,
    median 20k, clipped to [1k, 500k]; films 128^2..1024^2; half spectral), 32 spp, depth
    6. Aggregate pixel-samples per second of the plain loop (one Renderer after another)
    against one tuned Batch of all 64, device-timed on the context's stream, with every
    image compared bit for bit (identical images have equal RMSE against any reference)."""
    import numpy as np

    cases = []
    for sc, p in batch_cases(lr, scenes):
        s = lr.RenderSettings.of(p["side"], p["side"], BATCH_SPP)
        s.spectral = 1 if p["spectral"] else 0
        s.max_bounces = BATCH_BOUNCES
        s.light_tracing = 0.0
        cases.append((sc, s))
    samples = sum(s.c.width * s.c.height * BATCH_SPP for _, s in cases)
    triangles = sum(sc.triangle_count() for sc, _ in cases)
    renderers = [lr.Renderer.create(ctx, sc, s) for sc, s in cases]
    dist.barrier()
    ctx.synchronize()
    ctx.timer_start()
    for r in renderers:
        r.finish()
    loop_ms = dist.max(ctx.timer_stop())
    alone = [r.read() for r in renderers]
    for r in renderers:
        r.destroy()
    uploads = [lr.GpuScene.upload(ctx, sc) for sc, _ in cases]
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=BATCH_POOL, max_bounces=BATCH_BOUNCES, capacity=len(cases)))
    members = [b.add(gs, sc, s) for gs, (sc, s) in zip(uploads, cases)]
    tuning = b.tune()
    dist.barrier()
    ctx.synchronize()
    ctx.timer_start()
    b.finish()
    batch_ms = dist.max(ctx.timer_stop())
    identical = all(np.array_equal(b.read(m).view(np.uint32), img.view(np.uint32)) for m, img in zip(members, alone))
    passes = b.stats().passes
    # The same batch kept busy for `sustain` seconds (each member 32 more samples at a
    # time), as a server is: the rate the device holds under its power limit.
    sustain = 20.0
    dist.barrier()
    ctx.synchronize()
    clocks = Clocks(dist.local)
    clocks.ready()
    shaded0 = b.stats().shaded
    t0 = time.perf_counter()
    ctx.timer_start()
    while time.perf_counter() - t0 < sustain:
        for m in members:
            b.set_samples(m, b.info(m)[2] + BATCH_SPP)
        b.finish()
    sustained_ms = dist.max(ctx.timer_stop())
    sustained_samples = b.stats().shaded - shaded0
    sustained_clocks = clocks.stop()
    b.destroy()
    for gs in uploads:
        gs.destroy()
    for sc, _ in cases:
        sc.close()
    loop_rate = dist.sum(samples) / (loop_ms / 1e3) / 1e6
    batch_rate = dist.sum(samples) / (batch_ms / 1e3) / 1e6
    return {
        "workload": ("64 scenes of the incoherent generator, triangles log-normal (median 20k, clipped to "
                     f"[1k, 500k]; {triangles:,} in all), films "
                     "128^2/256^2/512^2/1024^2, half spectral, 32 spp, depth 6, seed 0xBA7C4"),
        "unit": "Msamples/s (pixel-samples, all scenes)",
        "pixel_samples": samples,
        "loop_ms": loop_ms, "batched_ms": batch_ms,
        "loop_value": loop_rate, "batched_value": batch_rate, "speedup": loop_ms / batch_ms,
        "identical_images": identical, "pool": BATCH_POOL, "passes": passes, "tuning": tuning,
        "sustained": {"seconds": sustained_ms / 1e3,
                      "value": dist.sum(sustained_samples) / (sustained_ms / 1e3) / 1e6,
                      "clocks": sustained_clocks,
                      "note": "the tuned batch kept busy (32 more samples a member at a time) for 20 s"},
        "timing": "device (CUDA events on the context stream), renderers and batch members made beforehand",
    }


def cornell(lr, scenes, ctx, dist, samples: int = 16, warmup: int = 3) -> dict:
    """The reference's Cornell benchmark configuration (tests/cornell/main.lucb: the box
    with a clear-coated blue box, a smooth glass ball, a rough gold ball, a white cube and
    an orange plastic ball; 12 bounces, camera at (0, 1, 3.9), 50.5 mm on a 36 mm film) at
    512^2 and 1024^2, spectral and RGB, with light tracing at its default 0.5 and without:
    ms a sample, timed with CUDA events on the context's stream around `samples` passes
    after `warmup`. The reference publishes ms a sample for these configurations on an
    M4 Max (Metal), which is not a B200 number: recorded beside, never divided by."""
    meshes, cams, lights, mats = scenes.glossy_cornell(4)
    cams = [lr.camera((0.0, 1.0, 3.9), (0.0, 0.0, 0.0), focal_length=50.5, horizontal_aperture=36.0)]
    sc = lr.compile_scene(meshes, cams, lights, mats)
    lines = []
    for size, spectral, tracing in [(512, True, 0.5), (512, True, 0.0), (1024, True, 0.5), (1024, False, 0.5)]:
        s = lr.RenderSettings.of(size, size, warmup + samples)
        s.max_bounces = 12
        s.spectral = 1 if spectral else 0
        s.light_tracing = tracing
        s.seed = 0
        r = lr.Renderer.create(ctx, sc, s)
        for _ in range(warmup):
            r.advance_one()
        r.wait()
        s0 = r.stats()
        dist.barrier()
        ctx.synchronize()
        ctx.timer_start()
        for _ in range(samples):
            r.advance_one()
        r.join()
        ms = dist.max(ctx.timer_stop())
        r.finish()
        s1 = r.stats()
        r.destroy()
        rays = (s1.closest_rays - s0.closest_rays) + (s1.shadow_rays - s0.shadow_rays)
        lines.append({"size": size, "spectral": spectral, "light_tracing": tracing, "ms_per_sample": ms / samples,
                      "mrays_s": rays / (ms / 1e3) / 1e6})
    return {"triangles": int(sc.info.triangle_count), "max_bounces": 12, "samples": samples, "lines": lines,
            "reference_m4_max_ms": {"1024 spectral": 8.1, "1024 rgb": 7.1, "512 path tracing only": 3.14}}


def refit(lr, scenes, ctx, dist, repeats: int = 10) -> dict:
    """Moved geometry on the 1,048,576-triangle scene: the device refit with the points
    already in device memory (a simulation's output), against the reference's route for
    moved geometry -- a host compile of the moved mesh (its binned-SAH rebuild) and an
    upload. Two poses alternate, so every refit moves every point."""
    import numpy as np

    meshes, mats, lights, cam = scenes.incoherent_scene()
    sc = lr.compile_scene(meshes, [cam], lights, mats)
    gs = lr.GpuScene.upload(ctx, sc)
    a = sc.arrays()
    base = a["positions"].astype(np.float64)
    poses = [(base + amount * np.sin(0.7 * base[:, [1, 2, 0]])).astype(np.float32) for amount in (0.05, 0.1)]
    buffers = []
    for pose in poses:
        buffers.append(ctx.alloc(pose.nbytes))
        ctx.upload(buffers[-1], pose)
    points, triangles = len(base), len(a["indices"])
    for k in range(3):
        gs.refit(ctx, (buffers[k % 2], points), device=True)
    times = []
    for k in range(repeats):
        ctx.synchronize()
        ctx.timer_start()
        gs.refit(ctx, (buffers[k % 2], points), device=True)
        times.append(ctx.timer_stop())
    refit_ms = dist.max(statistics.median(times))
    info = gs.info
    entries = (int(sc.info.node_count) - 1) // 2
    # Bytes a refit must move at least once: the points and indices read, the triangle
    # records written, both copies of the BVH2's boxes, the 4-wide nodes' boxes and the
    # compressed 8-wide nodes (96 bytes each) written.
    algorithmic = (12 * points + 12 * triangles + 48 * triangles + 96 * entries + 96 * int(info.wide4_nodes) +
                   96 * int(info.wide8_nodes))
    for b in buffers:
        ctx.free(b)
    gs.destroy()
    # The reference's route: compile the moved mesh again (BVH2 rebuilt on the host) and upload it.
    moved = lr.MeshData(poses[1], a["indices"][np.argsort(a["order"])])
    start = time.perf_counter()
    rebuilt = lr.compile_scene([moved], [cam], lights, mats)
    compile_s = time.perf_counter() - start
    start = time.perf_counter()
    gs2 = lr.GpuScene.upload(ctx, rebuilt)
    upload_s = time.perf_counter() - start
    gs2.destroy()
    rebuilt.close()
    build_info = device_build(lr, scenes, ctx, dist, sc, meshes, cam, lights, mats)
    sc.close()
    hbm = measured_peaks().get("hbm_gbs") or 6650.0
    achieved = algorithmic / (refit_ms / 1e3) / 1e9
    return {"workload": "every point of the 1,048,576-triangle scene moved (two poses alternating), points in "
                        "device memory; BVH2, 4- and 8-wide boxes, triangle records refit",
            "triangles": triangles, "points": points, "device_refit_ms": refit_ms,
            "algorithmic_bytes": algorithmic, "achieved_gbs": achieved, "hbm_frac": achieved / hbm,
            "host_compile_ms": compile_s * 1e3, "host_upload_ms": upload_s * 1e3,
            "speedup_vs_host_rebuild": (compile_s + upload_s) * 1e3 / refit_ms,
            "timing": "device refit: CUDA events on the context's stream around the call (it waits for the new "
                      "root box between launches), median of 10; host rebuild: wall clock",
            "device_build": build_info}


def device_build(lr, scenes, ctx, dist, sc, meshes, cam, lights, mats, repeats: int = 5) -> dict:
    """The 1,048,576-triangle scene's BVH2 built on the device (lr_gpu_scene_build on a tree-less
    compile) against the host's binned-SAH compile and upload, and the closest-hit rate of both
    trees on the same 2^22 incoherent rays resident in device memory."""
    start = time.perf_counter()
    flat = lr.compile_scene(meshes, [cam], lights, mats, trees=False)
    flat_compile_s = time.perf_counter() - start
    start = time.perf_counter()
    full = lr.compile_scene(meshes, [cam], lights, mats)
    sah_compile_s = time.perf_counter() - start
    uploaded = lr.GpuScene.upload(ctx, full)
    for _ in range(2):
        lr.GpuScene.build(ctx, flat).destroy()
    times = []
    for _ in range(repeats):
        ctx.synchronize()
        ctx.timer_start()
        built = lr.GpuScene.build(ctx, flat)
        times.append(ctx.timer_stop())
        built.destroy()
    build_ms = dist.max(statistics.median(times))
    built = lr.GpuScene.build(ctx, flat)
    rays = scenes.incoherent_rays(1 << 22, seed=9)
    d_rays, d_hits = ctx.alloc(rays.nbytes), ctx.alloc(len(rays) * 16)
    ctx.upload(d_rays, rays)
    rates = {}
    for name, gs in (("device_built", built), ("host_sah", uploaded)):
        for _ in range(3):
            lr._check(lr.lib.lr_trace_rays_device(ctx.handle, gs.handle, d_rays, len(rays), d_hits, 0))
        ms = []
        for _ in range(5):
            ctx.synchronize()
            ctx.timer_start()
            lr._check(lr.lib.lr_trace_rays_device(ctx.handle, gs.handle, d_rays, len(rays), d_hits, 0))
            ms.append(ctx.timer_stop())
        rates[name] = len(rays) / (dist.max(statistics.median(ms)) / 1e3) / 1e6
    ctx.free(d_rays)
    ctx.free(d_hits)
    built.destroy()
    uploaded.destroy()
    full.close()
    flat.close()
    return {"device_build_ms": build_ms, "tree_less_compile_ms": flat_compile_s * 1e3,
            "host_sah_compile_ms": sah_compile_s * 1e3,
            "closest_mrays_device_built": rates["device_built"], "closest_mrays_host_sah": rates["host_sah"],
            "timing": "device build: CUDA events around lr_gpu_scene_build (its copies of the triangles "
                      "included), median of 5; closest: 2^22 incoherent rays in device memory, CUDA events, "
                      "median of 5; compiles: wall clock"}


def overhead(lr, scenes, ctx, dist) -> dict:
    """Launch overhead (the analogue of the reference's tests/gpu/overhead.lucb:9-39):
    chains of 10, 100 and 400 dependent empty launches, one by one and as one CUDA graph,
    microseconds a launch on the device and on the host's clock; and the fixed cost of a
    pass -- a renderer of an 8 x 8 film of the Cornell box at depth 6, whose passes hold
    64 paths, so nearly all of a pass's time is its launches and their tails -- in ms a
    pass, device-timed over 200 passes after 20."""
    chains = {}
    for count in (10, 100, 400):
        for graph in (False, True):
            device_us, host_us = ctx.launch_overhead(count, graph)
            chains[f"{count}_{'graph' if graph else 'stream'}"] = {"device_us": device_us, "host_us": host_us}
    sc = lr.compile_scene(scenes.cornell_meshes(True), [scenes.cornell_camera()], [scenes.cornell_light()],
                          scenes.cornell_materials())
    s = lr.RenderSettings.of(8, 8, 220)
    s.max_bounces = BOUNCES
    s.light_tracing = 0.0
    r = lr.Renderer.create(ctx, sc, s)
    for _ in range(20):
        r.advance_one()
    r.wait()
    dist.barrier()
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(200):
        r.advance_one()
    r.join()
    ms = dist.max(ctx.timer_stop())
    r.destroy()
    sc.close()
    return {"launch_chains": chains, "empty_pass_ms": ms / 200.0,
            "kernels_per_pass": 1 + 3 * (BOUNCES + 1) + 5,
            "timing": "chains: best of 5, CUDA events and the host clock; passes: CUDA events on the context "
                      "stream over 200 passes of 64 paths (two lanes, graphs)"}


def cpu_intersection(arrays, scenes, oracle, cores: int) -> dict:
    """The reference's CPU intersection on the 1M-triangle scene, on all host cores: its
    f64 brute force (tests/gpu/main.lucb:82-119, every ray against every triangle) on a
    seeded subset of 4,096 incoherent rays, and the restatement of trace_closest (BVH2)
    over 2^22 incoherent rays, repeated until two seconds have passed."""
    rays = scenes.incoherent_rays(1 << 22, seed=5)
    t0 = time.perf_counter()
    oracle.nearest_f64(arrays["positions"], arrays["indices"], arrays["faces"], rays[:4096], threads=cores)
    brute = time.perf_counter() - t0
    traced, t0 = 0, time.perf_counter()
    while traced == 0 or time.perf_counter() - t0 < 2.0:
        oracle.trace(arrays["nodes"], arrays["positions"], arrays["indices"], rays, threads=cores)
        traced += len(rays)
    bvh = time.perf_counter() - t0
    return {
        "brute_force_f64": {"value": 4096 / brute / 1e6, "unit": "Mrays/s", "cores": cores,
                            "sample": f"4,096 incoherent rays x {len(arrays['indices']):,} triangles, {brute:.1f} s"},
        "bvh2_closest": {"value": traced / bvh / 1e6, "unit": "Mrays/s", "cores": cores,
                         "sample": f"{traced:,} incoherent rays (2^22 a round), {bvh:.1f} s"},
    }


def main():
    args = parse()
    spectral = not args.rgb
    dist = Dist(args.gpus)
    if args.impl == "reference":
        return reference_arm(args, dist, spectral)

    import numpy as np

    import luce_render_b200 as lr
    from luce_render_b200 import scenes

    ctx = lr.Context(dist.local)
    W, K = max(3, args.warmup), args.steps
    if args.cornell_only or args.refit_only:
        info = cornell(lr, scenes, ctx, dist, samples=K, warmup=W) if args.cornell_only else refit(lr, scenes, ctx, dist)
        if dist.rank == 0:
            print(json.dumps({"cornell" if args.cornell_only else "refit": info, "n_gpus": dist.world}))
        ctx.close()
        dist.close()
        return
    sc, lights, mats = build_scene(lr, scenes)
    info = sc.info
    if args.trace_only:
        # The headline renderer alone (two lanes, graphs): what a profiler captures.
        if args.width:
            os.environ["LUCE_RENDER_B200_BVH_WIDTH"] = str(args.width)
        if args.refill >= 0:
            os.environ["LUCE_RENDER_B200_REFILL"] = str(args.refill)
        r = lr.Renderer.create(ctx, sc, settings_for(lr, W + K, spectral))
        for _ in range(W):
            r.advance_one()
        r.wait()
        s0 = r.stats()
        ctx.synchronize()
        ctx.timer_start()
        for _ in range(K):
            r.advance_one()
        r.join()
        ms = ctx.timer_stop()
        r.finish()
        s1 = r.stats()
        r.destroy()
        rays = (s1.closest_rays - s0.closest_rays) + (s1.shadow_rays - s0.shadow_rays)
        if dist.rank == 0:
            print(json.dumps({"trace_only": {"mrays_s": rays / (ms / 1e3) / 1e6, "ms_per_step": ms / K, "steps": K,
                                             "width": args.width or 2, "refill_at": max(args.refill, 0)},
                              "n_gpus": dist.world}))
        ctx.close()
        dist.close()
        return

    # Work per ray, counted by the traversal kernels on one pass of the same workload.
    counter = lr.Renderer.create(ctx, sc, settings_for(lr, 1, spectral, profile=2))
    counter.finish()
    cs = counter.stats()
    counter.destroy()
    closest_nodes = cs.closest_nodes / max(1, cs.closest_rays)
    closest_tests = cs.closest_tests / max(1, cs.closest_rays)
    shadow_nodes = cs.shadow_nodes / max(1, cs.shadow_rays)
    shadow_tests = cs.shadow_tests / max(1, cs.shadow_rays)

    # Kernel durations: a renderer that records CUDA events after every kernel (one pass
    # at a time on one stream), for the roofline and the per-kernel shares.
    r = lr.Renderer.create(ctx, sc, settings_for(lr, W + K, spectral, profile=1))
    for _ in range(W):
        r.advance_one()
    r.wait()
    p0, t0 = r.stats(), r.kernel_times()
    for _ in range(K):
        r.advance_one()
    r.finish()
    p1, t1 = r.stats(), r.kernel_times()
    r.destroy()
    kernel_ms = t1 - t0
    profiled_closest = p1.closest_rays - p0.closest_rays

    # Device-timed region: the renderer as it runs (passes taking turns on two streams),
    # CUDA events on the context's stream joined after the last pass.
    r = lr.Renderer.create(ctx, sc, settings_for(lr, W + K, spectral, profile=0))
    for _ in range(W):
        r.advance_one()
    r.wait()
    s0 = r.stats()
    clocks = Clocks(dist.local)
    clocks.ready()
    dist.barrier()
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(K):
        r.advance_one()
    r.join()
    ms = ctx.timer_stop()
    clock_info = clocks.stop()
    r.finish()
    s1 = r.stats()
    r.destroy()
    closest = s1.closest_rays - s0.closest_rays
    shadow = s1.shadow_rays - s0.shadow_rays
    slowest = dist.max(ms)
    rays_all = dist.sum(closest + shadow)
    value = rays_all / (slowest / 1e3) / 1e6

    # Roofline of the dominant kernel (closest hit): algorithmic bytes per ray
    # 48 + 64 N_int + 48 N_tri (ray in and hit out, both children's boxes per interior
    # visit, three indices and three vertices per triangle test).
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    launches = K * (BOUNCES + 1)
    closest_bytes = profiled_closest * (48.0 + 64.0 * closest_nodes + 48.0 * closest_tests)
    closest_s = kernel_ms[1] / 1e3
    achieved = closest_bytes / closest_s / 1e9 if closest_s > 0 else None
    roofline = {
        "kernel": "closest_kernel (intersect closest)",
        # The scene (~100 MB) stays in the 126 MB L2: DRAM moves a few percent of the
        # algorithmic bytes, and the kernel waits on L1/L2 latency with few lanes of a
        # warp active (divergent incoherent traversal). Reported against HBM as the
        # roofline asks; the bound the counters show is latency.
        "bound": "hbm",
        "bound_observed": "latency (L2-resident scene; divergent traversal; ncu summary in profiles/)",
        "achieved": achieved,
        "peak": hbm if hbm else 6650.0,
        "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm else "fallback 6.65 TB/s",
        "unit": "GB/s",
        "frac": (achieved / (hbm if hbm else 6650.0)) if achieved else None,
        "traffic": None,  # DRAM bytes a launch: from ncu only (profiles/), not measured in this run
        "algorithmic_bytes_per_launch": closest_bytes / launches,
        "launch_ms": kernel_ms[1] / launches,
        "bytes_per_ray": 48.0 + 64.0 * closest_nodes + 48.0 * closest_tests,
        "interior_visits_per_ray": closest_nodes,
        "triangle_tests_per_ray": closest_tests,
        "shadow_interior_visits_per_ray": shadow_nodes,
        "shadow_triangle_tests_per_ray": shadow_tests,
        "kernel_share": kernel_ms[1] / max(1e-9, kernel_ms.sum()),
    }

    # End to end through the public API: each step one pass and its image read back into
    # pinned host memory (the pass takes no new input: the scene stays resident). The reads
    # are Renderer.read_ticket into two host buffers in turn, each copy running beside the
    # next pass; before a buffer is used again its last copy has landed (read_landed), and
    # the timed region ends when the last copy has landed.
    e2e_r = lr.Renderer.create(ctx, sc, settings_for(lr, W + K, spectral, profile=0))
    hosts = [lr.PinnedArray((HEIGHT, WIDTH, 4), np.float32) for _ in range(2)]
    for step in range(W):
        e2e_r.advance_one()
        e2e_r.read_async(hosts[step % 2].array)
    e2e_r.read_wait()
    e0 = e2e_r.stats()
    dist.barrier()
    start = time.perf_counter()
    tickets = [0, 0]
    for step in range(K):
        e2e_r.advance_one()
        while tickets[step % 2] and not e2e_r.read_landed(tickets[step % 2]):
            time.sleep(2e-5)  # the copy that last filled this buffer
        tickets[step % 2] = e2e_r.read_ticket(hosts[step % 2].array)
    e2e_r.read_wait()
    e2e_s = time.perf_counter() - start
    e1 = e2e_r.stats()
    e2e_r.destroy()
    e2e_rays = dist.sum((e1.closest_rays - e0.closest_rays) + (e1.shadow_rays - e0.shadow_rays))
    e2e_value = e2e_rays / dist.max(e2e_s) / 1e6

    # The same workload with light tracing at the reference's default share (0.5): light
    # paths and their camera connections count among the rays.
    lt = lr.Renderer.create(ctx, sc, settings_for(lr, W + K, spectral, light_tracing=0.5))
    for _ in range(W):
        lt.advance_one()
    lt.wait()
    l0 = lt.stats()
    dist.barrier()
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(K):
        lt.advance_one()
    lt.join()
    lt_ms = dist.max(ctx.timer_stop())
    lt.finish()
    l1 = lt.stats()
    lt.destroy()
    lt_rays = dist.sum((l1.closest_rays - l0.closest_rays) + (l1.shadow_rays - l0.shadow_rays))
    traced_info = {"light_tracing": 0.5, "value": lt_rays / (lt_ms / 1e3) / 1e6, "unit": "Mrays/s",
                   "ms_per_step": lt_ms / K,
                   "rays_per_step": lt_rays / K / dist.world,
                   "note": "light paths (0.5 x the pixels a sample) from the scene's rect lights, their camera "
                           "connections splatted; rays include the light paths' closest and connection rays"}

    cornell_info = None if args.skip_cornell else cornell(lr, scenes, ctx, dist)
    batch_info = None if args.skip_batched else batched(lr, scenes, ctx, dist)
    served_info = None if args.skip_served else served(lr, scenes, dist, args.served_seconds)
    refit_info = None if args.skip_refit else refit(lr, scenes, ctx, dist)
    overhead_info = overhead(lr, scenes, ctx, dist)

    cpu = None
    if dist.rank == 0 and dist.world == 1:
        from oracle import oracle

        ref = CpuReference(spectral, oracle)
        ref.calibrate(4.0)
        mrays, secs, rays = ref.run(3)
        cpu = {"value": mrays, "unit": "Mrays/s", "cores": ref.cores, "kind": "port",
               "sample": f"3 strips of {ref.pixels} pixels x 1 spp of the same frame ({rays} closest+shadow rays, "
                         f"{secs:.1f} s wall on {ref.cores} threads): the f64 restatement of the reference's "
                         f"estimator and BVH2 traversal"}
        cpu.update(cpu_intersection(ref.arrays, scenes, oracle, ref.cores))

    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": dist.world, "steps": K, "warmup": W,
            "ms_per_step": slowest / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded generator of the workload's shapes)",
            "config": config_of(spectral, dist.world),
            "closest_mrays_s": dist.sum(closest) / (slowest / 1e3) / 1e6,
            "shadow_mrays_s": dist.sum(shadow) / (slowest / 1e3) / 1e6,
            "spp_per_s": K / (slowest / 1e3),
            "kernel_ms_per_step": {n: kernel_ms[i] / K for i, n in enumerate(lr.KERNEL_NAMES) if kernel_ms[i] > 0},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": WIDTH * HEIGHT * 16},
            # a pass: camera; closest, shade and shadow each round; finish, fold, the two
            # adaptive phases and convert (the launch list in profiles/ counts the same)
            "gpu_launches": K * (1 + 3 * (BOUNCES + 1) + 5),
            "clocks": clock_info,
            "light_traced": traced_info,
            "cornell": cornell_info,
            "batched": batch_info,
            "served": served_info,
            "refit": refit_info,
            "overhead": overhead_info,
        }
        print(json.dumps(line))
    ctx.close()
    dist.close()


def reference_arm(args, dist, spectral: bool):
    """The reference's path on the host cores: its CPU restatement (the oracle port; the
    reference itself runs only on Vulkan/Metal, unavailable here), timed on the same
    workload, a bounded strip of pixels per step. The scene is compiled, its BVH built
    and its camera frame made by the oracle alone: this process maps no library of the
    CUDA path (the line lists what it mapped)."""
    if dist.rank != 0:
        dist.close()
        return
    from oracle import oracle

    info_triangles = 1 << 20
    W, K = max(3, args.warmup), args.steps
    ref = CpuReference(spectral, oracle)
    if len(ref.arrays["indices"]) != info_triangles:
        raise RuntimeError("the oracle compiled another workload")
    # A step is a strip sized to about 4 s (less when many steps are asked for), so the
    # whole run stays within a few minutes; warm-up steps are a quarter of that.
    seconds = min(4.0, 150.0 / max(1, K + W / 4))
    ref.calibrate(seconds)
    pixels = ref.pixels
    ref.pixels = max(256, pixels // 4)
    ref.run(W)
    ref.pixels = pixels
    mrays, secs, rays = ref.run(K)
    cores = ref.cores
    line = {
        "impl": "reference", "metric": METRIC, "value": mrays, "unit": "Mrays/s", "n_gpus": dist.world, "steps": K,
        "warmup": W, "ms_per_step": secs * 1e3 / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator of the workload's shapes)",
        "config": config_of(spectral, dist.world),
        "cpu_baseline": {"value": mrays, "unit": "Mrays/s", "cores": cores, "kind": "port",
                         "sample": f"{K} strips of {pixels} pixels x 1 spp of the 1920x1080 frame ({rays} closest+"
                                   f"shadow rays, {secs:.1f} s on {cores} threads)"},
        "e2e": {"value": mrays, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "native_so_loaded": mapped_libraries(),
    }
    print(json.dumps(line))
    dist.close()


if __name__ == "__main__":
    main()
