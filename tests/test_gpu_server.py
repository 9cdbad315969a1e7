"""The serving loop (lr_server) through the C ABI: render sessions and probes submitted
together, admitted by slots and a memory budget tight enough to force evictions, come
out exactly as they do alone -- each render bit for bit a Renderer's image, each probe
bit for bit lr_probe's result."""
import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes
import render_cases

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _upload_estimate(sc):
    info = sc.info
    return int(info.triangle_count) * 256 + int(info.point_count) * 16 + (1 << 20)


def test_results_same_alone_and_in_the_mix(ctx):
    cs = render_cases.cases()
    alone = [render_cases.alone(ctx, sc, s) for sc, s in cs]
    # Probe frames through each scene's camera, and what lr_probe returns for them.
    probe_frames, probe_want = [], []
    for index, (sc, s) in enumerate(cs):
        frame = lr.ray_frame(sc.camera(), 40 + 8 * index, 30 + 4 * index)
        gs = lr.GpuScene.upload(ctx, sc)
        probe_want.append(lr.probe(ctx, gs, frame))
        gs.destroy()
        probe_frames.append(frame)
    # A pool of 4096 paths and room for the largest scene and session, so that scenes
    # take turns on the device.
    pool = 4096
    wave = pool * 16 * 15 + (1 << 20)
    biggest_scene = max(_upload_estimate(sc) for sc, _ in cs)
    biggest_session = max(s.c.width * s.c.height * 32 + (1 << 20) for _, s in cs)
    # The static probe array (LR_PROBE_STATIC_PIXELS face ids and distances) counts
    # against the budget from the server's start.
    budget = wave + biggest_scene + biggest_session + lr.PROBE_STATIC_PIXELS * 8
    server = lr.Server(lr.ServerSettings.default(budget_bytes=budget, capacity=2, pool=pool, max_bounces=12))
    try:
        ids = [server.add_scene(sc) for sc, _ in cs]
        renders, probes = [], []
        for round_ in range(2):
            for index, (sc, s) in enumerate(cs):
                rgba = np.full((s.c.height, s.c.width, 4), np.nan, np.float32)
                renders.append((server.submit_render(ids[index], s, rgba=rgba), index, rgba))
                frame = probe_frames[index]
                n = int(frame.width) * int(frame.height)
                faces, dist = np.zeros(n, np.uint32), np.zeros(n, np.float32)
                probes.append((server.submit_probe(ids[index], frame, faces, dist), index, faces, dist))
        for rid, index, rgba in renders:
            server.wait(rid, 300.0)
            info = server.info(rid)
            assert info["state"] == "done" and info["samples_done"] == cs[index][1].c.samples
            assert 0 <= info["submitted"] <= info["admitted"] <= info["first"] <= info["finished"]
            assert np.array_equal(_bits(rgba), _bits(alone[index])), (rid, index)
        for rid, index, faces, dist in probes:
            server.wait(rid, 300.0)
            assert server.info(rid)["state"] == "done"
            assert np.array_equal(faces, probe_want[index][0]) and np.array_equal(_bits(dist), _bits(probe_want[index][1]))
        st = server.stats()
        assert st["sessions_done"] == len(renders) and st["probes_done"] == len(probes) and st["failed"] == 0
        assert st["evictions"] > 0 and st["uploads"] > len(cs)
        assert st["pixel_samples"] == sum(2 * s.c.width * s.c.height * s.c.samples for _, s in cs)
        assert st["bytes_in_use"] <= budget
        # The render thread's own account: it queued passes and its host time adds up to
        # no more than the server's life.
        assert st["passes"] > 0
        spent = sum(st[k] for k in ("seconds_advance", "seconds_wait", "seconds_progress", "seconds_admit",
                                    "seconds_tune"))
        assert all(st[k] >= 0.0 for k in ("seconds_advance", "seconds_wait", "seconds_progress", "seconds_admit",
                                          "seconds_tune"))
        assert 0.0 < spent <= st["seconds"] + 1e-3
    finally:
        server.destroy()
        for sc, _ in cs:
            sc.close()


def test_queue_timeouts_and_stop(ctx):
    sc = lr.compile_scene(scenes.cornell_meshes(materials=True), [scenes.cornell_camera()],
                          [scenes.cornell_light()], scenes.cornell_materials())
    server = lr.Server(lr.ServerSettings.default(capacity=1, pool=1 << 16, max_bounces=8))
    try:
        sid = server.add_scene(sc)
        long = render_cases.settings(256, 256, 4000, 8, True)
        first = server.submit_render(sid, long)
        queued = server.submit_render(sid, render_cases.settings(32, 32, 2, 2, False))
        with pytest.raises(lr.RenderError) as e:
            server.wait(queued, 0.05)
        assert e.value.code == 504
        assert server.info(queued)["state"] == "queued"
        # A probe is served while the long session occupies the render thread.
        frame = scenes.cornell_frame(64, 64)
        faces, dist = np.zeros(64 * 64, np.uint32), np.zeros(64 * 64, np.float32)
        pid = server.submit_probe(sid, frame, faces, dist)
        server.wait(pid, 60.0)
        assert server.info(first)["state"] == "running"
        assert np.count_nonzero(faces != 0xFFFFFFFF) > 0
    finally:
        server.destroy()  # ends the running and queued sessions with LR_STOPPED
        sc.close()
