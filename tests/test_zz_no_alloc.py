"""lr_probe_static, the probe that allocates no device memory, against lr_probe.

Named to be collected last, so that it runs both alone and after every other GPU test
in one process: its static scratch is set up on the first call, whatever ran before.
Both probes compute the same kernel on the same rays, so the tolerance is zero: faces
and distances are compared bit for bit, on two calls in a row.
"""
import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def _same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(_bits(a[1]), _bits(b[1]))


@pytest.mark.parametrize("reference", [False, True])
def test_static_probe_equals_probe(ctx, reference):
    sc = lr.compile_scene(scenes.cornell_meshes())
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        # A viewport, then the largest frame the scratch holds (2048 x 1024 pixels).
        for width, height in ((640, 480), (2048, 1024)):
            frame = scenes.cornell_frame(width, height)
            want = lr.probe(ctx, gs, frame, reference=reference)
            first = lr.probe_static(ctx, gs, frame, reference=reference)
            second = lr.probe_static(ctx, gs, frame, reference=reference)
            assert _same(first, want), (width, height)
            assert _same(second, want), (width, height)
            assert np.count_nonzero(want[0] != 0xFFFFFFFF) > width * height // 16
    finally:
        gs.destroy()
        sc.close()


def test_static_probe_on_a_larger_scene(ctx):
    # A scene of about 200k triangles seen from its camera and from inside, alternating
    # with lr_probe so that each static call follows one that used stream-ordered scratch.
    meshes, _, _, cam = scenes.scene_of_size(200_000, seed=17)
    sc = lr.compile_scene(meshes, [cam])
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        frames = (lr.ray_frame(sc.camera(0), 1280, 720),
                  lr.look_frame((1.0, 2.0, 3.0), (0.3, -0.2, -1.0), (0.0, 1.0, 0.0), 0.6, 1280, 720))
        for index, frame in enumerate(frames):
            want = lr.probe(ctx, gs, frame)
            assert _same(lr.probe_static(ctx, gs, frame), want), index
            assert _same(lr.probe_static(ctx, gs, frame), want), index
            assert np.count_nonzero(want[0] != 0xFFFFFFFF) > 0, index
    finally:
        gs.destroy()
        sc.close()


def test_static_probe_refuses_frames_beyond_its_scratch(ctx):
    sc = lr.compile_scene(scenes.cornell_meshes())
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        assert lr.PROBE_STATIC_PIXELS == 2048 * 1024
        with pytest.raises(lr.RenderError) as error:
            lr.probe_static(ctx, gs, scenes.cornell_frame(2048, 1025))
        assert error.value.code == 401 and "lr_probe" in str(error.value)
        # The refusal leaves the context usable.
        frame = scenes.cornell_frame(64, 64)
        assert _same(lr.probe_static(ctx, gs, frame), lr.probe(ctx, gs, frame))
    finally:
        gs.destroy()
        sc.close()


def test_static_probe_allocates_nothing(ctx):
    # What the entry point exists for: after its first call on the device (its set-up,
    # which may load the module and so reserve the static array), calls take nothing from
    # the device -- its free bytes stay the same and the stream-ordered pool hands out
    # nothing -- while lr_probe, on the same frame, does draw its 16 MiB of scratch from
    # that pool (the measurement sees an allocation when there is one).
    sc = lr.compile_scene(scenes.cornell_meshes())
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        frame = scenes.cornell_frame(2048, 1024)
        first = lr.probe_static(ctx, gs, frame)
        before = ctx.memory(reset_high=True)
        for _ in range(3):
            assert _same(lr.probe_static(ctx, gs, frame), first)
        after = ctx.memory()
        assert after["free"] == before["free"], (before, after)
        assert after["pool_used"] == before["pool_used"] and after["pool_high"] <= before["pool_used"], (before, after)
        lr.probe(ctx, gs, frame)
        control = ctx.memory()
        assert control["pool_high"] >= before["pool_used"] + 2048 * 1024 * 8, (before, control)
    finally:
        gs.destroy()
        sc.close()
