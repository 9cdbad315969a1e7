"""The BVH2 built on the device (lr_gpu_scene_build, the analogue of the reference's
GpuScene.upload(accelerate = true) with compile_scene(trees = false), device.lucb:41-89,
scene.lucb:111-129).

The tree differs from the host's binned SAH, but the watertight path's answers do not
depend on the tree: closest-hit ids, distances and barycentrics equal the FP32 brute force
over the same triangles bit for bit (ties in t to the smaller source id), any-hit agrees on
which rays hit, and probes equal an upload's probes of the same scene bit for bit.
"""
import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def _rays(frame, n=8192, spread=3.0, seed=7):
    rng = np.random.default_rng(seed)
    extra = np.zeros((n, 8), np.float32)
    extra[:, 0:3] = rng.uniform(-spread, spread, (n, 3))
    d = rng.normal(size=(n, 3))
    extra[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    extra[:, 7] = 3e38
    return np.concatenate([orc.probe_rays(frame.pack()), extra])


def _check_exact(ctx, gs, sc, rays):
    a = sc.arrays()
    prim, t, u, v = orc.brute_watertight(a["positions"], a["indices"], a["order"], rays)
    hits = lr.trace_rays(ctx, gs, rays)
    assert np.array_equal(lr.hit_ids(hits), prim)
    assert np.array_equal(_bits(hits[:, 0]), _bits(t))
    hit = prim >= 0
    assert np.array_equal(_bits(hits[hit, 2]), _bits(u[hit])) and np.array_equal(_bits(hits[hit, 3]), _bits(v[hit]))
    anyh = lr.trace_rays(ctx, gs, rays, any_hit=True)
    assert np.array_equal(lr.hit_ids(anyh) >= 0, hit)
    return int(hit.sum())


@pytest.mark.parametrize("trees", [False, True])
def test_device_build_cornell_equals_brute_force(ctx, trees):
    sc = lr.compile_scene(scenes.cornell_meshes(), trees=trees)
    gs = lr.GpuScene.build(ctx, sc)
    try:
        frame = scenes.cornell_frame(128, 96)
        assert _check_exact(ctx, gs, sc, _rays(frame)) > 2000
        # A request for a wide BVH takes the BVH2: the device build has no collapses.
        assert lr.hit_ids(lr.trace_rays(ctx, gs, _rays(frame), width=8)).shape[0] == 128 * 96 + 8192
    finally:
        gs.destroy()
        sc.close()


def test_device_build_probe_equals_upload(ctx):
    # A scene of about 200k triangles: the device build of the tree-less compile against the
    # upload of the host-built one, from the scene's camera and from inside it.
    meshes, _, _, cam = scenes.scene_of_size(200_000, seed=17)
    flat = lr.compile_scene(meshes, [cam], trees=False)
    full = lr.compile_scene(meshes, [cam])
    built, uploaded = lr.GpuScene.build(ctx, flat), lr.GpuScene.upload(ctx, full)
    try:
        frames = (lr.ray_frame(full.camera(0), 640, 360),
                  lr.look_frame((1.0, 2.0, 3.0), (0.3, -0.2, -1.0), (0.0, 1.0, 0.0), 0.6, 640, 360))
        for index, frame in enumerate(frames):
            faces, dist = lr.probe(ctx, built, frame)
            want_faces, want_dist = lr.probe(ctx, uploaded, frame)
            assert np.array_equal(faces, want_faces), index
            assert np.array_equal(_bits(dist), _bits(want_dist)), index
            assert np.count_nonzero(want_faces != 0xFFFFFFFF) > 0, index
        # Random rays through the whole scene, against the upload (the brute force at this size
        # would take minutes on the host; the upload's answers equal it in test_gpu_trace).
        rays = _rays(frames[0], n=1 << 16, spread=50.0, seed=3)
        got, want = lr.trace_rays(ctx, built, rays), lr.trace_rays(ctx, uploaded, rays)
        assert np.array_equal(lr.hit_ids(got), lr.hit_ids(want))
        assert np.array_equal(_bits(got[:, 0]), _bits(want[:, 0]))
    finally:
        built.destroy()
        uploaded.destroy()
        flat.close()
        full.close()


def test_device_build_small_and_empty(ctx):
    # One triangle (the root is a leaf), two (one interior node), and no triangles.
    p = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0], [-1, -1, -1], [1, -1, -1], [0, 1, -1]], np.float32)
    frame = lr.look_frame((0.0, 0.0, 3.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 0.5, 32, 32)
    for tris in ([[0, 1, 2]], [[0, 1, 2], [3, 4, 5]]):
        sc = lr.compile_scene([lr.MeshData(p, np.array(tris, np.uint32))], trees=False)
        gs = lr.GpuScene.build(ctx, sc)
        try:
            assert _check_exact(ctx, gs, sc, _rays(frame, n=1024)) > 0
        finally:
            gs.destroy()
            sc.close()
    sc = lr.compile_scene([], trees=False)
    gs = lr.GpuScene.build(ctx, sc)
    try:
        faces, _ = lr.probe(ctx, gs, frame)
        assert np.all(faces == 0xFFFFFFFF)
    finally:
        gs.destroy()
        sc.close()


def test_device_build_refits_and_refuses_renders(ctx):
    sc = lr.compile_scene(scenes.cornell_meshes(materials=True), [scenes.cornell_camera()],
                          [scenes.cornell_light()], scenes.cornell_materials(), trees=False)
    gs = lr.GpuScene.build(ctx, sc)
    try:
        # A refit of the device-built tree stays exact for the moved points.
        moved = (sc.arrays()["positions"] * np.float32(1.1)).astype(np.float32)
        sc.move_points(moved)
        gs.refit(ctx, moved)
        assert _check_exact(ctx, gs, sc, _rays(scenes.cornell_frame(64, 64), n=2048)) > 1024
        # Renders take uploads only: the upload of a tree-less scene and a batch member on a
        # device build are refused.
        with pytest.raises(lr.RenderError) as e:
            lr.GpuScene.upload(ctx, sc)
        assert e.value.code == 400
        b = lr.Batch(ctx, lr.BatchSettings.default(pool=1 << 14, max_bounces=4, capacity=1))
        try:
            with pytest.raises(lr.RenderError) as e:
                b.add(gs, sc, lr.RenderSettings.of(16, 16, 1))
            assert e.value.code == 400
        finally:
            b.destroy()
    finally:
        gs.destroy()
        sc.close()
