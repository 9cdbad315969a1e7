"""Refitting an uploaded scene on the device after its points move (lr_gpu_scene_refit,
lr_renderer_refit): the triangle records, flat normals and every BVH's boxes again, the
topology kept.

- Points unchanged: every query answers bit for bit as before the refit.
- Points moved: the watertight path (BVH2, 4- and 8-wide) equals the FP32 brute force over
  the moved triangles bit for bit; the reference path equals the oracle's restatement of
  trace_closest on the host refit of the same tree (lr_scene_move_points), bit for bit, and
  so do its counted interior visits and triangle tests -- so the device's exact boxes are
  the host's; points given in device memory refit the same.
- A scene whose root is a leaf (at most 16 triangles) refits too.
- A renderer refit after its points move renders, bit for bit, what a renderer made afresh
  from the moved scene renders.
"""
import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def _deform(p, amount=0.08):
    p = np.asarray(p, np.float64)
    return (p + amount * np.sin(3.0 * p[:, [1, 2, 0]])).astype(np.float32)


def _rays(sc, w=96, h=64):
    frame = lr.ray_frame(sc.camera(0), w, h)
    rng = np.random.default_rng(7)
    extra = np.zeros((8192, 8), np.float32)
    extra[:, 0:3] = rng.uniform(-3.0, 3.0, (8192, 3))
    d = rng.normal(size=(8192, 3))
    extra[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    extra[:, 7] = 3e38
    return frame, np.concatenate([orc.probe_rays(frame.pack()), extra])


def _exact(ctx, gs, a, rays):
    prim, t, u, v = orc.brute_watertight(a["positions"], a["indices"], a["order"], rays)
    for width in (2, 4, 8):
        hits = lr.trace_rays(ctx, gs, rays, width=width)
        assert np.array_equal(lr.hit_ids(hits), prim), width
        assert np.array_equal(_bits(hits[:, 0]), _bits(t)), width
        hit = prim >= 0
        assert np.array_equal(_bits(hits[hit, 2]), _bits(u[hit])) and np.array_equal(_bits(hits[hit, 3]), _bits(v[hit]))
        anyh = lr.trace_rays(ctx, gs, rays, any_hit=True, width=width)
        assert np.array_equal(lr.hit_ids(anyh) >= 0, hit), width


def _reference(ctx, gs, a, frame, rays):
    lr.trace_counts(ctx)
    hits = lr.trace_rays(ctx, gs, rays, reference=True, count=True)
    nodes, tests = lr.trace_counts(ctx)
    ref, counts = orc.trace(a["nodes"], a["positions"], a["indices"], rays)
    assert counts.dropped == 0
    assert (nodes, tests) == (counts.interior, counts.triangles)
    slot = ref["triangle"].astype(np.int64)
    want = np.where(slot == 0xFFFFFFFF, -1, a["order"][np.minimum(slot, len(a["order"]) - 1)].astype(np.int64))
    assert np.array_equal(lr.hit_ids(hits), want.astype(np.int32))
    assert np.array_equal(_bits(hits[:, 0]), _bits(ref["t"]))
    faces, dist = lr.probe(ctx, gs, frame, reference=True)
    n = frame.width * frame.height
    want_faces = np.where(slot[:n] == 0xFFFFFFFF, 0xFFFFFFFF, a["faces"][np.minimum(slot[:n], len(a["faces"]) - 1)])
    assert np.array_equal(faces, want_faces.astype(np.uint32))
    assert np.array_equal(_bits(dist), _bits(ref["t"][:n]))


def test_refit_unchanged_points_answers_the_same(ctx):
    meshes, cams = scenes.probe_test_scene()
    sc = lr.compile_scene(meshes, cams)
    a = sc.arrays()
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        frame, rays = _rays(sc)
        before = [lr.trace_rays(ctx, gs, rays, width=w) for w in (2, 4, 8)] + [lr.trace_rays(ctx, gs, rays, reference=True)]
        gs.refit(ctx, a["positions"])
        after = [lr.trace_rays(ctx, gs, rays, width=w) for w in (2, 4, 8)] + [lr.trace_rays(ctx, gs, rays, reference=True)]
        for x, y in zip(before, after):
            assert np.array_equal(_bits(x), _bits(y))
    finally:
        gs.destroy()


@pytest.mark.parametrize("device", [False, True])
def test_refit_moved_points(ctx, device):
    meshes, cams = scenes.probe_test_scene()
    sc = lr.compile_scene(meshes, cams)
    gs = lr.GpuScene.upload(ctx, sc)
    buffer = None
    try:
        moved = _deform(sc.arrays()["positions"])
        sc.move_points(moved)
        a = sc.arrays()
        if device:
            buffer = ctx.alloc(moved.nbytes)
            ctx.upload(buffer, moved)
            gs.refit(ctx, (buffer, len(moved)), device=True)
        else:
            gs.refit(ctx, moved)
        frame, rays = _rays(sc)
        _exact(ctx, gs, a, rays)
        _reference(ctx, gs, a, frame, rays)
    finally:
        if buffer is not None:
            ctx.free(buffer)
        gs.destroy()


def test_refit_leaf_root(ctx):
    p, t, f = scenes.grid(2.0, 1)  # one quad: 2 triangles, the root a leaf
    sc = lr.compile_scene([lr.MeshData(p, t, faces=f, face_count=1)],
                          [lr.camera((0.0, 2.0, 0.0), (-1.5707963, 0.0, 0.0))])
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        moved = sc.arrays()["positions"].copy()
        moved[:, 1] += np.array([0.1, -0.2, 0.3, 0.05], np.float32)
        sc.move_points(moved)
        gs.refit(ctx, moved)
        a = sc.arrays()
        frame, rays = _rays(sc, 32, 32)
        _exact(ctx, gs, a, rays)
        _reference(ctx, gs, a, frame, rays)
    finally:
        gs.destroy()


def test_refit_rejects_other_point_counts(ctx):
    sc = lr.compile_scene(scenes.cornell_meshes())
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        with pytest.raises(lr.RenderError) as e:
            gs.refit(ctx, sc.arrays()["positions"][:-1])
        assert e.value.code == 400
    finally:
        gs.destroy()


@pytest.mark.parametrize("spectral", [False, True])
def test_renderer_refit_equals_fresh_renderer(ctx, spectral):
    # The Cornell box with an emissive quad: the light tree's emitters move too.
    meshes = scenes.cornell_meshes(materials=True)
    p, t, f = scenes.grid(0.3, 1)
    glow = lr.OpenPbr.lambert((0.8, 0.8, 0.8), emission=6.0)
    meshes.append(lr.MeshData(p, t, faces=f, face_count=1, face_materials=[len(scenes.cornell_materials()) + 1],
                              transform=lr.placement((0.1, 0.3, 0.0), (np.pi, 0.0, 0.0))))
    mats = scenes.cornell_materials() + [glow]
    cams, lights = [scenes.cornell_camera()], [scenes.cornell_light()]
    s = lr.RenderSettings.of(48, 40, 4)
    s.spectral = 1 if spectral else 0
    s.max_bounces = 5
    s.seed = 3
    sc = lr.compile_scene(meshes, cams, lights, mats)
    r = lr.Renderer.create(ctx, sc, s)
    try:
        for _ in range(3):
            r.advance()  # passes in flight when the points move
        moved = _deform(sc.arrays()["positions"], 0.03)
        sc.move_points(moved)
        r.refit(sc)
        r.finish()
        assert r.samples_done() == 4
        got = r.read()
    finally:
        r.destroy()
    fresh = lr.Renderer.create(ctx, sc, s)
    try:
        fresh.finish()
        want = fresh.read()
    finally:
        fresh.destroy()
    assert np.array_equal(_bits(got), _bits(want))


def test_batch_member_follows_a_refit(ctx):
    # A batch member borrowing an upload that is refit before its passes traces the moved
    # geometry: the Cornell box grown by a fifth (past its old root box) renders, bit for
    # bit, what a renderer made from the moved scene renders. Its loaded records do not
    # depend on the points here (a rect light, no light paths).
    sc = lr.compile_scene(scenes.cornell_meshes(materials=True), [scenes.cornell_camera()],
                          [scenes.cornell_light()], scenes.cornell_materials())
    s = lr.RenderSettings.of(40, 32, 3)
    s.max_bounces = 4
    s.light_tracing = 0.0
    s.seed = 11
    gs = lr.GpuScene.upload(ctx, sc)
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=1 << 16, max_bounces=8, capacity=2))
    try:
        m = b.add(gs, sc, s)
        moved = (sc.arrays()["positions"] * np.float32(1.2)).astype(np.float32)
        sc.move_points(moved)
        gs.refit(ctx, moved)
        b.finish()
        got = b.read(m)
    finally:
        b.destroy()
        gs.destroy()
    fresh = lr.Renderer.create(ctx, sc, s)
    try:
        fresh.finish()
        want = fresh.read()
    finally:
        fresh.destroy()
    assert np.array_equal(_bits(got), _bits(want))


def test_refit_empty_scene(ctx):
    sc = lr.compile_scene([])
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        gs.refit(ctx, np.zeros((0, 3), np.float32))
        hits = lr.trace_rays(ctx, gs, scenes.random_rays(64))
        assert np.all(lr.hit_ids(hits) == -1)
    finally:
        gs.destroy()
