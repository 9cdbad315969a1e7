"""The integrator's own traversal against the brute force, hit for hit.

The renderer's closest-hit and shadow kernels (trace.cu) are the ones the headline
Mrays/s times. With settings.profile = 3 every pass records, per round, each ray it traced
and the triangle traversal's answer (before the analytic lights); these tests take those
records and compare them with:

- the oracle's FP32 watertight brute force over all triangles (oracle/trace.c
  `or_brute_watertight`): closest-hit ids, t, u and v bit for bit, exact-t ties going to
  the smaller id on both sides; shadow rays blocked exactly when the brute force finds a
  triangle closer than their reach;
- on the 1,048,576-triangle scene, where a brute force over every ray of a pass would take
  hours of host time, every recorded ray also against lr_trace_rays (the ray queries that
  tests/test_gpu_trace.py holds bit-exact to the brute force), and a seeded subset of each
  round directly against the brute force.

Reference: shaders/intersect_closest.comp:45-76 and intersect_shadow.comp:28-92 trace
with shaders/bvh.glsl:51-122; the acceptance rule of tests/gpu/main.lucb:61-78 asks for
equal ids, which the watertight path meets bit for bit.
"""
import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def _records(ctx, sc, settings):
    settings.profile = 3
    r = lr.Renderer.create(ctx, sc, settings)
    try:
        r.finish()
        assert r.samples_done() == settings.samples
        rounds = settings.max_bounces + 1
        return [(r.recorded_rays(k), r.recorded_rays(k, shadow=True)) for k in range(rounds)]
    finally:
        r.destroy()


def _closest_equal(a, rays, got):
    prim, t, u, v = orc.brute_watertight(a["positions"], a["indices"], a["order"], rays)
    ids = got[:, 1].view(np.int32)
    assert np.array_equal(ids, prim), f"{np.count_nonzero(ids != prim)} of {len(ids)} ids differ"
    hit = prim >= 0
    assert np.array_equal(_bits(got[hit, 0]), _bits(t[hit])), "hit distances differ"
    assert np.array_equal(_bits(got[hit, 2]), _bits(u[hit])) and np.array_equal(_bits(got[hit, 3]), _bits(v[hit]))
    return np.count_nonzero(hit)


def _shadow_equal(a, rays, got):
    traced = got[:, 0] >= 0.0
    prim, _, _, _ = orc.brute_watertight(a["positions"], a["indices"], a["order"], rays[traced])
    blocked = got[traced, 0] == 1.0
    assert np.array_equal(blocked, prim >= 0), f"{np.count_nonzero(blocked != (prim >= 0))} shadow rays differ"
    return np.count_nonzero(traced)


@pytest.mark.parametrize("spectral,refill", [(True, 0), (False, 0), (True, 16)])
def test_cornell_pass_hits_equal_brute_force(ctx, spectral, refill, monkeypatch):
    # The 34-triangle Cornell box with its rect light at 256 x 256, one sample, eight
    # bounces: every recorded ray of every round, closest and shadow, light tracing on;
    # grid-stride traversal, and warps refilling at 16 idle lanes.
    monkeypatch.setenv("LUCE_RENDER_B200_REFILL", str(refill))
    sc = lr.compile_scene(scenes.cornell_meshes(True), [scenes.cornell_camera()], [scenes.cornell_light()],
                          scenes.cornell_materials())
    a = sc.arrays()
    s = lr.RenderSettings.of(256, 256, 1)
    s.spectral = 1 if spectral else 0
    s.max_bounces = 8
    try:
        records = _records(ctx, sc, s)
        (rays0, hits0), _ = records[0]
        assert len(rays0) >= 256 * 256  # the camera's rays, then the light paths'
        closest = shadow = 0
        for (rays, hits), (srays, shits) in records:
            if len(rays):
                closest += len(rays)
                _closest_equal(a, rays, hits)
            if len(srays):
                shadow += _shadow_equal(a, srays, shits)
        assert closest > 2 * 256 * 256 and shadow > 256 * 256, (closest, shadow)
    finally:
        sc.close()


@pytest.mark.parametrize("refill", [0, 8])
def test_million_triangle_pass_hits_equal_queries_and_brute_force(ctx, refill, monkeypatch):
    # The 1,048,576-triangle workload at 320 x 240, one sample, six bounces, spectral:
    # every ray of every round against lr_trace_rays; 4,096 rays of rounds 0 and 1 and
    # 4,096 shadow rays of round 0 against the brute force. Grid-stride traversal, and
    # warps refilling at 8 idle lanes.
    monkeypatch.setenv("LUCE_RENDER_B200_REFILL", str(refill))
    meshes, mats, lights, cam = scenes.incoherent_scene()
    sc = lr.compile_scene(meshes, [cam], lights, mats)
    a = sc.arrays()
    gs = lr.GpuScene.upload(ctx, sc)
    s = lr.RenderSettings.of(320, 240, 1)
    s.max_bounces = 6
    rng = np.random.default_rng(0x5EED)
    try:
        records = _records(ctx, sc, s)
        total = 0
        for k, ((rays, hits), (srays, shits)) in enumerate(records):
            if len(rays):
                total += len(rays)
                want = lr.trace_rays(ctx, gs, rays)
                assert np.array_equal(_bits(hits), _bits(want)), f"round {k}: closest hits differ from lr_trace_rays"
            traced = shits[:, 0] >= 0.0
            if np.any(traced):
                anyh = lr.trace_rays(ctx, gs, srays[traced], any_hit=True)
                assert np.array_equal(shits[traced, 0] == 1.0, lr.hit_ids(anyh) >= 0), f"round {k}: shadows differ"
            if k < 2:
                pick = rng.choice(len(rays), size=min(4096, len(rays)), replace=False)
                assert _closest_equal(a, rays[pick], hits[pick]) > 0
            if k == 0:
                pick = rng.choice(np.flatnonzero(traced), size=min(4096, int(traced.sum())), replace=False)
                _shadow_equal(a, srays[pick], shits[pick])
        assert total >= 65536 * 2, total
    finally:
        gs.destroy()
        sc.close()
