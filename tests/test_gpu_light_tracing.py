"""Light tracing (shaders/connect.glsl, light_paths.glsl, light_emit.comp) through the C
ABI: light paths from the light tree's emitters, connected to the camera and splatted,
with the camera paths' two techniques weighed against them by the power heuristic.

- The f64 oracle's restatement of the same estimator over the same samples: 8x8-block
  means within 3 sigma of a block mean's standard error.
- Closed forms (tests/gpu/integrator.lucb): the area light and emissive quad within the
  reference's 2 %, the emitting enclosure within 3 sigma.
- The three-technique estimator is unbiased: the same image as camera paths alone within
  3 sigma, and splats add in fixed point, so a render repeats bit for bit.
"""
import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes, testscenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _render(ctx, meshes, cams, lights, mats, w, h, spp, bounces, spectral, tracing, material=None, pool=0):
    sc = lr.compile_scene(meshes, cams, lights, mats)
    s = lr.RenderSettings.of(w, h, spp)
    s.spectral = 1 if spectral else 0
    s.max_bounces = bounces
    s.light_tracing = tracing
    s.pool = pool
    s.c.material = material if material is not None else lr.OpenPbr.lambert()
    r = lr.Renderer.create(ctx, sc, s)
    try:
        r.finish()
        assert r.samples_done() == spp
        return sc, r.read(), r.stats()
    finally:
        r.destroy()


def _blocks(x, b):
    h, w = x.shape[:2]
    return x[: h // b * b, : w // b * b].reshape(h // b, b, w // b, b, -1)


def _cornell():
    return (scenes.cornell_meshes(True), [scenes.cornell_camera()], [scenes.cornell_light()],
            scenes.cornell_materials())


@pytest.mark.parametrize("spectral", [False, True])
def test_matches_f64_oracle_cornell(ctx, spectral):
    w = h = 48
    spp, bounces = 16, 6
    meshes, cams, lights, mats = _cornell()
    sc, img, st = _render(ctx, meshes, cams, lights, mats, w, h, spp, bounces, spectral, 0.5)
    frame = lr.ray_frame(sc.camera(), w, h)
    job = orc.RenderJob(sc.arrays(), lights, [lr.OpenPbr.lambert()] + mats, frame, bounces, spectral,
                        light_tracing=0.5)
    mean, var, _ = job.traced(spp)
    camera_part, _, _ = job.region(spp, 0, 0, w * h)
    mean, var, camera_part = (x.reshape(h, w, 3) for x in (mean, var, camera_part))
    gpu = img[..., :3].astype(np.float64)
    g = _blocks(gpu, 8).mean((1, 3))
    o = _blocks(mean, 8).mean((1, 3))
    sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
    assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), np.max(np.abs(g - o) / (sem + 1e-12))
    # Both draw the same samples: nearly every pixel agrees to f32 rounding, splats included
    # (here about 30 % of the image: light paths carry much of what the box's walls bounce).
    relative = np.abs(gpu - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.mean(relative < 1e-3) >= 0.99, np.mean(relative < 1e-3)
    assert (mean - camera_part).sum() / mean.sum() > 0.1
    # Light paths were traced: more closest rays than the camera paths alone make.
    _, _, st0 = _render(ctx, meshes, cams, lights, mats, w, h, spp, bounces, spectral, 0.0)
    assert st.closest_rays > st0.closest_rays and st.shaded == st0.shaded == w * h * spp


@pytest.mark.parametrize("spectral", [False, True])
def test_closed_forms(ctx, spectral):
    for scene in (testscenes.area_light_scene, testscenes.emissive_quad_scene):
        meshes, cams, lights, mats = scene()
        _, img, _ = _render(ctx, meshes, cams, lights, mats, 32, 32, 256, 1, spectral, 0.5,
                            material=lr.OpenPbr.lambert((0.5, 0.5, 0.5)))
        measured = img[14:18, 14:18, :3].reshape(-1, 3).mean(0)
        # integrator.lucb:765: Y within 2 %
        assert abs(measured[1] / testscenes.AREA_LIGHT_EXPECTED - 1.0) <= 0.02, (scene.__name__, measured)
    # The emitting enclosure: every triangle an emitter of the light tree.
    _, img, _ = _render(ctx, scenes.furnace_meshes(4), [lr.camera((0.0, 0.0, 0.0))], [], [], 32, 32, 64, 8, spectral,
                        0.5, material=scenes.furnace_material(0.8, 1.0))
    v = img[..., :3].reshape(-1, 3).astype(np.float64)
    expected = (1.0 - 0.8 ** 9) / 0.2
    sem = v.std(0) / np.sqrt(len(v))
    assert np.all(np.abs(v.mean(0) - expected) <= 3.0 * sem + 2e-4 * expected), (v.mean(0), sem)


def test_unbiased_against_camera_paths_alone(ctx):
    w = h = 48
    spp = 64
    meshes, cams, lights, mats = _cornell()
    _, with_lt, _ = _render(ctx, meshes, cams, lights, mats, w, h, spp, 6, True, 0.5)
    sc, without, _ = _render(ctx, meshes, cams, lights, mats, w, h, spp, 6, True, 0.0)
    # Per-block spread from the oracle's per-sample variance of the camera-only image.
    frame = lr.ray_frame(sc.camera(), w, h)
    _, var = orc.render(sc.arrays(), lights, [lr.OpenPbr.lambert()] + mats, frame, 16, 6, True)
    sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
    a = _blocks(with_lt[..., :3].astype(np.float64), 8).mean((1, 3))
    b = _blocks(without[..., :3].astype(np.float64), 8).mean((1, 3))
    assert np.all(np.abs(a - b) <= 3.0 * np.sqrt(2.0) * sem + 1e-6), np.max(np.abs(a - b) / (sem + 1e-12))


def test_splats_repeat_bit_for_bit(ctx):
    meshes, cams, lights, mats = _cornell()
    runs = [_render(ctx, meshes, cams, lights, mats, 40, 30, 4, 5, True, 1.0, pool=700)[1] for _ in range(2)]
    assert np.array_equal(runs[0].view(np.uint32), runs[1].view(np.uint32))
    # Light paths land where the camera paths' pixels did not reach on their own.
    assert np.all(np.isfinite(runs[0]))
