"""Dome lights through the C ABI (shaders/lights.glsl:89-174, shade_miss.comp:12-51,
light_emit.comp:31-62, src/render/environment.lucb): a lat-long image around the scene,
sampled by importance (rows, then the row's texels), or a uniform colour without one.

- The reference's closed forms (tests/gpu/integrator.lucb:495-582): the dome furnace (a
  white sphere under a white dome, white within 1 % over the frame and 2 % on the sphere)
  and the dome sun (a grey floor under a sky whose sun is 1/512 of its texels reflects
  albedo / pi x the image's irradiance within 2 %), spectral and RGB.
- The f64 oracle over the same samples on a glossy scene under the sun sky's dome, or a dome
  of one colour, with light tracing (light paths from afar start on the disk facing the
  dome): 8x8-block means within 3 sigma and most pixels within f32 rounding.
"""
import math

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes, testscenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _render(ctx, sc, w, h, spp, bounces, spectral, material, tracing=0.0, background=(0.0, 0.0, 0.0)):
    s = lr.RenderSettings.of(w, h, spp)
    s.spectral = 1 if spectral else 0
    s.max_bounces = bounces
    s.light_tracing = tracing
    s.background = background
    s.c.material = material
    r = lr.Renderer.create(ctx, sc, s)
    try:
        r.finish()
        assert r.samples_done() == spp
        return r.read()
    finally:
        r.destroy()


@pytest.mark.parametrize("spectral", [False, True])
def test_dome_furnace(ctx, spectral):
    meshes, cams, lights, mats = testscenes.dome_furnace_scene(4)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    white = lr.OpenPbr.standard()
    white.base_color[:] = [1.0, 1.0, 1.0]
    img = _render(ctx, sc, 64, 48, 64, 64, spectral, white)
    mean = img[..., :3].reshape(-1, 3).mean(0)
    center = img[16:32, 24:40, :3].reshape(-1, 3).mean(0)
    # tests/gpu/integrator.lucb:515.
    assert abs(mean[1] - 1.0) <= 0.01, mean
    assert abs(center[1] - 1.0) <= 0.02 and abs(center[0] - 1.0) <= 0.03, center


@pytest.mark.parametrize("spectral", [False, True])
def test_dome_sun(ctx, spectral):
    meshes, cams, lights, mats, irradiance = testscenes.dome_sun_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    img = _render(ctx, sc, 32, 32, 256, 1, spectral, lr.OpenPbr.lambert((0.5, 0.5, 0.5)))
    measured = img[..., :3].reshape(-1, 3).mean(0)
    expected = 0.5 / math.pi * irradiance
    # tests/gpu/integrator.lucb:581.
    assert abs(measured[1] / expected - 1.0) < 0.02, (measured, expected)


def _blocks(x, b):
    h, w = x.shape[:2]
    return x[: h // b * b, : w // b * b].reshape(h // b, b, w // b, b, -1)


@pytest.mark.parametrize("spectral,textured", [(False, True), (True, True), (True, False)])
def test_gpu_matches_f64_oracle_dome(ctx, spectral, textured):
    # The sun sky's dome, or a dome of one colour (sampled uniformly over the sphere).
    meshes, cams, lights, mats, background = scenes.caustic_scene()
    sky, _ = testscenes.sun_sky()
    lights = [lr.light(lr.LIGHT_DOME, rotation=(0.0, 0.7, 0.0), intensity=0.5, image=sky if textured else None,
                       color=(1.0, 0.9, 0.7))]
    sc = lr.compile_scene(meshes, cams, lights, mats)
    w, h, spp, bounces = 48, 32, 32, 6
    library = [lr.OpenPbr.lambert()] + mats
    img = _render(ctx, sc, w, h, spp, bounces, spectral, library[0], tracing=0.5, background=background)
    frame = lr.ray_frame(sc.camera(), w, h)
    job = orc.RenderJob(sc.arrays(), lights, library, frame, bounces, spectral, background=background,
                        light_tracing=0.5)
    # The dome starts light paths on the disk facing it (the glass ball casts caustics).
    assert job.light_paths > 0 and job.desc.emit_share > 0.0
    mean, var, _ = job.traced(spp)
    mean, var = mean.reshape(h, w, 3), var.reshape(h, w, 3)
    gpu = img[..., :3].astype(np.float64)
    g = _blocks(gpu, 8).mean((1, 3))
    o = _blocks(mean, 8).mean((1, 3))
    sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
    assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), np.max(np.abs(g - o) / (sem + 1e-12))
    relative = np.abs(gpu - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.mean(relative < 1e-3) >= 0.95, np.mean(relative < 1e-3)


def test_reload_with_another_dome_image(ctx):
    # Renderer.reload with the same geometry under another sky (the sun moved, a brighter
    # dome), passes in flight: the image equals a renderer made for the new sky, bit for bit.
    meshes, cams, _, mats, background = scenes.caustic_scene()
    sky, _ = testscenes.sun_sky()
    moved_sun = np.full_like(sky, 0.5)
    moved_sun[4:6, 10:12] = 300.0
    s = lr.RenderSettings.of(32, 24, 6)
    s.spectral = 1
    s.max_bounces = 4
    s.light_tracing = 0.5
    s.background = background
    s.c.material = lr.OpenPbr.lambert()

    def compiled(image, intensity):
        dome = lr.light(lr.LIGHT_DOME, rotation=(0.0, 0.7, 0.0), intensity=intensity, image=image)
        return lr.compile_scene(meshes, cams, [dome], mats)

    first, second = compiled(sky, 0.5), compiled(moved_sun, 0.8)
    r = lr.Renderer.create(ctx, first, s)
    try:
        r.advance()
        r.advance()
        r.reload(second, s)
        r.finish()
        got = r.read()
    finally:
        r.destroy()
    fresh = lr.Renderer.create(ctx, second, s)
    try:
        fresh.finish()
        want = fresh.read()
    finally:
        fresh.destroy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
