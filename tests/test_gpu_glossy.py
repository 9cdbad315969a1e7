"""OpenPBR's glossy lobes through the C ABI: GGX specular over EON diffuse with
Kulla-Conty compensation, F82-tint metal, the coat with darkening, rough refraction into
and out of transmissive objects (shaders/openpbr.glsl, microfacet.glsl, tables.comp).

- The albedo tables made on the device against the oracle's f64 tables (same nodes, same
  32 x 32 grid): within f32 rounding.
- The reference's furnaces (tests/gpu/integrator.lucb:111-167): under a white sky a white
  metal of any roughness, a white base under a clear coat and a closed sphere of smooth
  glass are white within the reference's 2 %.
- The f64 oracle's restatement over the same samples, on the benchmark's layout (coat,
  glass, gold, rough plastic): 8x8-block means within 3 sigma, camera paths alone and with
  light tracing, RGB and spectral; and a glass ball under a sun, its light paths starting
  from afar (lights.glsl:283-308).
"""
import math

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes, testscenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _render(ctx, sc, w, h, spp, bounces, spectral, material=None, background=(0.0, 0.0, 0.0), tracing=0.0, seed=1):
    s = lr.RenderSettings.of(w, h, spp)
    s.spectral = 1 if spectral else 0
    s.max_bounces = bounces
    s.light_tracing = tracing
    s.seed = seed
    s.background = background
    s.c.material = material if material is not None else lr.OpenPbr.lambert()
    r = lr.Renderer.create(ctx, sc, s)
    try:
        r.finish()
        assert r.samples_done() == spp
        return r.read()
    finally:
        r.destroy()


def _blocks(x, b):
    h, w = x.shape[:2]
    return x[: h // b * b, : w // b * b].reshape(h // b, b, w // b, b, -1)


def test_albedo_tables_match_oracle(ctx):
    gpu = lr.albedo_tables(ctx).astype(np.float64)
    ref = orc.albedo_tables()
    assert gpu.shape == ref.shape
    assert np.max(np.abs(gpu - ref)) <= 2e-5, np.max(np.abs(gpu - ref))


FURNACES = [("metal", True, 0.5), ("metal", False, 1.0), ("coat", True, 0.3), ("coat", False, 0.3),
            ("glass", False, 0.0), ("glass", True, 0.0)]


@pytest.mark.parametrize("kind,spectral,roughness", FURNACES)
def test_glossy_furnaces(ctx, kind, spectral, roughness):
    if kind == "metal":
        m = scenes.openpbr(base_color=(1.0, 1.0, 1.0), base_metalness=1.0, specular_roughness=roughness)
    elif kind == "coat":
        m = scenes.openpbr(base_color=(1.0, 1.0, 1.0), coat_weight=1.0, coat_roughness=roughness)
    else:
        m = scenes.openpbr(base_color=(1.0, 1.0, 1.0), transmission_weight=1.0, specular_roughness=roughness)
    meshes, cams = scenes.furnace_sphere(4)
    sc = lr.compile_scene(meshes, cams)
    img = _render(ctx, sc, 64, 48, 64, 64, spectral, material=m, background=(1.0, 1.0, 1.0))
    center = img[16:32, 24:40, :3].reshape(-1, 3).mean(0)
    # tests/gpu/integrator.lucb:131 and :165: the sphere's centre within 2 %.
    assert abs(center[1] - 1.0) <= 0.02, (kind, spectral, center)
    # and the whole frame, sky and sphere, stays white on average
    assert abs(img[..., 1].mean() - 1.0) <= 0.02, img[..., 1].mean()


def _oracle_case(ctx, spectral, tracing, w, h, spp, bounces):
    meshes, cams, lights, mats = scenes.glossy_cornell(2)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    img = _render(ctx, sc, w, h, spp, bounces, spectral, tracing=tracing)
    frame = lr.ray_frame(sc.camera(), w, h)
    mean, var = orc.render(sc.arrays(), lights, [lr.OpenPbr.lambert()] + mats, frame, spp, bounces, spectral,
                           light_tracing=tracing)
    return img[..., :3].astype(np.float64), mean, var


@pytest.mark.parametrize("spectral", [False, True])
def test_gpu_matches_f64_oracle_glossy_cornell(ctx, spectral):
    w = h = 64
    spp = 16
    gpu, mean, var = _oracle_case(ctx, spectral, 0.0, w, h, spp, 8)
    g = _blocks(gpu, 8).mean((1, 3))
    o = _blocks(mean, 8).mean((1, 3))
    sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
    assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), np.max(np.abs(g - o) / (sem + 1e-12))
    # The same samples: most pixels agree to f32 rounding (a mirror or glass chain can
    # part where a ray grazes an edge).
    relative = np.abs(gpu - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.mean(relative < 1e-3) >= 0.95, np.mean(relative < 1e-3)


@pytest.mark.parametrize("spectral", [False, True])
def test_gpu_matches_f64_oracle_glossy_light_tracing(ctx, spectral):
    w = h = 48
    spp = 16
    gpu, mean, var = _oracle_case(ctx, spectral, 0.5, w, h, spp, 6)
    g = _blocks(gpu, 8).mean((1, 3))
    o = _blocks(mean, 8).mean((1, 3))
    sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
    assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), np.max(np.abs(g - o) / (sem + 1e-12))
    relative = np.abs(gpu - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.mean(relative < 1e-3) >= 0.95, np.mean(relative < 1e-3)


def test_glossy_light_tracing_is_unbiased(ctx):
    # With and without light paths the glossy box's image has the same mean. Camera paths
    # alone find the glass ball's caustic rarely (a heavy tail), light paths often, so the
    # two spread differently: sixteen seeds of each give every 16x16 block's mean and its
    # standard error from the seeds' spread.
    meshes, cams, lights, mats = scenes.glossy_cornell(2)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    w = h = 32
    spp, seeds = 64, 16
    luma = np.array([0.2722287168, 0.6740817658, 0.0536895174])

    def blocks(tracing):
        imgs = np.stack([_render(ctx, sc, w, h, spp, 6, False, tracing=tracing, seed=1 + k)[..., :3]
                         for k in range(seeds)]).astype(np.float64)
        b = (imgs @ luma).reshape(seeds, 2, 16, 2, 16).mean((2, 4))
        return b.mean(0), b.std(0, ddof=1) / math.sqrt(seeds)

    traced, se_traced = blocks(0.5)
    camera, se_camera = blocks(0.0)
    assert np.all(np.abs(traced - camera) <= 4.0 * np.sqrt(se_traced ** 2 + se_camera ** 2) + 1e-6), (traced, camera)
    # Light paths carry the caustic with less noise than camera paths alone.
    assert se_traced.mean() < se_camera.mean()


@pytest.mark.parametrize("spectral", [False, True])
def test_gpu_matches_f64_oracle_light_paths_from_afar(ctx, spectral):
    # A sun with a size and a glass ball: light paths start on the disk facing the sun,
    # camera paths weigh their BSDF rays to the sun and their light samples against them.
    meshes, cams, lights, mats, background = scenes.caustic_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    w, h, spp = 48, 32, 32
    img = _render(ctx, sc, w, h, spp, 6, spectral, background=background, tracing=0.5)
    frame = lr.ray_frame(sc.camera(), w, h)
    job = orc.RenderJob(sc.arrays(), lights, [lr.OpenPbr.lambert()] + mats, frame, 6, spectral, background=background,
                        light_tracing=0.5)
    assert job.light_paths > 0 and job.desc.emitter_count == 0
    mean, var, _ = job.traced(spp)
    camera_part, _, _ = job.region(spp, 0, 0, w * h)
    mean, var, camera_part = (x.reshape(h, w, 3) for x in (mean, var, camera_part))
    gpu = img[..., :3].astype(np.float64)
    g = _blocks(gpu, 8).mean((1, 3))
    o = _blocks(mean, 8).mean((1, 3))
    sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
    assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), np.max(np.abs(g - o) / (sem + 1e-12))
    relative = np.abs(gpu - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.mean(relative < 1e-3) >= 0.95, np.mean(relative < 1e-3)
    # The light paths from afar carry part of the image (the caustic under the ball).
    assert (mean - camera_part).sum() / mean.sum() > 0.02


@pytest.mark.parametrize("spectral", [False, True])
def test_cutouts(ctx, spectral):
    # integrator.lucb:170-192: the half-transparent emitting sphere in the dark shows 2.25
    # (the reference's tolerance 0.05).
    meshes, cams, lights, mats = testscenes.cutout_sphere_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    img = _render(ctx, sc, 32, 32, 256, 8, spectral, material=testscenes.cutout_material())
    center = img[12:20, 12:20, 1].mean()
    assert abs(center - testscenes.CUTOUT_SPHERE_EXPECTED) <= 0.05, center
    # integrator.lucb:292-333: a veil at opacity one half passes half the light (0.015).
    means = []
    for opacity in (0.5, 0.0):
        meshes, cams, lights, mats = testscenes.veil_scene(opacity)
        sc = lr.compile_scene(meshes, cams, lights, mats)
        img = _render(ctx, sc, 32, 32, 256, 1, spectral, material=lr.OpenPbr.lambert((0.5, 0.5, 0.5)))
        means.append(img[14:18, 14:18, 1].mean())
    assert abs(means[0] / means[1] - 0.5) <= 0.015, means


def test_cutouts_match_f64_oracle(ctx):
    # The veil over the floor at depth 3 (rays pass through at the same bounce, shadow rays
    # walk through), with light tracing: 8x8-block means within 3 sigma of the oracle's.
    meshes, cams, lights, mats = testscenes.veil_scene(0.5)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    w, h, spp = 48, 32, 32
    base = lr.OpenPbr.lambert((0.5, 0.5, 0.5))
    for tracing in (0.0, 0.5):
        img = _render(ctx, sc, w, h, spp, 3, False, material=base, tracing=tracing)
        frame = lr.ray_frame(sc.camera(), w, h)
        mean, var = orc.render(sc.arrays(), lights, [base] + mats, frame, spp, 3, False, light_tracing=tracing)
        g = _blocks(img[..., :3].astype(np.float64), 8).mean((1, 3))
        o = _blocks(mean, 8).mean((1, 3))
        sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
        assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), (tracing, np.max(np.abs(g - o) / (sem + 1e-12)))


def test_dispersion(ctx):
    # integrator.lucb:135-167 (kind 3, 1,024 samples): dispersive glass under a white sky
    # stays white within 2 %; and over the benchmark's box, against the oracle's image.
    m = scenes.openpbr(base_color=(1.0, 1.0, 1.0), transmission_weight=1.0, specular_roughness=0.0,
                       transmission_dispersion_scale=1.0, transmission_dispersion_abbe_number=10.0)
    meshes, cams = scenes.furnace_sphere(4)
    sc = lr.compile_scene(meshes, cams)
    img = _render(ctx, sc, 64, 48, 1024, 64, True, material=m, background=(1.0, 1.0, 1.0))
    center = img[16:32, 24:40, :3].reshape(-1, 3).mean(0)
    assert abs(center[1] - 1.0) <= 0.02, center
    meshes, cams, lights, mats = scenes.glossy_cornell(2)
    mats = list(mats)
    mats[4] = m  # the glass ball disperses
    sc = lr.compile_scene(meshes, cams, lights, mats)
    w = h = 48
    spp = 32
    for tracing in (0.0, 0.5):
        img = _render(ctx, sc, w, h, spp, 6, True, tracing=tracing)
        frame = lr.ray_frame(sc.camera(), w, h)
        mean, var = orc.render(sc.arrays(), lights, [lr.OpenPbr.lambert()] + mats, frame, spp, 6, True,
                               light_tracing=tracing)
        g = _blocks(img[..., :3].astype(np.float64), 8).mean((1, 3))
        o = _blocks(mean, 8).mean((1, 3))
        sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
        assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), (tracing, np.max(np.abs(g - o) / (sem + 1e-12)))
