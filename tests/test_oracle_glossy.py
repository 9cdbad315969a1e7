"""The f64 oracle's OpenPBR lobes pinned on CPU before the GPU is compared with them.

- The albedo tables (tables.comp) against their closed ends -- a smooth mirror reflects
  everything, a smooth dielectric at normal incidence reflects ((eta - 1) / (eta + 1))^2 --
  and against an independent estimate of the same integral (uniform directions over the
  hemisphere, not visible normals).
- The reference's furnaces (tests/gpu/integrator.lucb:111-167): a white metal of any
  roughness, a white base under a clear coat and a closed sphere of smooth glass, under a
  white sky, are white within 2 %.
- Light tracing with glossy lobes leaves the image unbiased: the glossy Cornell box is the
  same with and without light paths within 3 sigma, and so is a glass ball under a sun
  whose light paths all start from afar (on the disk facing the sun).
"""
import math

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes, testscenes
from oracle import oracle as orc


def _ggx_albedo_uniform(mu, roughness, eta, n=400_000, seed=5):
    # E(mu) = integral of F D G2 / (4 mu) over the hemisphere, by uniform directions.
    rng = np.random.default_rng(seed)
    alpha = max(roughness * roughness, 1e-4)
    z = rng.random(n)
    phi = 2.0 * math.pi * rng.random(n)
    s = np.sqrt(1.0 - z * z)
    wi = np.stack([s * np.cos(phi), s * np.sin(phi), z], 1)
    wo = np.array([math.sqrt(1.0 - mu * mu), 0.0, mu])
    h = wi + wo
    h /= np.linalg.norm(h, axis=1, keepdims=True)
    k = (h[:, 0] / alpha) ** 2 + (h[:, 1] / alpha) ** 2 + h[:, 2] ** 2
    d = 1.0 / (math.pi * alpha * alpha * k * k)

    def lam(v):
        return 0.5 * (-1.0 + np.sqrt(1.0 + alpha * alpha * (v[..., 0] ** 2 + v[..., 1] ** 2) / v[..., 2] ** 2))

    g2 = 1.0 / (1.0 + lam(wi) + lam(wo[None, :]))
    f = 1.0
    if eta > 0:
        c = np.abs(h @ wo)
        g = np.sqrt(eta * eta - 1.0 + c * c)
        a = (g - c) / (g + c)
        b = (c * (g + c) - 1.0) / (c * (g - c) + 1.0)
        f = 0.5 * a * a * (1.0 + b * b)
    value = f * d * g2 / (4.0 * mu) * 2.0 * math.pi  # pdf 1 / (2 pi)
    return value.mean(), value.std() / math.sqrt(n)


def test_albedo_table_ends_and_independent_estimate():
    assert orc.table_albedo(1.0, 0.0, -1.0) == pytest.approx(1.0, abs=1e-6)
    assert orc.table_albedo(1.0, 0.0, 1.5) == pytest.approx(0.04, abs=1e-6)
    assert orc.table_albedo(1.0, 0.0, 2.0) == pytest.approx(1.0 / 9.0, abs=1e-6)
    for mu, r, eta in [(0.8, 0.5, -1.0), (0.5, 0.8, -1.0), (0.3, 1.0, -1.0), (0.7, 0.6, 1.5)]:
        table = orc.table_albedo(mu, r, eta)
        mc, sem = _ggx_albedo_uniform(mu, r, eta)
        # The 32 x 32 stratified grid against 400k uniform directions.
        assert abs(table - mc) <= 4.0 * sem + 2e-3, (mu, r, eta, table, mc, sem)
    t = orc.albedo_tables()
    assert t.shape == (orc.ALBEDO_TABLE_SIZE,)
    ggx = t[:1024].reshape(32, 32)  # [roughness][mu]
    assert np.all(ggx <= 1.0 + 1e-9) and np.all(ggx[31] < ggx[0] + 1e-12)
    assert np.all(np.diff(t[1024:1056]) <= 1e-12)  # the average falls with roughness


def _furnace(material, spectral, samples=16, w=32, h=24, bounces=64):
    meshes, cams = scenes.furnace_sphere(4)
    sc = lr.compile_scene(meshes, cams)
    frame = lr.ray_frame(sc.camera(), w, h)
    mean, var = orc.render(sc.arrays(), [], [material], frame, samples, bounces, spectral, background=(1.0, 1.0, 1.0))
    window = mean[h // 2 - 4:h // 2 + 4, w // 2 - 4:w // 2 + 4]
    sem = math.sqrt(var[h // 2 - 4:h // 2 + 4, w // 2 - 4:w // 2 + 4, 1].mean() / (64 * samples))
    return window.reshape(-1, 3).mean(0), sem


@pytest.mark.parametrize("kind,spectral", [("metal", True), ("metal", False), ("coat", True), ("glass", False),
                                           ("glass", True)])
def test_oracle_glossy_furnaces(kind, spectral):
    if kind == "metal":
        m = scenes.openpbr(base_color=(1.0, 1.0, 1.0), base_metalness=1.0,
                           specular_roughness=0.5 if spectral else 1.0)
    elif kind == "coat":
        m = scenes.openpbr(base_color=(1.0, 1.0, 1.0), coat_weight=1.0, coat_roughness=0.3)
    else:
        m = scenes.openpbr(base_color=(1.0, 1.0, 1.0), transmission_weight=1.0, specular_roughness=0.0)
    center, sem = _furnace(m, spectral)
    assert abs(center[1] - 1.0) <= 0.02 + 3.0 * sem, (kind, spectral, center, sem)


def test_oracle_glossy_light_tracing_is_unbiased():
    meshes, cams, lights, mats = scenes.glossy_cornell(2)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    frame = lr.ray_frame(sc.camera(), 32, 32)
    library = [lr.OpenPbr.lambert()] + mats
    a, va = orc.render(sc.arrays(), lights, library, frame, 32, 6, False, light_tracing=0.5)
    b, vb = orc.render(sc.arrays(), lights, library, frame, 32, 6, False)
    blocks = lambda x: x.reshape(4, 8, 4, 8, 3).mean((1, 3))
    sem = np.sqrt((blocks(va) + blocks(vb)) / (64 * 32))
    assert np.all(np.abs(blocks(a) - blocks(b)) <= 3.5 * sem + 1e-9), np.max(np.abs(blocks(a) - blocks(b)) / sem)


def test_oracle_light_paths_from_afar():
    # A sun with a size over a glass ball (loading.lucb:127-146): light paths start on the
    # disk facing it (no emitters of the light tree here, so all of them), and the image is
    # the camera paths' alone within 4 sigma.
    meshes, cams, lights, mats, background = scenes.caustic_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    w, h = 48, 32
    frame = lr.ray_frame(sc.camera(), w, h)
    library = [lr.OpenPbr.lambert()] + mats
    job = orc.RenderJob(sc.arrays(), lights, library, frame, 6, False, background=background, light_tracing=0.5)
    assert job.light_paths == w * h // 2 and job.desc.emitter_count == 0 and job.desc.emit_share == 1.0
    # The disk covers the casters: the glass ball of radius 0.5 at (0, 0.5, 0).
    assert job.desc.emit_radius >= 0.5 * math.sqrt(3.0) - 1e-3
    a, va = orc.render(sc.arrays(), lights, library, frame, 256, 6, False, background=background, light_tracing=0.5)
    b, vb = orc.render(sc.arrays(), lights, library, frame, 256, 6, False, background=background)
    blocks = lambda x: x.reshape(2, 16, 3, 16, 3).mean((1, 3))
    sem = np.sqrt((blocks(va) + blocks(vb)) / (256 * 256))
    assert np.all(np.abs(blocks(a) - blocks(b)) <= 4.0 * sem), np.max(np.abs(blocks(a) - blocks(b)) / sem)
    # Without a caster nothing starts from afar: no emitters, so no light paths at all.
    plain = [scenes.openpbr(base_color=(0.8, 0.8, 0.8), specular_weight=0.0)] * 3
    job = orc.RenderJob(sc.arrays(), lights, [lr.OpenPbr.lambert()] + plain, frame, 6, False, light_tracing=0.5)
    assert job.light_paths == 0 and job.desc.emit_share == 0.0


def test_oracle_cutouts():
    # integrator.lucb:170-192: the half-transparent emitting sphere shows 2.25.
    meshes, cams, lights, mats = testscenes.cutout_sphere_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    frame = lr.ray_frame(sc.camera(), 32, 32)
    mean, var = orc.render(sc.arrays(), lights, [testscenes.cutout_material()], frame, 64, 8, False)
    center = mean[12:20, 12:20, 1].mean()
    assert abs(center - testscenes.CUTOUT_SPHERE_EXPECTED) <= 0.05, center
    # integrator.lucb:292-333: a veil at opacity one half passes half the light.
    means = []
    for opacity in (0.5, 0.0):
        meshes, cams, lights, mats = testscenes.veil_scene(opacity)
        sc = lr.compile_scene(meshes, cams, lights, mats)
        frame = lr.ray_frame(sc.camera(), 32, 32)
        mean, _ = orc.render(sc.arrays(), lights, [lr.OpenPbr.lambert((0.5, 0.5, 0.5))] + mats, frame, 128, 1, False)
        means.append(mean[14:18, 14:18, 1].mean())
    assert abs(means[0] / means[1] - 0.5) <= 0.015, means


def test_oracle_dispersive_glass_furnace():
    # integrator.lucb:135-167 (kind 3): a closed sphere of smooth dispersive glass under a
    # white sky is white: its wavelengths split at the first hit and the hero carries the
    # sample (openpbr.glsl:182-194).
    m = scenes.openpbr(base_color=(1.0, 1.0, 1.0), transmission_weight=1.0, specular_roughness=0.0,
                       transmission_dispersion_scale=1.0, transmission_dispersion_abbe_number=10.0)
    center, sem = _furnace(m, True, samples=256)
    assert abs(center[1] - 1.0) <= 0.02 + 3.0 * sem, (center, sem)
