"""Dome lights in the f64 oracle, pinned on CPU before the GPU is compared with them
(shaders/lights.glsl:89-174, src/render/environment.lucb, src/render/lights.lucb:61-99).

- The image's sampling tables as environment_of builds them: every row's cumulative
  weights and the rows' own rise to 1, the weights' sum is the texels' total, and the
  dome's record says where the texels and weights start.
- The reference's closed forms (tests/gpu/integrator.lucb:495-582): a white sphere under a
  white dome with no image is white (the furnace through the dome's light samples and BSDF
  hits under MIS); a grey floor under a dome whose image holds a small sun 400 times
  brighter than the sky reflects albedo / pi x the image's irradiance.
"""
import math
import struct

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import testscenes
from oracle import oracle as orc


def _bits(x) -> int:
    return struct.unpack("<I", struct.pack("<f", float(x)))[0]


def test_environment_tables():
    sky, _ = testscenes.sun_sky(64, 32)
    sky[0, :] = 0.0  # an empty row: uniform within it
    lights = [lr.light(lr.LIGHT_RECT, position=(0.0, 2.0, 0.0)),
              lr.light(lr.LIGHT_DOME, intensity=2.0, image=sky),
              lr.light(lr.LIGHT_DOME, intensity=1.0)]
    rows, power, n = orc.pack_lights(lights, 3.0, with_image=True)
    assert n == 3
    records = rows[: n * 28].reshape(n, 28)
    dome, plain = records[1], records[2]
    assert dome[3] == 4.0 and plain[3] == 4.0
    assert _bits(plain[7]) == 0  # a dome without an image shines its colour evenly
    texel_base, width, height, cdf_base = (_bits(dome[7]), _bits(dome[11]), _bits(dome[15]), _bits(dome[27]))
    assert (width, height) == (64, 32) and texel_base == n * 7
    texels = rows[texel_base * 4: texel_base * 4 + width * height * 4].reshape(height, width, 4)
    cdf = rows[cdf_base: cdf_base + width * height + height]
    per_row = cdf[: width * height].reshape(height, width)
    assert np.all(np.diff(per_row, axis=1) >= 0.0) and np.allclose(per_row[:, -1], 1.0, atol=1e-6)
    assert np.allclose(per_row[0], (np.arange(width) + 1) / width)  # the empty row
    assert np.all(np.diff(cdf[width * height:]) >= 0.0) and cdf[-1] == pytest.approx(1.0, abs=1e-6)
    # Weights: luminance x sin theta of the ACEScg texels; their sum in the record.
    sin_theta = np.sin(np.pi * (np.arange(height) + 0.5) / height)
    lum = texels[..., :3].astype(np.float64) @ np.array([0.2722287168, 0.6740817658, 0.0536895174])
    assert np.allclose(texels[..., 3], lum * sin_theta[:, None], rtol=1e-5, atol=1e-7)
    assert dome[0] == pytest.approx(texels[..., 3].astype(np.float64).sum(), rel=1e-5)
    # Power by the mean luminance over the sphere (the textured dome) or 1 (the plain one),
    # shares of the domes' power.
    mean = (lum * sin_theta[:, None]).sum() / (sin_theta.sum() * width)
    expected = np.array([2.0 * mean, 1.0]) * math.pi ** 2 * 9.0
    assert power == pytest.approx(expected.sum(), rel=1e-5)
    assert dome[25] == pytest.approx(expected[0] / expected.sum(), rel=1e-5)
    assert plain[26] == pytest.approx(1.0, abs=1e-6)


@pytest.mark.parametrize("spectral", [False, True])
def test_oracle_dome_furnace(spectral):
    meshes, cams, lights, mats = testscenes.dome_furnace_scene(3)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    w, h = 32, 24
    frame = lr.ray_frame(sc.camera(), w, h)
    white = lr.OpenPbr.standard()
    white.base_color[:] = [1.0, 1.0, 1.0]
    mean, _ = orc.render(sc.arrays(), lights, [white], frame, 16, 64, spectral)
    # tests/gpu/integrator.lucb:515: the frame within 1 %, the sphere within 2 %.
    assert abs(mean[..., 1].mean() - 1.0) <= 0.01, mean[..., 1].mean()
    center = mean[8:16, 12:20].reshape(-1, 3).mean(0)
    assert np.all(np.abs(center - 1.0) <= 0.02), center


@pytest.mark.parametrize("spectral", [False, True])
def test_oracle_dome_sun(spectral):
    meshes, cams, lights, mats, irradiance = testscenes.dome_sun_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    frame = lr.ray_frame(sc.camera(), 32, 32)
    mean, _ = orc.render(sc.arrays(), lights, [lr.OpenPbr.lambert((0.5, 0.5, 0.5))], frame, 256, 1, spectral)
    expected = 0.5 / math.pi * irradiance
    # tests/gpu/integrator.lucb:581: within 2 %.
    assert abs(mean[..., 1].mean() / expected - 1.0) < 0.02, (mean[..., 1].mean(), expected)


@pytest.mark.parametrize("textured", [True, False])
def test_oracle_dome_light_paths_are_unbiased(textured):
    # Light paths from afar start on the disk facing the dome (its image by importance, or
    # uniform over the sphere for a dome of one colour); with and without them, the image of
    # glossy objects under the dome has the same mean.
    from luce_render_b200 import scenes
    meshes, cams, _, mats, background = scenes.caustic_scene()
    sky, _ = testscenes.sun_sky()
    lights = [lr.light(lr.LIGHT_DOME, rotation=(0.0, 0.7, 0.0), intensity=0.5, image=sky if textured else None)]
    sc = lr.compile_scene(meshes, cams, lights, mats)
    w, h, spp = 32, 24, 64
    frame = lr.ray_frame(sc.camera(), w, h)
    library = [lr.OpenPbr.lambert()] + mats
    means = []
    for tracing in (0.0, 0.5):
        job = orc.RenderJob(sc.arrays(), lights, library, frame, 6, False, background=background,
                            light_tracing=tracing)
        assert (job.light_paths > 0) == (tracing > 0.0)
        if tracing > 0.0:
            assert job.desc.emit_share == pytest.approx(1.0)  # no emitters: every light path from afar
            mean, var, _ = job.traced(spp)
        else:
            mean, var, _ = job.region(spp, 0, 0, w * h)
        means.append((mean.mean(0), np.sqrt(var.mean(0) / (w * h * spp))))
    (a, sa), (b, sb) = means
    assert np.all(np.abs(a - b) <= 4.0 * np.sqrt(sa ** 2 + sb ** 2)), (a, b, sa, sb)
