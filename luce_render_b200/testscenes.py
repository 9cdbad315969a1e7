"""Scenes of the reference's closed-form integrator checks (tests/gpu/integrator.lucb),
rebuilt from this package's own primitives: a 20 x 20 floor of 8 divisions under a
1 x 1 light at height 1, seen from the side; the same light as an emissive quad; a
coloured (or blackbody) 2 x 2 light over a white floor; cut-outs; and dome lights."""
from __future__ import annotations

import math

import numpy as np

from . import (LIGHT_DOME, LIGHT_RECT, MeshData, OpenPbr, camera, light, placement)
from .scenes import grid


def corner_irradiance(x: float, y: float, h: float) -> float:
    """Irradiance under the corner of an x by y rectangle of radiance 1 at height h
    (integrator.lucb:252-255)."""
    a = math.sqrt(x * x + h * h)
    b = math.sqrt(y * y + h * h)
    return 0.5 * (x / a * math.atan(y / a) + y / b * math.atan(x / b))


AREA_LIGHT_EXPECTED = 0.5 / math.pi * 4.0 * 4.0 * corner_irradiance(0.5, 0.5, 1.0)


def _floor():
    p, t, f = grid(20.0, 8)
    return MeshData(p, t, faces=f, face_count=64)


def side_camera():
    """At (0, 0.5, 3), pitched down toward the origin, 200 mm on a 36 mm back."""
    pitch = -math.atan2(0.5, 3.0)
    return camera((0.0, 0.5, 3.0), (pitch, 0.0, 0.0), focal_length=200.0, horizontal_aperture=36.0)


def area_light_scene():
    """integrator.lucb:743-769: a 1 x 1 rect light of radiance 4 at height 1 over the floor."""
    lamp = light(LIGHT_RECT, position=(0.0, 1.0, 0.0), rotation=(-0.5 * math.pi, 0.0, 0.0), intensity=4.0,
                 width=1.0, height=1.0, normalize=False, visible=False)
    return [_floor()], [side_camera()], [lamp], []


def emissive_quad_scene():
    """integrator.lucb:259-289: the same square as an emissive mesh (luminance 4, base
    weight 0), sampled through the light tree."""
    p, t, f = grid(1.0, 1)
    glow = OpenPbr.lambert((0.8, 0.8, 0.8), emission=4.0)
    glow.base_weight = 0.0
    quad = MeshData(p, t, faces=f, face_count=1, face_materials=[1], transform=placement((0.0, 1.0, 0.0)))
    return [_floor(), quad], [side_camera()], [], [glow]


def colored_light_scene(color=(1.0, 0.4, 0.1), kelvin: float = 0.0):
    """integrator.lucb:773-798: a 2 x 2 light of intensity 10 (normalized) at height 2."""
    pitch = -math.atan2(2.0, 4.0)
    cam = camera((0.0, 2.0, 4.0), (pitch, 0.0, 0.0), focal_length=35.0, horizontal_aperture=36.0)
    lamp = light(LIGHT_RECT, position=(0.0, 2.0, 0.0), rotation=(-0.5 * math.pi, 0.0, 0.0), color=color,
                 intensity=10.0, temperature=kelvin, width=2.0, height=2.0, normalize=True, visible=False)
    return [_floor()], [cam], [lamp], []


def cutout_sphere_scene():
    """integrator.lucb:170-192: a sphere emitting 3 nits at opacity one half, in the dark,
    seen from (0, 1, 4) through 100 mm: half the rays stop at its front and see 3, a
    quarter pass to its back face and see 3 there, so it shows 2.25. The sphere is this
    package's icosphere (level 4); its material is the default, so the settings carry it
    (cutout_material)."""
    from .scenes import icosphere
    p, t, n = icosphere(4, 1.0)
    cam = camera((0.0, 1.0, 4.0), (-math.atan2(1.0, 4.0), 0.0, 0.0), focal_length=100.0, horizontal_aperture=36.0)
    return [MeshData(p, t, normals=n)], [cam], [], []


CUTOUT_SPHERE_EXPECTED = 2.25


def cutout_material(opacity: float = 0.5, emission: float = 3.0) -> OpenPbr:
    m = OpenPbr.lambert((0.0, 0.0, 0.0), emission=emission)
    m.geometry_opacity = opacity
    return m


def veil_scene(opacity: float):
    """integrator.lucb:292-333: the area light's floor under a 3 x 3 veil at height 0.5
    (opacity `opacity`, base weight 0, library material 1), seen from below the veil at
    (0, 0.3, 3): at opacity one half the floor under the light gets exactly half of what it
    gets through a fully transparent veil (shadow rays walk through cut-outs keeping
    1 - opacity, BSDF rays pass at random, MIS weighs both)."""
    p, t, f = grid(3.0, 1)
    veil = OpenPbr.lambert((0.8, 0.8, 0.8))
    veil.base_weight = 0.0
    veil.geometry_opacity = opacity
    sheet = MeshData(p, t, faces=f, face_count=1, face_materials=[1], transform=placement((0.0, 0.5, 0.0)))
    pitch = -math.atan2(0.3, 3.0)
    cam = camera((0.0, 0.3, 3.0), (pitch, 0.0, 0.0), focal_length=200.0, horizontal_aperture=36.0)
    lamp = light(LIGHT_RECT, position=(0.0, 1.0, 0.0), rotation=(-0.5 * math.pi, 0.0, 0.0), intensity=4.0,
                 width=1.0, height=1.0, normalize=False, visible=False)
    return [_floor(), sheet], [cam], [lamp], [veil]


# ---- dome lights (integrator.lucb:495-582) -----------------------------------------------


def dome_furnace_scene(level: int = 4):
    """integrator.lucb:495-518: a white sphere under a white dome with no image (intensity
    1, visible, turned about +Y): the furnace again, lit by the dome's light samples and BSDF
    hits under MIS instead of the background. The sphere is this package's icosphere; its
    material is the settings' default."""
    from .scenes import furnace_sphere
    meshes, cams = furnace_sphere(level)
    sky = light(LIGHT_DOME, rotation=(0.3, 1.0, 0.0), intensity=1.0, visible=True)
    return meshes, cams, [sky], []


def sun_sky(width: int = 64, height: int = 32):
    """integrator.lucb:520-549: a dim grey sky (0.5) with a 2 x 2-texel sun 400 times
    brighter, as linear Rec.709 (height x width x 3), and the irradiance a floor facing +Y
    receives from it (cos theta integrated over each texel in 8 x 8 pieces)."""
    sky = np.full((height, width, 3), 0.5, np.float32)
    sky[8:10, 40:42] = 200.0
    irradiance = 0.0
    for y in range(height):
        for sy in range(8):
            theta = math.pi * (y + (sy + 0.5) / 8.0) / height
            c = math.cos(theta)
            if c <= 0.0:
                continue
            row = float(sky[y, :, 1].astype(np.float64).sum())
            irradiance += row * c * math.sin(theta) * (math.pi / height / 8.0) * (2.0 * math.pi / width)
    return sky, irradiance


def dome_sun_scene():
    """integrator.lucb:551-582: a 20 x 20 floor under the sun sky's dome (+Y up), seen
    straight down from height 4 (50 mm on a 36 mm film): with one bounce, what the floor
    reflects straight up is albedo / pi x the image's irradiance, which needs the image
    sampled by importance (the sun is 1/512 of the texels). Returns (meshes, cameras,
    lights, materials, irradiance)."""
    sky, irradiance = sun_sky()
    cam = camera((0.0, 4.0, 0.0), (-0.5 * math.pi, 0.0, 0.0), focal_length=50.0, horizontal_aperture=36.0)
    dome = light(LIGHT_DOME, intensity=1.0, visible=False, image=sky)
    return [_floor()], [cam], [dome], [], irradiance
