"""Render cases shared by the batch and server tests: (compiled scene, settings) pairs of
uneven sizes, spectral and RGB, depths 2 to 8, Lambertian, glossy and cut-out, lit by
rect, distant, emissive and dome lights, with and without light tracing, and the image a
Renderer makes of each."""
import luce_render_b200 as lr
from luce_render_b200 import scenes, testscenes


def settings(width, height, samples, bounces, spectral, seed=1, material=None, background=(0.0, 0.0, 0.0)):
    s = lr.RenderSettings.of(width, height, samples)
    s.spectral = 1 if spectral else 0
    s.max_bounces = bounces
    s.light_tracing = 0.0
    s.seed = seed
    s.background = background
    s.c.material = material if material is not None else lr.OpenPbr.lambert()
    return s


def cases():
    """(compiled scene, settings) pairs of uneven sizes, modes and depths."""
    out = []
    sc = lr.compile_scene(scenes.cornell_meshes(materials=True), [scenes.cornell_camera()],
                          [scenes.cornell_light()], scenes.cornell_materials())
    out.append((sc, settings(48, 40, 4, 6, False, seed=3)))
    sc = lr.compile_scene(scenes.furnace_meshes(4), [lr.camera((0.0, 0.0, 0.0))])
    out.append((sc, settings(32, 32, 3, 8, True, material=scenes.furnace_material(0.8, 1.0))))
    meshes, cams, lights, mats = testscenes.emissive_quad_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    out.append((sc, settings(24, 20, 5, 2, True, seed=7, material=lr.OpenPbr.lambert((0.5, 0.5, 0.5)))))
    meshes, materials, lights, cam = scenes.scene_of_size(20_000, seed=11)
    sc = lr.compile_scene(meshes, [cam], lights, materials)
    out.append((sc, settings(64, 36, 2, 6, False, seed=5, background=(0.1, 0.2, 0.3))))
    meshes, cams, lights, mats = testscenes.colored_light_scene(kelvin=3200.0)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    out.append((sc, settings(16, 16, 6, 3, True, seed=9)))
    # With light tracing: light paths share the pool and splat on the film.
    sc = lr.compile_scene(scenes.cornell_meshes(materials=True), [scenes.cornell_camera()],
                          [scenes.cornell_light()], scenes.cornell_materials())
    traced = settings(40, 32, 3, 4, False, seed=13)
    traced.light_tracing = 0.5
    out.append((sc, traced))
    # Glossy: coat, glass, gold and rough plastic, alone and with light tracing.
    meshes, cams, lights, mats = scenes.glossy_cornell(2)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    out.append((sc, settings(36, 28, 3, 6, False, seed=17)))
    glossy_traced = settings(28, 24, 2, 5, True, seed=19)
    glossy_traced.light_tracing = 0.5
    out.append((sc, glossy_traced))
    # Adaptive sampling: checks after samples 4 and 8 stop converged pixels.
    meshes, cams, lights, mats = testscenes.area_light_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    adaptive = settings(32, 24, 8, 2, False, seed=29, material=lr.OpenPbr.lambert((0.5, 0.5, 0.5)))
    adaptive.noise_threshold = 0.05
    adaptive.adaptive_minimum = 4
    out.append((sc, adaptive))
    # Cut-outs: 8 rounds more than the bounces, shadow rays walking through the veil.
    meshes, cams, lights, mats = testscenes.veil_scene(0.5)
    sc = lr.compile_scene(meshes, cams, lights, mats)
    out.append((sc, settings(24, 24, 4, 2, False, seed=23, material=lr.OpenPbr.lambert((0.5, 0.5, 0.5)))))
    # A dome light with an image over glossy objects, with light paths from afar.
    meshes, cams, lights, mats, background = scenes.caustic_scene()
    sky, _ = testscenes.sun_sky()
    dome = lr.light(lr.LIGHT_DOME, rotation=(0.0, 0.7, 0.0), intensity=0.5, image=sky)
    sc = lr.compile_scene(meshes, cams, [dome], mats)
    domed = settings(32, 24, 3, 5, True, seed=31, background=background)
    domed.light_tracing = 0.5
    out.append((sc, domed))
    return out


def alone(ctx, sc, s):
    """The image a Renderer of its own makes."""
    r = lr.Renderer.create(ctx, sc, s)
    try:
        r.finish()
        assert r.samples_done() == s.c.samples
        return r.read()
    finally:
        r.destroy()
