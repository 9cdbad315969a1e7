"""The interactive state model (integrator.lucb:455-582, tests/gpu/interactive.lucb and
display.lucb) through the C ABI: restarts through other views and sizes, with passes in
flight; reloads with another light or other materials over the same geometry; another
scene in the same renderer; and the display image. Each render is compared with a
renderer made afresh for the same view, scene and settings: bit for bit, since a
restarted, reloaded or replaced renderer starts its samples over and light paths' splats
add in fixed point."""
import math

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes

pytestmark = pytest.mark.gpu


def _scene(key: float, lift: float = 0.0, ball=(0.6, 0.6, 0.6)):
    sp, st, sn = scenes.icosphere(3, 0.6)
    p, t, f = scenes.grid(10.0, 4)
    meshes = [lr.MeshData(sp, st, normals=sn, faces=np.zeros(len(st), np.uint32), face_count=1, face_materials=[1],
                          transform=lr.placement((0.0, lift, 0.0))),
              lr.MeshData(p, t, faces=f, face_count=16, face_materials=[2] * 16, transform=lr.placement((0.0, -0.6, 0.0)))]
    lights = [lr.light(lr.LIGHT_RECT, position=(0.5, 3.0, 1.0), rotation=(-0.5 * math.pi, 0.0, 0.0), intensity=key,
                       width=1.5, height=1.5)]
    mats = [scenes.openpbr(base_color=ball, specular_roughness=0.3),
            scenes.openpbr(base_color=(0.6, 0.6, 0.6), specular_weight=0.0)]
    return lr.compile_scene(meshes, [], lights, mats)


def _view(eye, w, h):
    e = np.array(eye, np.float64)
    forward = -e / np.linalg.norm(e)
    return lr.look_frame(tuple(e), tuple(forward), (0.0, 1.0, 0.0), math.tan(math.radians(20.0)), w, h)


def _settings(w=48, h=32, samples=12):
    s = lr.RenderSettings.of(w, h, samples)
    s.max_bounces = 4
    return s


def _fresh(ctx, sc, frame, s):
    r = lr.Renderer.create(ctx, sc, s, frame)
    r.finish()
    img = r.read()
    r.destroy()
    return img


def test_restarts(ctx):
    sc = _scene(6.0)
    a, b, half = _view((0.0, 1.5, 4.0), 48, 32), _view((3.0, 2.5, 1.0), 48, 32), _view((0.0, 1.5, 4.0), 24, 16)
    s = _settings()
    fresh = _fresh(ctx, sc, a, s)
    r = lr.Renderer.create(ctx, sc, s, b)
    try:
        r.finish()
        assert r.samples_done() == 12
        r.restart(a)
        assert r.samples_done() == 0
        r.finish()
        assert np.array_equal(r.read(), fresh), "restarted through another view"
        # A smaller view shows at its own size; growing back renders as before.
        r.restart(half)
        r.finish()
        assert r.shown_size() == (24, 16)
        assert np.array_equal(r.read(), _fresh(ctx, sc, half, _settings(24, 16))), "a smaller view"
        r.restart(a)
        r.finish()
        assert r.shown_size() == (48, 32)
        assert np.array_equal(r.read(), fresh), "back from a smaller view"
        # Restarted mid-render: the passes in flight count for nothing.
        r.restart(b)
        r.advance()
        r.advance()
        r.restart(a)
        r.finish()
        assert r.samples_done() == 12
        assert np.array_equal(r.read(), fresh), "restarted with passes in flight"
        # A view larger than the renderer's buffers: made again.
        big = _view((0.0, 1.5, 4.0), 96, 64)
        r.restart(big)
        r.finish()
        assert np.array_equal(r.read(), _fresh(ctx, sc, big, _settings(96, 64))), "a larger view"
        with pytest.raises(lr.RenderError) as e:
            ortho = _view((0.0, 1.5, 4.0), 48, 32)
            ortho.orthographic = 1
            r.restart(ortho)
        assert e.value.code == 400
    finally:
        r.destroy()


def test_reload_and_replace(ctx):
    sc = _scene(6.0)
    a = _view((0.0, 1.5, 4.0), 48, 32)
    s = _settings()
    r = lr.Renderer.create(ctx, sc, s, a)
    try:
        r.finish()
        before = r.read()
        # A light twice as bright over the same geometry: as a renderer made for it, and
        # about twice the light (tests/gpu/interactive.lucb:91-103).
        brighter = _scene(12.0)
        r.reload(brighter, s)
        assert r.samples_done() == 0
        r.finish()
        again = r.read()
        assert np.array_equal(again, _fresh(ctx, brighter, a, s)), "reloaded with a brighter light"
        ratio = again[..., :3].mean() / before[..., :3].mean()
        assert abs(ratio - 2.0) <= 0.02, ratio
        # Other materials (the triangles' shading uploaded again), with passes in flight.
        red = _scene(6.0, ball=(0.8, 0.1, 0.1))
        r.set_samples(40)
        r.advance()
        r.advance()
        r.reload(red, s)
        r.finish()
        assert np.array_equal(r.read(), _fresh(ctx, red, a, s)), "reloaded with other materials"
        # Other settings (more bounces) over the same geometry.
        deeper = _settings()
        deeper.max_bounces = 7
        r.reload(red, deeper)
        r.finish()
        assert np.array_equal(r.read(), _fresh(ctx, red, a, deeper)), "reloaded with more bounces"
        # Other geometry is not a reload.
        moved = _scene(6.0, lift=0.1)
        with pytest.raises(lr.RenderError) as e:
            r.reload(moved, s)
        assert e.value.code == 400
        # Other geometry in the same renderer, through another view.
        b = _view((3.0, 2.5, 1.0), 48, 32)
        r.replace_scene(moved, s, b)
        r.finish()
        assert np.array_equal(r.read(), _fresh(ctx, moved, b, s)), "another scene in the same renderer"
    finally:
        r.destroy()


def _neutral(c):
    # film_convert.comp:20-34
    start, desaturation = 0.8 - 0.04, 0.15
    x = c.min(-1, keepdims=True)
    offset = np.where(x < 0.08, x - 6.25 * x * x, 0.04)
    c = c - offset
    peak = c.max(-1, keepdims=True)
    d = 1.0 - start
    new_peak = 1.0 - d * d / (peak + d - start)
    g = 1.0 - 1.0 / (desaturation * (peak - new_peak) + 1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        mapped = c * (new_peak / peak) * (1.0 - g) + new_peak * g
    return np.where(peak < start, c, mapped)


def test_display(ctx):
    sc = _scene(6.0)
    a = _view((0.0, 1.5, 4.0), 48, 32)
    r = lr.Renderer.create(ctx, sc, _settings(), a)
    try:
        assert r.shown_size() == (0, 0)
        r.finish()
        to709 = np.array([[1.70505, -0.62179, -0.08326], [-0.13026, 1.14080, -0.01055], [-0.02400, -0.12897, 1.15297]])
        image = r.read()[..., :3].astype(np.float64)
        for exposure, view in ((0.0, 0), (1.5, 0), (1.0, 1)):
            r.set_display(exposure, view)
            r.finish()  # a conversion of its own: every sample is taken
            shown = r.read_display().astype(np.float64)
            assert shown.shape == (32, 48, 4)
            want = np.maximum(image @ to709.T * 2.0 ** exposure, 0.0)
            if view == 1:
                want = _neutral(want)
            want = np.minimum(want, 1.0)
            assert np.max(np.abs(shown[..., :3] - want)) <= 2e-3, (exposure, view)
        # Restarted mid-render: every display image shown is one whole view's.
        b = _view((3.0, 2.5, 1.0), 24, 16)
        r.set_display(0.0, 0)
        r.restart(b)
        r.advance()
        w, h = r.shown_size()
        assert (w, h) in ((48, 32), (24, 16))
        r.finish()
        assert r.shown_size() == (24, 16)
    finally:
        r.destroy()
