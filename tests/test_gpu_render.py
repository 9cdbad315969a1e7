"""The CUDA integrator through the C ABI against closed forms and the f64 oracle.

- Closed forms (tests/gpu/integrator.lucb): the emitting Lambertian enclosure
  L = Le (1 - rho^(D+1)) / (1 - rho) (D = 8: 4.3289; D large: Le / (1 - rho) = 5), the
  irradiance under a rect light and under the same square as an emissive mesh
  (0.5 / pi * 4 * 4 * corner_irradiance(0.5, 0.5, 1)), spectral against RGB. Each is
  checked within 3 sigma of the Monte Carlo standard error, and within the reference's
  own relative tolerance where it states one.
- The f64 host accumulation of the same estimator over the same Sobol samples
  (oracle/integrator.c): block means of the GPU image within 3 sigma of the oracle's.
"""
import math

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes, testscenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _render(ctx, meshes, cams, lights, materials, width, height, samples, bounces, spectral, material=None,
            background=(0.0, 0.0, 0.0), seed=1):
    sc = lr.compile_scene(meshes, cams, lights, materials)
    s = lr.RenderSettings.of(width, height, samples)
    s.spectral = 1 if spectral else 0
    s.max_bounces = bounces
    s.light_tracing = 0.0
    s.seed = seed
    s.background = background
    s.c.material = material if material is not None else lr.OpenPbr.lambert()
    r = lr.Renderer.create(ctx, sc, s)
    r.finish()
    assert r.samples_done() == samples
    img = r.read()
    r.destroy()
    return sc, img


def _mean_sem(values):
    v = np.asarray(values, np.float64).reshape(-1, values.shape[-1])
    return v.mean(0), v.std(0, ddof=1) / math.sqrt(len(v))


@pytest.mark.parametrize("spectral", [False, True])
def test_furnace_enclosure(ctx, spectral):
    # A closed icosphere (20,480 triangles) of albedo 0.8 emitting 1, the camera inside:
    # emission is counted at hits 0..D, so L = (1 - 0.8^(D+1)) / 0.2.
    for bounces, samples in ((8, 64), (64, 16)):
        _, img = _render(ctx, scenes.furnace_meshes(5), [lr.camera((0.0, 0.0, 0.0))], [], [], 64, 64, samples,
                         bounces, spectral, material=scenes.furnace_material(0.8, 1.0))
        mean, sem = _mean_sem(img[..., :3])
        expected = (1.0 - 0.8 ** (bounces + 1)) / 0.2
        # Spectral: XYZ under E through the film matrix, whose white is exact to 1e-6, and
        # the observer's integrals summed at 1 nm against the sampled continuous density.
        bias = 2e-4 * expected if spectral else 1e-6
        assert np.all(np.abs(mean - expected) <= 3.0 * sem + bias), (bounces, mean, sem, expected)


@pytest.mark.parametrize("spectral", [False, True])
def test_area_light_irradiance(ctx, spectral):
    meshes, cams, lights, mats = testscenes.area_light_scene()
    _, img = _render(ctx, meshes, cams, lights, mats, 32, 32, 256, 1, spectral,
                     material=lr.OpenPbr.lambert((0.5, 0.5, 0.5)))
    window = img[14:18, 14:18, :3]
    measured = window.reshape(-1, 3).mean(0)
    expected = testscenes.AREA_LIGHT_EXPECTED
    # The reference's rule (integrator.lucb:765): Y within 2%, X within 3%.
    assert abs(measured[1] / expected - 1.0) <= 0.02 and abs(measured[0] / expected - 1.0) <= 0.03, measured


@pytest.mark.parametrize("spectral", [False, True])
def test_emissive_quad_through_light_tree(ctx, spectral):
    meshes, cams, lights, mats = testscenes.emissive_quad_scene()
    _, img = _render(ctx, meshes, cams, lights, mats, 32, 32, 256, 1, spectral,
                     material=lr.OpenPbr.lambert((0.5, 0.5, 0.5)))
    measured = img[14:18, 14:18, :3].reshape(-1, 3).mean(0)
    assert abs(measured[1] / testscenes.AREA_LIGHT_EXPECTED - 1.0) <= 0.02, measured


@pytest.mark.parametrize("kelvin", [0.0, 3000.0])
def test_spectral_agrees_with_rgb(ctx, kelvin):
    color = (1.0, 0.4, 0.1) if kelvin == 0.0 else (1.0, 1.0, 1.0)
    means = []
    for spectral in (True, False):
        meshes, cams, lights, mats = testscenes.colored_light_scene(color, kelvin)
        _, img = _render(ctx, meshes, cams, lights, mats, 48, 32, 64, 4, spectral,
                         material=lr.OpenPbr.lambert((0.9, 0.9, 0.9)))
        means.append(img[0:32, 8:40, :3].reshape(-1, 3).mean(0))
    s, r = means
    # integrator.lucb:793-796
    assert abs(s[0] / r[0] - 1) <= 0.03 and abs(s[1] / r[1] - 1) <= 0.03 and abs(s[2] / r[2] - 1) <= 0.06, (s, r)


def _blocks(x, b):
    h, w = x.shape[:2]
    return x[: h // b * b, : w // b * b].reshape(h // b, b, w // b, b, -1)


@pytest.mark.parametrize("spectral", [False, True])
def test_gpu_matches_f64_oracle_cornell(ctx, spectral):
    w = h = 64
    spp, bounces = 16, 8
    meshes = scenes.cornell_meshes(True)
    cams = [scenes.cornell_camera()]
    lights = [scenes.cornell_light()]
    mats = scenes.cornell_materials()
    sc, img = _render(ctx, meshes, cams, lights, mats, w, h, spp, bounces, spectral)
    frame = lr.ray_frame(sc.camera(), w, h)
    mean, var = orc.render(sc.arrays(), lights, [lr.OpenPbr.lambert()] + mats, frame, spp, bounces, spectral)
    gpu = img[..., :3].astype(np.float64)
    # 8x8-pixel blocks: the GPU's block mean against the oracle's within 3 sigma of the
    # standard error of a block mean (both draw the same samples, so most paths agree).
    b = 8
    g = _blocks(gpu, b).mean((1, 3))
    o = _blocks(mean, b).mean((1, 3))
    sem = np.sqrt(_blocks(var, b).mean((1, 3)) / (b * b * spp))
    assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), np.max(np.abs(g - o) / (sem + 1e-12))
    # and the whole image's mean
    assert np.all(np.abs(gpu.mean((0, 1)) - mean.mean((0, 1))) <= 3.0 * np.sqrt(var.mean((0, 1)) / (w * h * spp)) + 1e-6)


def test_gpu_matches_f64_oracle_lights(ctx):
    # Sphere, disk and distant lights with a size and a delta sun over a 16-triangle floor,
    # with a grey background: NEE by power among the distant lights, tree for the rest.
    p, t, f = scenes.grid(8.0, 2)
    meshes = [lr.MeshData(p, t, faces=f, face_count=4)]
    sp, st, sn = scenes.icosphere(2, 0.6)
    meshes.append(lr.MeshData(sp, st, normals=sn, transform=lr.placement((0.8, 0.6, -0.5))))
    lights = [lr.light(lr.LIGHT_SPHERE, position=(-1.0, 2.0, 0.5), intensity=3.0, radius=0.3),
              lr.light(lr.LIGHT_DISK, position=(1.0, 2.5, 1.0), rotation=(-1.2, 0.3, 0.0), intensity=5.0, radius=0.5,
                       color=(0.9, 0.6, 0.3)),
              lr.light(lr.LIGHT_DISTANT, rotation=(-0.9, 0.5, 0.0), intensity=1.5, angle=4.0),
              lr.light(lr.LIGHT_DISTANT, rotation=(-1.3, -0.4, 0.0), intensity=0.7, angle=0.0)]
    cams = [lr.camera((0.0, 2.0, 5.0), (-0.35, 0.0, 0.0), focal_length=30.0)]
    w, h, spp, bounces = 48, 32, 16, 4
    for spectral in (False, True):
        sc, img = _render(ctx, meshes, cams, lights, [], w, h, spp, bounces, spectral,
                          background=(0.05, 0.07, 0.1))
        frame = lr.ray_frame(sc.camera(), w, h)
        mean, var = orc.render(sc.arrays(), lights, [lr.OpenPbr.lambert()], frame, spp, bounces, spectral,
                               background=(0.05, 0.07, 0.1))
        g = _blocks(img[..., :3].astype(np.float64), 8).mean((1, 3))
        o = _blocks(mean, 8).mean((1, 3))
        sem = np.sqrt(_blocks(var, 8).mean((1, 3)) / (64 * spp))
        assert np.all(np.abs(g - o) <= 3.0 * sem + 1e-6), (spectral, np.max(np.abs(g - o) / (sem + 1e-12)))


def test_renderer_api_progress_and_errors(ctx):
    sc = lr.compile_scene(scenes.cornell_meshes(), [scenes.cornell_camera()], [scenes.cornell_light()])
    s = lr.RenderSettings.of(64, 48, 3)
    s.max_bounces = 3
    # Camera paths alone: light paths' sampler numbers follow the band, so an image with
    # light tracing depends on the pool size (as the reference's does).
    s.light_tracing = 0.0
    rough = lr.OpenPbr.lambert()
    rough.base_diffuse_roughness = 2.0
    s.c.material = rough
    with pytest.raises(lr.RenderError) as e:
        lr.Renderer.create(ctx, sc, s)  # EON's roughness is 0 to 1
    assert e.value.code == 400
    s.c.material = lr.OpenPbr.lambert()
    s.pool = 1000  # bands of 1,000 paths: 4 passes a sample
    r = lr.Renderer.create(ctx, sc, s)
    assert r.samples_done() == 0
    more = True
    while more:
        more = r.advance()
    assert r.samples_done() == 3
    first = r.read()
    r.set_samples(5)
    r.finish()
    assert r.samples_done() == 5
    st = r.stats()
    assert st.passes == 5 * 4 and st.closest_rays >= 5 * 64 * 48
    with pytest.raises(lr.RenderError) as e:
        bad = np.empty(10, np.float32)
        lr._check(lr.lib.lr_renderer_read(r.handle, lr._fptr(bad), 10))
    assert e.value.code == 400
    r.destroy()
    # The same render in one band (no pool limit) gives the same image.
    s.pool = 0
    s.samples = 3
    r2 = lr.Renderer.create(ctx, sc, s)
    r2.finish()
    assert np.array_equal(r2.read(), first)
    r2.destroy()
    with pytest.raises(lr.RenderError):
        bad = lr.RenderSettings.of(0, 10, 1)
        bad.c.material = lr.OpenPbr.lambert()
        lr.Renderer.create(ctx, sc, bad)


def test_renderer_read_async_is_the_image_of_its_pass(ctx):
    # A read queued after a pass holds that pass's image however many passes follow
    # before it is waited for: the same bits as a render of that many samples.
    sc = lr.compile_scene(scenes.cornell_meshes(True), [scenes.cornell_camera()], [scenes.cornell_light()],
                          scenes.cornell_materials())
    s = lr.RenderSettings.of(96, 64, 6)
    s.max_bounces = 4
    s.light_tracing = 0.0
    s.c.material = lr.OpenPbr.lambert()
    hosts = [lr.PinnedArray((64, 96, 4), np.float32) for _ in range(3)]
    r = lr.Renderer.create(ctx, sc, s)
    r.advance_one()
    r.read_async(hosts[0].array)
    r.advance_one()
    r.advance_one()
    r.read_async(hosts[1].array)
    r.finish()
    r.read_async(hosts[2].array)
    r.read_wait()
    final = r.read()
    r.destroy()
    for samples, got in ((1, hosts[0].array), (3, hosts[1].array), (6, hosts[2].array)):
        s.samples = samples
        want = lr.Renderer.create(ctx, sc, s)
        want.finish()
        assert np.array_equal(got, want.read()), samples
        want.destroy()
    assert np.array_equal(hosts[2].array, final)
    for h in hosts:
        h.close()


def test_renderer_read_tickets_land_in_order(ctx):
    # Ticketed reads into two buffers in turn, each reused once its last copy has landed:
    # every copy holds its pass's image, and a ticket lands no earlier than those before it.
    sc = lr.compile_scene(scenes.cornell_meshes(True), [scenes.cornell_camera()], [scenes.cornell_light()],
                          scenes.cornell_materials())
    s = lr.RenderSettings.of(96, 64, 4)
    s.max_bounces = 4
    s.light_tracing = 0.0
    s.c.material = lr.OpenPbr.lambert()
    hosts = [lr.PinnedArray((64, 96, 4), np.float32) for _ in range(2)]
    r = lr.Renderer.create(ctx, sc, s)
    tickets, seen, last = [0, 0], [], 0
    for step in range(4):
        r.advance_one()
        if tickets[step % 2]:
            for _ in range(1000000):
                if r.read_landed(tickets[step % 2]):
                    break
            assert r.read_landed(tickets[step % 2])
            seen.append((step - 2, hosts[step % 2].array.copy()))
        tickets[step % 2] = r.read_ticket(hosts[step % 2].array)
        assert tickets[step % 2] > last
        last = tickets[step % 2]
    r.read_wait()
    assert r.read_landed(tickets[0]) and r.read_landed(tickets[1])
    seen += [(2, hosts[0].array.copy()), (3, hosts[1].array.copy())]
    r.destroy()
    for step, got in seen:
        s.samples = step + 1
        want = lr.Renderer.create(ctx, sc, s)
        want.finish()
        assert np.array_equal(got, want.read()), step
        want.destroy()
    for h in hosts:
        h.close()


def test_adaptive_sampling(ctx):
    # tests/gpu/integrator.lucb:334-358: a sphere under an area light, half the frame empty
    # sky: with adaptive sampling the image is the same within 1 % (it stops sampling only
    # where the image is clean) and at least a third of the pixels stop early.
    sp, st, sn = scenes.icosphere(4, 1.0)
    cam = lr.camera((1.5, 1.0, 5.0), (-math.atan2(1.0, math.hypot(1.5, 5.0)), math.atan2(1.5, 5.0), 0.0),
                    focal_length=35.0, horizontal_aperture=36.0)
    key = lr.light(lr.LIGHT_RECT, position=(1.0, 4.0, 1.0), rotation=(-1.2, 0.3, 0.0), intensity=20.0, width=2.0,
                   height=2.0, normalize=True, visible=False)
    sc = lr.compile_scene([lr.MeshData(sp, st, normals=sn)], [cam], [key])
    sums, stopped, images = [], 0, []
    for threshold in (0.01, 0.0):
        s = lr.RenderSettings.of(64, 48, 64)
        s.spectral = 0
        s.noise_threshold = threshold
        r = lr.Renderer.create(ctx, sc, s)
        r.finish()
        img = r.read()
        images.append(img)
        sums.append(img[..., 1].astype(np.float64).sum())
        if threshold > 0.0:
            stopped = r.converged_pixels()
        r.destroy()
    assert abs(sums[0] / sums[1] - 1.0) <= 0.01, sums
    assert stopped >= 64 * 48 // 3, stopped
    # The sky (nothing hit) converges at the first check and stays black.
    sky = images[1][..., :3].sum(-1) == 0.0
    assert sky.sum() > 0 and np.all(images[0][sky][:, :3] == 0.0)
