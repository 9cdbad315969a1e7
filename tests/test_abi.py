"""The C-ABI library loads and exports every entry point include/*.h declares; the
ctypes harness binds each of them; host-only calls behave (no GPU needed)."""
import re
from pathlib import Path

import numpy as np
import pytest

import luce_render_b200 as lr

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names.update(re.findall(r"\b(lr_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    names = declared_symbols()
    assert len(names) > 30
    missing = [n for n in names if getattr(lr.lib, n, None) is None]
    assert not missing, missing


def test_harness_binds_every_declared_symbol():
    assert set(declared_symbols()) <= set(lr.exported_symbols())


def test_version_and_error_text():
    assert b"sm_100a" in lr.lib.lr_version()
    with pytest.raises(lr.RenderError) as e:
        lr.compile_scene([lr.MeshData([[0, 0, 0]], [[0, 1, 2]])])
    assert e.value.code == 400 and "point" in e.value.message


def test_settings_defaults_match_render_settings_of():
    # RenderSettings.of (integrator.lucb:84-85)
    s = lr.RenderSettings.of(640, 480, 32)
    assert (s.width, s.height, s.samples, s.max_bounces, s.spectral, s.camera) == (640, 480, 32, 12, 1, -1)
    assert (s.pool, s.seed, s.software_bvh, s.adaptive_minimum) == (0, 1, 0, 16)
    assert (s.diffuse_bounces, s.glossy_bounces, s.transmission_bounces) == (1024, 1024, 1024)
    assert s.light_tracing == 0.5 and s.clamp_indirect == 0.0 and s.noise_threshold == 0.0
    m = s.material
    assert m.specular_weight == 1.0 and abs(m.specular_roughness - 0.3) < 1e-12 and list(m.base_color) == [0.8] * 3


def test_scene_compile_polygons_materials_and_placement():
    p, t, f = (np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32),
               np.array([[0, 1, 2], [0, 2, 3]], np.uint32), np.array([0, 0], np.uint32))
    meshes = [lr.MeshData(p, t, faces=f, face_count=1, face_materials=[2]),
              lr.MeshData(p, t, faces=f, face_count=1, face_materials=[7], transform=lr.placement((0, 0, 5)))]
    sc = lr.compile_scene(meshes, materials=[lr.OpenPbr.lambert(), lr.OpenPbr.lambert()])
    a = sc.arrays()
    info = sc.info
    assert info.triangle_count == 4 and info.face_count == 2 and info.point_count == 8
    src = np.empty_like(a["faces"])
    src[a["order"]] = a["faces"]
    assert src.tolist() == [0, 0, 1, 1]
    mats = np.empty(4, np.uint32)
    mats[a["order"]] = a["shading"][:, 3]
    # a polygon naming a material the library lacks falls back to the default (0)
    assert mats.tolist() == [2, 2, 0, 0]
    assert a["positions"][4:, 2].tolist() == [5.0] * 4


def test_empty_scene_and_bad_light():
    sc = lr.compile_scene([])
    assert sc.triangle_count() == 0 and len(sc.arrays()["nodes"]) == 1
    bad = lr.light(9)
    with pytest.raises(lr.RenderError):
        lr.compile_scene([], lights=[bad])


def test_dome_image_checks():
    # A dome's image is height x width x 3 (the harness checks the shape); an image with
    # no pixels is refused by the compile; the compiled scene keeps its own copy.
    with pytest.raises(ValueError):
        lr.light(lr.LIGHT_DOME, image=np.zeros((4, 4), np.float32))
    empty = lr.light(lr.LIGHT_DOME, image=np.zeros((2, 3, 3), np.float32))
    empty.image_width = 0
    with pytest.raises(lr.RenderError) as e:
        lr.compile_scene([], lights=[empty])
    assert e.value.code == 400
    sky = np.ones((2, 4, 3), np.float32)
    dome = lr.light(lr.LIGHT_DOME, image=sky)
    sc = lr.compile_scene([], lights=[dome])
    sky[:] = np.nan  # the caller's buffer may change or go once the compile returns
    assert sc.info.light_count == 1


def test_standard_material_is_the_libraries():
    # OpenPbr.standard fills materials.lucb:46-53's values in Python (describing a scene
    # maps no library); lr_openpbr_standard is the ABI's own copy of them.
    import ctypes as C
    ours = lr.OpenPbr.standard()
    theirs = lr.OpenPbr()
    lr.lib.lr_openpbr_standard(C.byref(theirs))
    assert bytes(ours) == bytes(theirs)


def test_describing_a_workload_maps_no_library():
    # The scene generators and descriptions run without the C library (the benchmark's
    # CPU reference arm builds its workload this way and maps only the oracle).
    import subprocess
    import sys
    code = ("import luce_render_b200 as lr; from luce_render_b200 import scenes; "
            "scenes.incoherent_scene(spheres=2, tori=2); scenes.cornell_meshes(True); scenes.cornell_materials(); "
            "assert lr.lib._dll is None; "
            "assert 'libluce_render_b200' not in open('/proc/self/maps').read()")
    subprocess.run([sys.executable, "-c", code], check=True, cwd=str(ROOT))
