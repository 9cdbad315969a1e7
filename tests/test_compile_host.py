"""compile_scene without trees (scene.lucb:111-129, `trees = false`): no host BVH2, the
triangles in the meshes' order, the same triangles, polygons and shading words as the
compile with trees, only permuted by its leaf order."""
import ctypes as C

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes


def test_tree_less_compile_keeps_the_meshes_order():
    meshes = scenes.cornell_meshes(materials=True)
    full = lr.compile_scene(meshes, [scenes.cornell_camera()], [scenes.cornell_light()], scenes.cornell_materials())
    flat = lr.compile_scene(meshes, [scenes.cornell_camera()], [scenes.cornell_light()], scenes.cornell_materials(),
                            trees=False)
    try:
        a, b = full.arrays(), flat.arrays()
        T = len(a["order"])
        assert flat.info.node_count == 0 and flat.info.bvh_depth == 0 and full.info.node_count > 0
        assert np.array_equal(b["order"], np.arange(T, dtype=np.uint32))
        assert np.array_equal(b["positions"], a["positions"])
        # The host tree's leaf slot s holds source triangle order[s].
        for key in ("indices", "faces", "shading"):
            assert np.array_equal(b[key][a["order"]], a[key]), key
    finally:
        full.close()
        flat.close()


def test_tree_less_compile_moves_points():
    meshes, _, _, cam = scenes.scene_of_size(5_000, seed=5)
    sc = lr.compile_scene(meshes, [cam], trees=False)
    try:
        p = sc.arrays()["positions"] * np.float32(2.0)
        sc.move_points(p)
        assert np.array_equal(sc.arrays()["positions"], p)
    finally:
        sc.close()


def test_compile_rejects_unknown_flags():
    out = C.c_void_p()
    assert lr.lib.lr_scene_compile_ex(None, 0, None, 0, None, 0, None, 0, 2, C.byref(out)) == lr.INVALID
    assert "flags" in lr.lib.lr_last_error().decode()
