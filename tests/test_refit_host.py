"""Moving a compiled scene's points with its triangles kept (lr_scene_move_points): the
BVH2 refit in place on the host, what lr_gpu_scene_refit does on the device.

- Points unchanged: nodes and shading stay bit for bit.
- Points moved: every node's box is the minimum and maximum of its triangles' corners (a
  numpy refit of the same tree), children inside parents; flat normals are those a fresh
  compile of the moved mesh gives the same triangle; and the oracle's restatement of
  trace_closest on the refit tree passes the reference's acceptance rule against the f64
  brute force.
"""
import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes
from oracle import oracle as orc


def _deform(p, amount=0.08):
    p = np.asarray(p, np.float64)
    return (p + amount * np.sin(3.0 * p[:, [1, 2, 0]])).astype(np.float32)


def _numpy_refit(nodes, positions, indices):
    lo = np.empty((len(nodes), 3), np.float32)
    hi = np.empty((len(nodes), 3), np.float32)
    for n in range(len(nodes) - 1, -1, -1):
        first, count = int(nodes["first"][n]), int(nodes["count"][n])
        if count:
            corners = positions[indices[first:first + count].reshape(-1)]
            lo[n], hi[n] = corners.min(0), corners.max(0)
        else:
            lo[n] = np.minimum(lo[first], lo[first + 1])
            hi[n] = np.maximum(hi[first], hi[first + 1])
    return lo, hi


def test_unmoved_points_change_nothing():
    meshes, cams = scenes.probe_test_scene()
    sc = lr.compile_scene(meshes, cams)
    before = sc.arrays()
    sc.move_points(before["positions"])
    after = sc.arrays()
    for key in ("positions", "indices", "shading", "order"):
        assert np.array_equal(before[key], after[key]), key
    assert before["nodes"].tobytes() == after["nodes"].tobytes()


def test_moved_points_refit_the_tree():
    meshes, cams = scenes.probe_test_scene()
    sc = lr.compile_scene(meshes, cams)
    a0 = sc.arrays()
    moved = _deform(a0["positions"])
    sc.move_points(moved)
    a = sc.arrays()
    assert np.array_equal(a["positions"], moved)
    assert np.array_equal(a["indices"], a0["indices"]) and np.array_equal(a["order"], a0["order"])
    assert np.array_equal(a["nodes"]["first"], a0["nodes"]["first"])
    assert np.array_equal(a["nodes"]["count"], a0["nodes"]["count"])
    lo, hi = _numpy_refit(a["nodes"], moved, a["indices"])
    assert np.array_equal(a["nodes"]["lo"], lo) and np.array_equal(a["nodes"]["hi"], hi)
    # Flat normals: the cube and the floor were compiled without authored normals; a fresh
    # compile of the moved points gives each source triangle the same code.
    fresh_meshes = []
    start = 0
    for m in meshes:
        count = len(m.positions)
        fresh_meshes.append(lr.MeshData(moved[start:start + count], m.indices, faces=m.faces, face_count=m.face_count,
                                        normals=m.normals))
        start += count
    fresh = lr.compile_scene(fresh_meshes, cams).arrays()
    by_source = np.empty_like(fresh["shading"])
    by_source[fresh["order"]] = fresh["shading"]
    assert np.array_equal(a["shading"], by_source[a["order"]])
    # The refit tree traces correctly: the reference's acceptance rule against f64 brute force.
    frame = lr.ray_frame(sc.camera(0), 96, 64)
    rays = orc.probe_rays(frame.pack())
    ref, counts = orc.trace(a["nodes"], a["positions"], a["indices"], rays)
    assert counts.dropped == 0
    face, distance, margin = orc.nearest_f64(a["positions"], a["indices"], a["faces"], rays)
    slot = ref["triangle"]
    got = np.where(slot == 0xFFFFFFFF, -1, a["faces"][np.minimum(slot, len(a["faces"]) - 1)].astype(np.int64))
    agrees = (got == face) & ((face < 0) | (np.abs(ref["t"].astype(np.float64) - distance) <= 1e-4 * distance))
    assert np.count_nonzero(~agrees & (margin > 1e-3)) == 0
    assert np.count_nonzero(face >= 0) > len(rays) // 2


def test_move_points_rejects_other_counts():
    sc = lr.compile_scene(scenes.cornell_meshes())
    p = sc.arrays()["positions"]
    with pytest.raises(lr.RenderError) as e:
        sc.move_points(p[:-1])
    assert e.value.code == 400
    bad = p.copy()
    bad[0, 0] = np.nan
    with pytest.raises(lr.RenderError):
        sc.move_points(bad)


def test_move_points_of_an_empty_scene():
    sc = lr.compile_scene([])
    sc.move_points(np.zeros((0, 3), np.float32))
    assert sc.triangle_count() == 0 and len(sc.arrays()["nodes"]) == 1
