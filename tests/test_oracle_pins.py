"""The oracle pinned against the reference's own golden table and known-answer tests
(src/render/tests.lucb), and the product's host side held to the same answers.
CPU only."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes, testscenes
from oracle import oracle as orc

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_sobol_table_matches_reference_generator():
    table = json.loads((GOLDEN / "sobol_directions.json").read_text())["directions"]
    assert orc.sobol_directions().tolist() == table


def test_sample4_is_24_bit_and_stratified():
    # sampler.glsl:47-55: four dimensions, top 24 bits; the first dimension of a
    # pixel's first 2^k samples covers the 2^k strata exactly once (Owen-scrambled Sobol).
    vals = np.array([orc.sample4_bits(1, 77, i, 0) for i in range(256)])
    assert vals.max() < (1 << 24)
    for d in range(2):
        strata = np.sort(vals[:, d] >> 16)
        assert np.array_equal(strata, np.arange(256))


def check_bvh(nodes, positions, indices):
    """check_bvh (tests.lucb:9-28)."""
    count = len(indices)
    seen = np.zeros(count, np.int64)
    for n in nodes:
        if n["count"] == 0:
            if count == 0:
                continue
            for child in (n["first"], n["first"] + 1):
                inner = nodes[child]
                assert np.all(inner["lo"] >= n["lo"]) and np.all(inner["hi"] <= n["hi"])
            continue
        for slot in range(n["first"], n["first"] + n["count"]):
            seen[slot] += 1
            for k in range(3):
                p = positions[indices[slot][k]]
                assert np.all(p >= n["lo"]) and np.all(p <= n["hi"])
    assert np.all(seen == 1)


def test_cube_compiles_to_12_triangles_of_6_faces():
    # tests.lucb:30-41, through the product's compile_scene and the oracle's build.
    p, t, f = scenes.cube(2.0)
    sc = lr.compile_scene([lr.MeshData(p, t, faces=f, face_count=6)])
    a = sc.arrays()
    assert sc.triangle_count() == 12 and sc.point_count() == 8
    assert np.array_equal(np.bincount(a["faces"], minlength=6), [2] * 6)
    check_bvh(a["nodes"], a["positions"], a["indices"])
    nodes, order = orc.build_bvh(p, t)
    assert np.array_equal(nodes.view(np.uint8), a["nodes"].view(np.uint8))


def test_instances_placed_and_leaves_at_most_16():
    # tests.lucb:43-61: a 40x40 grid and a copy 5 units up.
    p, t, f = scenes.grid(10.0, 40)
    sc = lr.compile_scene([lr.MeshData(p, t, faces=f, face_count=1600),
                           lr.MeshData(p, t, faces=f, face_count=1600, transform=lr.placement((0.0, 5.0, 0.0)))])
    a = sc.arrays()
    assert sc.triangle_count() == 2 * 2 * 40 * 40
    assert a["positions"][:, 1].max() == 5.0
    assert a["nodes"]["count"].max() <= 16 and len(a["nodes"]) > 100
    check_bvh(a["nodes"], a["positions"], a["indices"])


def test_camera_frame_fits_film_horizontally():
    # tests.lucb:63-81: 36 mm across at 18 mm is 90 deg horizontally.
    cam = lr.camera((0.0, 0.0, 5.0), focal_length=18.0, horizontal_aperture=36.0)
    for frame in (lr.ray_frame(cam, 200, 100),):
        origin, left = frame.ray(0.0, 50.0)
        assert origin[2] == 5.0 and abs(left[0] + 1.0) < 1e-9 and abs(left[2] + 1.0) < 1e-9
        _, center = frame.ray(100.0, 50.0)
        assert abs(center[0]) < 1e-9 and abs(center[1]) < 1e-9 and center[2] == -1.0
        _, top = frame.ray(100.0, 0.0)
        assert abs(top[1] - 0.5) < 1e-9
    status, f = orc.frame_of_camera(cam.matrix, 0, 18.0, 36.0, 0.0, 5.0, 200, 100)
    assert status == 0
    o, d = orc.frame_ray(f, 0.0, 50.0)
    assert o[2] == 5.0 and abs(d[0] + 1.0) < 1e-9 and abs(d[2] + 1.0) < 1e-9
    assert np.array_equal(orc.frame_pack(f), lr.ray_frame(cam, 200, 100).pack())


def test_orthographic_view_looks_along_forward():
    # tests.lucb:83-91
    frame = lr.look_frame((0.0, 10.0, 0.0), (0.0, -1.0, 0.0), (0.0, 0.0, -1.0), 2.0, 200, 100, orthographic=True)
    assert frame.orthographic
    corner, along = frame.ray(0.0, 0.0)
    assert abs(corner[0] + 4.0) < 1e-9 and abs(corner[2] + 2.0) < 1e-9 and corner[1] == 10.0
    assert along[1] == -1.0 and along[0] == 0.0
    middle, _ = frame.ray(100.0, 50.0)
    assert abs(middle[0]) < 1e-9 and abs(middle[2]) < 1e-9
    status, f = orc.look_frame((0.0, 10.0, 0.0), (0.0, -1.0, 0.0), (0.0, 0.0, -1.0), 2.0, 200, 100, True)
    assert status == 0 and np.array_equal(orc.frame_pack(f), frame.pack())


def test_invalid_frames_raise_400():
    with pytest.raises(lr.RenderError) as e:
        lr.look_frame((0, 0, 0), (0, 0, -1), (0, 1, 0), 0.0, 10, 10)
    assert e.value.code == 400
    with pytest.raises(lr.RenderError) as e:
        lr.ray_frame(lr.camera((0, 0, 0)), 0, 10)
    assert e.value.code == 400


def test_spectrum_fit_round_trips_through_the_film():
    # tests.lucb:93-109
    to_acescg = orc.film_matrix()
    white = orc.fit_spectrum((1.0, 1.0, 1.0))
    assert white[0] == 0 and white[1] == 0 and white[2] == 0 and abs(white[3] * 0.5 - 1.0) < 1e-12
    back = to_acescg @ np.ones(3)
    assert np.all(np.abs(back - 1.0) < 1e-6)
    integrals = orc.cmf_integrals()
    lam = np.arange(360.0, 831.0, 1.0)
    obs = np.array([orc.cmf(l) for l in lam])
    for color in [(0.8, 0.2, 0.1), (0.05, 0.5, 0.2), (0.1, 0.2, 0.9), (0.9, 0.9, 0.2)]:
        c0, c1, c2, scale = orc.fit_spectrum(color)
        x = (lam - 360.0) / 470.0
        z = (c0 * x + c1) * x + c2
        s = scale * (0.5 + z / (2.0 * np.sqrt(1.0 + z * z)))
        xyz = (obs * s[:, None]).sum(0) / integrals
        rgb = to_acescg @ xyz
        assert np.all(np.abs(rgb - np.array(color)) < 0.01)


def test_blackbody_hues():
    # tests.lucb:111-122
    to_acescg = orc.film_matrix()
    n = to_acescg @ (orc.blackbody_xyz(5455.0) / orc.blackbody_xyz(5455.0)[1])
    assert np.all(np.abs(n - 1.0) < 0.06)
    w = to_acescg @ (orc.blackbody_xyz(3000.0) / orc.blackbody_xyz(3000.0)[1])
    assert w[0] > 1.2 * w[1] and w[1] > w[2]
    k = to_acescg @ (orc.blackbody_xyz(9000.0) / orc.blackbody_xyz(9000.0)[1])
    assert k[2] > k[1] > k[0]


def test_octahedral_normals_round_trip():
    # tests.lucb:126-144
    for d in [(0.3, -0.5, 0.8), (-1.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.6, 0.6, -0.5)]:
        e = np.array(d) / np.linalg.norm(d)
        assert np.linalg.norm(orc.octahedral_decode(orc.octahedral(e)) - e) < 1e-3


def test_sphere_shading_normals_point_outward():
    # tests.lucb:134-153: compiled shading normals of a sphere point away from its centre.
    p, t, n = scenes.icosphere(2, 1.0)
    sc = lr.compile_scene([lr.MeshData(p, t, normals=n, transform=lr.placement((0.0, 1.0, 0.0)))])
    a = sc.arrays()
    for tri in range(sc.triangle_count()):
        for k in range(3):
            pos = a["positions"][a["indices"][tri][k]] - np.array([0.0, 1.0, 0.0])
            normal = orc.octahedral_decode(int(a["shading"][tri][k]))
            assert normal @ pos > 0.9


def test_light_tree_trails_and_energy():
    # tests.lucb:155-183: a 9x9 grid, every triangle emitting.
    p, t, f = scenes.grid(4.0, 9)
    sc = lr.compile_scene([lr.MeshData(p, t, faces=f, face_count=81)])
    a = sc.arrays()
    glowing = orc.material_standard()
    glowing.emission_luminance = 2.0
    tree = orc.light_tree(a["positions"], a["indices"], a["shading"], np.zeros(0, np.float32), [glowing])
    count = tree["emitter_count"]
    assert count == sc.triangle_count() == 162
    records, links, nodes = tree["records"], tree["links"], tree["nodes"]
    total = 0.0
    for index in range(count):
        trail, depth = records[index * 4 + 1], records[index * 4 + 2]
        assert depth <= 8
        node = 0
        for level in range(depth):
            node = int(links[node][0]) + int((trail >> level) & 1)
        assert links[node][1] == 0x80000000 and links[node][0] == index
        code = records[index * 4]
        assert code & 0x80000000 and records[count * 4 + (code & 0x7FFFFFFF)] == index
        total += float(nodes[node][3])
    assert abs(float(nodes[0][3]) / total - 1.0) < 1e-4


def test_oracle_light_tracing_is_unbiased():
    # The three-technique estimator (connect.glsl) in f64: the area light's closed form
    # within the reference's 2 % with light paths, and the Cornell box's image the same as
    # camera paths alone within 3 sigma; the light paths contribute through their splats.

    meshes, cams, lights, mats = testscenes.area_light_scene()
    sc = lr.compile_scene(meshes, cams, lights, mats)
    frame = lr.ray_frame(sc.camera(), 32, 32)
    library = [lr.OpenPbr.lambert((0.5, 0.5, 0.5))] + list(mats)
    mean, _ = orc.render(sc.arrays(), lights, library, frame, 128, 1, False, light_tracing=0.5)
    assert abs(mean[14:18, 14:18, 1].mean() / testscenes.AREA_LIGHT_EXPECTED - 1.0) <= 0.02
    job = orc.RenderJob(sc.arrays(), lights, library, frame, 1, False, light_tracing=0.5)
    assert job.light_paths == 512
    camera_part, _, _ = job.region(32, 0, 0, 32 * 32)
    traced, _, _ = job.traced(32)
    assert traced.sum() > camera_part.sum()  # splats add what the weights took away
    sc = lr.compile_scene(scenes.cornell_meshes(True), [scenes.cornell_camera()], [scenes.cornell_light()],
                          scenes.cornell_materials())
    frame = lr.ray_frame(sc.camera(), 32, 32)
    library = [lr.OpenPbr.lambert()] + scenes.cornell_materials()
    a, va = orc.render(sc.arrays(), [scenes.cornell_light()], library, frame, 32, 5, True, light_tracing=0.5)
    b, vb = orc.render(sc.arrays(), [scenes.cornell_light()], library, frame, 32, 5, True)
    blocks = lambda x: x.reshape(4, 8, 4, 8, 3).mean((1, 3))
    sem = np.sqrt((blocks(va) + blocks(vb)) / (64 * 32))
    assert np.all(np.abs(blocks(a) - blocks(b)) <= 3.0 * sem + 1e-9)


def _source_order_indices(a):
    # The compiled scene keeps triangles in leaf order; the build takes them in source order.
    indices = np.empty_like(a["indices"])
    indices[a["order"]] = a["indices"]
    return indices


@pytest.mark.parametrize("which", ["cornell", "icosphere", "million"])
def test_bvh_equals_oracle_build_node_for_node(which):
    # The product's binned-SAH build (csrc/bvh.cpp) against the oracle's restatement of
    # bvh.lucb:66-217, byte for byte: nodes (boxes, links, counts) and leaf order. The
    # traversal work the roofline counts (interior visits, triangle tests) is counted on
    # this tree, so it is the reference's tree.
    if which == "cornell":
        sc = lr.compile_scene(scenes.cornell_meshes(True), [scenes.cornell_camera()], [scenes.cornell_light()],
                              scenes.cornell_materials())
        expect = 34
    elif which == "icosphere":
        sc = lr.compile_scene(scenes.furnace_meshes(5))
        expect = 20480
    else:
        meshes, mats, lights, cam = scenes.incoherent_scene()
        sc = lr.compile_scene(meshes, [cam], lights, mats)
        expect = 1 << 20
    try:
        a = sc.arrays()
        assert sc.triangle_count() == expect
        nodes, order = orc.build_bvh(a["positions"], _source_order_indices(a))
        assert len(nodes) == len(a["nodes"])
        assert np.array_equal(nodes.view(np.uint8), a["nodes"].view(np.uint8))
        assert np.array_equal(order, a["order"])
    finally:
        sc.close()


def _compiled_equal(meshes, library, cams=(), lights=(), mats=()):
    sc = lr.compile_scene(meshes, cams, lights, mats)
    try:
        a = sc.arrays()
        o = orc.compile_meshes(meshes, library)
        for key in ("positions", "indices", "shading", "faces", "order"):
            assert np.array_equal(np.asarray(a[key]).reshape(-1).view(np.uint32),
                                  np.asarray(o[key]).reshape(-1).view(np.uint32)), key
        assert np.array_equal(a["nodes"].view(np.uint8), o["nodes"].view(np.uint8))
    finally:
        sc.close()


@pytest.mark.parametrize("which", ["cornell", "icosphere", "million"])
def test_scene_compile_equals_oracle_compile(which):
    # csrc/scene.cpp (placement, polygons, octahedral normals, materials, BVH, leaf order)
    # against the oracle's restatement of scene.lucb's compile_scene, bit for bit.
    if which == "cornell":
        mats = scenes.cornell_materials()
        _compiled_equal(scenes.cornell_meshes(True), len(mats), [scenes.cornell_camera()], [scenes.cornell_light()],
                        mats)
    elif which == "icosphere":
        _compiled_equal(scenes.furnace_meshes(5), 0)
    else:
        meshes, mats, lights, cam = scenes.incoherent_scene()
        _compiled_equal(meshes, len(mats), [cam], lights, mats)


def test_scene_compile_edge_cases_equal_oracle():
    # Per-corner normals, polygons of two triangles, a mirroring placement (the normals'
    # cofactors take the determinant's sign), a singular one, unknown materials (-> 0).
    p, t, f = scenes.cube(2.0)
    rng = np.random.default_rng(3)
    corner_normals = rng.normal(size=(len(t) * 3, 3)).astype(np.float32)
    mirror = lr.placement((1.0, 2.0, 3.0), (0.3, 0.2, 0.1), (-1.0, 2.0, 0.5))
    flat = np.zeros(12)
    flat[0], flat[4], flat[9] = 1.0, 1.0, 4.0  # z axis zero: singular
    meshes = [lr.MeshData(p, t, faces=f, face_count=6, face_materials=[0, 1, 2, 3, 9, 1]),
              lr.MeshData(p, t, normals=corner_normals, normals_per_corner=True, transform=mirror),
              lr.MeshData(p, t, normals=p, faces=f, face_count=6, transform=flat),
              lr.MeshData(p, t, transform=mirror)]
    mats = [lr.OpenPbr.lambert(), lr.OpenPbr.lambert((0.2, 0.3, 0.4)), lr.OpenPbr.lambert((0.9, 0.1, 0.1))]
    _compiled_equal(meshes, len(mats), mats=mats)
