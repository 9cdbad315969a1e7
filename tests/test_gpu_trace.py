"""Parity of the CUDA traversal with the oracle, through the C ABI (probe, ray queries).

- The default (watertight) path: every closest hit -- triangle id, t, u, v -- equals an
  FP32 brute force over all triangles running the same watertight test, bit for bit
  (ties in t go to the smaller id on both sides, so exact-t ties agree too); any-hit
  agrees with "the closest hit exists".
- The reference path (LR_TRACE_REFERENCE): equal, bit for bit, to the oracle's
  restatement of shaders/bvh.glsl's trace_closest / trace_any on the same BVH.
- The reference's own acceptance rule (tests/gpu/main.lucb:61-78): polygon ids equal and
  |dt| <= 1e-4 t against the f64 brute force, forgiving near-ties (margin <= 1e-3).
"""
import math

import numpy as np
import pytest

import luce_render_b200 as lr
from luce_render_b200 import scenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _upload(ctx, meshes, cams=()):
    sc = lr.compile_scene(meshes, cams)
    return sc, sc.arrays(), lr.GpuScene.upload(ctx, sc)


def _as_bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def cornell(ctx):
    sc, a, gs = _upload(ctx, scenes.cornell_meshes())
    yield sc, a, gs
    gs.destroy()
    sc.close()


def _check_exact(ctx, a, gs, rays):
    hits = lr.trace_rays(ctx, gs, rays)
    prim, t, u, v = orc.brute_watertight(a["positions"], a["indices"], a["order"], rays)
    got = lr.hit_ids(hits)
    assert np.array_equal(got, prim), f"{np.count_nonzero(got != prim)} ids differ"
    hit = prim >= 0
    assert np.array_equal(_as_bits(hits[:, 0]), _as_bits(t))
    assert np.array_equal(_as_bits(hits[hit, 2]), _as_bits(u[hit]))
    assert np.array_equal(_as_bits(hits[hit, 3]), _as_bits(v[hit]))
    anyh = lr.trace_rays(ctx, gs, rays, any_hit=True)
    assert np.array_equal(lr.hit_ids(anyh) >= 0, hit)
    return hits, prim, t


def _check_reference(ctx, a, gs, rays):
    hits = lr.trace_rays(ctx, gs, rays, reference=True)
    ref, counts = orc.trace(a["nodes"], a["positions"], a["indices"], rays)
    assert counts.dropped == 0
    slot = ref["triangle"].astype(np.int64)
    want = np.where(slot == 0xFFFFFFFF, -1, a["order"][np.minimum(slot, len(a["order"]) - 1)].astype(np.int64))
    assert np.array_equal(lr.hit_ids(hits), want.astype(np.int32))
    assert np.array_equal(_as_bits(hits[:, 0]), _as_bits(ref["t"]))
    m = slot != 0xFFFFFFFF
    assert np.array_equal(_as_bits(hits[m, 2]), _as_bits(ref["u"][m]))
    assert np.array_equal(_as_bits(hits[m, 3]), _as_bits(ref["v"][m]))
    anyh = lr.trace_rays(ctx, gs, rays, any_hit=True, reference=True)
    refany, _ = orc.trace(a["nodes"], a["positions"], a["indices"], rays, any_hit=True)
    assert np.array_equal(lr.hit_ids(anyh) >= 0, refany.astype(bool))


def test_cornell_primary_rays_exact(ctx, cornell):
    sc, a, gs = cornell
    rays = scenes.frame_rays(scenes.cornell_frame(256, 256))
    _check_exact(ctx, a, gs, rays)


def test_cornell_random_rays_exact(ctx, cornell):
    sc, a, gs = cornell
    _check_exact(ctx, a, gs, scenes.random_rays(65536))


def test_cornell_reference_traversal(ctx, cornell):
    sc, a, gs = cornell
    _check_reference(ctx, a, gs, scenes.frame_rays(scenes.cornell_frame(256, 256)))
    _check_reference(ctx, a, gs, scenes.random_rays(65536))


def test_probe_matches_oracle_bitwise(ctx, cornell):
    sc, a, gs = cornell
    frame = scenes.cornell_frame(256, 256)
    block = frame.pack()
    rays = orc.probe_rays(block)
    assert np.array_equal(rays, scenes.frame_rays(frame))
    # reference path: the restated probe.comp + trace_closest
    faces, dist = lr.probe(ctx, gs, frame, reference=True)
    ref, _ = orc.trace(a["nodes"], a["positions"], a["indices"], rays)
    slot = ref["triangle"]
    want = np.where(slot == 0xFFFFFFFF, 0xFFFFFFFF, a["faces"][np.minimum(slot, len(a["faces"]) - 1)])
    assert np.array_equal(faces, want.astype(np.uint32))
    assert np.array_equal(_as_bits(dist), _as_bits(ref["t"]))
    # default path: the watertight brute force
    faces, dist = lr.probe(ctx, gs, frame)
    prim, t, _, _ = orc.brute_watertight(a["positions"], a["indices"], a["order"], rays)
    slot_of = np.empty_like(a["order"])
    slot_of[a["order"]] = np.arange(len(a["order"]), dtype=np.uint32)
    want = np.where(prim < 0, 0xFFFFFFFF, a["faces"][slot_of[np.maximum(prim, 0)]])
    assert np.array_equal(faces, want.astype(np.uint32))
    assert np.array_equal(_as_bits(dist), _as_bits(t))


def _reference_rule(frame, faces, dist, a):
    """compare (tests/gpu/main.lucb:61-78) against the f64 brute force."""
    w, h = frame.width, frame.height
    rays = np.zeros((w * h, 8), np.float32)
    for y in range(h):
        for x in range(w):
            o, d = frame.ray(x + 0.5, y + 0.5)
            rays[y * w + x, 0:3] = o
            rays[y * w + x, 4:7] = d
            rays[y * w + x, 7] = 3e38
    face, distance, margin = orc.nearest_f64(a["positions"], a["indices"], a["faces"], rays)
    got_none = faces == 0xFFFFFFFF
    agrees = (got_none & (face < 0)) | (~got_none & (face >= 0) & (faces.astype(np.int64) == face) &
                                        (np.abs(dist.astype(np.float64) - distance) <= 1e-4 * distance))
    differ = np.count_nonzero(~agrees & (margin > 1e-3))
    hits = np.count_nonzero(face >= 0)
    return hits, differ


@pytest.mark.parametrize("reference", [False, True])
def test_probe_reference_acceptance_rule(ctx, reference):
    meshes, cams = scenes.probe_test_scene()
    sc, a, gs = _upload(ctx, meshes, cams)
    try:
        for index in range(2):
            frame = lr.ray_frame(sc.camera(index), 96, 64)
            faces, dist = lr.probe(ctx, gs, frame, reference=reference)
            hits, differ = _reference_rule(frame, faces, dist, a)
            assert hits > (96 * 64) // 2 and differ == 0, (index, hits, differ)
    finally:
        gs.destroy()
        sc.close()


def test_edge_cases(ctx):
    # An empty scene: every ray misses; one triangle (the root is a leaf).
    empty = lr.compile_scene([])
    gs = lr.GpuScene.upload(ctx, empty)
    rays = scenes.random_rays(1000)
    hits = lr.trace_rays(ctx, gs, rays)
    assert np.all(lr.hit_ids(hits) == -1) and np.all(hits[:, 0] == np.float32(3e38))
    gs.destroy()
    one = lr.compile_scene([lr.MeshData([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 2]])])
    a = one.arrays()
    gs = lr.GpuScene.upload(ctx, one)
    r = np.array([[0.25, 0.25, 1, 0, 0, 0, -1, 3e38], [0.25, 0.25, 1, 0, 0, 0, 1, 3e38],
                  [0.6, 0.6, 1, 0, 0, 0, -1, 3e38], [0.25, 0.25, 1, 0, 0, 0, -1, 0.5],
                  [0.25, 0.25, 1, 2.0, 0, 0, -1, 3e38], [0.0, 0.0, 1, 0, 0, 0, -1, 3e38]], np.float32)
    hits = lr.trace_rays(ctx, gs, r)
    prim, t, _, _ = orc.brute_watertight(a["positions"], a["indices"], a["order"], r)
    assert np.array_equal(lr.hit_ids(hits), prim)
    assert lr.hit_ids(hits).tolist()[:5] == [0, -1, -1, -1, -1]
    assert np.array_equal(_as_bits(hits[:, 0]), _as_bits(t))
    gs.destroy()
    # Axis-parallel rays and a ray grazing shared edges of a grid (watertightness: a
    # ray through a shared vertex or edge hits some triangle).
    p, tt, f = scenes.grid(4.0, 4)
    g = lr.compile_scene([lr.MeshData(p, tt, faces=f, face_count=16)])
    ga = g.arrays()
    gs = lr.GpuScene.upload(ctx, g)
    xs = np.linspace(-2.0, 2.0, 9)
    r = np.array([[x, 1.0, z, 0, 0, -1, 0, 3e38] for x in xs for z in xs], np.float32)
    hits = lr.trace_rays(ctx, gs, r)
    prim, t, _, _ = orc.brute_watertight(ga["positions"], ga["indices"], ga["order"], r)
    assert np.array_equal(lr.hit_ids(hits), prim)
    assert np.all(prim >= 0), "a ray through a shared edge or vertex fell through"
    gs.destroy()


@pytest.fixture(scope="module")
def incoherent(ctx):
    meshes, mats, lights, cam = scenes.incoherent_scene()
    sc, a, gs = _upload(ctx, meshes)
    yield sc, a, gs
    gs.destroy()
    sc.close()


def test_million_triangles_exact_subset(ctx, incoherent):
    sc, a, gs = incoherent
    assert sc.triangle_count() == 1 << 20
    rays = scenes.incoherent_rays(2048)
    _check_exact(ctx, a, gs, rays)


def test_million_triangles_reference_traversal(ctx, incoherent):
    sc, a, gs = incoherent
    _check_reference(ctx, a, gs, scenes.incoherent_rays(1 << 18, seed=7))


def test_traversal_work_counts_match_oracle(ctx, incoherent, cornell):
    # The reference path's interior visits and triangle tests equal the oracle's
    # restatement of trace_closest / trace_any exactly (the work the roofline's
    # algorithmic bytes are counted from); the watertight path, over boxes widened by a
    # few ulps of the scene scale, does at least that work and not much more.
    for fixture, rays in ((incoherent, scenes.incoherent_rays(1 << 16, seed=5)),
                          (cornell, scenes.random_rays(1 << 16))):
        sc, a, gs = fixture
        lr.trace_counts(ctx)
        for any_hit in (False, True):
            lr.trace_rays(ctx, gs, rays, any_hit=any_hit, reference=True, count=True)
            nodes, tests = lr.trace_counts(ctx)
            _, counts = orc.trace(a["nodes"], a["positions"], a["indices"], rays, any_hit=any_hit)
            assert (nodes, tests) == (counts.interior, counts.triangles)
            lr.trace_rays(ctx, gs, rays, any_hit=any_hit, count=True, width=2)
            enodes, etests = lr.trace_counts(ctx)
            if not any_hit:
                assert counts.interior <= enodes <= 1.05 * counts.interior
                assert counts.triangles <= etests <= 1.05 * counts.triangles


def test_bvh_widths_agree_bit_for_bit(ctx, incoherent, cornell):
    # The 4- and 8-wide collapses reach the same leaves and keep the same tie rule, so
    # closest and any hits equal the BVH2 path's exactly; they visit fewer nodes.
    for fixture, rays in ((incoherent, scenes.incoherent_rays(1 << 18, seed=9)),
                          (cornell, scenes.random_rays(1 << 16, seed=3))):
        sc, a, gs = fixture
        info = gs.info
        assert info.width in (2, 4, 8)
        base = lr.trace_rays(ctx, gs, rays, width=2, count=True)
        base_nodes, base_tests = lr.trace_counts(ctx)
        base_any = lr.trace_rays(ctx, gs, rays, width=2, any_hit=True)
        for w in (4, 8):
            hits = lr.trace_rays(ctx, gs, rays, width=w, count=True)
            nodes, tests = lr.trace_counts(ctx)
            assert np.array_equal(_as_bits(hits), _as_bits(base)), w
            anyh = lr.trace_rays(ctx, gs, rays, width=w, any_hit=True)
            assert np.array_equal(lr.hit_ids(anyh) >= 0, lr.hit_ids(base_any) >= 0), w
            if sc.triangle_count() > 1000:
                assert nodes < base_nodes, (w, nodes, base_nodes)


@pytest.mark.parametrize("leaf", [4, 16])
def test_wide_trees_with_whole_subtree_leaves_agree(ctx, incoherent, leaf, monkeypatch):
    # Wide trees that take BVH2 subtrees of up to `leaf` triangles whole as leaves (one
    # contiguous range of the leaf order each) reach the same triangles: closest and any
    # hits equal the BVH2 path's bit for bit.
    sc, a, _ = incoherent
    monkeypatch.setenv("LUCE_RENDER_B200_WIDE_LEAF", str(leaf))
    gs = lr.GpuScene.upload(ctx, sc)
    try:
        rays = scenes.incoherent_rays(1 << 17, seed=21)
        base = lr.trace_rays(ctx, gs, rays, width=2)
        base_any = lr.trace_rays(ctx, gs, rays, width=2, any_hit=True)
        for w in (4, 8):
            assert np.array_equal(_as_bits(lr.trace_rays(ctx, gs, rays, width=w)), _as_bits(base)), w
            anyh = lr.trace_rays(ctx, gs, rays, width=w, any_hit=True)
            assert np.array_equal(lr.hit_ids(anyh) >= 0, lr.hit_ids(base_any) >= 0), w
    finally:
        gs.destroy()


def test_million_triangles_properties_at_full_size(ctx, incoherent):
    # 2^21 incoherent rays: any-hit agrees with the existence of a closest hit, and
    # every closest hit re-tested alone (the oracle's watertight test on that one
    # triangle) gives the same t.
    sc, a, gs = incoherent
    rays = scenes.incoherent_rays(1 << 21, seed=11)
    hits = lr.trace_rays(ctx, gs, rays)
    anyh = lr.trace_rays(ctx, gs, rays, any_hit=True)
    ids = lr.hit_ids(hits)
    assert np.array_equal(ids >= 0, lr.hit_ids(anyh) >= 0)
    pick = np.flatnonzero(ids >= 0)[:: 97]
    src = np.empty_like(a["indices"])
    src[a["order"]] = a["indices"]
    for i in pick[:2000]:
        tri = src[ids[i]]
        pts = a["positions"][tri]
        prim, t, _, _ = orc.brute_watertight(pts, np.array([[0, 1, 2]], np.uint32), None, rays[i:i + 1])
        assert prim[0] == 0 and np.float32(t[0]) == hits[i, 0]
