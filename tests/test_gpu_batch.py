"""Batches (lr_batch) through the C ABI: every member's image equals, bit for bit, the
image a Renderer of its own makes of the same scene, frame and settings -- alone or in
the mix, whatever the pool size, and with members joining and leaving between passes.
Each path's arithmetic depends only on its member, pixel and sample, and a pixel takes
its samples in order, so the tolerance is zero."""
import numpy as np
import pytest

import luce_render_b200 as lr
import render_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cases(ctx):
    cs = render_cases.cases()
    uploads = [lr.GpuScene.upload(ctx, sc) for sc, _ in cs]
    alone = [render_cases.alone(ctx, sc, s) for sc, s in cs]
    yield cs, uploads, alone
    for gs in uploads:
        gs.destroy()
    for sc, _ in cs:
        sc.close()


def _bits(img):
    return np.ascontiguousarray(img, np.float32).view(np.uint32)


@pytest.mark.parametrize("pool", [1 << 21, 1500, 333])
def test_members_equal_their_renderers(ctx, cases, pool):
    # A pool larger than all films together (one pass a sample for everyone), one that
    # splits the larger films over passes, and one smaller than every film but the last.
    cs, uploads, alone = cases
    # 12 bounces of room: 11 rounds for the cut-out case (2 bounces + 1 + 8).
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=pool, max_bounces=12, capacity=16))
    try:
        members = [b.add(gs, sc, s) for gs, (sc, s) in zip(uploads, cs)]
        b.finish()
        for m, (sc, s), want in zip(members, cs, alone):
            assert b.samples_done(m) == s.c.samples
            got = b.read(m)
            assert np.array_equal(_bits(got), _bits(want)), m
        st = b.stats()
        total_paths = sum(s.c.width * s.c.height * s.c.samples for _, s in cs)
        assert st.shaded == total_paths
        if pool >= 1 << 21:
            assert st.passes == max(s.c.samples for _, s in cs)
    finally:
        b.destroy()


def test_members_join_and_leave(ctx, cases):
    cs, uploads, alone = cases
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=700, max_bounces=8, capacity=3))
    try:
        first = b.add(uploads[0], *cs[0])
        leaving = b.add(uploads[3], *cs[3])
        for _ in range(5):
            b.advance()
        # A member joins while passes are in flight; another leaves part way.
        late = b.add(uploads[1], *cs[1])
        for _ in range(3):
            b.advance()
        b.remove(leaving)
        with pytest.raises(lr.RenderError):
            b.info(leaving)
        # Its slot is taken again once its passes have finished.
        again = b.add(uploads[4], *cs[4])
        b.finish()
        for m, i in ((first, 0), (late, 1), (again, 4)):
            assert np.array_equal(_bits(b.read(m)), _bits(alone[i])), i
    finally:
        b.destroy()


def test_more_samples_later(ctx, cases):
    # set_samples after a finish continues each pixel's sample sequence.
    cs, uploads, alone = cases
    sc, s = cs[2]
    fewer = render_cases.settings(24, 20, 2, 2, True, seed=7, material=lr.OpenPbr.lambert((0.5, 0.5, 0.5)))
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=100, max_bounces=4, capacity=2))
    try:
        m = b.add(uploads[2], sc, fewer)
        b.finish()
        assert b.info(m) == (2, 2, 2)
        b.set_samples(m, s.c.samples)
        b.finish()
        assert b.samples_done(m) == s.c.samples
        assert np.array_equal(_bits(b.read(m)), _bits(alone[2]))
    finally:
        b.destroy()


def test_batch_limits(ctx, cases):
    cs, uploads, _ = cases
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=4096, max_bounces=4, capacity=1))
    try:
        with pytest.raises(lr.RenderError) as e:
            b.add(uploads[0], *cs[0])  # 6 bounces > 4
        assert e.value.code == 401
        b.add(uploads[2], *cs[2])
        with pytest.raises(lr.RenderError) as e:
            b.add(uploads[4], *cs[4])  # full
        assert e.value.code == 401
    finally:
        b.destroy()
    with pytest.raises(lr.RenderError):
        lr.Batch(ctx, lr.BatchSettings.default(pool=0))


@pytest.mark.parametrize("refill", [32, 8, 1])
def test_refilling_warps_equal_grid_stride(ctx, cases, refill, monkeypatch):
    # Traversal warps that hand idle lanes new queue entries once `refill` lanes are idle
    # make the images the grid-stride walks make: a ray's result depends on it alone.
    cs, uploads, alone = cases
    monkeypatch.setenv("LUCE_RENDER_B200_REFILL", str(refill))
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=1500, max_bounces=12, capacity=16))
    try:
        members = [b.add(gs, sc, s) for gs, (sc, s) in zip(uploads, cs)]
        b.finish()
        for m, want in zip(members, alone):
            assert np.array_equal(_bits(b.read(m)), _bits(want)), m
    finally:
        b.destroy()


@pytest.mark.parametrize("thin", [-1, 1, 3])
def test_thin_rounds_on_the_wide_tree_equal(ctx, cases, thin, monkeypatch):
    # Passes that trace their rounds from `thin` on over the compressed 8-wide tree (-1:
    # none) make the images the BVH2 alone makes: the closest hit does not depend on the tree.
    cs, uploads, alone = cases
    monkeypatch.setenv("LUCE_RENDER_B200_THIN", str(thin))
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=1500, max_bounces=12, capacity=16))
    try:
        members = [b.add(gs, sc, s) for gs, (sc, s) in zip(uploads, cs)]
        b.finish()
        for m, want in zip(members, alone):
            assert np.array_equal(_bits(b.read(m)), _bits(want)), m
    finally:
        b.destroy()


def test_ticketed_reads_land_the_images(ctx, cases):
    # Reads queued with tickets while the other members' passes still run land the same
    # images a waiting read gives; each ticket lands, and later tickets land after earlier.
    cs, uploads, alone = cases
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=1500, max_bounces=12, capacity=16))
    pinned = []
    try:
        members = [b.add(gs, sc, s) for gs, (sc, s) in zip(uploads, cs)]
        tickets = []

        def read_finished():
            for m, (sc, s) in zip(members, cs):
                if any(t[0] == m for t in tickets) or b.info(m)[0] < s.c.samples:
                    continue
                buf = lr.PinnedArray((s.c.height, s.c.width, 4), np.float32)
                pinned.append(buf)
                tickets.append((m, b.read_ticket(m, buf.array), buf))

        for _ in range(100000):
            more = b.advance()
            read_finished()
            if not more:
                break
        b.finish()
        read_finished()
        assert len(tickets) == len(members)
        for k, (m, t, buf) in enumerate(tickets):
            for _ in range(10000):
                if b.read_landed(t):
                    break
            assert b.read_landed(t)
            assert all(b.read_landed(tickets[j][1]) for j in range(k))
            assert np.array_equal(_bits(buf.array), _bits(alone[members.index(m)])), m
    finally:
        b.destroy()
        for buf in pinned:
            buf.close()


def test_tuning_changes_speed_not_images(ctx, cases):
    cs, uploads, alone = cases
    b = lr.Batch(ctx, lr.BatchSettings.default(pool=2048, max_bounces=12, capacity=16))
    try:
        members = [b.add(gs, sc, s) for gs, (sc, s) in zip(uploads, cs)]
        for _ in range(3):
            b.advance()
        t = b.tune()
        assert t["width"] in (2, 4, 8) and t["fill"] in (512, 1024, 2048)
        assert t["refill_at"] in (0, 32, 16, 8) and t["bin_interval"] in (0, 1, 2) and t["thin_from"] in (-1, 2, 3, 4)
        assert t["candidates"] >= 4 and t["paths_per_ms"] > 0
        # The cases hold scenes under 16k triangles and one of about 20k.
        assert t["class_members"][0] >= 1 and t["class_members"][1] == 1 and t["class_members"][2] == 0
        assert all(w in (2, 4, 8) for w in t["class_width"][:2]) and t["class_width"][2] == 0
        st = b.stats()
        b.finish()
        for m, want in zip(members, alone):
            assert np.array_equal(_bits(b.read(m)), _bits(want)), m
        # Trial passes add no paths to the count of finished work.
        assert b.stats().shaded == sum(s.c.width * s.c.height * s.c.samples for _, s in cs)
        assert st.shaded <= b.stats().shaded
    finally:
        b.destroy()
