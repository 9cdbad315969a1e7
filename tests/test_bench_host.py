"""bench.py's host logic on the CPU: the replicas' reduction over ranks (two gloo ranks,
as torchrun launches them), the served arrival stream and the latency percentiles."""
import os
import socket

import numpy as np
import pytest

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    d = bench.Dist(world)
    d.barrier()
    # Each replica reports its own rays and time; the line takes the sum and the max.
    rays, ms = 1000.0 * (rank + 1), 10.0 + rank
    out.put((rank, d.sum(rays), d.max(ms)))
    d.close()


def test_replicas_reduce_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 3000.0, 11.0), (1, 3000.0, 11.0)]


def test_single_rank_needs_no_process_group():
    for key in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(key, None)
    d = bench.Dist(1)
    assert d.world == 1 and d.sum(5.0) == 5.0 and d.max(2.0) == 2.0
    d.barrier()
    d.close()


def test_arrival_stream_shape():
    a = bench.arrival_stream(60.0, 64)
    times = np.array([x[0] for x in a])
    assert np.all(np.diff(times) > 0) and times[-1] < 60.0
    assert abs(len(a) / 60.0 - 200.0) < 10.0  # Poisson at 200 a second
    probes = [x for x in a if x[1] == "probe"]
    renders = [x for x in a if x[1] == "render"]
    assert abs(len(probes) / len(a) - 0.2) < 0.02
    px = np.array([w * h for _, _, _, w, h in probes])
    assert px.min() >= 900 and px.max() <= 2_000_000
    spp = np.array([s for _, _, _, s, _ in renders])
    assert spp.min() >= 16 and spp.max() <= 256
    assert all(0 <= x[2] < 64 for x in a)
    assert a == bench.arrival_stream(60.0, 64)  # seeded


def test_percentiles():
    p = bench.percentiles([0.001 * i for i in range(1, 101)])
    assert p["count"] == 100 and abs(p["p50_ms"] - 50.5) < 1e-9 and abs(p["p99_ms"] - 99.01) < 1e-6
    assert bench.percentiles([])["p50_ms"] is None


@pytest.mark.parametrize("count", [64])
def test_batch_plan_distribution(count):
    from luce_render_b200 import scenes

    plan = scenes.batch_plan(count)
    tris = np.array([p["triangles"] for p in plan])
    assert tris.min() >= 1000 and tris.max() <= 500000
    assert 5000 < np.median(tris) < 80000
    assert set(p["side"] for p in plan) <= {128, 256, 512, 1024}
    assert sum(p["spectral"] for p in plan) == count // 2
