"""Multi-process (world size 2, gloo on CPU) checks of the replica plumbing
bench.py uses under torchrun: rendezvous, barrier, max over ranks and the
whole-job aggregate (every rank's units over the slowest rank's time)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from wgpufft_b200.replicas import Replicas
    rep = Replicas(backend="gloo", timeout_s=30)
    rep.barrier()
    seconds = 1.0 + rank  # rank 1 is the slow one
    lines = 20000.0
    m = rep.max(seconds)
    rate = rep.aggregate_rate(lines, seconds)
    q.put((rank, m, rate))
    rep.close()


def test_two_rank_aggregation_with_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, rate in res:
        assert m == pytest.approx(2.0)
        assert rate == pytest.approx(2 * 20000.0 / 2.0)


def test_single_process_is_identity():
    from wgpufft_b200.replicas import Replicas
    os.environ.pop("WORLD_SIZE", None)
    rep = Replicas()
    assert rep.world == 1 and rep.max(3.0) == 3.0
    assert rep.aggregate_rate(10.0, 2.0) == 5.0
    rep.close()


def _partition_worker(rank, world, port, q):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist

    from wgpufft_b200 import workloads as W
    from wgpufft_b200.replicas import Replicas, partition_lines
    rep = Replicas(backend="gloo", timeout_s=30)
    lengths = W.mixed_lengths()
    mine = partition_lines(lengths, world)[rank]
    everyone = [None] * world
    dist.all_gather_object(everyone, mine)
    q.put((rank, mine, everyone, int(lengths[mine[0]:mine[1]].sum())))
    rep.close()


def test_two_rank_partition_owns_every_line_once():
    # the bench's strong-scaling split: each rank takes one contiguous run of
    # lines; the runs are the same on every rank, cover every line exactly
    # once and hold about equal points
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_partition_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from wgpufft_b200 import workloads as W
    n = len(W.mixed_lengths())
    runs = res[0][2]
    assert all(r[2] == runs for r in res)
    assert [r[1] for r in res] == [tuple(x) for x in runs]
    owned = [i for a, b in runs for i in range(a, b)]
    assert owned == list(range(n))
    pts = [r[3] for r in res]
    assert max(pts) / min(pts) < 1.01


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8, 64])
def test_partition_properties(world):
    import numpy as np

    from wgpufft_b200.replicas import partition_lines
    rng = np.random.default_rng(world)
    for lengths in (rng.integers(1, 70000, 997), np.array([7]), np.array([], dtype=np.int64),
                    np.full(5, 100)):
        runs = partition_lines(lengths, world)
        assert len(runs) == world
        assert runs[0][0] == 0 and runs[-1][1] == len(lengths)
        for (a, b), (c, d) in zip(runs, runs[1:]):
            assert b == c and a <= b
        if len(lengths) >= 4 * world and world > 1:
            pts = [int(lengths[a:b].sum()) for a, b in runs]
            assert max(pts) <= lengths.sum() / world + lengths.max()
