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
