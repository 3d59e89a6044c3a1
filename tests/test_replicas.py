"""The multi-rank path of bench.py on CPU: two ranks over gloo.

The timestep does not shard across GPUs here (replicas only), so the only
collectives are the barrier around the timed region and the max over ranks
of the per-rank step time.  These tests run those helpers, exactly as
bench.py calls them, in two spawned processes, and check that every rank
sees the slowest rank's time.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, dist, barrier, max_over_ranks = bench.init_replicas("gloo")
    assert (w, r, local) == (world, rank, rank)
    barrier()
    # each replica reports its own step time; the line carries the slowest
    t = max_over_ranks(100.0 + 10.0 * rank)
    barrier()
    out.put((rank, t))
    dist.destroy_process_group()


def test_two_replicas_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 110.0, 1: 110.0}


def test_single_process_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, dist, barrier, max_over_ranks = bench.init_replicas("gloo")
    assert (w, r, local, dist) == (1, 0, 0, None)
    barrier()
    assert max_over_ranks(3.5) == 3.5


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
