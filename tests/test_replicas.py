"""Multi-GPU plan on the host, with 2 gloo ranks on CPU: replicas only.

Each rank serves its own seeded request stream (no data exchange); the step time is the
slowest rank's, taken with one all-reduce; the reported value is the sum of all ranks'
solves over that time.  Nothing here touches a GPU.
"""
import datetime
import os
import socket
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import __graft_entry__ as ge
        sv = ge.load_package().serving
        reqs = sv.make_stream(count=3, rate=2000.0, seed=bench.stream_seed(rank), device="cpu",
                              edges=(16,))
        digest = float(sum(float(r.sigma.sum()) + 31.0 * float(r.rhs.abs().sum()) for r in reqs))
        ms = 10.0 * (rank + 1)  # this rank's device time of a step
        slowest = bench.max_over_ranks(torch, ms, "cpu")
        digests = [None] * world
        dist.all_gather_object(digests, digest)
        q.put((rank, slowest, digests))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    # every rank sees the slowest rank's time
    assert [o[1] for o in out] == [20.0, 20.0]
    # the ranks' streams are different (own seeds) and every rank agrees on them
    assert out[0][2] == out[1][2]
    assert out[0][2][0] != out[0][2][1]


def test_single_process_time_is_own():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(torch, 12.5, "cpu") == 12.5
    assert bench.stream_seed(0) != bench.stream_seed(1)
