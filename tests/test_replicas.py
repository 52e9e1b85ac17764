"""Multi-GPU plumbing of bench.py on CPU: N independent replicas synchronise through a
gloo process group (barrier, max over ranks of the timed region, whole-job value),
world size 2 on 127.0.0.1.  No data-path collective exists (one solve per GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    elapsed = bench.max_over_ranks(w, 1.0 + rank)  # rank 1 is the slowest
    out.put((rank, elapsed))
    import torch.distributed as dist
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_take_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(100)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 2.0, 1: 2.0}
