"""The multi-rank path of bench.py on CPU: two gloo ranks, each solving its
own subgames (weak scaling), reduce the step time with a max and the solve
count with a sum; no other collective touches the data path."""
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


def _rank(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    import torch.distributed as dist
    w, r, loc = bench.dist_init()
    assert dist.get_backend() == "gloo"
    step_ms = 10.0 * (r + 1)
    bench.barrier()
    q.put((r, w, bench.dist_max(step_ms), bench.dist_sum(3)))
    dist.destroy_process_group()


def test_two_rank_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, mx, sm in res:
        assert w == 2 and mx == 20.0 and sm == 6.0
