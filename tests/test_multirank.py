"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (127.0.0.1) take disjoint instance
shards, agree on the job's step time as the max over ranks, and no rank exchanges instance data."""
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
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = bench.shard(rank, 3)
    allv = [None] * world
    dist.all_gather_object(allv, mine)
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, allv, ms))


def test_two_gloo_ranks_shard_instances_and_take_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, allv, ms in out:
        flat = [i for v in allv for i in v]
        assert sorted(flat) == list(range(6))        # disjoint, complete
        assert ms == pytest.approx(15.0)              # slowest rank's time
