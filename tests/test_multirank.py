"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (127.0.0.1) take disjoint instance
shards, agree on the job's step time as the max over ranks, learn of a bad run status on any
rank, and no rank exchanges instance data."""
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
    # a status set on rank 1 alone reaches rank 0 too; a clean job stays clean everywhere
    st_bad = bench.job_status(4 if rank == 1 else 0, world, device="cpu")
    st_ok = bench.job_status(0, world, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, allv, ms, st_bad, st_ok))


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
    for rank, allv, ms, st_bad, st_ok in out:
        flat = [i for v in allv for i in v]
        assert sorted(flat) == list(range(6))        # disjoint, complete
        assert ms == pytest.approx(15.0)              # slowest rank's time
        assert st_bad == 4 and st_ok == 0            # every rank stops together


class _FakeNet:
    """Stands in for ScheduleGNN on CPU: a parameter vector pulled towards a per-problem target
    (the problem's n), mean squared loss over the problems of a step, plain gradient steps."""

    def __init__(self, dim=5):
        import numpy as np
        self.theta = np.zeros(dim)
        self.param_count = dim

    def train_step(self, problems, tk, ts, lr=0.0, lambda_spins=0.2, want_grads=True):
        import numpy as np
        t = np.array([[float(p.n)] * self.param_count for p in problems])
        d = self.theta[None, :] - t
        return float(np.mean(np.sum(d * d, axis=1))), (2.0 * d.mean(axis=0)).astype(np.float32)

    def apply_grads(self, g, lr=1e-3):
        self.theta = self.theta - lr * g


def _dp_rank(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist

    from tessera_b200 import instances, learned
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    probs = [instances.dense_er(n, 10 + n, T=1.0) for n in range(4, 15)]
    net = _FakeNet()
    losses = learned.train_data_parallel(net, probs, np.zeros((len(probs), 16)), [np.ones(p.n) for p in probs],
                                         epochs=3, batch=4, lr=0.1, seed=5)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, net.theta.tolist(), losses))


def test_data_parallel_training_matches_one_process():
    """learned.train_data_parallel on two gloo ranks: the replicas stay identical and follow the
    same trajectory as one process taking full-batch steps (the gradient all-reduce is weighted
    by the share sizes, so uneven shares average correctly)."""
    import numpy as np

    from tessera_b200 import instances, learned
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_dp_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=180) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.allclose(out[0][1], out[1][1], rtol=0, atol=0)
    # serial reference: same batch order, full-batch mean gradient
    probs = [instances.dense_er(n, 10 + n, T=1.0) for n in range(4, 15)]
    net = _FakeNet()
    rng = np.random.Generator(np.random.PCG64(5))
    idx = np.arange(len(probs))
    for _ in range(3):
        rng.shuffle(idx)
        for s in range(0, len(idx), 4):
            _, g = net.train_step([probs[i] for i in idx[s:s + 4]], None, None)
            net.apply_grads(g.astype(np.float64), lr=0.1)
    assert np.allclose(out[0][1], net.theta, rtol=1e-6, atol=1e-6)
    assert learned.spin_targets([np.ones(2)]).tolist() == [1.0, 1.0]


def _ragged_problems():
    from tessera_b200 import instances
    probs = [instances.dense_er(4 + (7 * k) % 13, 70 + k, T=0.5 + 0.1 * (k % 4), dt=0.1, chi=8 << (k % 3))
             for k in range(37)]
    probs += instances.batch_3_regular(count=8, T=0.2, dt=0.05, nmin=32, nmax=40)
    return probs


def _stub_runner(probs, fail=False):
    """Stands in for ffi.anneal_batch on CPU: one record per problem, computed from it alone."""
    if fail:
        raise RuntimeError("injected failure")
    from tessera_b200 import shard
    return [{"name": p.name, "n": p.n, "cost": shard.instance_cost(p)} for p in probs]


def _ragged_rank(rank, world, port, q):
    import torch.distributed as dist

    from tessera_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    probs = _ragged_problems()
    out = shard.run_ragged(probs, runner=_stub_runner)
    try:
        shard.run_ragged(probs, runner=lambda ps: _stub_runner(ps, fail=(rank == 1)))
        failed = None
    except shard.ShardError as e:
        failed = e.failures
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out, failed))


def test_ragged_batch_partitioned_by_cost_and_gathered():
    """tessera_b200.shard on two gloo ranks: a ragged batch (dense instances of n 4..16 with bond
    caps 8..32 and 3-regular instances of n 32..40, deliberately uneven costs) is partitioned by
    estimated cost with the largest rank load within 15% of the best any partition can reach
    (the mean load or the largest instance, whichever is larger); the gathered records, on
    every rank, equal a one-process run in the original order; and a failure on one rank raises
    on both, naming that rank."""
    from tessera_b200 import shard
    probs = _ragged_problems()
    costs = [shard.instance_cost(p) for p in probs]
    parts = shard.partition(costs, 2)
    assert sorted(i for p in parts for i in p) == list(range(len(probs)))
    assert max(costs) / min(costs) > 100  # the batch really is ragged
    assert shard.imbalance(costs, parts) < 1.15
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_ragged_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted((q.get(timeout=180) for _ in ps), key=lambda t: t[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    local = shard.run_ragged(probs, runner=_stub_runner)  # no process group: one process
    for rank, recs, failed in out:
        assert recs == local
        assert failed is not None and set(failed) == {1} and "injected failure" in failed[1]
