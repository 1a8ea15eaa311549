"""Replica (multi-GPU) host logic on two CPU processes with the gloo backend: every unit is
processed exactly once across ranks, the timing reduction is the maximum over ranks, and the
whole-job rate is the units of all ranks over the slowest rank's time."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from mossquantum_b200 import replicas as R
    r, w, lr = R.rank_info()
    units = R.shard(range(11), r, w)
    results = R.gather_results([(u, u * u) for u in units])
    t_max = R.max_over_ranks(0.5 + r)           # rank 1 is the slow one
    out[rank] = (sorted(results), t_max, R.aggregate_rate(len(units), w, t_max), (r, w, lr))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_on_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        results, t_max, rate, info = res[rank]
        assert results == [(u, u * u) for u in range(11)]       # each unit exactly once
        assert t_max == 1.5                                     # max over ranks
        assert info == (rank, world, rank)
    # rank 0 processed 6 units, rank 1 five: rate uses each rank's own count times world
    assert res[0][2] == pytest.approx(2 * 6 / 1.5) and res[1][2] == pytest.approx(2 * 5 / 1.5)


def test_shard_partitions():
    from mossquantum_b200.replicas import shard
    parts = [shard(range(10), r, 3) for r in range(3)]
    assert sorted(x for p in parts for x in p) == list(range(10))
    with pytest.raises(ValueError):
        shard(range(3), 3, 3)
