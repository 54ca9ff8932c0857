"""World-size-2 check of the replica path on CPU (gloo): job sharding covers
every job exactly once and the measurement reduction returns the max time
and the total work on every rank."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from deconlib_b200.replicas import aggregate, shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    jobs = list(range(11))
    mine = shard(jobs, rank, world)
    ms, units = aggregate(10.0 + 5.0 * rank, 100.0 * len(mine))
    out[rank] = (mine, ms, units)
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    jobs = sorted(out[0][0] + out[1][0])
    assert jobs == list(range(11))
    for r in range(world):
        assert out[r][1] == 15.0
        assert out[r][2] == 1100.0


def test_shard_rejects_bad_rank():
    from deconlib_b200.replicas import shard

    with pytest.raises(ValueError):
        shard([1, 2], 2, 2)
