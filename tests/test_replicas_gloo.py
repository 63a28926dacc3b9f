"""Replica / shard logic of the multi-GPU bench on CPU: two gloo ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from opentelemac_b200.replicas import shard_instances


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, out):
    import torch.distributed as dist
    from opentelemac_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = replicas.shard_instances(sizes, world, rank)
    load = float(sum(sizes[k] for k in mine))
    mx = replicas.max_over_ranks(load)
    tot = replicas.sum_over_ranks(len(mine))
    out[rank] = (mine, load, mx, tot)
    dist.barrier()
    dist.destroy_process_group()


def test_shards_cover_and_balance():
    rng = np.random.default_rng(4)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(200000), 256)).astype(int)
    for world in (1, 2, 4, 8):
        parts = [shard_instances(sizes, world, r) for r in range(world)]
        allk = sorted(k for p in parts for k in p)
        assert allk == list(range(256))
        loads = [sizes[p].sum() for p in parts]
        assert max(loads) <= 1.05 * np.mean(loads) + sizes.max()


def test_two_gloo_ranks():
    sizes = [5000, 3000, 2500, 2000, 1000, 800, 600, 100]
    ctx = mp.get_context("spawn")   # no fork: the oracle's OpenMP threads may be alive
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    mine0, load0, mx0, tot0 = res[0]
    mine1, load1, mx1, tot1 = res[1]
    assert sorted(mine0 + mine1) == list(range(len(sizes)))
    assert mx0 == mx1 == max(load0, load1)
    assert tot0 == tot1 == len(sizes)
