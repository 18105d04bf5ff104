"""Band-apply sharding over ranks (bench.py --gpus N): world-size-2 gloo
processes on CPU.  Each rank owns the bands of its k-points; the union of
the ranks' partial H psi (oracle on CPU as the stand-in compute) must equal
the unsharded result, and the max-over-ranks timing reduction is checked."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from tc_b200 import abi, synth
        from oracle import oracle as O
        O.set_threads(1)
        s = synth.small("TC", nk=2)
        own = bench.shard_owned(s, world, rank)
        h2, h3 = O.apply(s, abi.TERMS_TC, owned=own)
        t = torch.from_numpy(np.concatenate([h2.view(np.float64), h3.view(np.float64)]))
        dist.all_reduce(t)                               # union of disjoint shards
        m = torch.tensor([float(own.sum()), float(rank + 1)])
        dist.all_reduce(m[1:], op=dist.ReduceOp.MAX)     # max-over-ranks timing
        masks = [torch.zeros(own.size, dtype=torch.uint8) for _ in range(world)]
        dist.all_gather(masks, torch.from_numpy(own))
        if rank == 0:
            q.put((t.numpy(), [x.numpy() for x in masks], float(m[1])))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_reproduces_full_apply():
    from tc_b200 import abi, synth
    from oracle import oracle as O
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    t, masks, tmax = res
    s = synth.small("TC", nk=2)
    h2, h3 = O.apply(s, abi.TERMS_TC)
    full = np.concatenate([h2.view(np.float64), h3.view(np.float64)])
    assert np.abs(t - full).max() <= 1e-13 * np.abs(full).max()
    stack = np.stack(masks)
    assert np.all(stack.sum(0) == 1)              # every band owned exactly once
    assert stack[0].sum() > 0 and stack[1].sum() > 0
    assert tmax == 2.0
