"""Multi-rank host logic (tc_b200.sharding, bench.py --gpus N) with
world-size-2 gloo processes on CPU.
- Band-apply sharding: each rank owns the bands of its k-points; the union of
  the ranks' partial H psi (oracle on CPU as the stand-in compute) equals the
  unsharded result, and the max-over-ranks timing reduction is checked.
- Occupied-pair stage of tc3a2a4b2b5: the protocol of sharded_qp_stage
  (partial share -> in-place all_reduce of the device buffer -> finish) on a
  stand-in context whose buffer is a CPU tensor.  The numbers of the split
  itself (partial grids of two ranks summing to the whole stage) are checked
  on the GPU in tests/test_gpu_sharding.py."""
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
        from tc_b200 import abi, sharding, synth
        from oracle import oracle as O
        O.set_threads(1)
        s = synth.small("TC", nk=2)
        own = sharding.owned_mask(s, world, rank)
        h2, h3 = O.apply(s, abi.TERMS_TC, owned=own)
        t2, t3 = torch.from_numpy(h2.copy()), torch.from_numpy(h3.copy())
        sharding.reduce_h([t2, t3])                      # union of disjoint shards (all()'s reduction)
        t = torch.from_numpy(np.concatenate([t2.numpy().view(np.float64), t3.numpy().view(np.float64)]))
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


class _FakeCtx:
    """stand-in for tc_b200.context.Context: the partial buffer of rank r holds
    (r + 1) * [0, 1, 2, ...]; the calls are logged in order"""

    def __init__(self, n):
        import torch
        self.buf = torch.zeros(n, dtype=torch.float64)
        self.log = []

    def qp_partial(self, rank, world):
        import torch
        self.log.append(("partial", rank, world))
        self.buf[:] = (rank + 1) * torch.arange(self.buf.numel(), dtype=torch.float64)
        return 12345, self.buf.numel() * 8

    def qp_finish(self):
        self.log.append(("finish", float(self.buf[1])))


def _qp_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from tc_b200 import sharding
        ctx = _FakeCtx(7)
        sharding.sharded_qp_stage(ctx, view=lambda ptr, nbytes: ctx.buf)
        q.put((rank, ctx.log, ctx.buf.numpy().copy()))
    finally:
        dist.destroy_process_group()


def test_two_rank_qp_stage_protocol():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_qp_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, log, buf in res:
        # each rank computed its own share, then finished on the summed buffer
        assert log == [("partial", rank, world), ("finish", 3.0)]
        assert np.array_equal(buf, 3.0 * np.arange(7))
