"""Multi-process path on CPU: world_size-2 gloo ranks shard an ensemble by
cell count (no collective on the data path) and gather per-instance results."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from aeromhd_cuda_b200.ensemble import draw_configs, shard
        cfgs = draw_configs(64, seed=9)
        mine = shard(cfgs, world, rank)
        # the per-instance "result" a rank reports: (index, cells); gathered once at the end
        res = torch.tensor([[k, cfgs[k].nx * cfgs[k].ny] for k in mine], dtype=torch.int64)
        n = torch.tensor([len(mine)])
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(sizes, n)
        m = int(max(s.item() for s in sizes))
        pad = torch.full((m, 2), -1, dtype=torch.int64)
        pad[: len(mine)] = res
        gathered = [torch.zeros_like(pad) for _ in range(world)]
        dist.all_gather(gathered, pad)
        # max-over-ranks timing reduction used by the benchmark
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            allres = torch.cat(gathered)
            out_q.put((allres[allres[:, 0] >= 0].tolist(), float(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_ensemble_gathers_every_instance():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    idx = sorted(int(k) for k, _ in res)
    assert idx == list(range(64))
    assert tmax == 2.0
    from aeromhd_cuda_b200.ensemble import draw_configs
    cfgs = draw_configs(64, seed=9)
    assert all(c == cfgs[int(k)].nx * cfgs[int(k)].ny for k, c in res)
