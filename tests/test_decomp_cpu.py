"""Row-split grid (aeromhd_cuda_b200.decomp) on CPU: the split run loop --
halo exchange with the neighbouring ranks, CFL max reduction, finish -- run as
2 and 3 gloo ranks with the oracle standing in for the GPU stages, gathered,
equals the same loop on one rank bit for bit (periodic and outflow x
boundaries, Powell source on)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from aeromhd_cuda_b200.decomp import HaloExchange, SplitLoop, all_reduce_max, neighbours, split_rows


def test_split_rows_and_neighbours():
    assert split_rows(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert split_rows(8, 1) == [(0, 8)]
    with pytest.raises(ValueError):
        split_rows(5, 3)
    assert neighbours(0, 3, True) == (2, 1) and neighbours(2, 3, True) == (1, 0)
    assert neighbours(0, 3, False) == (None, 1) and neighbours(2, 3, False) == (1, None)
    assert neighbours(0, 1, True) == (None, None)


def _cfg(bcx):
    from aeromhd_cuda_b200.config import Config
    return Config(nx=22, ny=12, x_min=0.0, x_max=1.1, y_min=0.0, y_max=0.6, t_end=1.0, cfl=0.3, gamma=5.0 / 3.0,
                  B_transverse=0.4, powell_source=True, bc_x_type=bcx, bc_y_type="periodic")


def _initial(cfg):
    rng = np.random.default_rng(4)
    from oracle import oracle as O
    nxt, nyt = cfg.nx + 4, cfg.ny + 4
    W = np.zeros((10, nxt, nyt))
    x = (np.arange(nxt) - 1.5)[:, None] / cfg.nx
    y = (np.arange(nyt) - 1.5)[None, :] / cfg.ny
    W[0] = 1.0 + 0.5 * (x > 0.4) + 0.05 * np.sin(2 * np.pi * y)
    W[1] = 0.3 * np.cos(2 * np.pi * y) + 0.01 * rng.standard_normal((nxt, nyt))
    W[2] = 0.2 * np.sin(2 * np.pi * x)
    W[4], W[5], W[6] = 0.5, 0.4 * np.sin(2 * np.pi * x), 0.1
    W[7] = 1.0 + 0.1 * np.cos(2 * np.pi * (x + y))
    W[9] = (x > 0.4) + 0 * y
    return O.prim_to_cons(W, cfg.gamma)


def _run(cfg, U, rank, world, steps, group=None):
    from split_oracle import OracleBackend
    from aeromhd_cuda_b200.config import BC_PERIODIC, bc_x_code
    r0, r1 = split_rows(cfg.nx, world)[rank]
    b = OracleBackend(cfg, r0, r1)
    b.state(0).copy_(torch.from_numpy(U[:, r0:r1 + 4]))
    loop = SplitLoop(b, HaloExchange(rank, world, bc_x_code(cfg) == BC_PERIODIC, group), all_reduce_max(group))
    loop.init(0.0, cfg.t_end, 0, 1 << 40)
    for _ in range(steps):
        loop.step()
    return b


def _worker(rank, world, port, bcx, steps, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg = _cfg(bcx)
        b = _run(cfg, _initial(cfg), rank, world, steps)
        parts = [None] * world
        dist.all_gather_object(parts, (rank, b.state(0).numpy().copy(), dict(b.c)))
        if rank == 0:
            q.put(parts)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,bcx", [(2, "periodic"), (2, "extrapolation"), (3, "periodic")])
def test_split_loop_equals_single_block(world, bcx):
    steps = 6
    cfg = _cfg(bcx)
    one = _run(cfg, _initial(cfg), 0, 1, steps)
    ref = one.state(0).numpy()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, bcx, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    parts = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rows = split_rows(cfg.nx, world)
    # boundary energy: the ranks' physical sides add up to the single block's
    e_split = sum(c["e_bnd"] for _, _, c in parts)
    if bcx == "periodic":
        assert e_split == one.c["e_bnd"] == 0.0
    else:
        assert one.c["e_bnd"] != 0.0
        assert abs(e_split - one.c["e_bnd"]) <= 1e-12 * abs(one.c["e_bnd"]), (e_split, one.c["e_bnd"])
    for rank, U, c in parts:
        r0, r1 = rows[rank]
        assert c["step"] == one.c["step"] == steps
        assert c["t"] == one.c["t"] and c["dt"] == one.c["dt"]
        # interior rows and the y ghost columns of the block
        assert np.array_equal(U[:, 2:-2], ref[:, r0 + 2:r1 + 2]), rank
        # ghost rows: the neighbours' rows (cut) or the boundary fill (physical), as in the single block
        assert np.array_equal(U, ref[:, r0:r1 + 4]), rank
