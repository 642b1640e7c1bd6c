"""One grid split over GPUs by x rows (domain decomposition).

Rank r owns interior rows [r0, r1) of the global grid (contiguous blocks,
sizes differing by at most one) with the full y extent, stored in its own
padded state with the usual 2 ghost rows and columns.  One run-loop step is
the device loop taken apart (amhd_advance_stage / amhd_advance_finish):

    stage 1, 2, 3 -- each on the local grid (y ghosts and the physical x
                     boundaries filled locally), then the 2 rows next to each
                     rank boundary are exchanged: every rank sends its first
                     two interior rows to the rank on its left and its last two
                     to the rank on its right, and receives theirs into its x
                     ghost rows (periodic x: rank 0 and the last rank are
                     neighbours)
    CFL maxima    -- max-all-reduce of ctl->red[4] (ordered float64 bits, so an
                     int64 max is exact) over the ranks
    finish        -- t, step, and the next dt / ch / psi damping from the
                     global maxima, identical on every rank; the boundary
                     energy (solver.py:225-240, :316-317) of the block's
                     physical x sides only (the cut sides are masked), so the
                     sum over the ranks is the whole grid's

Every cell's arithmetic sees the same inputs as in the unsplit grid, so the
split run reproduces the single-grid run bit for bit (state, t, dt).  The
exchange is point-to-point (torch.distributed isend/irecv: NCCL over NVLink
between GPUs, gloo between CPU processes in tests); each rank talks to two
neighbours only.  The boundary energy is accumulated per rank on the sides
that are physical boundaries; its sum over the ranks equals the unsplit
grid's to rounding (the two sides are added per rank instead of per step).

The reference runs one grid on one GPU; this has no counterpart there.
"""
from __future__ import annotations

from dataclasses import replace
from typing import Callable, List, Optional, Tuple

import numpy as np
import torch

NG = 2


def split_rows(nx: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous blocks of interior rows, one per rank, sizes differing by at most one
    (the first nx % world ranks get the extra row)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if nx < 2 * world:
        raise ValueError(f"{nx} rows cannot give each of {world} ranks the 2 rows a halo needs")
    base, extra = divmod(nx, world)
    out, r0 = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((r0, r0 + n))
        r0 += n
    return out


def cut_sides(r0: int, r1: int, nx: int) -> int:
    """Mask of a block's x sides that are cuts between blocks rather than the
    grid's boundary: bit 0 its first row (r0 > 0), bit 1 its last (r1 < nx)."""
    return (1 if r0 > 0 else 0) | (2 if r1 < nx else 0)


def neighbours(rank: int, world: int, periodic: bool) -> Tuple[Optional[int], Optional[int]]:
    """(left, right) ranks across the cut rows; None at a physical x boundary."""
    left = rank - 1 if rank > 0 else (world - 1 if periodic and world > 1 else None)
    right = rank + 1 if rank < world - 1 else (0 if periodic and world > 1 else None)
    return left, right


class HaloExchange:
    """Exchange of the 2 rows on each side of this rank's block (all 10 planes,
    ghost columns included) with the neighbouring ranks.  World 1: the periodic
    wrap is a local copy; physical boundaries are left to the local fill."""

    TAG_RIGHTWARD, TAG_LEFTWARD = 17, 18

    def __init__(self, rank: int, world: int, periodic: bool, group=None):
        self.rank, self.world, self.periodic, self.group = rank, world, periodic, group
        self.left, self.right = neighbours(rank, world, periodic)

    def __call__(self, U: torch.Tensor, n: int) -> None:
        """U: [10][>= n+4][m] state of this rank (storage rows), n interior rows."""
        if self.world == 1:
            if self.periodic:
                U[:, 0:NG].copy_(U[:, n:n + NG])
                U[:, n + NG:n + 2 * NG].copy_(U[:, NG:2 * NG])
            return
        import torch.distributed as dist
        ops = []
        # per peer, messages are posted in the same order on both sides: the
        # rightward one (sender's last rows -> receiver's left ghosts) first
        recv_l = recv_r = None
        if self.right is not None:
            ops.append(dist.P2POp(dist.isend, U[:, n:n + NG].contiguous(), self.right, self.group,
                                  self.TAG_RIGHTWARD))
        if self.left is not None:
            ops.append(dist.P2POp(dist.isend, U[:, NG:2 * NG].contiguous(), self.left, self.group,
                                  self.TAG_LEFTWARD))
        if self.left is not None:
            recv_l = torch.empty_like(U[:, 0:NG])
            ops.append(dist.P2POp(dist.irecv, recv_l, self.left, self.group, self.TAG_RIGHTWARD))
        if self.right is not None:
            recv_r = torch.empty_like(U[:, 0:NG])
            ops.append(dist.P2POp(dist.irecv, recv_r, self.right, self.group, self.TAG_LEFTWARD))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        if recv_l is not None:
            U[:, 0:NG].copy_(recv_l)
        if recv_r is not None:
            U[:, n + NG:n + 2 * NG].copy_(recv_r)


def all_reduce_max(group=None) -> Callable[[torch.Tensor], None]:
    def reduce(t: torch.Tensor) -> None:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return reduce


class SplitLoop:
    """The run loop of one rank: local stages, halo exchanges, global CFL maxima.

    backend: control_init_split(t, t_end, step, max_steps), stage(s), finish(advance),
    state(k) -> [10][n+4][m] view of U (0), U1 (1), U2 (2), red() -> int64[4] view of
    the CFL maxima, n (interior rows)."""

    def __init__(self, backend, exchange: Callable[[torch.Tensor, int], None],
                 reduce_max: Callable[[torch.Tensor], None]):
        self.b, self.exchange, self.reduce_max = backend, exchange, reduce_max

    def init(self, t: float, t_end: float, step: int, max_steps: int) -> None:
        b = self.b
        b.control_init_split(t, t_end, step, max_steps)
        self.exchange(b.state(0), b.n)
        self.reduce_max(b.red())
        b.finish(0)

    def step(self) -> None:
        b = self.b
        for s in (1, 2, 3):
            b.stage(s)
            self.exchange(b.state(s % 3), b.n)
        self.reduce_max(b.red())
        b.finish(1)


class GpuBackend:
    """Stages of one rank's block on its GPU through the C ABI."""

    def __init__(self, cfg, r0: int, r1: int):
        from . import _lib
        from ._tensors import ptr, stream_ptr
        from .solver import MHDSolver
        self._lib, self._ptr, self._stream = _lib, ptr, stream_ptr
        self.n = r1 - r0
        self.cut_x = cut_sides(r0, r1, cfg.nx)
        local = replace(cfg, nx=self.n, x_min=cfg.x_min + r0 * cfg.dx, x_max=cfg.x_min + r1 * cfg.dx)
        self.solver = MHDSolver(local)
        s = self.solver
        g = s._grid()
        g.dx = cfg.dx  # the global spacing, bit for bit (not re-derived from the block's extent)
        self.grid = g
        self.buffers = (s._U, s._U1, s._U2)
        off = _lib.Control.red.offset
        self._red = s._ctl.view(-1)[off:off + 32].view(torch.int64)

    def state(self, k: int) -> torch.Tensor:
        return self.buffers[k]

    def red(self) -> torch.Tensor:
        return self._red

    def control_init_split(self, t, t_end, step, max_steps):
        s = self.solver
        self._lib.call("amhd_control_init_split", self.grid, self._ptr(s._U), self._ptr(s._ctl), float(t),
                       float(t_end), int(step), int(max_steps), self._stream())

    def stage(self, k: int) -> None:
        s = self.solver
        self._lib.call("amhd_advance_stage", self.grid, int(k), self._ptr(s._U), self._ptr(s._U1),
                       self._ptr(s._U2), self._ptr(s._ctl), self._stream())

    def finish(self, advance: int) -> None:
        s = self.solver
        self._lib.call("amhd_advance_finish", self.grid, self._ptr(s._U), self._ptr(s._ctl), int(advance),
                       int(self.cut_x), self._stream())

    def control(self):
        from ._tensors import read_controls
        return read_controls(self.solver._ctl)[0]


class DecomposedSolver:
    """A grid split over the ranks of a process group by x rows, one GPU per rank.

    cfg: the global Config.  set_global_state / gather_state move whole-grid
    states ([10][nx+4][ny+4]); advance(n) runs n steps of the split loop."""

    def __init__(self, cfg, group=None):
        import torch.distributed as dist
        from .config import BC_PERIODIC, bc_x_code
        cfg.validate()
        self.cfg = cfg
        self.group = group
        on = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if on else 0
        self.world = dist.get_world_size(group) if on else 1
        self.rows = split_rows(cfg.nx, self.world)
        self.r0, self.r1 = self.rows[self.rank]
        self.backend = GpuBackend(cfg, self.r0, self.r1)
        periodic = bc_x_code(cfg) == BC_PERIODIC
        self.loop = SplitLoop(self.backend, HaloExchange(self.rank, self.world, periodic, group),
                              all_reduce_max(group))
        self.t, self.step = 0.0, 0
        self._ready = False

    @property
    def U(self) -> torch.Tensor:
        """This rank's block with its ghost rows and columns."""
        return self.backend.state(0)

    def set_global_state(self, U) -> None:
        """Load this rank's rows (and their ghost rows) from a whole-grid state."""
        U = torch.as_tensor(U)
        want = (10, self.cfg.nx + 2 * NG, self.cfg.ny + 2 * NG)
        if tuple(U.shape) != want:
            raise ValueError(f"global state must have shape {want}, got {tuple(U.shape)}")
        self.backend.state(0).copy_(U[:, self.r0:self.r1 + 2 * NG].to(self.backend.state(0)))
        self._ready = False

    def gather_state(self) -> Optional[torch.Tensor]:
        """The whole-grid state on rank 0 (None elsewhere); ghost rows of the cut
        boundaries come from the owning ranks."""
        import torch.distributed as dist
        mine = self.backend.state(0)[:, NG:NG + self.r1 - self.r0].contiguous()
        if self.world == 1:
            return self.backend.state(0).clone()
        nmax = max(b - a for a, b in self.rows)
        pad = torch.zeros((10, nmax, mine.shape[2]), dtype=mine.dtype, device=mine.device)
        pad[:, :mine.shape[1]] = mine
        parts = [torch.empty_like(pad) for _ in range(self.world)] if self.rank == 0 else None
        dist.gather(pad, parts, dst=0, group=self.group)
        # the x ghost rows of the whole grid: from the first and the last rank
        edge = torch.cat([self.backend.state(0)[:, :NG], self.backend.state(0)[:, -NG:]], dim=1)
        edges = [torch.empty_like(edge) for _ in range(self.world)] if self.rank == 0 else None
        dist.gather(edge.contiguous(), edges, dst=0, group=self.group)
        if self.rank != 0:
            return None
        rows = [parts[r][:, :b - a] for r, (a, b) in enumerate(self.rows)]
        return torch.cat([edges[0][:, :NG]] + rows + [edges[-1][:, NG:]], dim=1)

    def advance(self, n_steps: int, t_end: Optional[float] = None, max_steps: Optional[int] = None) -> None:
        cfg = self.cfg
        if not self._ready:
            self.loop.init(self.t, cfg.t_end if t_end is None else t_end, self.step,
                           cfg.max_steps if max_steps is None else max_steps)
            self._ready = True
        for _ in range(n_steps):
            self.loop.step()
        c = self.backend.control()
        self.t, self.step = float(c.t), int(c.step)

    def boundary_energy(self) -> float:
        """The whole grid's cumulative boundary energy (solver.py:225-240, :316-317):
        the sum over the ranks of each block's physical sides.  A collective:
        every rank calls it."""
        import torch.distributed as dist
        e = torch.tensor([float(self.backend.control().e_bnd)], dtype=torch.float64, device=self.U.device)
        if self.world > 1:
            dist.all_reduce(e, op=dist.ReduceOp.SUM, group=self.group)
        return float(e.item())
