"""Batched ensemble of independent shock-accelerated-interface runs on one GPU.

Every instance keeps its own grid size, physics parameters and time step; all
of them advance together, one persistent launch per SSP-RK3 stage over a work
list of (instance, tile) pairs, plus one launch that finishes every
instance's CFL reduction and clock.  A run of steps is captured once as a
CUDA graph and replayed.  Instances that reach their end time stop (their
tiles return at once) while the others continue.

Layout: the three ensemble states are single device buffers; instance k
occupies ``10 * rows_k * pitch_k`` elements at ``offset_k`` in each (its own
padded layout, 16-byte aligned), described by an ``amhd_instance`` table in
device memory.

No counterpart in the reference, which runs one grid per ``MHDSolver``;
instance i of an ensemble produces exactly the state the single-grid solver
produces for it (the same kernels over the same tiles).
"""
from __future__ import annotations

import ctypes
from dataclasses import replace
from typing import List, Sequence

import numpy as np
import torch

from . import _lib, initial_conditions
from ._tensors import NG, control_tensor, read_controls, stream_ptr, torch_dtype, write_controls
from .config import Config, bc_x_code, bc_y_code
from .physics import prim_to_cons


def draw_configs(n: int = 256, seed: int = 0, t_end: float = 3.0, precision: str = "fp32",
                 ny_choices: Sequence[int] = (32, 64, 128, 256), noise_amp: float = 1e-3) -> List[Config]:
    """Seeded parameter draws of the uneven shock-interface ensemble:
    Ny in ny_choices, Nx = 4 Ny on [0,4]x[0,1]; Mach ~ U[2,5]; density ratio ~
    U[1.5,5]; mode k in 1..8, amplitude ~ U[0.01,0.08]; B = (B0 + B1 sin(2 pi m y), 0, 0)
    with B0, B1 ~ U[0,0.3], m in 1..6."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        ny = int(rng.choice(ny_choices))
        out.append(Config(
            nx=4 * ny, ny=ny, x_min=0.0, x_max=4.0, y_min=0.0, y_max=1.0, t_end=t_end, cfl=0.4, gamma=5.0 / 3.0,
            mach=float(rng.uniform(2.0, 5.0)), density_ratio=float(rng.uniform(1.5, 5.0)),
            perturbation_mode=int(rng.integers(1, 9)), perturbation_amp=float(rng.uniform(0.01, 0.08)),
            bx0=float(rng.uniform(0.0, 0.3)), b1=float(rng.uniform(0.0, 0.3)), b_mode=int(rng.integers(1, 7)),
            ic="shock_interface", interface_x=1.0, shock_x=0.5, perturbation_shape="cos", interface_cells=2.0,
            noise_amp=noise_amp, seed=seed * 100003 + k, powell_mode="on", bc_x_type="extrapolation",
            bc_y_type="periodic", precision=precision))
    return out


def pack_layout(configs: Sequence[Config], dtype_code: int):
    """Element offset, pitch and rows of every instance in the packed buffers,
    each start 16-byte aligned; returns (layouts, total elements)."""
    es = 4 if dtype_code == _lib.AMHD_F32 else 8
    align = 16 // es
    layouts, off = [], 0
    for c in configs:
        pitch, rows = _lib.padded_layout(c.nx, c.ny, dtype_code)
        layouts.append((off, pitch, rows))
        off += 10 * rows * pitch
        off = (off + align - 1) // align * align
    return layouts, off


MARCH_COLS = 28  # interior columns of one warp-marching work item (32 lanes minus a 2-column halo each side)


def valid_geometry(tile_x: int) -> bool:
    """4, 8, 16: tiled stage kernel; -1024..-4: warp-marching kernel, -tile_x rows per item."""
    return tile_x in (4, 8, 16) or -1024 <= tile_x <= -4


def work_shape(tile_x: int) -> tuple:
    """(rows, columns) of one work item of the stage kernel for this geometry."""
    if not valid_geometry(tile_x):
        raise ValueError("tile_x must be 4, 8, 16 (tiled kernel) or -1024..-4 (marching kernel rows)")
    return (tile_x, 32) if tile_x > 0 else (-tile_x, MARCH_COLS)


def march_pack(ny: int) -> int:
    """Row chunks of the last column strip that share one warp-marching item
    (amhd_march_pack): the strip's ny mod 28 columns plus a 2-column halo on
    each side in 8 lanes (4 chunks) or 16 lanes (2); 1 when the strip is full or
    wider than 12 columns."""
    rem = ny % MARCH_COLS
    return 1 if rem == 0 else 4 if rem <= 4 else 2 if rem <= 12 else 1


def march_items(nx: int, ny: int, rows: int, pack: int) -> int:
    """Work items of an nx x ny instance in chunks of `rows` rows (amhd_march_items):
    chunks x strips unpacked; packed, the full-width strips' items, then
    ceil(full-height chunks / pack) items of the last strip and one for a short
    last chunk."""
    chunks, strips = -(-nx // rows), -(-ny // MARCH_COLS)
    if pack <= 1:
        return chunks * strips
    full = nx // rows
    return (strips - 1) * chunks + -(-full // pack) + (1 if nx % rows else 0)


def tile_counts(configs: Sequence[Config], tile_x: int, pack: bool = False) -> np.ndarray:
    """Work items per instance; pack (marching kernel): the last strip's row
    chunks share warps (march_pack)."""
    r, c_ = work_shape(tile_x)
    if tile_x < 0 and pack:
        return np.array([march_items(c.nx, c.ny, r, march_pack(c.ny)) for c in configs], dtype=np.int64)
    return np.array([((c.nx + r - 1) // r) * ((c.ny + c_ - 1) // c_) for c in configs], dtype=np.int64)


def work_list(counts: Sequence[int], order: str = "instance"):
    """(tile_order, tile_inst, first_tile) of a packed ensemble.

    Tiles are numbered instance by instance (instance k owns ids first_tile[k] ..
    first_tile[k] + counts[k] - 1, taken in that order); tile_inst maps an id to
    its instance; tile_order is the id taken at each work position:
      instance       instance by instance (neighbouring tiles share halo lines in L2)
      largest_first  the instances with most tiles first
      interleave     round robin over instances
    """
    counts = np.asarray(counts, dtype=np.int64)
    first = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    n_tiles = int(counts.sum())
    tile_inst = np.repeat(np.arange(len(counts), dtype=np.int32), counts)
    if order == "instance":
        seq = [np.arange(first[k], first[k] + counts[k]) for k in range(len(counts))]
        tile_order = np.concatenate(seq) if seq else np.zeros(0, np.int64)
    elif order == "largest_first":
        ks = np.argsort(-counts, kind="stable")
        tile_order = np.concatenate([np.arange(first[k], first[k] + counts[k]) for k in ks])
    elif order == "interleave":
        m = int(counts.max())
        grid = np.full((m, len(counts)), -1, dtype=np.int64)
        for k in range(len(counts)):
            grid[: counts[k], k] = np.arange(first[k], first[k] + counts[k])
        flat = grid.reshape(-1)
        tile_order = flat[flat >= 0]
    else:
        raise ValueError(f"unknown order {order!r}")
    assert len(tile_order) == n_tiles
    return tile_order.astype(np.int32), tile_inst, first.astype(np.int32)


def shard(configs: Sequence[Config], world: int, rank: int) -> List[int]:
    """Instances of this rank: longest-processing-time greedy over cell counts,
    so that every GPU gets about the same number of zone updates per step."""
    cells = np.array([c.nx * c.ny for c in configs])
    load = np.zeros(world)
    owner = np.empty(len(configs), dtype=np.int64)
    for k in np.argsort(-cells, kind="stable"):
        r = int(np.argmin(load))
        owner[k] = r
        load[r] += cells[k]
    return [k for k in range(len(configs)) if owner[k] == rank]


class _GridView:
    """The coordinate attributes initial_conditions needs, for one instance."""

    def __init__(self, cfg: Config, device):
        self.cfg = cfg
        self.nx_tot, self.ny_tot = cfg.nx + 2 * NG, cfg.ny + 2 * NG
        self.device = device
        self.x = torch.as_tensor(cfg.x_min + (np.arange(self.nx_tot) - NG + 0.5) * cfg.dx, device=device)
        self.y = torch.as_tensor(cfg.y_min + (np.arange(self.ny_tot) - NG + 0.5) * cfg.dy, device=device)
        self.X, self.Y = torch.meshgrid(self.x, self.y, indexing="ij")


def default_tile_x(precision: str) -> int:
    """Rows per marching item an ensemble starts with: 32 in float32 (on the
    seeded 256-instance draw, 32-row items give 6.22 G zone-updates/s against
    6.09 G for the single-grid default of 24: the uneven instances leave fewer
    part-filled waves), the library default in float64.  Item height moves the
    seams between work items only, so results do not depend on it."""
    return -32 if precision == "fp32" else _lib.default_tile_x(precision)


class Ensemble:
    def __init__(self, configs: Sequence[Config], tile_x: int = 0, order: str = "instance", ctas: int = 0,
                 device=None, use_tma: bool | None = None, dynamic: bool = True, pack: bool = True):
        if not configs:
            raise ValueError("empty ensemble")
        precs = {c.precision for c in configs}
        if len(precs) != 1:
            raise ValueError("all instances must share one precision")
        for c in configs:
            c.validate()
        _lib.call("amhd_init")
        self.configs = [replace(c) for c in configs]
        self.precision = precs.pop()
        self.dtype = torch_dtype(self.precision)
        self.code = _lib.AMHD_F64 if self.dtype == torch.float64 else _lib.AMHD_F32
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.n = len(self.configs)
        tile_x = int(tile_x) or default_tile_x(self.precision)  # 0: the ensemble default
        self.tile_x = tile_x
        self.ctas = int(ctas)
        self.use_tma = use_tma  # None: the library default of the stage kernel in use (_lib.DEFAULT_TMA)
        self.layouts, off = pack_layout(self.configs, self.code)
        self.total = off
        self.U = torch.zeros(off, dtype=self.dtype, device=self.device)
        self.U1 = torch.zeros_like(self.U)
        self.U2 = torch.zeros_like(self.U)
        self.ctl = control_tensor(self.n, self.device)
        # work queue of a persistent marching grid: {next position, warps finished},
        # zero between launches (the kernel's last warp resets it)
        self.queue = torch.zeros(2, dtype=torch.int32, device=self.device)
        self.dynamic = bool(dynamic)
        self.pack = bool(pack)
        self._graphs = {}
        self.set_schedule(tile_x, order, ctas)

    # -------------------------------------------------------- schedule
    def set_schedule(self, tile_x: int, order: str = "instance", ctas: int = -1):
        """Stage-kernel geometry (tile_x: 4, 8, 16 rows x 32 columns per CTA of the
        tiled kernel, or negative: -tile_x rows x 28 columns per warp of the
        marching kernel), work-list order and grid size (chosen by autotune).
        ctas: 0 (default) = a persistent grid of resident CTAs per SM x SM
        count (> 0: that many CTAs), one launch per RK stage; -1 = one CTA per
        tile (tiled) / per 4 work items (marching), the hardware handing CTAs
        to SMs as they free up.  On a persistent marching grid each warp takes
        the next free item from a device work queue when it finishes one
        (``dynamic``, the default): on the uneven 256-instance ensemble as fast
        as one CTA per 4 items (6.67 against 6.69 G zone-updates/s, measured
        before the last strips were packed); with dynamic=False warp w takes
        items w, w + warps, ... (20-30 % slower: the static split leaves warps
        idle at the end).  With ``pack`` (the constructor's, default on) the
        marching kernel runs 2 or 4 row chunks of an instance's narrow last
        column strip in one warp (march_pack): 7.39 against 6.63 G on that
        ensemble, identical results."""
        rows, cols = work_shape(tile_x)
        self.tile_x, self.order, self.ctas = int(tile_x), order, int(ctas)
        # marching items of the last column strips share warps unless rows are staged by TMA
        pack = tile_x < 0 and self.pack and not self.tma_staging()
        counts = tile_counts(self.configs, tile_x, pack)
        tile_order, tile_inst, first = work_list(counts, order)
        table = (_lib.Instance * self.n)()
        for k, c in enumerate(self.configs):
            inst = table[k]
            inst.grid = self._grid(k)
            inst.offset = self.layouts[k][0]
            inst.tiles_x = (c.nx + rows - 1) // rows
            inst.tiles_y = (c.ny + cols - 1) // cols
            inst.first_tile = int(first[k])
            inst.pack = march_pack(c.ny) if pack else 1
        self.n_tiles = int(counts.sum())
        self._table = table
        raw = np.frombuffer(bytes(table), dtype=np.uint8).copy()
        self.inst_dev = torch.from_numpy(raw).to(self.device)
        self.tile_inst = torch.from_numpy(tile_inst).to(self.device)
        self.tile_order = torch.from_numpy(tile_order).to(self.device)
        self.tmaps_dev = None
        if self.tma_staging():
            # TMA descriptors of every instance's box in U, U1, U2 for this work shape
            maps = torch.empty(3 * self.n * 128, dtype=torch.uint8)
            _lib.call("amhd_ensemble_tensormaps", ctypes.byref(table), self.n, self.code, self.tile_x,
                      self.U.data_ptr(), self.U1.data_ptr(), self.U2.data_ptr(), maps.data_ptr())
            self.tmaps_dev = maps.to(self.device)
        self._graphs = {}

    def tma_staging(self) -> bool:
        """Does the stage kernel stage its tiles (tiled) or rows (marching) with TMA?"""
        if self.use_tma is None:
            return bool(_lib.DEFAULT_TMA & (2 if self.tile_x < 0 else 1))
        return bool(self.use_tma)

    def _grid(self, k: int) -> _lib.Grid:
        c = self.configs[k]
        off, pitch, rows = self.layouts[k]
        g = _lib.Grid()
        g.nx, g.ny, g.pitch, g.dtype = c.nx, c.ny, pitch, self.code
        g.var_stride = rows * pitch
        g.dx, g.dy, g.gamma, g.cfl, g.glm_alpha = c.dx, c.dy, c.gamma, c.cfl, c.glm_alpha
        g.bc_x, g.bc_y = bc_x_code(c), bc_y_code(c)
        g.powell = int(c.powell_enabled())
        g.limiter = _lib.LIMITER_CODES[c.limiter]
        return g

    # ----------------------------------------------------------- state
    def state(self, k: int, buf: torch.Tensor | None = None) -> torch.Tensor:
        """[10, nx+4, ny+4] view of instance k's state."""
        c = self.configs[k]
        off, pitch, rows = self.layouts[k]
        b = self.U if buf is None else buf
        return b[off: off + 10 * rows * pitch].view(10, rows, pitch)[:, : c.nx + 2 * NG, : c.ny + 2 * NG]

    def cells(self) -> np.ndarray:
        return np.array([c.nx * c.ny for c in self.configs], dtype=np.int64)

    def initialize(self):
        """Each instance's configured initial condition (shock_interface or rmi)."""
        for k, c in enumerate(self.configs):
            gv = _GridView(c, self.device)
            W = initial_conditions.shock_interface(gv)[0] if c.ic == "shock_interface" else \
                initial_conditions.rmi(gv)[0]
            self.state(k).copy_(prim_to_cons(W, c.gamma).to(self.dtype))
        self._graphs = {}

    def start(self, t_end: float | None = None, max_steps: int = 1 << 62):
        """dt / GLM speed of every instance from its current state (run-loop head)."""
        t_end = float(self.configs[0].t_end if t_end is None else t_end)
        _lib.call("amhd_ensemble_init", ctypes.byref(self._table), self.inst_dev.data_ptr(), self.n, self.code,
                  self.U.data_ptr(), self.ctl.data_ptr(), t_end, int(max_steps), stream_ptr())

    def continue_to(self, t_end: float):
        """Keep every instance's t and step; run on to a new end time."""
        _lib.call("amhd_ensemble_continue", ctypes.byref(self._table), self.inst_dev.data_ptr(), self.n, self.code,
                  self.U.data_ptr(), self.ctl.data_ptr(), float(t_end), stream_ptr())

    def _advance_eager(self, n: int):
        _lib.call("amhd_ensemble_advance", self.inst_dev.data_ptr(), self.n, self.tile_inst.data_ptr(),
                  self.tile_order.data_ptr(), self.n_tiles, self.code, self.tile_x, self.U.data_ptr(),
                  self.U1.data_ptr(), self.U2.data_ptr(), self.ctl.data_ptr(), int(n),
                  self.n_tiles if self.ctas < 0 else self.ctas,
                  self.tmaps_dev.data_ptr() if self.tmaps_dev is not None else None,
                  self.queue.data_ptr() if self.uses_queue() else None, stream_ptr())

    def uses_queue(self) -> bool:
        """Does the stage kernel draw work items from the device queue?"""
        return self.dynamic and self.ctas >= 0 and self.tile_x < 0

    def advance(self, n: int, graph: bool = True):
        """n run-loop steps of every active instance (one graph replay)."""
        if not graph:
            self._advance_eager(n)
            return
        g = self._graphs.get(n)
        if g is None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._advance_eager(n)
            self._graphs[n] = g
        g.replay()

    def controls(self):
        return read_controls(self.ctl)

    def set_state(self, k: int, U) -> None:
        """Load instance k's conserved state ([10, nx+4, ny+4], ghosts included)."""
        v = self.state(k)
        src = torch.as_tensor(U)
        if tuple(src.shape) != tuple(v.shape):
            raise ValueError(f"instance {k}: state must have shape {tuple(v.shape)}, got {tuple(src.shape)}")
        v.copy_(src.to(device=self.device, dtype=self.dtype))
        self._graphs = {}

    def resume(self, t, step, e_bnd, t_end: float, max_steps: int = 1 << 62) -> None:
        """Continue every instance from its own saved time, step count and boundary
        energy (sequences of length n) toward t_end: dt and ch from the states, as
        at a loop head."""
        self.start(t_end=t_end, max_steps=max_steps)
        ctl = self.controls()
        for k, c in enumerate(ctl):
            c.t, c.step, c.e_bnd = float(t[k]), int(step[k]), float(e_bnd[k])
        write_controls(self.ctl, ctl)
        self.continue_to(t_end)

    def run(self, chunk: int = 50, max_chunks: int = 1 << 30):
        """Advance until every instance reached its end time; returns steps per instance."""
        for _ in range(max_chunks):
            self.advance(chunk)
            c = self.controls()
            for k, x in enumerate(c):
                _lib.check_control(x, f"Ensemble.run, instance {k}")
            if not any(x.active for x in c):
                break
        return np.array([x.step for x in self.controls()])
