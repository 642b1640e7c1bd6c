"""Autotuner for the fused stage kernel: kernel and work shape, work order and grid size.

The stage kernel's cost depends on the kernel and its work shape (tiled:
tile_x rows x 32 columns per CTA -- halo re-reads and the share of faces
computed twice fall with the tile size, while registers, shared memory and
wave quantisation favour small tiles on small grids; warp-marching, tile_x
negative: -tile_x rows x 28 columns per warp -- longer items amortise the
4-row start-up, shorter ones balance better), on the persistent grid size,
and for an ensemble on the order in which CTAs take the work items.  The tuner times a few
steps of every candidate on the GPU, on a scratch copy of the state, and keeps
the fastest; results are cached per problem signature (process memory and an
optional JSON file).

No counterpart in the reference (it has a single kernel launch shape).
"""
from __future__ import annotations

import hashlib
import json
import os
from dataclasses import asdict, dataclass
from typing import Callable, Dict, Iterable, List, Optional, Sequence

TILE_XS = (4, 8, 16, -16, -24, -32, -64)
ORDERS = ("instance", "interleave", "largest_first")
GRIDS = (-1, 0)  # -1: one CTA per tile; 0: persistent (resident CTAs per SM x SMs)


@dataclass(frozen=True)
class Candidate:
    tile_x: int
    order: str = "instance"
    ctas: int = -1


def candidates(ensemble: bool, precision: str = "fp32", tile_xs: Sequence[int] = TILE_XS,
               orders: Sequence[str] = ORDERS, grids: Sequence[int] = GRIDS) -> List[Candidate]:
    """Search space.  float64 tiles of 16 rows spill registers, so they are left out."""
    out = []
    for tx in tile_xs:
        if precision == "fp64" and tx == 16:
            continue
        for g in grids:
            for o in (orders if ensemble else ("instance",)):
                out.append(Candidate(tx, o, g))
    return out


def choose(timings: Dict[Candidate, float], rel_tie: float = 0.01) -> Candidate:
    """Fastest candidate; within rel_tie of the best, prefer the library's
    defaults (instance order, a persistent grid -- one launch per stage --,
    the marching kernel, then the shorter item or tile)."""
    if not timings:
        raise ValueError("no timings")
    best = min(timings.values())
    near = [c for c, t in timings.items() if t <= best * (1.0 + rel_tie)]
    return sorted(near, key=lambda c: (c.order != "instance", c.ctas != 0, c.tile_x > 0, abs(c.tile_x)))[0]


def signature(precision: str, sizes: Iterable[tuple], device_name: str = "") -> str:
    """Problem key: precision, the multiset of grid sizes, the device."""
    hist: Dict[str, int] = {}
    for nx, ny in sizes:
        k = f"{nx}x{ny}"
        hist[k] = hist.get(k, 0) + 1
    blob = json.dumps({"p": precision, "h": sorted(hist.items()), "d": device_name}, sort_keys=True)
    return hashlib.sha1(blob.encode()).hexdigest()[:16]


class Cache:
    def __init__(self, path: Optional[str] = None):
        self.path = path
        self.mem: Dict[str, dict] = {}
        if path and os.path.exists(path):
            try:
                with open(path) as f:
                    self.mem = json.load(f)
            except (OSError, ValueError):
                self.mem = {}

    def get(self, key: str) -> Optional[Candidate]:
        v = self.mem.get(key)
        return Candidate(**v["best"]) if v else None

    def put(self, key: str, best: Candidate, timings: Dict[Candidate, float]):
        self.mem[key] = {"best": asdict(best),
                         "timings": [[asdict(c), t] for c, t in sorted(timings.items(), key=lambda x: x[1])]}
        if self.path:
            os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.mem, f, indent=1)
            os.replace(tmp, self.path)


_CACHE = Cache(os.environ.get("AMHD_TUNE_CACHE"))


def tune(run_candidate: Callable[[Candidate], float], cands: Sequence[Candidate], key: Optional[str] = None,
         cache: Optional[Cache] = None) -> tuple:
    """Time every candidate with run_candidate (returns seconds) and pick one."""
    cache = cache or _CACHE
    if key is not None:
        hit = cache.get(key)
        if hit is not None:
            return hit, {}
    timings = {c: float(run_candidate(c)) for c in cands}
    best = choose(timings)
    if key is not None:
        cache.put(key, best, timings)
    return best, timings


# ------------------------------------------------------------- GPU drivers
def _time_steps(advance: Callable[[int], None], steps: int) -> float:
    import torch
    advance(1)  # warm-up (first launch configures the kernel)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    advance(steps)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3


def tune_ensemble(ens, steps: int = 3, cands: Optional[Sequence[Candidate]] = None, cache: Optional[Cache] = None):
    """Pick tile shape, work order and grid for an Ensemble; its state is restored after timing."""
    import torch
    cands = list(cands) if cands is not None else candidates(True, ens.precision)
    key = signature(ens.precision, [(c.nx, c.ny) for c in ens.configs], torch.cuda.get_device_name())
    saved = (ens.U.clone(), ens.ctl.clone())

    def run(c: Candidate) -> float:
        ens.set_schedule(c.tile_x, c.order, c.ctas)
        ens.U.copy_(saved[0])
        ens.ctl.copy_(saved[1])
        return _time_steps(lambda k: ens.advance(k, graph=False), steps)

    best, timings = tune(run, cands, key, cache)
    ens.set_schedule(best.tile_x, best.order, best.ctas)
    ens.U.copy_(saved[0])
    ens.ctl.copy_(saved[1])
    return best, timings


def tune_solver(solver, steps: int = 3, cands: Optional[Sequence[Candidate]] = None, cache: Optional[Cache] = None):
    """Pick tile shape and grid for single-grid calls (process-wide amhd_set_tiling)."""
    import torch
    from . import _lib
    cands = list(cands) if cands is not None else candidates(False, solver.cfg.precision)
    key = signature(solver.cfg.precision, [(solver.cfg.nx, solver.cfg.ny)], torch.cuda.get_device_name())
    saved = (solver.U.clone(), solver._ctl.clone(), solver.t, solver.step)
    solver._loop_init(1e30, 1 << 60)

    def run(c: Candidate) -> float:
        _lib.call("amhd_set_tiling", c.tile_x, 0 if c.ctas < 0 else 32)
        return _time_steps(lambda k: solver._advance_eager(k), steps)

    best, timings = tune(run, cands, key, cache)
    _lib.call("amhd_set_tiling", best.tile_x, 0 if best.ctas < 0 else 32)
    solver.U = saved[0]
    solver._ctl.copy_(saved[1])
    solver.t, solver.step = saved[2], saved[3]
    return best, timings
