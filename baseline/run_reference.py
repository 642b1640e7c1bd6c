"""Time the reference's own step loop, unchanged, on the Orszag-Tang vortex.

    python baseline/run_reference.py --backend torch --n 2048 --steps 5 --warmup 2   # GPU
    python baseline/run_reference.py --backend numpy --n 512 --steps 2 --warmup 1   # host cores

Drives the reference modules (imported through ``refshim.py``) the way its
own drivers do -- main.py:66-73: ``cons_to_prim`` -> ``compute_dt`` ->
``step_ssprk3`` -> advance t -- on the Orszag-Tang set-up of the benchmark
(periodic unit square, gamma 5/3, CFL 0.4, no Powell source), in float64 as
the reference computes.  The initial state is built with the reference's own
``prim_to_cons`` on its own grid (``MHDSolver.X``/``Y``).  Prints one JSON
line: zone-updates/s (interior cells x steps / wall time of the timed steps),
ms per step, the stand-in used and the threads of the host.

With ``--check-steps S`` it instead advances S steps and writes the final
state to ``--out`` (.npy; the initial one to ``--out-initial``), for
comparison with this library's solver.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

import refshim  # noqa: E402


def orszag_tang(R, n: int, t_end: float = 1e30):
    C = R.config
    cfg = C.Config(nx=n, ny=n, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, t_end=t_end, cfl=0.4,
                   gamma=5.0 / 3.0, powell_source=False, bc_x_type="periodic", bc_y_type="periodic",
                   diag_interval=1 << 30, snapshot_times=[])
    s = R.solver.MHDSolver(cfg)
    xp = R.physics.xp
    g = cfg.gamma
    W = xp.zeros((C.NVAR, s.nx_tot, s.ny_tot))
    W[C.iRHO] = g * g
    W[C.iVX] = -xp.sin(2 * math.pi * s.Y)
    W[C.iVY] = xp.sin(2 * math.pi * s.X)
    W[C.iBX] = -xp.sin(2 * math.pi * s.Y)
    W[C.iBY] = xp.sin(4 * math.pi * s.X)
    W[C.iPR] = g
    W[C.iCLR] = xp.where(s.X < 0.5, 1.0, 0.0)
    s.U = R.physics.prim_to_cons(W, g)
    s.t, s.step = 0.0, 0
    return s


def one_step(R, s):
    """main.py:66-73: dt from the primitives, one SSP-RK3 step, t and step advanced."""
    cfg = s.cfg
    W = R.physics.cons_to_prim(s.U, cfg.gamma)
    s.dt = min(s.compute_dt(W), cfg.t_end - s.t)
    s.step_ssprk3()
    s.t += s.dt
    s.step += 1


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--backend", choices=["torch", "numpy"], default="torch")
    ap.add_argument("--device", default="cuda")
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--check-steps", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--out-initial", default=None)
    a = ap.parse_args(argv)
    try:
        R = refshim.load_reference(a.backend, a.device, quiet=True)
    except Exception as e:  # reference absent, or the stand-in cannot start
        print(json.dumps({"unavailable": f"{type(e).__name__}: {e}"}))
        return 0
    on_gpu = a.backend == "torch" and a.device.startswith("cuda")
    if on_gpu:
        import torch
        sync = torch.cuda.synchronize
    else:
        def sync():
            return None
    s = orszag_tang(R, a.n)
    if a.check_steps:
        if a.out_initial:
            np.save(a.out_initial, R.solver.to_numpy(s.U))
        for _ in range(a.check_steps):
            one_step(R, s)
        sync()
        np.save(a.out, R.solver.to_numpy(s.U))
        print(json.dumps({"steps": s.step, "t": s.t, "dt": s.dt, "glm_ch": s.cfg.glm_ch, "out": a.out}))
        return 0
    for _ in range(a.warmup):
        one_step(R, s)
    sync()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        one_step(R, s)
    sync()
    wall = time.perf_counter() - t0
    zu = a.n * a.n * a.steps / wall
    out = {"impl": "reference modules, unchanged", "stand_in": R.label, "backend": a.backend,
           "device": a.device if a.backend == "torch" else "cpu", "n": a.n, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": 1e3 * wall / a.steps, "zone_updates_per_s": zu, "dtype": "f64",
           "host_threads": os.cpu_count(), "finite": bool(np.isfinite(R.solver.to_numpy(s.U[0])).all()),
           "source": R.source}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
