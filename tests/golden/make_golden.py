"""Generate the golden vectors in this folder by running the reference itself.

    python tests/golden/make_golden.py            # needs the reference checkout

Every array written here is an output of the reference's own code (imported
unchanged through ``refshim``), on inputs that are stored beside it:

* ``hlld_faces.npz``  -- the reference's HLLD kernel (physics.py:43-276) on
  random face states covering all six flux regions, ch = 0 and ch > 0, x and y.
* ``conversions.npz`` -- cons_to_prim / prim_to_cons / muscl_x / muscl_y
  (physics.py:284-350) on a random state.
* ``steps.npz``       -- three drivers'-loop steps (cons_to_prim -> compute_dt
  -> step_ssprk3, main.py:66-73) on a small random smooth state for every
  x/y boundary kind, Powell source on and off; plus apply_bc, compute_rhs,
  enforce_scalar_bounds and the Powell source of the first case.
* ``brio_wu.npz``     -- Brio-Wu 800x4 (and 200x4) to t = 0.1 with the
  reference's own driver setup (main.py:34-73); final y-row of U.
* ``alfven.npz``      -- linear Alfven-wave convergence (main.py:126-191).
* ``contact.npz``     -- contact discontinuity (main.py:215-249).
* ``rmi.npz``         -- MHDSolver.initialize() (solver.py:109-156) on a
  48x24 grid, By = 0.5, characteristic x boundaries, Powell on; 40 steps of
  the run loop, then compute_diagnostics() (solver.py:335-444).
* ``orszag_tang.npz`` -- an Orszag-Tang 32x32 state driven through the
  reference's step loop for 30 steps.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refshim  # noqa: E402

R = refshim.load_reference()
Config = R.config.Config
phys = R.physics
MHDSolver = R.solver.MHDSolver


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}: {os.path.getsize(path) / 1024:.0f} KB")


def random_faces(rng, n):
    W = np.empty((10, n))
    W[0] = rng.uniform(0.05, 3.0, n)
    W[1] = rng.uniform(-6.0, 6.0, n)
    W[2] = rng.uniform(-2.0, 2.0, n)
    W[3] = rng.uniform(-1.0, 1.0, n)
    W[4] = rng.uniform(-2.0, 2.0, n)
    W[5] = rng.uniform(-2.0, 2.0, n)
    W[6] = rng.uniform(-1.0, 1.0, n)
    W[7] = rng.uniform(0.01, 2.0, n)
    W[8] = rng.uniform(-0.5, 0.5, n)
    W[9] = rng.uniform(0.0, 1.0, n)
    # a few degenerate faces: floors, zero field, identical sides
    W[0, :8] = [1e-14, 0.0, -1.0, 1.0, 1.0, 2.0, 1.0, 1.0]
    W[7, 8:16] = [0.0, -1.0, 1e-13, 1.0, 1.0, 1.0, 1.0, 1.0]
    W[4:7, 16:24] = 0.0
    return W


def hlld_kernel_raw(WL, WR, gamma, ch):
    """The reference kernel launched exactly as physics.py:353-367 does, keeping the per-face smax."""
    n = WL.shape[1]
    F = np.empty_like(WL)
    smax = np.empty(n)
    block = 256
    grid = (n + block - 1) // block
    phys._hlld_kernel((grid,), (block,), (WL, WR, F, smax, np.int32(n), np.float64(gamma), np.float64(ch),
                                          np.float64(R.config.FLOOR_RHO), np.float64(R.config.FLOOR_PR)))
    return F, smax


def make_hlld():
    rng = np.random.default_rng(20260101)
    n = 1024
    WL = random_faces(rng, n)
    WR = random_faces(rng, n)
    WR[:, 24:32] = WL[:, 24:32]
    out = dict(WL=WL, WR=WR, gamma=np.float64(5.0 / 3.0), chs=np.array([0.0, 2.5]))
    perm = [0, 2, 1, 3, 5, 4, 6, 7, 8, 9]
    for k, ch in enumerate(out["chs"]):
        F, smax = hlld_kernel_raw(np.ascontiguousarray(WL), np.ascontiguousarray(WR), out["gamma"], ch)
        out[f"Fx_{k}"], out[f"smaxx_{k}"] = F, smax
        Fy_max = phys.hlld_flux_y(WL, WR, out["gamma"], ch)
        Fr, smax_y = hlld_kernel_raw(np.ascontiguousarray(WL[perm]), np.ascontiguousarray(WR[perm]), out["gamma"], ch)
        assert np.array_equal(Fr[perm], Fy_max[0])
        out[f"Fy_{k}"], out[f"smaxy_{k}"] = Fr[perm], smax_y
    save("hlld_faces.npz", **out)


def random_state(rng, nxt, nyt, gamma, smooth=True):
    x = np.linspace(0.0, 1.0, nxt)[:, None]
    y = np.linspace(0.0, 1.0, nyt)[None, :]
    noise = (lambda a: a * rng.standard_normal((nxt, nyt)))
    W = np.zeros((10, nxt, nyt))
    W[0] = 1.0 + 0.3 * np.sin(2 * np.pi * (x + 2 * y)) + noise(0.05)
    W[1] = 0.5 * np.cos(2 * np.pi * y) + noise(0.05)
    W[2] = 0.3 * np.sin(2 * np.pi * x) + noise(0.02)
    W[3] = noise(0.1)
    W[4] = 0.7 + 0.1 * np.sin(2 * np.pi * y)
    W[5] = 0.5 * np.cos(2 * np.pi * x)
    W[6] = noise(0.2)
    W[7] = 1.0 + 0.2 * np.cos(2 * np.pi * (x - y))
    W[8] = noise(0.01)
    W[9] = np.clip(x + 0.1 * noise(1.0), 0.0, 1.0)
    if not smooth:
        W[0] += noise(0.2) ** 2
    return phys.prim_to_cons(W, gamma)


def make_conversions():
    rng = np.random.default_rng(7)
    U = random_state(rng, 20, 15, 1.4, smooth=False)
    U[7, 3, 4] = 0.0          # negative pressure -> floor
    U[0, 5, 6] = -1.0         # negative density -> floor
    W = phys.cons_to_prim(U, 1.4)
    U2 = phys.prim_to_cons(W, 1.4)
    WLx, WRx = phys.muscl_x(W)
    WLy, WRy = phys.muscl_y(W)
    save("conversions.npz", U=U, gamma=np.float64(1.4), W=W, U2=U2, WLx=WLx, WRx=WRx, WLy=WLy, WRy=WRy)


STEP_CASES = [(bx, by, B) for bx in ("periodic", "extrapolation", "characteristic")
              for by in ("periodic", "outflow") for B in (0.0, 0.5)]


def make_steps():
    rng = np.random.default_rng(11)
    out = {}
    for k, (bcx, bcy, By) in enumerate(STEP_CASES):
        cfg = Config(nx=10, ny=8, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.8, cfl=0.3, gamma=5.0 / 3.0,
                     B_transverse=By, powell_source=True, bc_x_type=bcx, bc_y_type=bcy, glm_alpha=1.5)
        s = MHDSolver(cfg)
        U0 = random_state(rng, s.nx_tot, s.ny_tot, cfg.gamma)
        s.U = U0.copy()
        dts, chs = [], []
        for _ in range(3):
            W = phys.cons_to_prim(s.U, cfg.gamma)
            s.dt = s.compute_dt(W)
            dts.append(s.dt)
            chs.append(cfg.glm_ch)
            s.step_ssprk3()
        out[f"U0_{k}"] = U0
        out[f"U3_{k}"] = s.U
        out[f"dt_{k}"] = np.array(dts)
        out[f"ch_{k}"] = np.array(chs)
        out[f"ebnd_{k}"] = np.float64(s._cumulative_boundary_energy)
        if k == 3:  # periodic/outflow, By=0.5: the single-routine goldens
            cfg.glm_ch = 2.0
            s._glm_ch_frozen = 2.0
            Ub = U0.copy()
            R_ = s.compute_rhs(Ub)
            out["rhs_U"] = U0
            out["rhs_Ubc"] = Ub
            out["rhs_R"] = R_
            out["rhs_S"] = s._compute_powell_source(Ub, phys.cons_to_prim(Ub, cfg.gamma))
            Uc = U0.copy()
            Uc[9] *= 1.7
            Uc[9, 2, 3] = -0.4
            out["bounds_in"] = Uc.copy()
            out["bounds_out"] = s.enforce_scalar_bounds(Uc)
    out["cases"] = np.array([f"{a}|{b}|{c}" for a, b, c in STEP_CASES])
    save("steps.npz", **out)


def run_driver_loop(solver, t_end, max_steps):
    cfg = solver.cfg
    while solver.t < t_end and solver.step < max_steps:
        W = phys.cons_to_prim(solver.U, cfg.gamma)
        dt_cfl = solver.compute_dt(W)
        solver.dt = min(dt_cfl, t_end - solver.t)
        if solver.dt <= 1e-16:
            break
        solver.step_ssprk3()
        solver.t += solver.dt
        solver.step += 1


def brio_wu_solver(nx):
    """main.py:39-63 setup."""
    cfg = Config(nx=nx, ny=4, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.05, t_end=0.1, cfl=0.30, gamma=2.0,
                 mach=1.0, B_transverse=0.0, interface_x=0.5, perturbation_amp=0.0, density_ratio=1.0,
                 diag_interval=10000, snapshot_times=[0.1], powell_source=False, use_char_bc=False,
                 bc_x_type="extrapolation", bc_y_type="periodic")
    s = MHDSolver(cfg)
    W = np.zeros((10, s.nx_tot, s.ny_tot))
    left = s.x < 0.5
    W[0] = np.where(left[:, None], 1.0, 0.125)
    W[7] = np.where(left[:, None], 1.0, 0.1)
    W[4] = 0.75
    W[5] = np.where(left[:, None], 1.0, -1.0)
    W[9] = np.where(left[:, None], 1.0, 0.0)
    s.U = phys.prim_to_cons(W, cfg.gamma)
    return s


def make_brio_wu():
    out = {}
    for nx in (200, 800):
        s = brio_wu_solver(nx)
        out[f"U0_{nx}"] = s.U[:, :, 2].copy()
        t0 = time.time()
        run_driver_loop(s, s.cfg.t_end, s.cfg.max_steps)
        print(f"  brio-wu {nx}: {s.step} steps, {time.time() - t0:.1f}s")
        assert np.all(s.U == s.U[:, :, 2:3]), "Brio-Wu must stay uniform in y"
        out[f"row_{nx}"] = s.U[:, :, 2].copy()
        out[f"steps_{nx}"] = np.int64(s.step)
        out[f"t_{nx}"] = np.float64(s.t)
        out[f"ch_{nx}"] = np.float64(s.cfg.glm_ch)
    out["reference_pass_800"] = np.bool_(R.main.brio_wu_test(nx=800, t_end=0.1, plot=False))
    save("brio_wu.npz", **out)


def make_alfven():
    """main.py:126-191, repeated step by step so the final By rows are kept."""
    resolutions = [32, 64, 128, 256]
    errors, steps = [], []
    out = {}
    rho0, p0, bx0, amp, gamma, lx = 1.0, 0.1, 1.0, 1e-6, 5.0 / 3.0, 1.0
    period = lx / (bx0 / np.sqrt(rho0))
    for nx in resolutions:
        cfg = Config(nx=nx, ny=4, x_min=0.0, x_max=lx, y_min=0.0, y_max=0.05, t_end=period, cfl=0.25, gamma=gamma,
                     mach=1.0, B_transverse=0.0, interface_x=0.5, perturbation_amp=0.0, density_ratio=1.0,
                     diag_interval=100000, snapshot_times=[period], powell_source=False, use_char_bc=False,
                     bc_x_type="periodic", bc_y_type="periodic")
        s = MHDSolver(cfg)
        x = s.x
        W = np.zeros((10, s.nx_tot, s.ny_tot))
        W[0] = rho0
        W[7] = p0
        W[4] = bx0
        W[5] = amp * np.sin(2.0 * np.pi / lx * x)[:, None] * np.ones(s.ny_tot)[None, :]
        W[2] = -amp * np.sin(2.0 * np.pi / lx * x)[:, None] * np.ones(s.ny_tot)[None, :] / np.sqrt(rho0)
        W_init = W.copy()
        s.U = phys.prim_to_cons(W, gamma)
        out[f"U0_{nx}"] = s.U[:, :, 2].copy()
        run_driver_loop(s, cfg.t_end, 100000)
        wf = phys.cons_to_prim(s.U, gamma)
        err = float(np.mean(np.abs(wf[5, 2:-2, 2] - W_init[5, 2:-2, 2])))
        errors.append(err)
        steps.append(s.step)
        out[f"row_{nx}"] = s.U[:, :, 2].copy()
    out["resolutions"] = np.array(resolutions)
    out["L1"] = np.array(errors)
    out["steps"] = np.array(steps)
    out["period"] = np.float64(period)
    out["reference_pass"] = np.bool_(R.main.linear_wave_convergence_test(plot=False))
    print("  alfven L1:", errors)
    save("alfven.npz", **out)


def make_contact():
    cfg = Config(nx=400, ny=4, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.01, t_end=0.2, cfl=0.30, gamma=5.0 / 3.0,
                 mach=1.0, B_transverse=0.0, interface_x=0.5, perturbation_amp=0.0, density_ratio=1.0,
                 diag_interval=100000, snapshot_times=[0.2], powell_source=False, use_char_bc=False,
                 bc_x_type="extrapolation", bc_y_type="periodic")
    s = MHDSolver(cfg)
    x = s.x
    W = np.zeros((10, s.nx_tot, s.ny_tot))
    W[0] = np.where(x[:, None] < 0.5, 1.0, 3.0)
    W[7] = 1.0
    W[1] = 1.0
    W[4] = 0.5
    W[9] = np.where(x[:, None] < 0.5, 0.0, 1.0)
    s.U = phys.prim_to_cons(W, cfg.gamma)
    out = dict(U0=s.U[:, :, 2].copy())
    run_driver_loop(s, cfg.t_end, cfg.max_steps)
    out.update(row=s.U[:, :, 2].copy(), steps=np.int64(s.step), t=np.float64(s.t),
               reference_pass=np.bool_(R.main.contact_discontinuity_test(plot=False)))
    save("contact.npz", **out)


def make_rmi():
    cfg = Config(nx=48, ny=24, t_end=0.25, cfl=0.30, mach=10.0, B_transverse=0.5, powell_source=True,
                 use_char_bc=True, bc_x_type="characteristic", bc_y_type="periodic", diag_interval=20)
    s = MHDSolver(cfg)
    s.initialize()
    out = dict(U_init=s.U.copy())
    out.update({f"rh_{k}": np.float64(v) for k, v in s._rh_results.items()})
    nsteps = 40
    run_driver_loop(s, cfg.t_end, nsteps)
    s.compute_diagnostics()
    out.update(U_final=s.U.copy(), steps=np.int64(s.step), t=np.float64(s.t), ch=np.float64(cfg.glm_ch),
               ebnd=np.float64(s._cumulative_boundary_energy))
    for name in ("mixing_width_integral", "mixing_width_thresh", "mixedness", "enstrophy", "enstrophy_local",
                 "perturbation_amp", "stag_pressure", "divB_max", "divB_L2", "energy_total",
                 "boundary_flux_cumulative"):
        out[f"diag_{name}"] = np.float64(getattr(s, f"diag_{name}")[-1])
    out["diag_mode_amps"] = np.asarray(s.diag_mode_amps[-1])
    # the initial-condition routine for the RH branch without a transverse field
    out["rh_hydro"] = np.array(phys.mhd_rankine_hugoniot(5.0 / 3.0, 3.0, 1.0, 1.0, 0.0))
    out["rh_mhd"] = np.array(phys.mhd_rankine_hugoniot(5.0 / 3.0, 10.0, 1.0, 1.0, 1.5))
    save("rmi.npz", **out)


def orszag_tang_prims(x, y, gamma):
    """Orszag-Tang vortex on [0,1]^2: rho=gamma^2, p=gamma, v=(-sin2pi y, sin2pi x), B=(-sin2pi y, sin4pi x)."""
    X, Y = np.meshgrid(x, y, indexing="ij")
    W = np.zeros((10,) + X.shape)
    W[0] = gamma * gamma
    W[1] = -np.sin(2 * np.pi * Y)
    W[2] = np.sin(2 * np.pi * X)
    W[4] = -np.sin(2 * np.pi * Y)
    W[5] = np.sin(4 * np.pi * X)
    W[7] = gamma
    W[9] = (X < 0.5).astype(float)
    return W


def make_orszag_tang():
    cfg = Config(nx=32, ny=32, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, t_end=0.5, cfl=0.4, gamma=5.0 / 3.0,
                 B_transverse=0.0, powell_source=False, bc_x_type="periodic", bc_y_type="periodic")
    s = MHDSolver(cfg)
    W = orszag_tang_prims(s.x, s.y, cfg.gamma)
    s.U = phys.prim_to_cons(W, cfg.gamma)
    out = dict(U0=s.U.copy())
    run_driver_loop(s, cfg.t_end, 30)
    out.update(U_final=s.U.copy(), steps=np.int64(s.step), t=np.float64(s.t), ch=np.float64(cfg.glm_ch))
    save("orszag_tang.npz", **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["hlld", "conversions", "steps", "brio_wu", "alfven", "contact", "rmi", "orszag_tang"]
    for w in which:
        print(f"== {w}")
        globals()[f"make_{w}"]()
