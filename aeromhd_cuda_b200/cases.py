"""The benchmark configurations as runnable cases.

    python -m aeromhd_cuda_b200.cases orszag_tang --n 512 --precision fp32
    python -m aeromhd_cuda_b200.cases cp_alfven --sizes 32 64 128 256 512 1024
    python -m aeromhd_cuda_b200.cases shock_interface --nx 2048 --ny 512 --t-end 3
    python -m aeromhd_cuda_b200.cases brio_wu
    python -m aeromhd_cuda_b200.cases reference_rmi        # main.py:446-474
    python -m aeromhd_cuda_b200.cases rmi_convergence      # main.py:294-396, :476-492
    python -m aeromhd_cuda_b200.cases function_by_function --n 2048   # solver.py:268-333, pass by pass

Each prints one JSON object (wall time, steps, zone-updates/s and the case's
accuracy figures).  Errors of the float32 path are measured against a float64
run of the same case on the GPU (itself bit-exact with the reference's
float64 arithmetic).
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np
import torch

from . import initial_conditions as ic
from .config import Config
from .solver import MHDSolver


def _timed_advance(s: MHDSolver, t_end: float, max_steps: int = 1 << 60, chunk: int = 200):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.advance(t_end=t_end, max_steps=max_steps, chunk=chunk)
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def rel_l1(a: torch.Tensor, b: torch.Tensor) -> float:
    a, b = a.double(), b.double()
    return float((a - b).abs().sum() / b.abs().sum().clamp_min(1e-300))


def interior(s: MHDSolver) -> torch.Tensor:
    return s.U[:, 2:-2, 2:-2]


VAR_NAMES = ("rho", "mx", "my", "mz", "Bx", "By", "Bz", "E", "psi", "rhoC")


def precision_errors(s32: MHDSolver, s64: MHDSolver) -> dict:
    """Relative L1 error (sum |a - b| / sum |b|) of a state against a reference
    state, per conserved variable.  A variable that is (nearly) zero in the
    reference -- m_z and B_z of a planar flow, rho C once the mixed fluid has
    left the domain -- has no scale of its own: it is measured against the
    density, sum |a - b| / sum |rho|, and reported under "<name>/rho"."""
    a, b = interior(s32), interior(s64)
    rho = float(b[0].double().abs().sum())
    out = {}
    for v in range(10):
        ref = float(b[v].double().abs().sum())
        diff = float((a[v].double() - b[v].double()).abs().sum())
        if ref > 1e-9 * rho:
            out[VAR_NAMES[v]] = diff / ref
        else:
            out[VAR_NAMES[v] + "/rho"] = diff / max(rho, 1e-300)
    return out


def state_errors(s32: MHDSolver, s64: MHDSolver) -> dict:
    """Relative L1 errors of a state against a reference state by physical
    quantity: the whole state (all ten planes, sum |dU| / sum |U|), density,
    energy, the momentum and field vectors (sum over cells of the component
    L1 norm of the difference over that of the reference vector), psi against
    the field it cleans (sum |d psi| / sum |B|) and the colour against the
    density.  A small transverse component (m_y, B_y of a planar shock) is
    judged against the vector it belongs to rather than against itself."""
    a, b = interior(s32).double(), interior(s64).double()
    d = (a - b).abs()
    s = lambda t: float(t.sum())
    babs = b.abs()
    return {"state": s(d) / s(babs), "rho": s(d[0]) / s(babs[0]), "E": s(d[7]) / s(babs[7]),
            "m": s(d[1:4]) / s(babs[1:4]), "B": s(d[4:7]) / s(babs[4:7]), "psi/|B|": s(d[8]) / s(babs[4:7]),
            "rhoC/rho": s(d[9]) / s(babs[0])}


def same_initial_state(s32: MHDSolver, s64: MHDSolver) -> None:
    """Start both solvers from the float64 state rounded once to float32, so
    that their difference comes from the arithmetic alone."""
    r = s64.U.float()
    s64.U = r.double()
    s32.U = r
    s32.t, s32.step = s64.t, s64.step


def precision_horizon(nx: int = 2048, ny: int = 512, t_end: float = 3.0, every: float = 0.5) -> dict:
    """Where the float32 error of the shocked interface comes from, over time.

    Three runs: A float64 from the initial state, B float64 from that state
    rounded once to float32, C float32 from the same rounded state.  C - B is
    the error of the float32 arithmetic and storage; B - A is how far a
    perturbation of one float32 rounding of the initial state carries in
    float64 alone -- the flow's own sensitivity, the floor below which no
    precision can bring the difference of two runs of an unstable flow.
    Both are reported per variable (precision_errors) every `every` of
    simulated time."""
    from dataclasses import replace
    cfg = lambda p: shock_interface_config(nx, ny, p, t_end)
    A, B, C = MHDSolver(cfg("fp64")), MHDSolver(cfg("fp64")), MHDSolver(cfg("fp32"))
    D = MHDSolver(replace(cfg("fp32"), fp32_compensation=True))
    for s in (A, B, C, D):
        s.initialize()
    same_initial_state(C, B)
    D.U = C.U.clone()
    out = {"case": "precision_horizon", "nx": nx, "ny": ny, "times": [], "fp32_vs_fp64": [],
           "fp64_vs_fp64_of_rounded_start": [], "fp32_vs_fp64_by_quantity": [], "magnitudes": [],
           "fp32_compensated_vs_fp64": [], "fp32_compensated_vs_fp64_by_quantity": []}
    t = 0.0
    while t < t_end - 1e-12:
        t = min(t_end, t + every)
        for s in (A, B, C, D):
            s.advance(t_end=t, chunk=200)
        out["times"].append(t)
        out["fp32_vs_fp64"].append(precision_errors(C, B))
        out["fp64_vs_fp64_of_rounded_start"].append(precision_errors(B, A))
        out["fp32_vs_fp64_by_quantity"].append(state_errors(C, B))
        out["fp32_compensated_vs_fp64"].append(precision_errors(D, B))
        out["fp32_compensated_vs_fp64_by_quantity"].append(state_errors(D, B))
        Ub = interior(B).double().abs()
        out["magnitudes"].append({VAR_NAMES[v]: float(Ub[v].mean()) for v in range(10)})
    return out


# --------------------------------------------------------------- Orszag-Tang
def orszag_tang_config(n: int, precision: str, t_end: float = 0.5, cfl: float = 0.4) -> Config:
    return Config(nx=n, ny=n, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, t_end=t_end, cfl=cfl, gamma=5.0 / 3.0,
                  powell_source=False, bc_x_type="periodic", bc_y_type="periodic", precision=precision)


def orszag_tang(n: int = 512, t_end: float = 0.5, precisions=("fp32", "fp64")) -> dict:
    out = {"case": "orszag_tang", "n": n, "t_end": t_end}
    runs = {}
    for p in precisions:
        s = MHDSolver(orszag_tang_config(n, p, t_end))
        s.set_primitive(ic.orszag_tang(s))
        wall = _timed_advance(s, t_end)
        d = s.device_diagnostics()
        runs[p] = s
        out[p] = {"steps": s.step, "t": s.t, "wall_s": wall, "zone_updates_per_s": n * n * s.step / wall,
                  "mass": d["mass"], "energy": d["energy"], "divB_L2": d["divB_L2"]}
    if "fp32" in runs and "fp64" in runs:
        out["fp32_vs_fp64"] = precision_errors(runs["fp32"], runs["fp64"])
        out["fp32_vs_fp64_by_quantity"] = state_errors(runs["fp32"], runs["fp64"])
        out["same_step_count"] = runs["fp32"].step == runs["fp64"].step
    return out


# ------------------------------------------------------------------ CP Alfven
def cp_alfven(sizes=(32, 64, 128, 256, 512, 1024), precision: str = "fp64", amp: float = 0.1,
              angle: float = 30.0, cfl: float = 0.4) -> dict:
    """Circularly polarised Alfven wave, one period; L1 error of B_perp against the exact solution."""
    lx, ly = ic.cp_alfven_box(angle)
    out = {"case": "cp_alfven", "precision": precision, "amp": amp, "angle_deg": angle, "sizes": list(sizes),
           "L1": [], "steps": [], "zone_updates_per_s": []}
    a = math.radians(angle)
    for n in sizes:
        cfg = Config(nx=n, ny=n, x_min=0.0, x_max=lx, y_min=0.0, y_max=ly, t_end=1.0, cfl=cfl, gamma=5.0 / 3.0,
                     powell_source=False, bc_x_type="periodic", bc_y_type="periodic", precision=precision)
        s = MHDSolver(cfg)
        W0 = ic.cp_alfven(s, amp=amp, angle_deg=angle)
        s.set_primitive(W0)
        wall = _timed_advance(s, 1.0)
        from .physics import cons_to_prim
        W = cons_to_prim(s.U, cfg.gamma).double()
        # B_perp = -Bx sin(a) + By cos(a), interior
        bp = (-W[4] * math.sin(a) + W[5] * math.cos(a))[2:-2, 2:-2]
        bp0 = (-W0[4] * math.sin(a) + W0[5] * math.cos(a))[2:-2, 2:-2]
        out["L1"].append(float((bp - bp0).abs().mean()))
        out["steps"].append(s.step)
        out["zone_updates_per_s"].append(n * n * s.step / wall)
    L1 = out["L1"]
    out["orders"] = [math.log(L1[i - 1] / L1[i]) / math.log(sizes[i] / sizes[i - 1]) for i in range(1, len(L1))]
    out["mean_order"] = float(np.mean(out["orders"])) if out["orders"] else None
    return out


# ------------------------------------------------------------ shock interface
def shock_interface_config(nx=2048, ny=512, precision="fp32", t_end=3.0, seed=0) -> Config:
    """Single shock-accelerated interface: [0,4]x[0,1], Mach 3 from x = 0.5, interface at
    x = 1 + 0.05 cos(2 pi 2 y), rho 1 | 3, p = 1, 2-cell tanh, uniform Bx = 0.1, seeded
    1e-3 density noise ahead of the shock; outflow in x, periodic in y; GLM + Powell."""
    return Config(nx=nx, ny=ny, x_min=0.0, x_max=4.0, y_min=0.0, y_max=1.0, t_end=t_end, cfl=0.4, gamma=5.0 / 3.0,
                  mach=3.0, density_ratio=3.0, interface_x=1.0, shock_x=0.5, perturbation_amp=0.05,
                  perturbation_mode=2, perturbation_shape="cos", interface_cells=2.0, bx0=0.1, noise_amp=1e-3,
                  seed=seed, ic="shock_interface", powell_mode="on", bc_x_type="extrapolation",
                  bc_y_type="periodic", diag_interval=200, snapshot_times=[], precision=precision)


def shock_interface(nx=2048, ny=512, t_end=3.0, precisions=("fp32", "fp64"), diag_every=0.25) -> dict:
    out = {"case": "shock_interface", "nx": nx, "ny": ny, "t_end": t_end}
    runs = {}
    for p in precisions:
        cfg = shock_interface_config(nx, ny, p, t_end)
        s = MHDSolver(cfg)
        s.initialize()
        d0 = s.device_diagnostics()
        hist = {"t": [0.0], "mixing_width": [d0["mixing_width_integral"]], "divB_L2": [d0["divB_L2"]],
                "mass": [d0["mass"]], "energy": [d0["energy"]]}
        wall = 0.0
        tt = 0.0
        while tt < t_end - 1e-12:
            tt = min(t_end, tt + diag_every)
            wall += _timed_advance(s, tt)
            d = s.device_diagnostics()
            hist["t"].append(s.t)
            hist["mixing_width"].append(d["mixing_width_integral"])
            hist["divB_L2"].append(d["divB_L2"])
            hist["mass"].append(d["mass"])
            hist["energy"].append(d["energy"])
        ebnd = s._cumulative_boundary_energy
        runs[p] = (s, hist)
        out[p] = {"steps": s.step, "t": s.t, "wall_s": wall, "zone_updates_per_s": nx * ny * s.step / wall,
                  "history": hist,
                  "mass_drift_rel": (hist["mass"][-1] - hist["mass"][0]) / hist["mass"][0],
                  "energy_drift_rel_raw": (hist["energy"][-1] - hist["energy"][0]) / hist["energy"][0],
                  "boundary_energy": ebnd,
                  "energy_drift_rel_corrected": (hist["energy"][-1] - ebnd - hist["energy"][0]) / hist["energy"][0]}
    if "fp32" in runs and "fp64" in runs:
        (a, ha), (b, hb) = runs["fp32"], runs["fp64"]
        mwa, mwb = np.array(ha["mixing_width"]), np.array(hb["mixing_width"])
        out["fp32_vs_fp64"] = {
            "final_state": precision_errors(a, b),
            "mixing_width_max_abs_diff_over_peak": float(np.max(np.abs(mwa - mwb)) / max(np.max(np.abs(mwb)), 1e-300)),
        }
    return out


# ------------------------------------------------------------------ Brio-Wu
def brio_wu(nx: int = 800, precision: str = "fp64", cfl: float = 0.3, limiter: str = "vanleer") -> dict:
    cfg = Config(nx=nx, ny=4, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.05, t_end=0.1, cfl=cfl, gamma=2.0,
                 B_transverse=0.0, powell_source=False, use_char_bc=False, bc_x_type="extrapolation",
                 bc_y_type="periodic", precision=precision, limiter=limiter)
    s = MHDSolver(cfg)
    s.set_primitive(ic.brio_wu(s))
    wall = _timed_advance(s, 0.1)
    from .physics import cons_to_prim
    W = cons_to_prim(s.U, cfg.gamma).double().cpu().numpy()
    rho, by, vx = W[0, 2:-2, 2], W[5, 2:-2, 2], W[1, 2:-2, 2]
    checks = {"rho_min_in_(0.1,0.2)": bool(0.1 < rho.min() < 0.2), "rho_max_in_(0.9,1.05)": bool(0.9 < rho.max() < 1.05),
              "levels>10": bool(len(np.unique(np.round(rho, 2))) > 10), "By_sign_change": bool(np.any(by[:-1] * by[1:] < 0)),
              "rho_min<0.18": bool(rho.min() < 0.18), "vx_range>0.5": bool(vx.max() - vx.min() > 0.5)}
    return {"case": "brio_wu", "nx": nx, "cfl": cfl, "limiter": limiter, "precision": precision, "steps": s.step,
            "wall_s": wall, "rho_range": [float(rho.min()), float(rho.max())], "checks": checks,
            "passed": all(checks.values())}


# The reference drivers' shocked-interface set-up (main.py:446-458): Mach 10,
# density ratio 3, mode-4 perturbation, characteristic x boundaries, Powell on.
REFERENCE_RMI = dict(nx=400, ny=200, x_min=0.0, x_max=6.0, y_min=0.0, y_max=2.0, t_end=0.25, cfl=0.30, mach=10.0,
                     interface_x=1.5, perturbation_amp=0.15, perturbation_mode=4, density_ratio=3.0,
                     interface_width=2.0, powell_source=True, use_char_bc=True, bc_x_type="characteristic",
                     bc_y_type="periodic", enable_smoothing=False, diag_interval=20,
                     snapshot_times=[0.0, 0.05, 0.10, 0.15, 0.20, 0.25])
REFERENCE_RMI_CASES = {"Hydro (B=0)": 0.0, "MHD (By=0.5)": 0.5, "MHD (By=1.5)": 1.5}   # main.py:460-464


def _peak_after(s: MHDSolver, values, t_skip: float = 0.03) -> float:
    """Peak of a diagnostic history after t_skip (main.py:329-336)."""
    t = np.asarray(s.diag_times)
    v = np.asarray(values)[t > t_skip]
    return float(v.max()) if len(v) else 0.0


def reference_rmi_cases(precision: str = "fp64", t_end: float = 0.25) -> dict:
    """The three shocked-interface runs of the reference drivers (main.py:466-474)
    with their diagnostic summary (main.py:500-520: peaks after t = 0.03)."""
    out = {"case": "reference_rmi", "precision": precision, "runs": {}}
    for label, by in REFERENCE_RMI_CASES.items():
        cfg = Config(**{**REFERENCE_RMI, "t_end": t_end, "B_transverse": by, "precision": precision})
        s = MHDSolver(cfg)
        s.initialize()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.run()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        out["runs"][label] = {"steps": s.step, "t": s.t, "wall_s": wall,
                              "mw_integral_peak": _peak_after(s, s.diag_mixing_width_integral),
                              "mw_thresh_peak": _peak_after(s, s.diag_mixing_width_thresh),
                              "mixedness_peak": _peak_after(s, s.diag_mixedness),
                              "enstrophy_local_peak": _peak_after(s, s.diag_enstrophy_local),
                              "divB_L2_final": float(s.diag_divB_L2[-1])}
    return out


def convergence_config(nx: int, ny: int, by: float, precision: str = "fp64") -> Config:
    """One resolution of the reference's grid-convergence study (main.py:476-492,
    :306-312): the driver set-up to t = 0.15, diagnostics every max(10, 4000 / nx) steps."""
    return Config(**{**REFERENCE_RMI, "t_end": 0.15, "snapshot_times": [0.0, 0.15], "nx": nx, "ny": ny,
                     "B_transverse": by, "diag_interval": max(10, 20 * 200 // nx), "precision": precision})


def rmi_convergence(by: float, resolutions=((100, 50), (200, 100), (400, 200)), precision: str = "fp64") -> dict:
    """run_convergence_study, main.py:294-396: peak integral / threshold mixing
    width and local enstrophy per resolution, and the convergence order of the
    integral mixing width from three successive resolutions (main.py:346-356)."""
    rows, dxs, mwi = [], [], []
    for nx, ny in resolutions:
        cfg = convergence_config(nx, ny, by, precision)
        s = MHDSolver(cfg)
        s.initialize()
        wall = _timed_advance_run(s)
        rows.append({"nx": nx, "ny": ny, "dx": cfg.dx, "steps": s.step, "wall_s": wall,
                     "mw_integral_peak": _peak_after(s, s.diag_mixing_width_integral),
                     "mw_thresh_peak": _peak_after(s, s.diag_mixing_width_thresh),
                     "enstrophy_local_peak": _peak_after(s, s.diag_enstrophy_local)})
        dxs.append(cfg.dx)
        mwi.append(rows[-1]["mw_integral_peak"])
    orders = []
    for i in range(2, len(mwi)):
        d, dp = abs(mwi[i] - mwi[i - 1]), abs(mwi[i - 1] - mwi[i - 2])
        if mwi[i] > 0 and mwi[i - 1] > 0 and d > 1e-14 and dp > 1e-14:
            orders.append(float(np.log(dp / d) / np.log(dxs[i - 1] / dxs[i])))
    return {"case": "rmi_convergence", "By": by, "precision": precision, "resolutions": rows,
            "mw_integral_order": orders}


def _timed_advance_run(s: MHDSolver) -> float:
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.run()
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def function_by_function(n: int = 2048, precision: str = "fp64", steps: int = 5) -> dict:
    """The reference's step structure (compute_rhs / step_ssprk3, solver.py:268-333)
    executed function by function on the GPU: ghost fill, cons->prim, MUSCL and
    HLLD in x and y as separate passes over the grid (this library's
    per-function kernels), the flux differences, the right-hand side and the RK
    combinations as torch array operations -- the shape of the reference's
    CuPy path, with one pass per function where CuPy takes several.  Timed on
    the Orszag-Tang n x n grid; the fused run loop does the same step in one
    pass per stage."""
    from . import physics as P
    s = MHDSolver(orszag_tang_config(n, precision, t_end=1e30))
    s.set_primitive(ic.orszag_tang(s))
    cfg, ng, nx, ny = s.cfg, 2, n, n

    def rhs(U, ch):
        s.apply_bc(U)
        W = P.cons_to_prim(U, cfg.gamma)
        WLx, WRx = P.muscl_x(W)
        Fx, _ = P.hlld_flux_x(WLx, WRx, cfg.gamma, ch, return_smax_array=True)
        WLy, WRy = P.muscl_y(W)
        Fy, _ = P.hlld_flux_y(WLy, WRy, cfg.gamma, ch, return_smax_array=True)
        R = torch.zeros_like(U)
        R[:, ng:ng + nx, ng:ng + ny] -= (Fx[:, 1:1 + nx, :] - Fx[:, 0:nx, :])[:, :, ng:ng + ny] / cfg.dx
        R[:, ng:ng + nx, ng:ng + ny] -= (Fy[:, :, 1:1 + ny] - Fy[:, :, 0:ny])[:, ng:ng + nx, :] / cfg.dy
        return R

    def step(U, dt, ch):
        U0 = U.clone()
        U1 = s.enforce_scalar_bounds(U0 + dt * rhs(U0, ch))
        U2 = s.enforce_scalar_bounds(0.75 * U0 + 0.25 * (U1 + dt * rhs(U1, ch)))
        return s.enforce_scalar_bounds((1.0 / 3.0) * U0 + (2.0 / 3.0) * (U2 + dt * rhs(U2, ch)))

    U = s.U.clone()
    dt = s.compute_dt(P.cons_to_prim(U, cfg.gamma))
    ch = cfg.glm_ch
    for _ in range(2):
        U = step(U, dt, ch)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        U = step(U, dt, ch)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"case": "function_by_function", "n": n, "precision": precision, "ms_per_step": ms,
            "zone_updates_per_s": n * n / (ms / 1e3)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["orszag_tang", "cp_alfven", "shock_interface", "brio_wu", "reference_rmi",
                                     "rmi_convergence", "function_by_function", "precision_horizon"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--t-end", type=float, default=None)
    ap.add_argument("--sizes", type=int, nargs="*", default=[32, 64, 128, 256, 512, 1024])
    ap.add_argument("--precision", default=None)
    ap.add_argument("--cfl", type=float, default=None)
    ap.add_argument("--limiter", default="vanleer")
    a = ap.parse_args(argv)
    precs = (a.precision,) if a.precision else ("fp32", "fp64")
    if a.case == "orszag_tang":
        r = orszag_tang(a.n, a.t_end or 0.5, precs)
    elif a.case == "cp_alfven":
        r = {p: cp_alfven(tuple(a.sizes), p) for p in precs}
    elif a.case == "shock_interface":
        r = shock_interface(a.nx, a.ny, a.t_end or 3.0, precs)
    elif a.case == "reference_rmi":
        r = {p: reference_rmi_cases(p, a.t_end or 0.25) for p in precs}
    elif a.case == "precision_horizon":
        r = precision_horizon(a.nx, a.ny, a.t_end or 3.0)
    elif a.case == "function_by_function":
        r = {p: function_by_function(a.n, p) for p in precs}
    elif a.case == "rmi_convergence":
        r = {p: [rmi_convergence(by, precision=p) for by in (0.0, 1.5)] for p in precs}
    else:
        r = {p: brio_wu(precision=p, cfl=a.cfl or 0.3, limiter=a.limiter) for p in precs}
    print(json.dumps(r))
    return 0


if __name__ == "__main__":
    sys.exit(main())
