"""Initial conditions, evaluated on the GPU over the full grid (ghosts included).

Each generator returns primitive variables ``W[10, nx+4, ny+4]`` (float64)
for a solver's cell centres; ``MHDSolver.set_primitive(W)`` converts and
loads them.

* :func:`rmi` -- the reference's shocked, perturbed density interface
  (``MHDSolver.initialize``, solver.py:109-156): Rankine-Hugoniot post-shock
  state left of ``interface_x - 0.3``, tanh-smoothed sinusoidal interface,
  transverse field ``B_transverse``, colour = interface fraction.
* :func:`shock_interface` -- a planar shock launched at ``shock_x`` into a
  light/heavy interface at ``interface_x + amp * cos|sin(2 pi k y / Ly)``,
  smoothed over ``interface_cells`` cells, in a field
  ``Bx = bx0 + b1 sin(2 pi m y / Ly)`` (parallel to the shock normal, so the
  jump is the hydrodynamic one), with seeded white-noise density
  perturbation of relative amplitude ``noise_amp`` in the unshocked gas.
* :func:`orszag_tang` -- rho = gamma^2, p = gamma, v = (-sin 2pi y, sin 2pi x),
  B = (-sin 2pi y, sin 4pi x) on a periodic box; colour = (x < 0.5).
* :func:`cp_alfven` -- circularly polarised Alfven wave (amplitude, angle to
  the x axis) on a periodic box of one wavelength along the wave vector.
* :func:`brio_wu`, :func:`linear_alfven`, :func:`contact` -- the reference's
  verification set-ups (main.py:51-61, :155-160, :231-237).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .config import iBX, iBY, iBZ, iCLR, iPR, iRHO, iVX, iVY, iVZ
from .physics import mhd_rankine_hugoniot


def _zeros(solver):
    return torch.zeros((10, solver.nx_tot, solver.ny_tot), dtype=torch.float64, device=solver.device)


def _sel(mask, a, b):
    """torch.where in float64 (python-float operands would otherwise give float32)."""
    def f64(v):
        return v if isinstance(v, torch.Tensor) else torch.tensor(float(v), dtype=torch.float64, device=mask.device)
    return torch.where(mask, f64(a), f64(b)).to(torch.float64)


def _xy(solver):
    X = solver.X.to(torch.float64)
    Y = solver.Y.to(torch.float64)
    return X, Y


def rmi(solver):
    """solver.py:109-156; returns (W, rh) with rh the Rankine-Hugoniot dict (solver.py:118)."""
    cfg = solver.cfg
    g, M = cfg.gamma, cfg.mach
    rho1, p1 = 1.0, 1.0
    by_pre = cfg.B_transverse
    rho2, p2, vx2, by2, vs = mhd_rankine_hugoniot(g, M, rho1, p1, by_pre)
    rh = {"rho2": rho2, "p2": p2, "vx2": vx2, "By2": by2, "vs": vs}
    rho_h = rho1 * cfg.density_ratio
    x_shock = cfg.interface_x - 0.3
    ly = cfg.y_max - cfg.y_min
    ky = 2 * np.pi * cfg.perturbation_mode / ly
    X, Y = _xy(solver)
    x_if = cfg.interface_x + cfg.perturbation_amp * torch.sin(ky * Y)
    delta = cfg.interface_width * cfg.dx
    phi = 0.5 * (1.0 + torch.tanh((X - x_if) / max(delta, 1e-10)))
    W = _zeros(solver)
    post = X < x_shock
    rho_pre = rho1 * (1 - phi) + rho_h * phi
    W[iRHO] = _sel(post, rho2, rho_pre)
    W[iVX] = _sel(post, vx2, 0.0)
    W[iBY] = _sel(post, by2, by_pre)
    W[iPR] = _sel(post, p2, p1)
    W[iCLR] = _sel(post, 0.0, phi)
    return W, rh


def shock_interface(solver):
    """Uniform-Bx shocked interface (light gas rho=1, p=1 at rest ahead of the shock)."""
    cfg = solver.cfg
    g, M = cfg.gamma, cfg.mach
    rho1, p1 = 1.0, 1.0
    rho2, p2, vx2, _, vs = mhd_rankine_hugoniot(g, M, rho1, p1, 0.0)
    rh = {"rho2": rho2, "p2": p2, "vx2": vx2, "By2": 0.0, "vs": vs}
    rho_h = rho1 * cfg.density_ratio
    x_shock = cfg.shock_x if cfg.shock_x is not None else cfg.interface_x - 0.3
    ly = cfg.y_max - cfg.y_min
    ky = 2 * np.pi * cfg.perturbation_mode / ly
    X, Y = _xy(solver)
    yy = Y - cfg.y_min
    shape = torch.cos if cfg.perturbation_shape == "cos" else torch.sin
    x_if = cfg.interface_x + cfg.perturbation_amp * shape(ky * yy)
    cells = cfg.interface_cells if cfg.interface_cells is not None else cfg.interface_width
    phi = 0.5 * (1.0 + torch.tanh((X - x_if) / max(cells * cfg.dx, 1e-10)))
    rho_pre = rho1 * (1 - phi) + rho_h * phi
    if cfg.noise_amp > 0:
        rng = np.random.default_rng(cfg.seed)
        xi = torch.from_numpy(rng.uniform(-1.0, 1.0, size=tuple(X.shape))).to(X.device)
        rho_pre = rho_pre * (1.0 + cfg.noise_amp * xi)
    post = X < x_shock
    W = _zeros(solver)
    W[iRHO] = _sel(post, rho2, rho_pre)
    W[iVX] = _sel(post, vx2, 0.0)
    W[iPR] = _sel(post, p2, p1)
    W[iBX] = cfg.bx0 + cfg.b1 * torch.sin(2 * np.pi * cfg.b_mode * yy / ly)
    W[iCLR] = _sel(post, 0.0, phi)
    if cfg.ic_frame == "post_shock":
        W[iVX] -= vx2
    return W, rh


def orszag_tang(solver):
    cfg = solver.cfg
    X, Y = _xy(solver)
    g = cfg.gamma
    W = _zeros(solver)
    W[iRHO] = g * g
    W[iVX] = -torch.sin(2 * np.pi * Y)
    W[iVY] = torch.sin(2 * np.pi * X)
    W[iBX] = -torch.sin(2 * np.pi * Y)
    W[iBY] = torch.sin(4 * np.pi * X)
    W[iPR] = g
    W[iCLR] = (X < 0.5).to(torch.float64)
    return W


def cp_alfven_box(angle_deg: float = 30.0):
    """Periodic box holding one wavelength along a wave vector at `angle_deg` to x."""
    a = math.radians(angle_deg)
    return 1.0 / math.cos(a), 1.0 / math.sin(a)


def cp_alfven(solver, amp: float = 0.1, angle_deg: float = 30.0, rho: float = 1.0, p: float = 0.1, b0: float = 1.0,
              t: float = 0.0):
    """Circularly polarised Alfven wave; exact solution at time t (it travels at v_A = b0/sqrt(rho))."""
    a = math.radians(angle_deg)
    ca, sa = math.cos(a), math.sin(a)
    X, Y = _xy(solver)
    va = b0 / math.sqrt(rho)
    xp = X * ca + Y * sa + va * t      # phase coordinate along k (wave moves towards -k)
    ph = 2 * np.pi * xp
    b_perp = amp * torch.sin(ph)
    b_z = amp * torch.cos(ph)
    v_perp = b_perp / math.sqrt(rho)
    v_z = b_z / math.sqrt(rho)
    W = _zeros(solver)
    W[iRHO] = rho
    W[iPR] = p
    W[iVX] = -v_perp * sa
    W[iVY] = v_perp * ca
    W[iVZ] = v_z
    W[iBX] = b0 * ca - b_perp * sa
    W[iBY] = b0 * sa + b_perp * ca
    W[iBZ] = b_z
    W[iCLR] = 0.5
    return W


def brio_wu(solver):
    """main.py:51-59"""
    left = (solver.x < 0.5)[:, None].expand(solver.nx_tot, solver.ny_tot)
    W = _zeros(solver)
    W[iRHO] = _sel(left, 1.0, 0.125)
    W[iPR] = _sel(left, 1.0, 0.1)
    W[iBX] = 0.75
    W[iBY] = _sel(left, 1.0, -1.0)
    W[iCLR] = _sel(left, 1.0, 0.0)
    return W


def linear_alfven(solver, amp: float = 1e-6, rho0: float = 1.0, p0: float = 0.1, bx0: float = 1.0):
    """main.py:155-160 (x-aligned linear Alfven wave on [0, 1])."""
    lx = solver.cfg.x_max - solver.cfg.x_min
    s = torch.sin(2.0 * np.pi / lx * solver.x)[:, None].expand(solver.nx_tot, solver.ny_tot)
    W = _zeros(solver)
    W[iRHO] = rho0
    W[iPR] = p0
    W[iBX] = bx0
    W[iBY] = amp * s
    W[iVY] = -amp * s / np.sqrt(rho0)
    return W


def contact(solver):
    """main.py:231-237"""
    left = (solver.x < 0.5)[:, None].expand(solver.nx_tot, solver.ny_tot)
    W = _zeros(solver)
    W[iRHO] = _sel(left, 1.0, 3.0)
    W[iPR] = 1.0
    W[iVX] = 1.0
    W[iBX] = 0.5
    W[iCLR] = _sel(left, 0.0, 1.0)
    return W
