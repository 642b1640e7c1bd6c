"""Parameter set of the solver: variable slots, floors and ``Config``.

The names, slot numbers, floors, fields and defaults are the reference's
(config.py:13-89) so that code written against the reference's ``Config``
runs unchanged.  Fields added here (all defaulted so that the reference's
behaviour is what you get when you leave them alone):

``precision``      "fp64" (default; results match the reference's float64
                   path) or "fp32" (fp32 state and fluxes, fp64 pressure
                   recovery, dt reduction and diagnostics).
``limiter``        "vanleer" (the reference's only limiter, physics.py:323-350)
                   or "minmod".
``powell_mode``    "auto" (the reference's gate ``powell_source and
                   B_transverse > 0``, solver.py:304), "on" or "off".
``ic``             initial condition used by ``MHDSolver.initialize``:
                   "rmi" (the reference's, solver.py:109-156) or
                   "shock_interface" (a uniform-Bx shocked interface, see
                   ``initial_conditions.shock_interface``).
``bx0``, ``shock_x``, ``perturbation_shape``, ``interface_cells``,
``noise_amp``, ``seed``, ``b1``, ``b_mode``, ``ic_frame``
                   parameters of the "shock_interface" initial condition
                   (``ic_frame`` "lab": unshocked gas at rest; "post_shock":
                   the frame of the shocked gas, which keeps the mixing layer
                   near where the shock meets it).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from enum import IntEnum
from typing import List, Optional


class ConsVar(IntEnum):
    RHO = 0
    MX = 1
    MY = 2
    MZ = 3
    BX = 4
    BY = 5
    BZ = 6
    EN = 7
    PSI = 8
    RHOC = 9


class PrimVar(IntEnum):
    RHO = 0
    VX = 1
    VY = 2
    VZ = 3
    BX = 4
    BY = 5
    BZ = 6
    PR = 7
    PSI = 8
    CLR = 9


NVAR = 10

RHO, MX, MY, MZ, BX, BY, BZ, EN, PSI, RHOC = (
    ConsVar.RHO, ConsVar.MX, ConsVar.MY, ConsVar.MZ, ConsVar.BX, ConsVar.BY, ConsVar.BZ, ConsVar.EN,
    ConsVar.PSI, ConsVar.RHOC)
iRHO, iVX, iVY, iVZ, iBX, iBY, iBZ, iPR, iPSI, iCLR = (
    PrimVar.RHO, PrimVar.VX, PrimVar.VY, PrimVar.VZ, PrimVar.BX, PrimVar.BY, PrimVar.BZ, PrimVar.PR,
    PrimVar.PSI, PrimVar.CLR)

FLOOR_RHO = 1e-12
FLOOR_PR = 1e-12

PRECISIONS = ("fp64", "fp32")
LIMITERS = ("vanleer", "minmod")


@dataclass
class Config:
    """Simulation parameters (reference fields first, in the reference's order)."""
    nx: int = 400
    ny: int = 200
    x_min: float = 0.0
    x_max: float = 6.0
    y_min: float = 0.0
    y_max: float = 2.0
    t_end: float = 0.25
    cfl: float = 0.30
    max_steps: int = 200000
    gamma: float = 5.0 / 3.0
    mach: float = 10.0
    interface_x: float = 1.5
    perturbation_amp: float = 0.15
    perturbation_mode: int = 4
    density_ratio: float = 3.0
    interface_width: float = 2.0
    B_transverse: float = 0.0
    glm_ch: float = 0.0
    glm_alpha: float = 1.5
    powell_source: bool = True
    use_char_bc: bool = True
    bc_x_type: str = "auto"
    bc_y_type: str = "periodic"
    enable_smoothing: bool = False
    diag_interval: int = 20
    snapshot_times: List[float] = field(default_factory=lambda: [0.0, 0.05, 0.10, 0.15, 0.20, 0.25])
    # ---- additions (defaults reproduce the reference) ----
    precision: str = "fp64"
    limiter: str = "vanleer"
    powell_mode: str = "auto"
    ic: str = "rmi"
    bx0: float = 0.0
    b1: float = 0.0
    b_mode: int = 1
    shock_x: Optional[float] = None
    perturbation_shape: str = "sin"
    interface_cells: Optional[float] = None
    noise_amp: float = 0.0
    seed: int = 0
    ic_frame: str = "lab"
    # float32 run loop: accumulate the base state compensated (a float32 low part
    # kept next to U, amhd_advance_compensated).  The low part starts at zero at
    # every loop start and is not part of U or of a checkpoint.
    fp32_compensation: bool = False

    @property
    def dx(self) -> float:
        return (self.x_max - self.x_min) / self.nx

    @property
    def dy(self) -> float:
        return (self.y_max - self.y_min) / self.ny

    def get_bc_x(self) -> str:
        if self.bc_x_type != "auto":
            return self.bc_x_type
        return "characteristic" if self.use_char_bc else "extrapolation"

    def powell_enabled(self) -> bool:
        """The reference's gate (solver.py:304) unless ``powell_mode`` overrides it."""
        if self.powell_mode == "on":
            return True
        if self.powell_mode == "off":
            return False
        return bool(self.powell_source and self.B_transverse > 0)

    def validate(self) -> None:
        if self.nx < 2 or self.ny < 2:
            raise ValueError(f"grid must be at least 2x2 interior cells, got {self.nx}x{self.ny}")
        if self.precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}, got {self.precision!r}")
        if self.limiter not in LIMITERS:
            raise ValueError(f"limiter must be one of {LIMITERS}, got {self.limiter!r}")
        if self.powell_mode not in ("auto", "on", "off"):
            raise ValueError(f"powell_mode must be auto/on/off, got {self.powell_mode!r}")
        if not (self.x_max > self.x_min and self.y_max > self.y_min):
            raise ValueError("empty domain")
        if self.gamma <= 1.0:
            raise ValueError("gamma must exceed 1")


# boundary codes shared with the C ABI (include/aeromhd.h)
BC_PERIODIC = 0
BC_EXTRAPOLATION = 1
BC_CHARACTERISTIC = 2


def bc_x_code(cfg: Config) -> int:
    kind = cfg.get_bc_x()
    if kind == "periodic":
        return BC_PERIODIC
    if kind == "characteristic":
        return BC_CHARACTERISTIC
    return BC_EXTRAPOLATION


def bc_y_code(cfg: Config) -> int:
    return BC_PERIODIC if cfg.bc_y_type == "periodic" else BC_EXTRAPOLATION
