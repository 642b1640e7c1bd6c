"""CPU float64 oracle for the AeroMHD-CUDA solver hot path.

TEST INFRASTRUCTURE ONLY.  The tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module as the checker; the product
package never imports it.

It wraps ``liboracle.so`` (built from ``amhd_oracle.c`` by :func:`build`)
with the reference's own Python call surface:

* ``cons_to_prim`` / ``prim_to_cons`` / ``muscl_x`` / ``muscl_y`` /
  ``hlld_flux_x`` / ``hlld_flux_y``  -- physics.py:284-379
* :class:`OracleSolver` -- the hot-path methods of ``MHDSolver``
  (``apply_bc``, ``enforce_scalar_bounds``, ``compute_dt``, ``compute_rhs``,
  ``step_ssprk3``, ``_compute_powell_source``,
  ``_compute_boundary_energy_flux``), solver.py:158-333, plus the drivers'
  step loop (main.py:66-73) as :meth:`OracleSolver.advance`.

Arrays are numpy float64 ``[10, nx_tot, ny_tot]`` exactly as in the reference.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "amhd_oracle.c")
LIB_PATH = os.path.join(HERE, "liboracle.so")

NVAR = 10
NG = 2
FLOOR_RHO = 1e-12
FLOOR_PR = 1e-12
RHO, MX, MY, MZ, BX, BY, BZ, EN, PSI, RHOC = range(10)

BC_PERIODIC, BC_EXTRAP, BC_CHARACTERISTIC = 0, 1, 2

_lib = None
_D = ctypes.c_double
_L = ctypes.c_long
_I = ctypes.c_int
_P = ctypes.c_void_p


def _src_hash() -> str:
    with open(SRC, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def build(force: bool = False) -> str:
    """Compile liboracle.so with gcc (OpenMP, no FMA contraction); skipped when the
    source hash recorded beside the library matches."""
    stamp = LIB_PATH + ".srchash"
    current = os.path.exists(LIB_PATH) and os.path.exists(stamp) and open(stamp).read().strip() == _src_hash()
    if force or not current:
        cmd = ["gcc", "-O2", "-std=c11", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
               "-shared", "-o", LIB_PATH, SRC, "-lm"]
        subprocess.check_call(cmd)
        with open(stamp, "w") as f:
            f.write(_src_hash())
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_cons_to_prim.argtypes = [_P, _P, _L, _D]
        L.orc_prim_to_cons.argtypes = [_P, _P, _L, _D]
        L.orc_muscl_x.argtypes = [_P, _I, _I, _P, _P]
        L.orc_muscl_y.argtypes = [_P, _I, _I, _P, _P]
        L.orc_hlld_flux_x.argtypes = [_P, _P, _P, _P, _L, _D, _D]
        L.orc_hlld_flux_y.argtypes = [_P, _P, _P, _P, _L, _D, _D]
        L.orc_apply_bc.argtypes = [_P, _I, _I, _I, _I]
        L.orc_enforce_scalar_bounds.argtypes = [_P, _L]
        L.orc_compute_dt.argtypes = [_P, _L, _D, _D, _D, _D, ctypes.POINTER(_D)]
        L.orc_compute_dt.restype = _D
        L.orc_boundary_energy_flux.argtypes = [_P, _I, _I, _D, _D, _I]
        L.orc_boundary_energy_flux.restype = _D
        L.orc_powell_source.argtypes = [_P, _I, _I, _D, _D, _P]
        L.orc_compute_rhs.argtypes = [_P, _I, _I, _D, _D, _D, _I, _I, _I, _D, _P, _P]
        L.orc_step_ssprk3.argtypes = [_P, _I, _I, _D, _D, _D, _I, _I, _I, _D, _D, _D, _P]
        L.orc_advance.argtypes = [_P, _I, _I, _D, _D, _D, _D, _D, _I, _I, _I, _D, _L, _P, _P]
        L.orc_advance.restype = _L
        _lib = L
    return _lib


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


# ---------------------------------------------------------------- physics.py
def cons_to_prim(U, gamma):
    """physics.py:284-301"""
    U = _f64(U)
    W = np.empty_like(U)
    lib().orc_cons_to_prim(_ptr(U), _ptr(W), U[0].size, float(gamma))
    return W


def prim_to_cons(W, gamma):
    """physics.py:304-320"""
    W = _f64(W)
    U = np.empty_like(W)
    lib().orc_prim_to_cons(_ptr(W), _ptr(U), W[0].size, float(gamma))
    return U


def muscl_x(W):
    """physics.py:323-335; returns (WL, WR) of shape [10, nx_tot-3, ny_tot]."""
    W = _f64(W)
    nv, nxt, nyt = W.shape
    WL = np.empty((nv, nxt - 3, nyt))
    WR = np.empty_like(WL)
    lib().orc_muscl_x(_ptr(W), nxt, nyt, _ptr(WL), _ptr(WR))
    return WL, WR


def muscl_y(W):
    """physics.py:338-350; returns (WL, WR) of shape [10, nx_tot, ny_tot-3]."""
    W = _f64(W)
    nv, nxt, nyt = W.shape
    WL = np.empty((nv, nxt, nyt - 3))
    WR = np.empty_like(WL)
    lib().orc_muscl_y(_ptr(W), nxt, nyt, _ptr(WL), _ptr(WR))
    return WL, WR


def _hlld(fn, WL, WR, gamma, ch):
    WL = _f64(WL)
    WR = _f64(WR)
    shape = WL.shape
    n = WL[0].size
    F = np.empty_like(WL)
    smax = np.empty(n)
    fn(_ptr(WL), _ptr(WR), _ptr(F), _ptr(smax), n, float(gamma), float(ch))
    return F.reshape(shape), float(np.max(smax)) if n else 0.0


def hlld_flux_x(WL, WR, gamma, ch):
    """physics.py:353-370 (returns (F, max smax))."""
    return _hlld(lib().orc_hlld_flux_x, WL, WR, gamma, ch)


def hlld_flux_y(WL, WR, gamma, ch):
    """physics.py:373-379"""
    return _hlld(lib().orc_hlld_flux_y, WL, WR, gamma, ch)


def hlld_face_smax(WL, WR, gamma, ch, y=False):
    """Per-face signal speeds (the kernel's smax array, physics.py:108-109)."""
    WL = _f64(WL)
    WR = _f64(WR)
    n = WL[0].size
    F = np.empty_like(WL)
    smax = np.empty(n)
    fn = lib().orc_hlld_flux_y if y else lib().orc_hlld_flux_x
    fn(_ptr(WL), _ptr(WR), _ptr(F), _ptr(smax), n, float(gamma), float(ch))
    return smax


# ------------------------------------------------------------------ config
def bc_x_code(cfg) -> int:
    """Config.get_bc_x (config.py:86-89) -> oracle code (solver.py:164-172)."""
    kind = cfg.bc_x_type if cfg.bc_x_type != "auto" else ("characteristic" if cfg.use_char_bc else "extrapolation")
    if kind == "periodic":
        return BC_PERIODIC
    if kind == "characteristic":
        return BC_CHARACTERISTIC
    return BC_EXTRAP


def bc_y_code(cfg) -> int:
    """solver.py:178-184: anything but "periodic" is zero-gradient."""
    return BC_PERIODIC if cfg.bc_y_type == "periodic" else BC_EXTRAP


def powell_enabled(cfg) -> bool:
    """solver.py:304 gate, with the optional explicit override ``powell_mode``."""
    mode = getattr(cfg, "powell_mode", "auto")
    if mode == "on":
        return True
    if mode == "off":
        return False
    return bool(cfg.powell_source and cfg.B_transverse > 0)


def _dx(cfg):
    return (cfg.x_max - cfg.x_min) / cfg.nx


def _dy(cfg):
    return (cfg.y_max - cfg.y_min) / cfg.ny


# ------------------------------------------------------------------ solver
class OracleSolver:
    """Hot-path methods of the reference MHDSolver (solver.py:72-333) on numpy."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.ng = NG
        self.nx_tot = cfg.nx + 2 * NG
        self.ny_tot = cfg.ny + 2 * NG
        self.x = cfg.x_min + (np.arange(self.nx_tot) - NG + 0.5) * _dx(cfg)
        self.y = cfg.y_min + (np.arange(self.ny_tot) - NG + 0.5) * _dy(cfg)
        self.U = np.zeros((NVAR, self.nx_tot, self.ny_tot))
        self.t = 0.0
        self.step = 0
        self.dt = 0.0
        self._glm_ch_frozen = 0.0
        self._cumulative_boundary_energy = 0.0

    # solver.py:158-197
    def apply_bc(self, U):
        assert U.dtype == np.float64 and U.flags.c_contiguous
        lib().orc_apply_bc(_ptr(U), self.nx_tot, self.ny_tot, bc_x_code(self.cfg), bc_y_code(self.cfg))
        return U

    # solver.py:199-204
    def enforce_scalar_bounds(self, U):
        assert U.dtype == np.float64 and U.flags.c_contiguous
        lib().orc_enforce_scalar_bounds(_ptr(U), U[0].size)
        return U

    # solver.py:206-223 (mutates cfg.glm_ch like the reference)
    def compute_dt(self, W):
        W = _f64(W)
        ch = _D(0.0)
        dt = lib().orc_compute_dt(_ptr(W), W[0].size, float(self.cfg.gamma), _dx(self.cfg), _dy(self.cfg),
                                  float(self.cfg.cfl), ctypes.byref(ch))
        self.cfg.glm_ch = ch.value
        return dt

    # solver.py:225-240
    def _compute_boundary_energy_flux(self, U):
        U = _f64(U)
        return lib().orc_boundary_energy_flux(_ptr(U), self.nx_tot, self.ny_tot, float(self.cfg.gamma),
                                              _dy(self.cfg), bc_x_code(self.cfg))

    # solver.py:242-266
    def _compute_powell_source(self, U, W):
        W = _f64(W)
        S = np.empty_like(W)
        lib().orc_powell_source(_ptr(W), self.nx_tot, self.ny_tot, _dx(self.cfg), _dy(self.cfg), _ptr(S))
        return S

    # solver.py:268-308 (fills U's ghosts in place, as the reference does)
    def compute_rhs(self, U):
        assert U.dtype == np.float64 and U.flags.c_contiguous
        cfg = self.cfg
        W = np.empty_like(U)
        R = np.empty_like(U)
        lib().orc_compute_rhs(_ptr(U), cfg.nx, cfg.ny, float(cfg.gamma), _dx(cfg), _dy(cfg), bc_x_code(cfg),
                              bc_y_code(cfg), int(powell_enabled(cfg)), float(self._glm_ch_frozen), _ptr(W),
                              _ptr(R))
        return R

    def psi_decay(self, dt):
        """solver.py:331-333 damping factor, evaluated exactly as the reference does."""
        cfg = self.cfg
        return np.exp(-cfg.glm_alpha * self._glm_ch_frozen * dt / min(_dx(cfg), _dy(cfg)))

    # solver.py:310-333
    def step_ssprk3(self):
        cfg = self.cfg
        dt = self.dt
        self._glm_ch_frozen = cfg.glm_ch
        U = np.ascontiguousarray(self.U, dtype=np.float64).copy()
        bflux = self._compute_boundary_energy_flux(U)
        self._cumulative_boundary_energy += bflux * dt
        decay = float(self.psi_decay(dt)) if self._glm_ch_frozen > 0 else 1.0
        work = np.empty((4,) + U.shape)
        lib().orc_step_ssprk3(_ptr(U), cfg.nx, cfg.ny, float(cfg.gamma), _dx(cfg), _dy(cfg), bc_x_code(cfg),
                              bc_y_code(cfg), int(powell_enabled(cfg)), float(dt), float(self._glm_ch_frozen),
                              decay, _ptr(work))
        self.U = U

    # main.py:66-73: the drivers' loop
    def advance(self, t_end=None, max_steps=None, on_step=None):
        cfg = self.cfg
        t_end = cfg.t_end if t_end is None else t_end
        max_steps = cfg.max_steps if max_steps is None else max_steps
        while self.t < t_end and self.step < max_steps:
            W = cons_to_prim(self.U, cfg.gamma)
            dt_cfl = self.compute_dt(W)
            self.dt = min(dt_cfl, t_end - self.t)
            if self.dt <= 1e-16:
                break
            self.step_ssprk3()
            self.t += self.dt
            self.step += 1
            if on_step is not None:
                on_step(self)
        return self

    def advance_native(self, t_end=None, max_steps=None):
        """The same loop entirely in C (decay from C's exp); for timing."""
        cfg = self.cfg
        t_end = cfg.t_end if t_end is None else t_end
        max_steps = cfg.max_steps if max_steps is None else max_steps
        U = np.ascontiguousarray(self.U, dtype=np.float64).copy()
        state = np.array([self.t, cfg.glm_ch, self._cumulative_boundary_energy])
        work = np.empty((4,) + U.shape)
        n = lib().orc_advance(_ptr(U), cfg.nx, cfg.ny, float(cfg.gamma), _dx(cfg), _dy(cfg), float(cfg.cfl),
                              float(cfg.glm_alpha), bc_x_code(cfg), bc_y_code(cfg), int(powell_enabled(cfg)),
                              float(t_end), int(max_steps - self.step), _ptr(state), _ptr(work))
        self.U = U
        self.t, cfg.glm_ch, self._cumulative_boundary_energy = float(state[0]), float(state[1]), float(state[2])
        self.step += int(n)
        return int(n)


def set_threads(n: int) -> None:
    """Set the OpenMP thread count used by liboracle.so."""
    os.environ["OMP_NUM_THREADS"] = str(n)
    try:
        omp = ctypes.CDLL("libgomp.so.1")
        omp.omp_set_num_threads(int(n))
    except OSError:
        pass


def max_threads() -> int:
    try:
        omp = ctypes.CDLL("libgomp.so.1")
        return int(omp.omp_get_max_threads())
    except OSError:
        return 1


__all__ = [
    "build", "lib", "cons_to_prim", "prim_to_cons", "muscl_x", "muscl_y", "hlld_flux_x", "hlld_flux_y",
    "OracleSolver", "bc_x_code", "bc_y_code", "powell_enabled", "set_threads", "max_threads",
]
