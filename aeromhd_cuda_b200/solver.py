"""Drop-in replacement of the reference's ``MHDSolver`` (solver.py:69-520).

Same constructor, attributes and methods; the state is a PyTorch CUDA tensor
``U[10, nx+4, ny+4]`` (a view into padded storage the fused kernels need),
and every method runs kernels of libaeromhd.so:

=====================================  ======================================
reference (solver.py)                  here
=====================================  ======================================
``apply_bc`` :158-197                  amhd_apply_bc (ghost fill, in place)
``enforce_scalar_bounds`` :199-204     amhd_enforce_scalar_bounds
``compute_dt`` :206-223                amhd_compute_dt (sets ``cfg.glm_ch``)
``_compute_boundary_energy_flux``      amhd_boundary_energy_flux
``_compute_powell_source`` :242-266    amhd_powell_source
``compute_rhs`` :268-308               amhd_compute_rhs (one fused launch)
``step_ssprk3`` :310-333               amhd_step_ssprk3 (3 fused launches)
``compute_diagnostics`` :335-444       amhd_diagnostics + host finish
``run`` :465-520                       device-resident loop (amhd_advance,
                                       replayed as a CUDA graph per chunk)
=====================================  ======================================

``precision="fp32"`` in the Config stores the state in float32 (float64
pressure recovery, CFL reduction and diagnostics); the default "fp64"
reproduces the reference's float64 results.
"""
from __future__ import annotations

import ctypes
import sys
import time

import numpy as np
import torch

from . import _lib, initial_conditions
from ._tensors import (as_cuda, control_tensor, is_padded, make_grid, padded_state, ptr, read_controls,
                       stream_ptr, torch_dtype)
from .config import (BC_PERIODIC, NVAR, Config, bc_x_code, bc_y_code, iBX, iBY, iBZ, iCLR, iPR, iRHO, iVX, iVY)
from .physics import cons_to_prim

DIAG_NAMES = ("mass", "energy", "divB_max", "divB_L2", "mixing_width_integral", "stag_pressure", "enstrophy")


def to_numpy(a):
    """Tensor (any device) or array -> numpy (solver.py:59-63)."""
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


class MHDSolver:
    """2-D ideal MHD solver: HLLD, MUSCL, SSP-RK3, GLM + Powell, on sm_100a."""

    def __init__(self, config: Config):
        if not torch.cuda.is_available():
            raise RuntimeError("MHDSolver needs a CUDA device; libaeromhd has no CPU path")
        config.validate()
        _lib.call("amhd_init")
        self.cfg = config
        self.ng = 2
        self.nx_tot = config.nx + 2 * self.ng
        self.ny_tot = config.ny + 2 * self.ng
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.dtype = torch_dtype(config.precision)

        self.x = torch.as_tensor(config.x_min + (np.arange(self.nx_tot) - self.ng + 0.5) * config.dx,
                                 device=self.device)
        self.y = torch.as_tensor(config.y_min + (np.arange(self.ny_tot) - self.ng + 0.5) * config.dy,
                                 device=self.device)
        self.X, self.Y = torch.meshgrid(self.x, self.y, indexing="ij")

        self._store, self._U = padded_state(config.nx, config.ny, self.dtype, self.device)
        self._store1, self._U1 = padded_state(config.nx, config.ny, self.dtype, self.device)
        self._store2, self._U2 = padded_state(config.nx, config.ny, self.dtype, self.device)
        self._ctl = control_tensor(1, self.device)
        # float32 run loop with compensation: low part of the base state (zero at every loop start)
        self._compensated = config.precision == "fp32" and bool(config.fp32_compensation)
        self._store_lo, self._U_lo = (padded_state(config.nx, config.ny, self.dtype, self.device)
                                      if self._compensated else (None, None))
        self._diag_out = torch.zeros(8, dtype=torch.float64, device=self.device)
        self._diag_rows = torch.zeros(7 * config.nx, dtype=torch.float64, device=self.device)
        self._diag_colour = torch.zeros(config.nx + config.ny, dtype=torch.float64, device=self.device)
        self._graphs = {}
        self._loop_ready = False

        self.t = 0.0
        self.step = 0
        self.dt = 0.0
        self._glm_ch_frozen = 0.0

        self.diag_times = []
        self.diag_mixing_width_integral = []
        self.diag_mixing_width_thresh = []
        self.diag_mixedness = []
        self.diag_enstrophy = []
        self.diag_enstrophy_local = []
        self.diag_perturbation_amp = []
        self.diag_mode_amps = []
        self.diag_stag_pressure = []
        self.diag_divB_max = []
        self.diag_divB_L2 = []
        self.diag_energy_total = []
        self.diag_mass_total = []
        self.diag_boundary_flux_cumulative = []
        self._ebnd_host = 0.0
        self.snapshots = {}
        self._rho_light = 1.0
        self._rho_heavy = 1.0
        self._rh_results = None

    # ------------------------------------------------------------------ state
    @property
    def U(self) -> torch.Tensor:
        return self._U

    @U.setter
    def U(self, value):
        v = as_cuda(value)
        if tuple(v.shape) != (NVAR, self.nx_tot, self.ny_tot):
            raise ValueError(f"U must have shape {(NVAR, self.nx_tot, self.ny_tot)}, got {tuple(v.shape)}")
        if v.data_ptr() != self._U.data_ptr():
            self._U.copy_(v.to(self.dtype))
        self._loop_ready = False

    @property
    def _cumulative_boundary_energy(self) -> float:
        return self._ebnd_host + float(read_controls(self._ctl)[0].e_bnd)

    @_cumulative_boundary_energy.setter
    def _cumulative_boundary_energy(self, value):
        self._ebnd_host = float(value)
        self._ctl.zero_()
        self._loop_ready = False

    def _grid(self, state: torch.Tensor | None = None) -> _lib.Grid:
        cfg = self.cfg
        return make_grid(self._U if state is None else state, cfg.gamma, cfg.dx, cfg.dy, cfg.cfl, cfg.glm_alpha,
                         bc_x_code(cfg), bc_y_code(cfg), cfg.powell_enabled(), _lib.LIMITER_CODES[cfg.limiter])

    def set_primitive(self, W):
        """Load primitive variables W[10, nx+4, ny+4] (prim_to_cons on the GPU)."""
        from .physics import prim_to_cons
        self.U = prim_to_cons(as_cuda(W, torch.float64), self.cfg.gamma)

    # ------------------------------------------------------------- set-up
    def initialize(self):
        """Shocked gas + perturbed density interface (solver.py:109-156)."""
        cfg = self.cfg
        if cfg.ic == "shock_interface":
            W, rh = initial_conditions.shock_interface(self)
        else:
            W, rh = initial_conditions.rmi(self)
        self._rh_results = rh
        self.set_primitive(W)
        self.t = 0.0
        self.step = 0
        self._cumulative_boundary_energy = 0.0
        self._rho_light = 1.0
        self._rho_heavy = 1.0 * cfg.density_ratio
        print(f"  Mach={cfg.mach:.1f}, Vs={rh['vs']:.3f}, rho2={rh['rho2']:.3f}, p2={rh['p2']:.3f}, "
              f"vx2={rh['vx2']:.3f}")
        print(f"  Grid: {cfg.nx}x{cfg.ny}, dx={cfg.dx:.4f}, precision={cfg.precision}, "
              f"BC x: {cfg.get_bc_x()}, BC y: {cfg.bc_y_type}, Powell: {cfg.powell_enabled()}")
        sys.stdout.flush()

    # --------------------------------------------------------- hot methods
    def apply_bc(self, U):
        """Ghost cells from the interior, in place (solver.py:158-197)."""
        U = as_cuda(U)
        _lib.call("amhd_apply_bc", self._grid(U), ptr(U), stream_ptr())
        if U.data_ptr() == self._U.data_ptr():
            self._loop_ready = False
        return U

    def enforce_scalar_bounds(self, U):
        """rho*C <- rho * clip(C, 0, 1) on every cell (solver.py:199-204)."""
        U = as_cuda(U)
        _lib.call("amhd_enforce_scalar_bounds", self._grid(U), ptr(U), stream_ptr())
        return U

    def compute_dt(self, W):
        """CFL time step from primitives W; sets cfg.glm_ch (solver.py:206-223)."""
        W = as_cuda(W)
        dt, ch = ctypes.c_double(), ctypes.c_double()
        _lib.call("amhd_compute_dt", self._grid(W), ptr(W), ptr(self._ctl), ctypes.byref(dt), ctypes.byref(ch),
                  stream_ptr())
        self.cfg.glm_ch = ch.value
        return dt.value

    def _compute_boundary_energy_flux(self, U):
        """Net x-boundary energy flux (solver.py:225-240)."""
        U = as_cuda(U)
        out = ctypes.c_double()
        _lib.call("amhd_boundary_energy_flux", self._grid(U), ptr(U), ptr(self._ctl), ctypes.byref(out),
                  stream_ptr())
        return out.value

    def _compute_powell_source(self, U, W):
        """Powell 8-wave source from primitives (solver.py:242-266)."""
        W = as_cuda(W)
        S = torch.empty_strided(W.size(), W.stride(), dtype=W.dtype, device=W.device)
        _lib.call("amhd_powell_source", self._grid(W), ptr(W), ptr(S), stream_ptr())
        return S

    def compute_rhs(self, U):
        """-div F (+ Powell) on the interior; fills U's ghosts in place (solver.py:268-308)."""
        U = as_cuda(U)
        if is_padded(U):
            work = U
        else:
            _, work = padded_state(self.cfg.nx, self.cfg.ny, U.dtype, self.device)
            work.copy_(U)
        _, R = padded_state(self.cfg.nx, self.cfg.ny, U.dtype, self.device)
        _lib.call("amhd_compute_rhs", self._grid(work), ptr(work), ptr(R), float(self._glm_ch_frozen), stream_ptr())
        if work is not U:
            U.copy_(work)
        return R

    def psi_decay(self, dt):
        cfg = self.cfg
        return float(np.exp(-cfg.glm_alpha * self._glm_ch_frozen * dt / min(cfg.dx, cfg.dy)))

    def step_ssprk3(self):
        """One SSP-RK3 step with self.dt and the frozen cfg.glm_ch (solver.py:310-333)."""
        dt = float(self.dt)
        self._glm_ch_frozen = self.cfg.glm_ch
        ch = float(self._glm_ch_frozen)
        decay = self.psi_decay(dt) if ch > 0 else 1.0
        _lib.call("amhd_step_ssprk3", self._grid(), ptr(self._U), ptr(self._U1), ptr(self._U2), dt, ch, decay,
                  ptr(self._ctl), stream_ptr())
        self._loop_ready = False

    # --------------------------------------------------------- diagnostics
    def device_diagnostics(self) -> dict:
        """float64 conserved-quantity diagnostics computed on the GPU."""
        cfg = self.cfg
        _lib.call("amhd_diagnostics", self._grid(), ptr(self._U), float(cfg.x_min), ptr(self._diag_out),
                  ptr(self._diag_rows), stream_ptr())
        vals = self._diag_out.cpu().numpy()
        return dict(zip(DIAG_NAMES, (float(v) for v in vals[:7])))

    def compute_diagnostics(self):
        """solver.py:335-444.  Every pass over the field runs on the GPU (sums,
        maxima, integral mixing width, per-row colour variance, per-column
        interface positions); the host finishes from nx + ny + 7 nx numbers."""
        cfg = self.cfg
        ng = self.ng
        d = self.device_diagnostics()
        nx_int, ny_int = cfg.nx, cfg.ny
        col = self._diag_colour
        _lib.call("amhd_diagnostics_colour", self._grid(), ptr(self._U), float(cfg.x_min), ptr(self._diag_rows),
                  ptr(col), ptr(col[nx_int:]), stream_ptr())
        rows = self._diag_rows.view(7, cfg.nx).cpu().numpy()
        colour = col.cpu().numpy()
        x_arr = to_numpy(self.x[ng:-ng])
        y_arr = to_numpy(self.y[ng:-ng])
        C_bar = rows[0] / ny_int

        mixed = np.where((C_bar > 0.01) & (C_bar < 0.99))[0]
        mw_thresh = float(x_arr[mixed[-1]] - x_arr[mixed[0]]) if len(mixed) > 1 else 0.0
        C_prime_sq = colour[:nx_int] / ny_int
        denom_mix = np.maximum(C_bar * (1.0 - C_bar), 1e-14)
        if len(mixed) > 1:
            num = float(np.trapezoid(C_prime_sq[mixed], x_arr[mixed]))
            den = float(np.trapezoid(denom_mix[mixed], x_arr[mixed]))
            mixedness = float(np.clip(1.0 - num / max(den, 1e-14), 0.0, 1.0))
        else:
            mixedness = 0.0

        # interface position per column: gradient-weighted centroid around the peak
        interface_pos = colour[nx_int:]
        valid = ~np.isnan(interface_pos)
        n_valid = int(np.sum(valid))
        if n_valid > ny_int // 2:
            pos = interface_pos[valid]
            pos_i = np.interp(y_arr, y_arr[valid], pos) if n_valid < ny_int else pos
            modes = np.fft.rfft(pos_i - np.mean(pos_i))
            mode_amps = 2.0 * np.abs(modes) / ny_int
            pert_amp = float(mode_amps[cfg.perturbation_mode]) if cfg.perturbation_mode < len(mode_amps) else 0.0
        else:
            mode_amps = np.zeros(ny_int // 2 + 1)
            pert_amp = 0.0

        enst = d["enstrophy"]
        enst_local = enst
        if n_valid > ny_int // 2:
            xc = float(np.mean(interface_pos[valid]))
            lo = max(np.searchsorted(x_arr, xc - 0.5), 0)
            hi = min(np.searchsorted(x_arr, xc + 0.5), nx_int)
            if hi - lo > 3:
                enst_local = float(np.sum(rows[4, lo:hi]) / ((hi - lo) * ny_int))

        self.diag_times.append(self.t)
        self.diag_mixing_width_integral.append(d["mixing_width_integral"])
        self.diag_mixing_width_thresh.append(mw_thresh)
        self.diag_mixedness.append(mixedness)
        self.diag_enstrophy.append(enst)
        self.diag_enstrophy_local.append(enst_local)
        self.diag_perturbation_amp.append(pert_amp)
        self.diag_mode_amps.append(mode_amps.copy())
        self.diag_stag_pressure.append(d["stag_pressure"])
        self.diag_divB_max.append(d["divB_max"])
        self.diag_divB_L2.append(d["divB_L2"])
        self.diag_energy_total.append(d["energy"])
        self.diag_mass_total.append(d["mass"])
        self.diag_boundary_flux_cumulative.append(self._cumulative_boundary_energy)

    def save_snapshot(self, label=None):
        """Primitive interior fields to host memory (solver.py:446-463)."""
        ng = self.ng
        W = cons_to_prim(self._U, self.cfg.gamma)
        key = label or f"t={self.t:.4f}"
        names = {"rho": iRHO, "p": iPR, "vx": iVX, "vy": iVY, "Bx": iBX, "By": iBY, "Bz": iBZ, "C": iCLR}
        snap = {k: to_numpy(W[v, ng:-ng, ng:-ng]) for k, v in names.items()}
        snap.update(t=self.t, x=to_numpy(self.x[ng:-ng]), y=to_numpy(self.y[ng:-ng]))
        self.snapshots[key] = snap

    # ------------------------------------------------------ device run loop
    def _loop_init(self, t_end: float, max_steps: int):
        """amhd_control_init: dt/ch of the current state, exactly as the loop head computes them."""
        self._ebnd_host = self._cumulative_boundary_energy
        if self._compensated:
            self._store_lo.zero_()  # U as given is exactly its float32 values
        _lib.call("amhd_control_init", self._grid(), ptr(self._U), ptr(self._ctl), float(self.t), float(t_end),
                  int(self.step), int(max_steps), stream_ptr())
        self._loop_ready = True

    def _advance_eager(self, n: int):
        if self._compensated:
            _lib.call("amhd_advance_compensated", self._grid(), ptr(self._U), ptr(self._U_lo), ptr(self._U1),
                      ptr(self._U2), ptr(self._ctl), int(n), stream_ptr())
        else:
            _lib.call("amhd_advance", self._grid(), ptr(self._U), ptr(self._U1), ptr(self._U2), ptr(self._ctl),
                      int(n), stream_ptr())

    def _advance(self, n: int, graph: bool = True):
        """n device-loop iterations: as a CUDA graph replay (captured on first use) or eagerly."""
        if not graph:
            self._advance_eager(n)
            return
        g = self._graphs.get(n)
        if g is None:
            self._advance_eager(0)  # argument checks outside capture
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._advance_eager(n)
            self._graphs[n] = g
        g.replay()

    def _read_loop_state(self):
        c = read_controls(self._ctl)[0]
        self.t = float(c.t)
        self.step = int(c.step)
        if c.step > 0 and c.last_dt > 0:
            self.dt = float(c.last_dt)
        self.cfg.glm_ch = float(c.ch)
        self._glm_ch_frozen = float(c.ch)
        return c

    def advance(self, t_end=None, max_steps=None, chunk: int = 64, graph: bool = True):
        """The drivers' loop (main.py:66-73) on the device: steps until t >= t_end,
        step >= max_steps or dt <= 1e-16, reading back only once per chunk."""
        cfg = self.cfg
        t_end = cfg.t_end if t_end is None else float(t_end)
        max_steps = cfg.max_steps if max_steps is None else int(max_steps)
        self._loop_init(t_end, max_steps)
        while True:
            self._advance(chunk, graph)
            c = self._read_loop_state()
            _lib.check_control(c, "MHDSolver.advance")
            if not c.active:
                break
        self._loop_ready = False
        return self

    def run(self):
        """solver.py:465-520 with the step loop resident on the GPU."""
        cfg = self.cfg
        print(f"\n--- Running (B200): B_y = {cfg.B_transverse}, precision={cfg.precision} ---")
        sys.stdout.flush()
        t0 = time.time()
        self.compute_diagnostics()
        self.save_snapshot(label="initial")
        if not (self.t < cfg.t_end and self.step < cfg.max_steps):
            self._finish_run(t0)
            return
        self._loop_init(cfg.t_end, cfg.max_steps)
        self._set_next_snapshot()
        while True:
            n = min(cfg.diag_interval - self.step % cfg.diag_interval, 200 - self.step % 200)
            self._advance(n)
            c = self._read_loop_state()
            _lib.check_control(c, "MHDSolver.run")
            if self.step % cfg.diag_interval == 0:
                self.compute_diagnostics()
            for st in cfg.snapshot_times:
                lbl = f"t~{st:.2f}"
                if abs(self.t - st) < 1.5 * self.dt and lbl not in self.snapshots:
                    self.save_snapshot(label=lbl)
            if self.step % 200 == 0:
                mwi = self.diag_mixing_width_integral[-1] if self.diag_mixing_width_integral else 0
                print(f"  Step {self.step:5d}  t={self.t:.4f}  dt={self.dt:.2e}  MW={mwi:.4f}  "
                      f"divB={self.diag_divB_max[-1] if self.diag_divB_max else 0:.1f}  "
                      f"E={self.diag_energy_total[-1] if self.diag_energy_total else 0:.2f}")
                sys.stdout.flush()
            if not c.active and not (c.flags & _lib.AMHD_FLAG_PAUSED):
                break
            self._set_next_snapshot()
        self._loop_ready = False
        self._finish_run(t0)

    def _set_next_snapshot(self):
        pending = [st for st in self.cfg.snapshot_times if f"t~{st:.2f}" not in self.snapshots]
        nxt = min(pending) if pending else float("inf")
        _lib.call("amhd_control_resume", ptr(self._ctl), 1, float(nxt), stream_ptr())

    def _finish_run(self, t0):
        self.compute_diagnostics()
        self.save_snapshot(label="final")
        elapsed = time.time() - t0
        if len(self.diag_energy_total) >= 2:
            e0, ef = self.diag_energy_total[0], self.diag_energy_total[-1]
            bf = self._cumulative_boundary_energy
            de_raw = abs(ef - e0) / max(abs(e0), 1e-14) * 100
            de_corr = abs(ef - bf - e0) / max(abs(e0), 1e-14) * 100
            print(f"  Energy drift: raw={de_raw:.2f}%, corrected={de_corr:.2f}%")
            print(f"  Boundary flux: {bf:.2f}")
        if self.diag_divB_max:
            print(f"  Final max|divB|: {self.diag_divB_max[-1]:.2f}, L2|divB|: {self.diag_divB_L2[-1]:.4f}")
        print(f"  Done: {self.step} steps, {elapsed:.1f}s")
        sys.stdout.flush()


__all__ = ["MHDSolver", "to_numpy", "BC_PERIODIC"]
