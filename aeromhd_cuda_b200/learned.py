"""Training data, training and evaluation of the learned coarse-grid corrector.

    python -m aeromhd_cuda_b200.learned --train-seeds 100 --test-seeds 64

Data: shocked-interface runs drawn like the batched ensemble (Mach, density
ratio, mode, amplitude, field), each on a coarse (nx x ny) and a 4x finer
grid, as GPU ensembles.  The corrector learns the error the coarse solver
makes over one correction interval `delta` starting from a good state: at
every start time t_k (0, 0.1, ... 2.9) the fine state is restricted onto the
coarse grid (4x4 block averages), the coarse solver advances it by delta, and
the pair (that coarse state, the fine state at t_k + delta restricted) is
kept; the target is their difference.  Runs use the frame of the shocked gas
so that the mixing layer stays in the domain until t = 3.  Seeds split 90/10
into training and validation; separate test seeds measure the result.

Use: a corrected coarse run adds the corrector's output every `delta` of
simulated time (all instances of an ensemble together).  It is measured
against the plain fine solve on mixing width, spectral energy and div B; an
instance falls back to the plain fine solve when its corrected run leaves the
trusted range (non-finite or far out-of-range corrections, a correction that
collapses the time step, a step count far above the plain coarse run's, div B
above a tolerance).

No counterpart in the reference.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from dataclasses import replace
from typing import List, Sequence

import numpy as np
import torch

from . import _lib
from ._tensors import ptr, stream_ptr, write_controls
from .corrector import Corrector
from .ensemble import Ensemble, draw_configs

T_SNAPS = tuple(round(0.1 * k, 10) for k in range(1, 31))   # evaluation snapshot times
T_STARTS = tuple(round(0.1 * k, 10) for k in range(0, 30))   # training start times
DELTA = 0.02                                                 # correction interval (5 per snapshot interval)


def paired_configs(seeds: Sequence[int], nyc: int = 64, factor: int = 4, precision: str = "fp32"):
    """Coarse (4 ny x ny) and fine (factor x) configurations of the same parameter draws."""
    coarse = []
    for s in seeds:
        c = draw_configs(1, seed=int(s), t_end=3.0, precision=precision, ny_choices=(nyc,), noise_amp=0.0)[0]
        coarse.append(replace(c, interface_x=3.0, shock_x=2.5, ic_frame="post_shock", seed=int(s)))
    fine = [replace(c, nx=c.nx * factor, ny=c.ny * factor) for c in coarse]
    return coarse, fine


def _interior(ens: Ensemble, k: int) -> torch.Tensor:
    return ens.state(k)[:, 2:-2, 2:-2]


def _load_restricted(ef: Ensemble, ec: Ensemble, factor: int, buf: torch.Tensor) -> None:
    """Every coarse instance := its fine instance restricted (interior) + boundary conditions."""
    for i in range(ec.n):
        c = ec.configs[i]
        _lib.call("amhd_nn_restrict", ef._grid(i), ptr(ef.state(i)), factor, ptr(buf), c.nx * c.ny, 0, 1,
                  stream_ptr())
        _interior(ec, i).copy_(buf.view(10, c.nx, c.ny))
        _lib.call("amhd_apply_bc", ec._grid(i), ptr(ec.state(i)), stream_ptr())


def _timed_run(e: Ensemble, wall: dict, key: str) -> None:
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e.run(chunk=64)
    torch.cuda.synchronize()
    wall[key] += time.perf_counter() - t0


def generate_pairs(seeds: Sequence[int], t_starts: Sequence[float] = T_STARTS, delta: float = DELTA, nyc: int = 64,
                   factor: int = 4, precision: str = "fp32", log=print):
    """Returns (X, Y, wall): X[k][seed] = the coarse state after `delta` of coarse
    evolution from the fine state at t_starts[k] restricted; Y[k][seed] = the fine
    state at t_starts[k] + delta restricted (interiors, float32)."""
    coarse, fine = paired_configs(seeds, nyc, factor, precision)
    ec, ef = Ensemble(coarse), Ensemble(fine)
    ef.initialize()
    nxc, nyc_ = coarse[0].nx, coarse[0].ny
    n = len(seeds)
    X = torch.empty((len(t_starts), n, 10, nxc, nyc_), dtype=torch.float32, device=ec.device)
    Y = torch.empty_like(X)
    buf = torch.empty((10, nxc * nyc_), dtype=torch.float32, device=ec.device)
    wall = {"coarse": 0.0, "fine": 0.0}
    ef.start(t_end=t_starts[0])
    zeros = [0] * n
    for k, ts in enumerate(t_starts):
        if k:
            ef.continue_to(ts)
            _timed_run(ef, wall, "fine")
        _load_restricted(ef, ec, factor, buf)
        ec.resume([ts] * n, zeros, [0.0] * n, ts + delta)
        _timed_run(ec, wall, "coarse")
        ef.continue_to(ts + delta)
        _timed_run(ef, wall, "fine")
        for i in range(n):
            X[k, i].copy_(_interior(ec, i))
            _lib.call("amhd_nn_restrict", ef._grid(i), ptr(ef.state(i)), factor, ptr(Y[k, i]), nxc * nyc_, 0, 1,
                      stream_ptr())
        if log and (k % 5 == 4 or k == len(t_starts) - 1):
            log(f"  pairs from t={ts:.1f}: {n} seeds, wall coarse {wall['coarse']:.1f}s fine {wall['fine']:.1f}s")
    return X, Y, wall


class Normaliser:
    def __init__(self, X: torch.Tensor, T: torch.Tensor):
        xs = X.transpose(0, 1).reshape(10, -1) if X.dim() == 4 else X.permute(2, 0, 1, 3, 4).reshape(10, -1)
        ts = T.transpose(0, 1).reshape(10, -1) if T.dim() == 4 else T.permute(2, 0, 1, 3, 4).reshape(10, -1)
        self.in_mean = xs.mean(1)
        self.in_std = xs.std(1).clamp_min(1e-6)
        tstd = ts.std(1)
        # channels the fine solution never corrects (e.g. m_z, B_z of these runs) get no correction
        self.active = tstd > 1e-7 * tstd.max().clamp_min(1e-30)
        self.out_std = torch.where(self.active, tstd, torch.ones_like(tstd))
        self.out_max = (ts.abs().amax(1) / self.out_std).clamp_min(1.0)

    @property
    def out_scale(self) -> torch.Tensor:
        return torch.where(self.active, self.out_std, torch.zeros_like(self.out_std))

    def inputs(self, X: torch.Tensor) -> torch.Tensor:
        """[S][10][H][W] -> normalised [10][S*H*W]"""
        x = (X - self.in_mean.view(1, 10, 1, 1)) / self.in_std.view(1, 10, 1, 1)
        return x.transpose(0, 1).reshape(10, -1).contiguous()

    def targets(self, T: torch.Tensor) -> torch.Tensor:
        t = T / self.out_std.view(1, 10, 1, 1)
        return t.transpose(0, 1).reshape(10, -1).contiguous()


def project_rows(T: torch.Tensor) -> torch.Tensor:
    """The mean over y (the last axis) of every x-row, broadcast back: the part of
    a correction that moves the row averages -- the mixing width and the other
    integral diagnostics are functions of those -- without the small-scale part
    in which the coarse and fine runs of a chaotic layer decorrelate."""
    return T.mean(dim=-1, keepdim=True).expand_as(T)


def train(X: torch.Tensor, Y: torch.Tensor, train_seeds: Sequence[int], val_seeds: Sequence[int], epochs: int = 20,
          batch: int = 16, lr: float = 1e-3, seed: int = 0, net: Corrector | None = None,
          norm: "Normaliser | None" = None, project_y: bool = False, log=print):
    """X, Y: [snap][seed][10][H][W]; seeds index the second axis.  Returns (net, norm, history).
    Given net and norm, continues training that network with its normalisation.
    project_y: the targets are the row averages of the corrections (project_rows),
    and so are the corrections the network applies (net.project_y)."""
    H, W = X.shape[-2], X.shape[-1]
    project_y = project_y or bool(getattr(net, "project_y", False))
    T = Y - X
    if project_y:
        T = project_rows(T)
    tr = X[:, list(train_seeds)].reshape(-1, 10, H, W)
    ttr = T[:, list(train_seeds)].reshape(-1, 10, H, W)
    va = X[:, list(val_seeds)].reshape(-1, 10, H, W)
    tva = T[:, list(val_seeds)].reshape(-1, 10, H, W)
    if net is None:
        norm = Normaliser(tr, ttr)
        net = Corrector(H, W, seed=seed, device=X.device)
        net.set_normalisation(norm.in_mean, norm.in_std, norm.out_scale)
        net.project_y = bool(project_y)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    hist = {"epoch": [], "train_loss": [], "val_loss": [], "wall_s": []}
    n = tr.shape[0]
    t0 = time.perf_counter()
    sched = lambda e: lr * 0.5 * (1 + math.cos(math.pi * e / max(epochs, 1)))  # cosine decay
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen)
        losses = []
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch].to(X.device)
            x = norm.inputs(tr[idx])
            t = norm.targets(ttr[idx])
            losses.append(net.train_step_graphed(x, t, batch, lr=sched(ep)))
        net.check_gemm_status()  # once per epoch: a GEMM that gave up invalidates the epoch
        tl = float(torch.stack([l.reshape(()) for l in losses]).mean()) if losses else float("nan")
        vl = []
        for b0 in range(0, va.shape[0], batch):
            xb, tb = va[b0:b0 + batch], tva[b0:b0 + batch]
            vl.append(net.loss(norm.inputs(xb), norm.targets(tb), xb.shape[0]) * xb.shape[0])
        vloss = float(sum(vl) / max(va.shape[0], 1))
        hist["epoch"].append(ep)
        hist["train_loss"].append(tl)
        hist["val_loss"].append(vloss)
        hist["wall_s"].append(time.perf_counter() - t0)
        if log:
            log(f"  epoch {ep:3d}  train {tl:.4e}  val {vloss:.4e}  ({time.perf_counter() - t0:.1f}s)")
    # baseline: the loss of predicting no correction
    hist["val_loss_zero_correction"] = float(norm.targets(tva).pow(2).mean())
    return net, norm, hist


def rollout_pairs(net: Corrector, norm: "Normaliser", seeds: Sequence[int], delta: float = DELTA, t_end: float = 3.0,
                  alpha: float = 1.0, scalar_mode: int = 3, every: int = 3, nyc: int = 64, factor: int = 4,
                  precision: str = "fp32", log=print):
    """Pairs from the corrector's own runs (to correct the drift it causes): a
    corrected coarse run and the fine run of each seed advance together from the
    same restricted initial state; at every `every`-th correction time the pair
    (corrected-run state before its correction, fine state restricted) is kept.
    Returns (X, Y) shaped like generate_pairs'."""
    coarse, fine = paired_configs(seeds, nyc, factor, precision)
    ef, ec = Ensemble(fine), Ensemble(coarse)
    ef.initialize()
    nxc, nyc_ = coarse[0].nx, coarse[0].ny
    buf = torch.empty((10, nxc * nyc_), dtype=torch.float32, device=ec.device)
    _load_restricted(ef, ec, factor, buf)
    n = len(seeds)
    m_total = int(round(t_end / delta))
    keep = [q for q in range(1, m_total + 1) if q % every == 0]
    X = torch.empty((len(keep), n, 10, nxc, nyc_), dtype=torch.float32, device=ec.device)
    Y = torch.empty_like(X)
    ef.start(t_end=delta)
    ec.start(t_end=delta)
    idx = np.arange(n)
    j = 0
    for q in range(1, m_total + 1):
        tc = q * delta
        ef.continue_to(tc)
        ef.run(chunk=64)
        ec.continue_to(tc)
        ec.run(chunk=32)
        if q % every == 0:
            for i in range(n):
                X[j, i].copy_(_interior(ec, i))
                _lib.call("amhd_nn_restrict", ef._grid(i), ptr(ef.state(i)), factor, ptr(Y[j, i]), nxc * nyc_, 0, 1,
                          stream_ptr())
            j += 1
        _apply_batch(net, norm, ec, idx, 8.0, alpha, 0.5, None, scalar_mode)
        if log and q % 30 == 0:
            log(f"  rollout pairs to t={tc:.2f}")
    return X, Y


def prolong_linear(Uc: torch.Tensor, factor: int) -> torch.Tensor:
    """Coarse interior [10][nx][ny] -> fine interior [10][f nx][f ny]: in every
    coarse cell a linear profile with minmod-limited slopes in x (one-sided at
    the two ends) and y (periodic); the sub-cell offsets average to zero, so
    each coarse cell's mean -- mass, momentum, energy, field -- is kept."""
    U = Uc.double()

    def minmod(a, b):
        return torch.where(a * b > 0, torch.sign(a) * torch.minimum(a.abs(), b.abs()), torch.zeros_like(a))

    sx = minmod(U - torch.cat([U[:, :1], U[:, :-1]], 1), torch.cat([U[:, 1:], U[:, -1:]], 1) - U)
    sy = minmod(U - U.roll(1, 2), U.roll(-1, 2) - U)
    off = (torch.arange(factor, dtype=torch.float64, device=U.device) + 0.5) / factor - 0.5
    f = (U[:, :, None, :, None] + sx[:, :, None, :, None] * off.view(1, 1, -1, 1, 1)
         + sy[:, :, None, :, None] * off.view(1, 1, 1, 1, -1))
    nx, ny = U.shape[1], U.shape[2]
    return f.reshape(10, nx * factor, ny * factor).to(Uc.dtype)


def closure_pairs(net: Corrector, norm: "Normaliser", seeds: Sequence[int], delta: float = DELTA,
                  t_end: float = 3.0, alpha: float = 1.0, scalar_mode: int = 3, every: int = 3, nyc: int = 64,
                  factor: int = 4, precision: str = "fp32", log=print):
    """Pairs along the corrector's own runs with targets consistent with them: at
    every `every`-th correction time the corrected coarse state is prolonged onto
    the fine grid (prolong_linear), the fine solver advances it by `delta` and the
    result is restricted; the coarse solver advances the same state by `delta`.
    The pair (coarse result, restricted fine result) is what the fine solver
    would have added over that interval from where the corrected run actually
    is -- a closure target -- instead of the distance to a fine trajectory the
    chaotic run has decorrelated from.  Returns (X, Y) shaped like
    generate_pairs'."""
    coarse, fine = paired_configs(seeds, nyc, factor, precision)
    ef, ec = Ensemble(fine), Ensemble(coarse)
    ef.initialize()
    nxc, nyc_ = coarse[0].nx, coarse[0].ny
    buf = torch.empty((10, nxc * nyc_), dtype=torch.float32, device=ec.device)
    _load_restricted(ef, ec, factor, buf)
    n = len(seeds)
    m_total = int(round(t_end / delta))
    keep = [q for q in range(1, m_total + 1) if q % every == 0]
    X = torch.empty((len(keep), n, 10, nxc, nyc_), dtype=torch.float32, device=ec.device)
    Y = torch.empty_like(X)
    ec.start(t_end=delta)
    idx = np.arange(n)
    zeros = [0] * n
    j = 0
    for q in range(1, m_total + 1):
        tc = q * delta
        if q % every == 0:
            for i in range(n):
                _interior(ef, i).copy_(prolong_linear(_interior(ec, i), factor))
                _lib.call("amhd_apply_bc", ef._grid(i), ptr(ef.state(i)), stream_ptr())
            ef.resume([tc - delta] * n, zeros, [0.0] * n, tc)
            ef.run(chunk=64)
            for i in range(n):
                _lib.call("amhd_nn_restrict", ef._grid(i), ptr(ef.state(i)), factor, ptr(Y[j, i]), nxc * nyc_, 0, 1,
                          stream_ptr())
        ec.continue_to(tc)
        ec.run(chunk=32)
        if q % every == 0:
            for i in range(n):
                X[j, i].copy_(_interior(ec, i))
            j += 1
        _apply_batch(net, norm, ec, idx, 8.0, alpha, 0.5, None, scalar_mode)
        if log and q % 30 == 0:
            log(f"  closure pairs to t={tc:.2f}")
    return X, Y


def _mixing_width(ens: Ensemble, k: int) -> float:
    c = ens.configs[k]
    out = torch.zeros(8, dtype=torch.float64, device=ens.device)
    rows = torch.zeros(7 * c.nx, dtype=torch.float64, device=ens.device)
    st = ens.state(k)
    _lib.call("amhd_diagnostics", ens._grid(k), ptr(st), float(c.x_min), ptr(out), ptr(rows), stream_ptr())
    v = out.cpu().numpy()
    return float(v[4]), float(v[3])   # integral mixing width, divB L2


def _ke_spectrum(U: torch.Tensor) -> torch.Tensor:
    """y-direction kinetic-energy spectrum, summed over x: sum_x |FFT_y(m / sqrt(rho))|^2 over mx, my, mz."""
    rho = U[0].double().clamp_min(1e-12)
    s = 0
    for v in (1, 2, 3):
        f = torch.fft.rfft(U[v].double() / rho.sqrt(), dim=1)
        s = s + (f.abs() ** 2).sum(0)
    return s


def _set_limits(e: Ensemble, cap: np.ndarray, stop: np.ndarray) -> None:
    """Per-instance step cap for the current interval; instances in `stop` are halted."""
    ctl = e.controls()
    for i, c in enumerate(ctl):
        if stop[i]:
            c.max_steps = int(c.step)
            c.active = 0
        else:
            c.max_steps = int(cap[i])
    write_controls(e.ctl, ctl)


def evaluate(net: Corrector, norm: Normaliser, seeds: Sequence[int], delta: float = DELTA, nyc: int = 64,
             factor: int = 4, t_snaps: Sequence[float] = T_SNAPS, divb_tol: float = 1.0, corr_sigma: float = 8.0,
             step_factor: float = 3.0, dt_drop: float = 0.5, max_wall: float = 900.0, alpha: float = 1.0,
             min_ratio: float = 0.5, scalar_mode: int = 1, runs_in=None, log=print) -> dict:
    """Fine, coarse and corrected runs of the held-out seeds to every snapshot
    time.  The corrected run adds the correction every `delta` of simulated
    time; an instance falls back (stops; its plain fine solve stands in) when
    a correction is non-finite or far outside the training range, when it makes
    the next dt drop below dt_drop x its value before the correction, or when
    the instance needs more than step_factor x the plain coarse run's steps
    between two snapshots.  max_wall bounds the corrected run's wall time.
    alpha scales the corrections; cells a correction would leave with less than
    min_ratio of their density or pressure are not corrected; scalar_mode: how
    the passive scalar is corrected (amhd_nn_apply_guarded).  runs_in: the
    fine and coarse results of an earlier call on the same seeds (reused)."""
    coarse, fine = paired_configs(seeds, nyc, factor)
    n = len(seeds)
    runs = {}
    walls = {}
    names = ("fine", "fine_restricted", "coarse", "corrected")
    mw = {name: np.zeros((len(t_snaps), n)) for name in names}
    divb = {name: np.zeros((len(t_snaps), n)) for name in names}
    coarse_steps = np.zeros((len(t_snaps), n), dtype=np.int64)
    fallback = np.zeros(n, dtype=bool)
    nxc, nycc = coarse[0].nx, coarse[0].ny
    buf = torch.empty((10, nxc * nycc), dtype=torch.float32, device="cuda")
    scratch = Ensemble(coarse)   # restricted fine states, for the coarse-grid reference values
    reasons = {"range": 0, "dt_drop": 0, "steps": 0, "wall": 0, "divB": 0}
    n_corr = 0
    rejected = torch.zeros(1, dtype=torch.int32, device="cuda")
    cells_corrected = 0
    if runs_in is not None:
        runs, walls, coarse_steps = dict(runs_in["runs"]), dict(runs_in["walls"]), runs_in["coarse_steps"]
        for name in ("fine", "fine_restricted", "coarse"):
            mw[name], divb[name] = runs_in["mw"][name], runs_in["divb"][name]
    ic = None
    for name, cfgs in (("fine", fine), ("coarse", coarse), ("corrected", coarse)):
        if name in runs:
            continue
        e = Ensemble(cfgs)
        if name == "fine":
            e.initialize()
        else:
            # the fine run's initial state restricted: both grids start from the same physical state
            if ic is None:
                ic = Ensemble(fine)
                ic.initialize()
            _load_restricted(ic, e, factor, buf)
        e.start(t_end=t_snaps[0])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t_prev = 0.0
        pending = None   # instances corrected last and their CFL dt before the correction
        for k, ts in enumerate(t_snaps):
            if name != "corrected":
                if k:
                    e.continue_to(ts)
                e.run(chunk=64)
                if name == "coarse":
                    coarse_steps[k] = [c.step for c in e.controls()]
            else:
                start = np.array([c.step for c in e.controls()], dtype=np.int64)
                interval = coarse_steps[k] - (coarse_steps[k - 1] if k else 0)
                cap = start + (step_factor * interval).astype(np.int64) + 40
                m = max(1, int(round((ts - t_prev) / delta)))
                for q in range(1, m + 1):
                    tc = ts if q == m else t_prev + q * (ts - t_prev) / m
                    e.continue_to(tc)           # dt / ch of the (corrected) states
                    if pending is not None:
                        due, dt_before = pending
                        ctl = e.controls()
                        dt_after = np.array([ctl[i].dt_cfl for i in due])
                        drop = (dt_after < dt_drop * dt_before) & ~fallback[due]
                        fallback[due[drop]] = True
                        reasons["dt_drop"] += int(drop.sum())
                        pending = None
                    _set_limits(e, cap, fallback)
                    e.run(chunk=32)
                    ctl = e.controls()
                    t_now = np.array([c.t for c in ctl])
                    over = (t_now < tc * (1 - 1e-12)) & ~fallback
                    if over.any():
                        fallback |= over
                        reasons["steps"] += int(over.sum())
                    if time.perf_counter() - t0 > max_wall:
                        left = ~fallback
                        fallback |= left
                        reasons["wall"] += int(left.sum())
                    due = np.nonzero(~fallback)[0]
                    if len(due):
                        dt_before = np.array([ctl[i].dt_cfl for i in due])
                        ok = _apply_batch(net, norm, e, due, corr_sigma, alpha, min_ratio, rejected, scalar_mode)
                        n_corr += 1
                        cells_corrected += int(sum(cfgs[i].nx * cfgs[i].ny for i in due[ok]))
                        fallback[due[~ok]] = True
                        reasons["range"] += int((~ok).sum())
                        pending = (due[ok], dt_before[ok])
                t_prev = ts
            for i in range(n):
                mw[name][k, i], divb[name][k, i] = _mixing_width(e, i)
            if name == "fine":
                _load_restricted(e, scratch, factor, buf)
                for i in range(n):
                    mw["fine_restricted"][k, i], divb["fine_restricted"][k, i] = _mixing_width(scratch, i)
        torch.cuda.synchronize()
        walls[name] = time.perf_counter() - t0
        runs[name] = e
        if log:
            log(f"  {name}: {walls[name]:.1f}s" + (f"  corrections {n_corr}, fallback {int(fallback.sum())}/{n} "
                                                    f"{reasons}" if name == "corrected" else ""))
    # div B gate on the corrected runs
    gate = ((divb["corrected"].max(0) > divb_tol) | ~np.isfinite(mw["corrected"]).all(0)) & ~fallback
    reasons["divB"] += int(gate.sum())
    fallback |= gate
    # spectral energy at the final time (fine restricted to the coarse grid)
    spec_err = np.zeros((2, n))
    for i in range(n):
        r = torch.empty((10, nxc, nycc), dtype=torch.float32, device=runs["fine"].device)
        g = runs["fine"]._grid(i)
        _lib.call("amhd_nn_restrict", g, ptr(runs["fine"].state(i)), factor, ptr(r), nxc * nycc, 0, 1, stream_ptr())
        ref = _ke_spectrum(r)
        for j, name in enumerate(("coarse", "corrected")):
            sp = _ke_spectrum(_interior(runs[name], i))
            spec_err[j, i] = float((sp - ref).abs().sum() / ref.sum().clamp_min(1e-300))
    def mw_err(name, ref):
        peak = np.maximum(np.abs(mw[ref]).max(0), 1e-12)
        return np.abs(mw[name] - mw[ref]).max(0) / peak

    # reference: the fine solution restricted onto the coarse grid (what a coarse
    # grid can represent); against the fine grid's own values as well
    err_c, err_k = mw_err("coarse", "fine_restricted"), mw_err("corrected", "fine_restricted")
    err_cf, err_kf = mw_err("coarse", "fine"), mw_err("corrected", "fine")
    err_final = np.where(fallback, 0.0, err_k)
    out = {
        "seeds": list(map(int, seeds)), "correction_interval": delta, "corrections": n_corr,
        "wall_s": walls, "speedup_corrected_vs_fine": walls["fine"] / max(walls["corrected"], 1e-12),
        "mixing_width_err_coarse": {"mean": float(err_c.mean()), "median": float(np.median(err_c)),
                                    "max": float(err_c.max())},
        "mixing_width_err_corrected": {"mean": float(err_k.mean()), "median": float(np.median(err_k)),
                                       "max": float(err_k.max())},
        "within_2pct": {"coarse": int((err_c <= 0.02).sum()), "corrected": int((err_k <= 0.02).sum()), "of": n},
        "within_5pct": {"coarse": int((err_c <= 0.05).sum()), "corrected": int((err_k <= 0.05).sum()), "of": n},
        "mixing_width_err_vs_fine_grid": {"coarse": float(err_cf.mean()), "corrected": float(err_kf.mean()),
                                          "fine_restricted": float(mw_err("fine_restricted", "fine").mean())},
        "spectral_energy_err": {"coarse": float(spec_err[0].mean()), "corrected": float(spec_err[1].mean())},
        "divB_L2_final": {k: float(v[-1].mean()) for k, v in divb.items()},
        "fallback_instances": int(fallback.sum()), "fallback_reasons": reasons, "alpha": alpha,
        "scalar_mode": scalar_mode,
        "min_ratio": min_ratio, "cells_not_corrected_fraction": float(rejected.item()) / max(cells_corrected, 1),
        "speedup_with_fallback_fine_solves": walls["fine"] / max(walls["corrected"] +
                                                                 fallback.mean() * walls["fine"], 1e-12),
        "mixing_width_err_with_fallback": {"mean": float(err_final.mean()), "max": float(err_final.max())},
    }
    out["_baseline"] = {"runs": {k: runs[k] for k in ("fine", "coarse")},
                        "walls": {k: walls[k] for k in ("fine", "coarse")}, "coarse_steps": coarse_steps,
                        "mw": {k: mw[k] for k in ("fine", "fine_restricted", "coarse")},
                        "divb": {k: divb[k] for k in ("fine", "fine_restricted", "coarse")}}
    return out


def _apply_batch(net: Corrector, norm: Normaliser, e: Ensemble, idx, corr_sigma: float, alpha: float = 1.0,
                 min_ratio: float = 0.5, rejected: torch.Tensor | None = None, scalar_mode: int = 1) -> np.ndarray:
    """One forward pass over the instances `idx`; each gets alpha x its correction
    (cells whose corrected density or pressure would fall below min_ratio of the
    current value keep their state) unless the correction is non-finite or far
    outside the training range (then it is marked for fallback).  Ghost cells
    are refreshed afterwards."""
    N = net.H * net.W
    B = len(idx)
    x = net._buf("eval.x", (10, B * N))
    for b, i in enumerate(idx):
        _lib.call("amhd_nn_pack", e._grid(i), ptr(e.state(i)), ptr(net.in_mean), ptr(net.in_istd), ptr(x), B * N,
                  int(b), stream_ptr())
    y = net.forward(x, B)
    net.check_gemm_status()  # an unwritten GEMM output must not reach the states
    if getattr(net, "project_y", False):
        y = project_rows(y.view(10, B, net.H, net.W)).reshape(10, B * N).contiguous()
    lim = (norm.out_max * corr_sigma).view(10, 1, 1)
    yb = y.view(10, B, N)
    good = (torch.isfinite(yb).all(dim=2).all(dim=0) & (yb.abs() <= lim).all(dim=2).all(dim=0)).cpu().numpy()
    for b, i in enumerate(idx):
        g = e._grid(i)
        if good[b]:
            _lib.call("amhd_nn_apply_guarded", g, ptr(e.state(i)), ptr(net.out_scale), ptr(y), B * N, int(b),
                      float(alpha), float(min_ratio), int(scalar_mode), ptr(rejected) if rejected is not None else None,
                      stream_ptr())
        _lib.call("amhd_apply_bc", g, ptr(e.state(i)), stream_ptr())
    return good


def save(path: str, net: Corrector, norm: Normaliser) -> None:
    """Weights and normalisation of a trained corrector (torch.save)."""
    torch.save({"params": net.host_params(), "H": net.H, "W": net.W, "project_y": bool(getattr(net, "project_y", 0)),
                "norm": {k: getattr(norm, k).detach().cpu() for k in ("in_mean", "in_std", "out_std", "active",
                                                                       "out_max")}}, path)


def load(path: str, device="cuda"):
    """(Corrector, Normaliser) from a file written by save()."""
    d = torch.load(path, map_location="cpu")
    norm = Normaliser.__new__(Normaliser)
    for k, v in d["norm"].items():
        setattr(norm, k, v.to(device))
    net = Corrector(int(d["H"]), int(d["W"]), params=d["params"], device=device)
    net.set_normalisation(norm.in_mean, norm.in_std, norm.out_scale)
    net.project_y = bool(d.get("project_y", False))
    return net, norm


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=100)
    ap.add_argument("--test-seeds", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--nyc", type=int, default=64)
    ap.add_argument("--delta", type=float, default=DELTA, help="correction interval (simulated time)")
    ap.add_argument("--alpha", default="1.0", help="comma-separated correction scales to evaluate")
    ap.add_argument("--min-ratio", type=float, default=0.5)
    ap.add_argument("--scalar-modes", default="1", help="comma-separated scalar correction modes (0, 1, 2)")
    ap.add_argument("--load", default=None, help="evaluate a saved corrector instead of generating and training")
    ap.add_argument("--dagger-rounds", type=int, default=0,
                    help="rounds of training on pairs from the corrector's own runs")
    ap.add_argument("--dagger-epochs", type=int, default=20)
    ap.add_argument("--dagger-mode", type=int, default=3, help="correction mode of those runs")
    ap.add_argument("--closure-rounds", type=int, default=0,
                    help="rounds of training on closure pairs along the corrector's own runs (closure_pairs)")
    ap.add_argument("--closure-every", type=int, default=3)
    ap.add_argument("--project-y", action="store_true",
                    help="train on and apply the row averages of the corrections (project_rows)")
    ap.add_argument("--save", default=None)
    a = ap.parse_args(argv)
    log = lambda m: print(m, file=sys.stderr, flush=True)
    wall_gen, n_pairs, hist = None, 0, None
    if a.load:
        net, norm = load(a.load)
    else:
        seeds = list(range(a.train_seeds))
        n_val = max(1, a.train_seeds // 10)
        log(f"generating {a.train_seeds} coarse/fine run pairs ...")
        X, Y, wall_gen = generate_pairs(seeds, delta=a.delta, nyc=a.nyc, log=log)
        n_pairs = int(X.shape[0] * X.shape[1])
        log("training ...")
        net, norm, hist = train(X, Y, range(n_val, a.train_seeds), range(n_val), epochs=a.epochs, batch=a.batch,
                                lr=a.lr, project_y=a.project_y, log=log)
        for r in range(a.dagger_rounds):
            log(f"rollout round {r + 1}: pairs from corrected runs ...")
            X2, Y2 = rollout_pairs(net, norm, seeds, delta=a.delta, scalar_mode=a.dagger_mode, nyc=a.nyc, log=log)
            X, Y = torch.cat([X, X2]), torch.cat([Y, Y2])
            del X2, Y2
            n_pairs = int(X.shape[0] * X.shape[1])
            net, norm, h2 = train(X, Y, range(n_val, a.train_seeds), range(n_val), epochs=a.dagger_epochs,
                                  batch=a.batch, lr=a.lr * 0.5, net=net, norm=norm, log=log)
            hist[f"round{r + 1}"] = h2
        for r in range(a.closure_rounds):
            log(f"closure round {r + 1}: fine evolution from the corrected runs' states ...")
            X2, Y2 = closure_pairs(net, norm, seeds, delta=a.delta, scalar_mode=a.dagger_mode,
                                   every=a.closure_every, nyc=a.nyc, log=log)
            X, Y = torch.cat([X, X2]), torch.cat([Y, Y2])
            del X2, Y2
            n_pairs = int(X.shape[0] * X.shape[1])
            net, norm, h2 = train(X, Y, range(n_val, a.train_seeds), range(n_val), epochs=a.dagger_epochs,
                                  batch=a.batch, lr=a.lr * 0.5, net=net, norm=norm, log=log)
            hist[f"closure{r + 1}"] = h2
        del X, Y
    log("evaluating on held-out seeds ...")
    test = list(range(10000, 10000 + a.test_seeds))
    evs, base = [], None
    for mode in (int(x) for x in a.scalar_modes.split(",")):
        for alpha in (float(x) for x in a.alpha.split(",")):
            log(f"  alpha = {alpha}, scalar mode {mode}")
            ev = evaluate(net, norm, test, delta=a.delta, nyc=a.nyc, alpha=alpha, min_ratio=a.min_ratio,
                          scalar_mode=mode, runs_in=base, log=log)
            base = ev.pop("_baseline")
            evs.append(ev)
    if a.save:
        save(a.save, net, norm)
    print(json.dumps({"data_generation_wall_s": wall_gen, "pairs": n_pairs,
                      "training": hist, "evaluation": evs, "params": sum(p["w"].numel() + p["b"].numel()
                                                                        for p in net.p.values())}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
