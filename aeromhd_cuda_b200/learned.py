"""Training data, training and evaluation of the learned coarse-grid corrector.

    python -m aeromhd_cuda_b200.learned --train-seeds 100 --test-seeds 64

Data: shocked-interface runs drawn like the batched ensemble (Mach, density
ratio, mode, amplitude, field), each run twice from the same parameters --
coarse (nx x ny) and 4x finer -- as two GPU ensembles; at every snapshot time
(0.1, 0.2, ... 3.0) the pair (coarse state, fine state restricted onto the
coarse grid) is kept.  Runs use the frame of the shocked gas so that the
mixing layer stays in the domain until t = 3.  Seeds split 90/10 into
training and validation; separate test seeds judge the result.

Use: during a coarse run the corrector is applied every `apply_every` coarse
steps of each instance.  It is judged against the plain fine solve on
mixing width, spectral energy and div B; an instance falls back to the plain
fine solve when its corrected run leaves the trusted range (non-finite
values, corrections far outside the training distribution, div B above a
tolerance).

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
from ._tensors import ptr, stream_ptr
from .corrector import Corrector
from .ensemble import Ensemble, draw_configs

T_SNAPS = tuple(round(0.1 * k, 10) for k in range(1, 31))


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


def generate_pairs(seeds: Sequence[int], t_snaps: Sequence[float] = T_SNAPS, nyc: int = 64, factor: int = 4,
                   precision: str = "fp32", log=print):
    """Returns (X, Y, wall): X[snap][seed] coarse interiors, Y[snap][seed] restricted fine interiors."""
    coarse, fine = paired_configs(seeds, nyc, factor, precision)
    ec, ef = Ensemble(coarse), Ensemble(fine)
    ec.initialize()
    ef.initialize()
    nxc, nyc_ = coarse[0].nx, coarse[0].ny
    n = len(seeds)
    X = torch.empty((len(t_snaps), n, 10, nxc, nyc_), dtype=torch.float32, device=ec.device)
    Y = torch.empty_like(X)
    wall = {"coarse": 0.0, "fine": 0.0}
    ec.start(t_end=t_snaps[0])
    ef.start(t_end=t_snaps[0])
    plane = nxc * nyc_
    for k, ts in enumerate(t_snaps):
        if k:
            ec.continue_to(ts)
            ef.continue_to(ts)
        for name, e in (("coarse", ec), ("fine", ef)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e.run(chunk=64)
            torch.cuda.synchronize()
            wall[name] += time.perf_counter() - t0
        for i in range(n):
            X[k, i].copy_(_interior(ec, i))
            g = ef._grid(i)
            out = Y[k, i]
            _lib.call("amhd_nn_restrict", g, ptr(ef.state(i)), factor, ptr(out), plane, 0, 1, stream_ptr())
        if log and (k % 5 == 4 or k == len(t_snaps) - 1):
            log(f"  pairs at t={ts:.1f}: {n} seeds, wall coarse {wall['coarse']:.1f}s fine {wall['fine']:.1f}s")
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


def train(X: torch.Tensor, Y: torch.Tensor, train_seeds: Sequence[int], val_seeds: Sequence[int], epochs: int = 20,
          batch: int = 16, lr: float = 1e-3, seed: int = 0, log=print):
    """X, Y: [snap][seed][10][H][W]; seeds index the second axis.  Returns (net, norm, history)."""
    H, W = X.shape[-2], X.shape[-1]
    T = Y - X
    tr = X[:, list(train_seeds)].reshape(-1, 10, H, W)
    ttr = T[:, list(train_seeds)].reshape(-1, 10, H, W)
    va = X[:, list(val_seeds)].reshape(-1, 10, H, W)
    tva = T[:, list(val_seeds)].reshape(-1, 10, H, W)
    norm = Normaliser(tr, ttr)
    net = Corrector(H, W, seed=seed, device=X.device)
    net.set_normalisation(norm.in_mean, norm.in_std, norm.out_scale)
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
            losses.append(net.train_step(x, t, batch, lr=sched(ep)))
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


def evaluate(net: Corrector, norm: Normaliser, seeds: Sequence[int], apply_every: int = 20, nyc: int = 64,
             factor: int = 4, t_snaps: Sequence[float] = T_SNAPS, divb_tol: float = 1.0, corr_sigma: float = 8.0,
             log=print) -> dict:
    coarse, fine = paired_configs(seeds, nyc, factor)
    n = len(seeds)
    runs = {}
    walls = {}
    mw = {name: np.zeros((len(t_snaps), n)) for name in ("fine", "coarse", "corrected")}
    divb = {name: np.zeros((len(t_snaps), n)) for name in ("fine", "coarse", "corrected")}
    fallback = np.zeros(n, dtype=bool)
    for name, cfgs in (("fine", fine), ("coarse", coarse), ("corrected", coarse)):
        e = Ensemble(cfgs)
        e.initialize()
        e.start(t_end=t_snaps[0])
        last = np.zeros(n, dtype=np.int64)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k, ts in enumerate(t_snaps):
            if k:
                e.continue_to(ts)
            if name != "corrected":
                e.run(chunk=64)
            else:
                while True:
                    e.advance(apply_every)
                    ctl = e.controls()
                    steps = np.array([c.step for c in ctl])
                    due = np.nonzero((steps // apply_every > last // apply_every) & ~fallback)[0]
                    if len(due):
                        ok = _apply_batch(net, norm, e, due, corr_sigma)
                        fallback[due[~ok]] = True
                    last = steps
                    if len(due):
                        e.continue_to(ts)
                    if not any(c.active for c in e.controls()):
                        break
            for i in range(n):
                mw[name][k, i], divb[name][k, i] = _mixing_width(e, i)
        torch.cuda.synchronize()
        walls[name] = time.perf_counter() - t0
        runs[name] = e
        if log:
            log(f"  {name}: {walls[name]:.1f}s")
    # div B gate on the corrected runs
    fallback |= (divb["corrected"].max(0) > divb_tol) | ~np.isfinite(mw["corrected"]).all(0)
    # spectral energy at the final time (fine restricted to the coarse grid)
    spec_err = np.zeros((2, n))
    nxc, nycc = coarse[0].nx, coarse[0].ny
    for i in range(n):
        r = torch.empty((10, nxc, nycc), dtype=torch.float32, device=runs["fine"].device)
        g = runs["fine"]._grid(i)
        _lib.call("amhd_nn_restrict", g, ptr(runs["fine"].state(i)), factor, ptr(r), nxc * nycc, 0, 1, stream_ptr())
        ref = _ke_spectrum(r)
        for j, name in enumerate(("coarse", "corrected")):
            sp = _ke_spectrum(_interior(runs[name], i))
            spec_err[j, i] = float((sp - ref).abs().sum() / ref.sum().clamp_min(1e-300))
    peak = np.maximum(np.abs(mw["fine"]).max(0), 1e-12)

    def mw_err(name):
        return np.abs(mw[name] - mw["fine"]).max(0) / peak

    err_c, err_k = mw_err("coarse"), mw_err("corrected")
    err_final = np.where(fallback, 0.0, err_k)
    out = {
        "seeds": list(map(int, seeds)), "apply_every": apply_every,
        "wall_s": walls, "speedup_corrected_vs_fine": walls["fine"] / max(walls["corrected"], 1e-12),
        "mixing_width_err_coarse": {"mean": float(err_c.mean()), "median": float(np.median(err_c)),
                                    "max": float(err_c.max())},
        "mixing_width_err_corrected": {"mean": float(err_k.mean()), "median": float(np.median(err_k)),
                                       "max": float(err_k.max())},
        "within_2pct": {"coarse": int((err_c <= 0.02).sum()), "corrected": int((err_k <= 0.02).sum()), "of": n},
        "spectral_energy_err": {"coarse": float(spec_err[0].mean()), "corrected": float(spec_err[1].mean())},
        "divB_L2_final": {k: float(v[-1].mean()) for k, v in divb.items()},
        "fallback_instances": int(fallback.sum()),
        "mixing_width_err_with_fallback": {"mean": float(err_final.mean()), "max": float(err_final.max())},
    }
    return out


def _apply_batch(net: Corrector, norm: Normaliser, e: Ensemble, idx, corr_sigma: float) -> np.ndarray:
    """One forward pass over the instances `idx`; each gets its correction unless it is
    non-finite or far outside the training range (then it is marked for fallback).
    Ghost cells are refreshed afterwards."""
    N = net.H * net.W
    B = len(idx)
    x = net._buf("eval.x", (10, B * N))
    for b, i in enumerate(idx):
        _lib.call("amhd_nn_pack", e._grid(i), ptr(e.state(i)), ptr(net.in_mean), ptr(net.in_istd), ptr(x), B * N,
                  int(b), stream_ptr())
    y = net.forward(x, B)
    lim = (norm.out_max * corr_sigma).view(10, 1, 1)
    yb = y.view(10, B, N)
    good = (torch.isfinite(yb).all(dim=2).all(dim=0) & (yb.abs() <= lim).all(dim=2).all(dim=0)).cpu().numpy()
    for b, i in enumerate(idx):
        g = e._grid(i)
        if good[b]:
            _lib.call("amhd_nn_apply", g, ptr(e.state(i)), ptr(net.out_scale), ptr(y), B * N, int(b), stream_ptr())
        _lib.call("amhd_apply_bc", g, ptr(e.state(i)), stream_ptr())
    return good


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=100)
    ap.add_argument("--test-seeds", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--nyc", type=int, default=64)
    ap.add_argument("--apply-every", type=int, default=20)
    ap.add_argument("--save", default=None)
    a = ap.parse_args(argv)
    log = lambda m: print(m, file=sys.stderr, flush=True)
    seeds = list(range(a.train_seeds))
    n_val = max(1, a.train_seeds // 10)
    log(f"generating {a.train_seeds} coarse/fine run pairs ...")
    X, Y, wall_gen = generate_pairs(seeds, nyc=a.nyc, log=log)
    log("training ...")
    net, norm, hist = train(X, Y, range(n_val, a.train_seeds), range(n_val), epochs=a.epochs, batch=a.batch,
                            lr=a.lr, log=log)
    log("evaluating on held-out seeds ...")
    test = list(range(10000, 10000 + a.test_seeds))
    ev = evaluate(net, norm, test, apply_every=a.apply_every, nyc=a.nyc, log=log)
    if a.save:
        torch.save({"params": net.host_params(), "in_mean": norm.in_mean.cpu(), "in_std": norm.in_std.cpu(),
                    "out_std": norm.out_std.cpu()}, a.save)
    print(json.dumps({"data_generation_wall_s": wall_gen, "pairs": int(X.shape[0] * X.shape[1]),
                      "training": hist, "evaluation": ev, "params": sum(p["w"].numel() + p["b"].numel()
                                                                        for p in net.p.values())}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
