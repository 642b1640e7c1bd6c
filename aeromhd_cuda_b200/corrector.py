"""Learned coarse-grid corrector.

A 4-level convolutional encoder-decoder (U-Net shape, 3x3 kernels, 32 -> 256
channels, ~0.63 M parameters) maps a coarse solution (the 9 conserved fields
plus psi, normalised per channel) to a correction that moves it toward the
fine-grid solution restricted onto the coarse grid (4x4 block averages).

Every convolution is an im2col + GEMM on the BF16 tensor cores with FP32
accumulation (amhd_nn_gemm: tcgen05.mma fed by TMA for the wide layers,
mma.sync m16n8k16 for the narrow first one); forward, backward (data and
weight gradients),
bias/ReLU, pooling, upsampling, the loss and Adam are the library's own
kernels (amhd_nn_* in include/aeromhd.h).  Weights keep an FP32 master copy;
their BF16 copy feeds the GEMMs.  PyTorch only allocates the buffers.

No counterpart in the reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np
import torch

from . import _lib
from ._tensors import make_grid, ptr, stream_ptr

BF16 = torch.bfloat16
F32 = torch.float32


@dataclass(frozen=True)
class ConvSpec:
    name: str
    cin: int
    cout: int
    k: int      # 3 or 1
    relu: bool


def architecture(ch=(32, 64, 128, 256), nin: int = 10, nout: int = 10) -> List[ConvSpec]:
    c1, c2, c3, c4 = ch
    return [
        ConvSpec("e1", nin, c1, 3, True), ConvSpec("e2", c1, c2, 3, True), ConvSpec("e3", c2, c3, 3, True),
        ConvSpec("e4", c3, c4, 3, True),
        ConvSpec("d3a", c4, c3, 1, False), ConvSpec("d3", c3, c3, 3, True),
        ConvSpec("d2a", c3, c2, 1, False), ConvSpec("d2", c2, c2, 3, True),
        ConvSpec("d1a", c2, c1, 1, False), ConvSpec("d1", c1, c1, 3, True),
        ConvSpec("out", c1, nout, 3, False),
    ]


def _round8(k: int) -> int:
    return (k + 7) // 8 * 8


def n_params(specs: List[ConvSpec]) -> int:
    return sum(s.cout * s.cin * s.k * s.k + s.cout for s in specs)


def init_params(specs: List[ConvSpec], seed: int = 0) -> Dict[str, Dict[str, torch.Tensor]]:
    """He-normal weights (the last layer scaled down so the initial correction is small), zero biases."""
    gen = torch.Generator().manual_seed(seed)
    out = {}
    for s in specs:
        fan_in = s.cin * s.k * s.k
        std = math.sqrt(2.0 / fan_in) * (0.1 if s.name == "out" else 1.0)
        w = torch.randn((s.cout, s.cin, s.k, s.k), generator=gen, dtype=torch.float32) * std
        out[s.name] = {"w": w, "b": torch.zeros(s.cout, dtype=torch.float32)}
    return out


class Corrector:
    """Network state on the GPU plus its forward / backward / Adam step."""

    def __init__(self, H: int, W: int, params: Optional[dict] = None, seed: int = 0, device="cuda",
                 channels=(32, 64, 128, 256)):
        if H % 8 or W % 8:
            raise ValueError("coarse grid must be divisible by 8 in both directions (3 pooling levels)")
        self.H, self.W = H, W
        self.device = torch.device(device)
        self.specs = architecture(channels)
        host = params if params is not None else init_params(self.specs, seed)
        self.p = {}
        for s in self.specs:
            w = host[s.name]["w"].reshape(s.cout, -1).to(self.device, F32).contiguous()
            b = host[s.name]["b"].to(self.device, F32).contiguous()
            self.p[s.name] = {"w": w, "b": b, "wb": w.to(BF16).contiguous(),
                              "gw": torch.zeros_like(w), "gb": torch.zeros_like(b),
                              "mw": torch.zeros_like(w), "vw": torch.zeros_like(w),
                              "mb": torch.zeros_like(b), "vb": torch.zeros_like(b)}
        self.t = 0
        self._adam = None      # (device table of amhd_nn_tensor, count, largest size, weight decay)
        self._hyper = torch.zeros(6, dtype=F32, device=self.device)  # lr, b1, b2, eps, c1, c2
        self._graphs: Dict[int, tuple] = {}
        self._ws: Dict[str, torch.Tensor] = {}
        self._pad_shapes: Dict[str, tuple] = {}  # workspaces whose padding rows are zeroed
        self._act: Dict[str, torch.Tensor] = {}
        self.in_mean = torch.zeros(10, device=self.device)
        self.in_istd = torch.ones(10, device=self.device)
        self.out_scale = torch.ones(10, device=self.device)

    # ------------------------------------------------------------ buffers
    def _buf(self, key: str, shape, dtype=F32) -> torch.Tensor:
        t = self._ws.get(key)
        n = int(np.prod(shape))
        if t is None or t.numel() < n or t.dtype != dtype:
            t = torch.empty(n, dtype=dtype, device=self.device)
            self._ws[key] = t
        return t[:n].view(*shape)

    def _padded_rows(self, key: str, rows: int, rows_p: int, N: int) -> torch.Tensor:
        """A BF16 [rows_p][N] workspace whose rows rows .. rows_p-1 are zero: zeroed
        when the buffer or its shape is new (the eager step before a graph
        capture), never inside a captured step."""
        t = self._buf(key, (rows_p, N), BF16)
        if rows_p > rows and self._pad_shapes.get(key) != (rows, rows_p, N, t.data_ptr()):
            t[rows:].zero_()
            self._pad_shapes[key] = (rows, rows_p, N, t.data_ptr())
        return t

    def host_params(self) -> dict:
        return {s.name: {"w": self.p[s.name]["w"].detach().cpu().reshape(s.cout, s.cin, s.k, s.k).clone(),
                         "b": self.p[s.name]["b"].detach().cpu().clone()} for s in self.specs}

    # ------------------------------------------------------------- layers
    def _conv_fwd(self, s: ConvSpec, X: torch.Tensor, B: int, H: int, W: int) -> torch.Tensor:
        N = B * H * W
        st = stream_ptr()
        K = s.cin * s.k * s.k
        Kp = _round8(K)  # GEMM operands with a row pitch of whole 16-byte pieces (the TMA path)
        wb = self.p[s.name]["wb"]
        if s.k == 3:
            col = self._padded_rows(f"{s.name}.col", K, Kp, N)
            _lib.call("amhd_nn_im2col3", ptr(X), s.cin, B, H, W, ptr(col), st)
        else:
            col = self._padded_rows(f"{s.name}.col", K, Kp, N)
            _lib.call("amhd_nn_cast_bf16", ptr(X), ptr(col), X.numel(), st)
        if Kp != K:
            wp = self._buf(f"{s.name}.wpad", (s.cout, Kp), BF16)
            _lib.call("amhd_nn_pad_cols", ptr(wb), s.cout, K, Kp, ptr(wp), st)
            wb = wp
        Y = self._buf(f"{s.name}.y", (s.cout, N))
        _lib.call("amhd_nn_gemm", 0, 0, s.cout, N, Kp, ptr(wb), Kp, ptr(col), N, ptr(Y), N, 1.0, 0.0, 1, st)
        _lib.call("amhd_nn_bias_act", ptr(Y), ptr(self.p[s.name]["b"]), s.cout, N, int(s.relu), st)
        return Y

    def _conv_bwd(self, s: ConvSpec, dY: torch.Tensor, Y: torch.Tensor, B: int, H: int, W: int,
                  need_dx: bool = True) -> Optional[torch.Tensor]:
        N = B * H * W
        st = stream_ptr()
        K = s.cin * s.k * s.k
        if s.relu:
            _lib.call("amhd_nn_relu_bwd", ptr(dY), ptr(Y), dY.numel(), st)
        P = self.p[s.name]
        _lib.call("amhd_nn_bias_grad", ptr(dY), s.cout, N, ptr(P["gb"]), st)
        dYb = self._buf(f"{s.name}.dyb", (s.cout, N), BF16)
        _lib.call("amhd_nn_cast_bf16", ptr(dY), ptr(dYb), dY.numel(), st)
        col = self._ws[f"{s.name}.col"][: K * N]  # the forward's columns (its first K rows)
        splits = max(1, min(64, N // 4096))
        # dW[cout][K] = dY[cout][N] x col[K][N]^T
        _lib.call("amhd_nn_gemm", 0, 1, s.cout, K, N, ptr(dYb), N, ptr(col), N, ptr(P["gw"]), K, 1.0, 0.0,
                  splits, st)
        if not need_dx:
            return None
        if s.k == 3:
            # the adjoint of the zero-padded 3x3 convolution: the same convolution of dY
            # with the transposed weights turned by 180 degrees (amhd_nn_flip3), one GEMM
            # of K = cout x 9 instead of a [cin x 9][N] product and its col2im gather
            Kg = _round8(s.cout * 9)
            colg = self._padded_rows(f"{s.name}.colg", s.cout * 9, Kg, N)
            _lib.call("amhd_nn_im2col3", ptr(dY), s.cout, B, H, W, ptr(colg), st)
            wt = self._buf(f"{s.name}.wt", (s.cin, Kg), BF16)
            _lib.call("amhd_nn_flip3", ptr(P["wb"]), s.cout, s.cin, Kg, ptr(wt), st)
            dX = self._buf(f"{s.name}.dx", (s.cin, N))
            _lib.call("amhd_nn_gemm", 0, 0, s.cin, N, Kg, ptr(wt), Kg, ptr(colg), N, ptr(dX), N, 1.0, 0.0, 1, st)
        else:
            dX = self._buf(f"{s.name}.dx", (s.cin, N))
            _lib.call("amhd_nn_gemm", 1, 0, s.cin, N, s.cout, ptr(P["wb"]), s.cin, ptr(dYb), N, ptr(dX), N,
                      1.0, 0.0, 1, st)
        return dX

    def _pool(self, key, X, C, B, H, W):
        Y = self._buf(key, (C, B * (H // 2) * (W // 2)))
        _lib.call("amhd_nn_pool2", ptr(X), C * B, H, W, ptr(Y), 0, stream_ptr())
        return Y

    def _pool_bwd_add(self, dY, C, B, H, W, into):
        dX = self._buf("poolbwd.tmp", (C, B * H * W))
        _lib.call("amhd_nn_pool2", ptr(dY), C * B, H, W, ptr(dX), 1, stream_ptr())
        _lib.call("amhd_nn_axpy", ptr(into), ptr(dX), 1.0, into.numel(), stream_ptr())

    def _up(self, key, X, C, B, h, w):
        Y = self._buf(key, (C, B * 4 * h * w))
        _lib.call("amhd_nn_up2", ptr(X), C * B, h, w, ptr(Y), 0, stream_ptr())
        return Y

    def _up_bwd(self, key, dY, C, B, h, w):
        dX = self._buf(key, (C, B * h * w))
        _lib.call("amhd_nn_up2", ptr(dY), C * B, h, w, ptr(dX), 1, stream_ptr())
        return dX

    def _add(self, key, a, b):
        out = self._buf(key, a.shape)
        out.copy_(a)
        _lib.call("amhd_nn_axpy", ptr(out), ptr(b), 1.0, out.numel(), stream_ptr())
        return out

    # ----------------------------------------------------------- network
    def forward(self, x: torch.Tensor, B: int) -> torch.Tensor:
        """x: [10][B*H*W] float32 (normalised input) -> correction [10][B*H*W] (normalised)."""
        H, W = self.H, self.W
        S = {s.name: s for s in self.specs}
        a = self._act
        a["x"] = x
        a["e1"] = self._conv_fwd(S["e1"], x, B, H, W)
        a["p1"] = self._pool("p1", a["e1"], S["e1"].cout, B, H, W)
        a["e2"] = self._conv_fwd(S["e2"], a["p1"], B, H // 2, W // 2)
        a["p2"] = self._pool("p2", a["e2"], S["e2"].cout, B, H // 2, W // 2)
        a["e3"] = self._conv_fwd(S["e3"], a["p2"], B, H // 4, W // 4)
        a["p3"] = self._pool("p3", a["e3"], S["e3"].cout, B, H // 4, W // 4)
        a["e4"] = self._conv_fwd(S["e4"], a["p3"], B, H // 8, W // 8)
        a["u3"] = self._up("u3", a["e4"], S["e4"].cout, B, H // 8, W // 8)
        a["d3a"] = self._conv_fwd(S["d3a"], a["u3"], B, H // 4, W // 4)
        a["s3"] = self._add("s3", a["d3a"], a["e3"])
        a["d3"] = self._conv_fwd(S["d3"], a["s3"], B, H // 4, W // 4)
        a["u2"] = self._up("u2", a["d3"], S["d3"].cout, B, H // 4, W // 4)
        a["d2a"] = self._conv_fwd(S["d2a"], a["u2"], B, H // 2, W // 2)
        a["s2"] = self._add("s2", a["d2a"], a["e2"])
        a["d2"] = self._conv_fwd(S["d2"], a["s2"], B, H // 2, W // 2)
        a["u1"] = self._up("u1", a["d2"], S["d2"].cout, B, H // 2, W // 2)
        a["d1a"] = self._conv_fwd(S["d1a"], a["u1"], B, H, W)
        a["s1"] = self._add("s1", a["d1a"], a["e1"])
        a["d1"] = self._conv_fwd(S["d1"], a["s1"], B, H, W)
        a["out"] = self._conv_fwd(S["out"], a["d1"], B, H, W)
        return a["out"]

    def backward(self, dout: torch.Tensor, B: int) -> None:
        """Gradients of every parameter from d(loss)/d(out); forward must have run on this batch."""
        H, W = self.H, self.W
        S = {s.name: s for s in self.specs}
        a = self._act
        d_d1 = self._conv_bwd(S["out"], dout, a["out"], B, H, W)
        d_s1 = self._conv_bwd(S["d1"], d_d1.clone(), a["d1"], B, H, W)
        d_e1 = d_s1.clone()
        d_u1 = self._conv_bwd(S["d1a"], d_s1, a["d1a"], B, H, W)
        d_d2 = self._up_bwd("d_d2", d_u1, S["d2"].cout, B, H // 2, W // 2)
        d_s2 = self._conv_bwd(S["d2"], d_d2, a["d2"], B, H // 2, W // 2)
        d_e2 = d_s2.clone()
        d_u2 = self._conv_bwd(S["d2a"], d_s2, a["d2a"], B, H // 2, W // 2)
        d_d3 = self._up_bwd("d_d3", d_u2, S["d3"].cout, B, H // 4, W // 4)
        d_s3 = self._conv_bwd(S["d3"], d_d3, a["d3"], B, H // 4, W // 4)
        d_e3 = d_s3.clone()
        d_u3 = self._conv_bwd(S["d3a"], d_s3, a["d3a"], B, H // 4, W // 4)
        d_e4 = self._up_bwd("d_e4", d_u3, S["e4"].cout, B, H // 8, W // 8)
        d_p3 = self._conv_bwd(S["e4"], d_e4, a["e4"], B, H // 8, W // 8)
        self._pool_bwd_add(d_p3, S["e3"].cout, B, H // 4, W // 4, d_e3)
        d_p2 = self._conv_bwd(S["e3"], d_e3, a["e3"], B, H // 4, W // 4)
        self._pool_bwd_add(d_p2, S["e2"].cout, B, H // 2, W // 2, d_e2)
        d_p1 = self._conv_bwd(S["e2"], d_e2, a["e2"], B, H // 2, W // 2)
        self._pool_bwd_add(d_p1, S["e1"].cout, B, H, W, d_e1)
        self._conv_bwd(S["e1"], d_e1, a["e1"], B, H, W, need_dx=False)

    def _adam_table(self, weight_decay: float):
        """Device records of every parameter tensor for amhd_nn_adam_multi (weights
        with their BF16 copies and weight decay, biases without)."""
        if self._adam is None or self._adam[3] != weight_decay:
            recs = []
            for s in self.specs:
                P = self.p[s.name]
                recs.append((P["w"], P["gw"], P["mw"], P["vw"], P["wb"], weight_decay))
                recs.append((P["b"], P["gb"], P["mb"], P["vb"], None, 0.0))
            table = (_lib.NNTensor * len(recs))()
            for r, (w, g, m, v, wb, wd) in zip(table, recs):
                r.w, r.g, r.m, r.v = ptr(w), ptr(g), ptr(m), ptr(v)
                r.w_bf16 = ptr(wb) if wb is not None else None
                r.n, r.weight_decay = w.numel(), wd
            dev = torch.frombuffer(bytearray(bytes(table)), dtype=torch.uint8).to(self.device)
            self._adam = (dev, len(recs), max(r[0].numel() for r in recs), weight_decay)
            self._graphs = {}
        return self._adam

    def _set_hyper(self, lr, beta1, beta2, eps) -> None:
        """The step's Adam scalars into device memory (read by the kernel, also inside a graph)."""
        t = np.float32(self.t)
        c1 = np.float32(1) / (np.float32(1) - np.power(np.float32(beta1), t))
        c2 = np.float32(1) / (np.float32(1) - np.power(np.float32(beta2), t))
        self._hyper.copy_(torch.tensor([lr, beta1, beta2, eps, c1, c2], dtype=F32))

    def _adam_launch(self, weight_decay: float) -> None:
        table, n, big, _ = self._adam_table(weight_decay)
        _lib.call("amhd_nn_adam_multi", ptr(table), n, big, ptr(self._hyper), stream_ptr())

    def adam_step(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
                  weight_decay: float = 0.0) -> None:
        """One Adam step of every parameter (one launch: amhd_nn_adam_multi)."""
        self.t += 1
        self._adam_table(weight_decay)
        self._set_hyper(lr, beta1, beta2, eps)
        self._adam_launch(weight_decay)

    def check_gemm_status(self) -> None:
        """Raise if a tensor-core GEMM of the work queued so far gave up its bounded
        wait (its output then was not written).  Synchronises; the training loop
        calls it once per epoch, loss() and correct_state() on every call."""
        _lib.check_gemm_status("corrector")

    def train_step(self, x: torch.Tensor, target: torch.Tensor, B: int, lr: float = 1e-3) -> torch.Tensor:
        """One Adam step on mean squared error; returns the loss (device scalar, before
        the step).  Asynchronous: check_gemm_status() reports a GEMM that gave up."""
        out = self.forward(x, B)
        dout = self._buf("dout", out.shape)
        loss = self._buf("loss", (1,))
        loss.zero_()
        _lib.call("amhd_nn_mse", ptr(out), ptr(target), out.numel(), ptr(dout), ptr(loss), stream_ptr())
        self.backward(dout, B)
        self.adam_step(lr)
        return loss

    def train_step_graphed(self, x: torch.Tensor, target: torch.Tensor, B: int, lr: float = 1e-3) -> torch.Tensor:
        """train_step replayed as one CUDA graph: forward, loss, backward and the
        Adam step captured once per batch size (after one eager step that sizes
        every buffer), then every call copies the batch into the graph's input
        buffers, writes the step's Adam scalars to device memory and replays.
        Same kernels and arithmetic as train_step; returns a copy of the loss."""
        g = self._graphs.get(B)
        if g is None:
            loss = self.train_step(x, target, B, lr)  # eager: sizes every workspace buffer
            xs = torch.empty_like(x)
            ts = torch.empty_like(target)
            self._adam_table(0.0)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                out = self.forward(xs, B)
                dout = self._buf("dout", out.shape)
                lbuf = self._buf("loss", (1,))
                lbuf.zero_()
                _lib.call("amhd_nn_mse", ptr(out), ptr(ts), out.numel(), ptr(dout), ptr(lbuf), stream_ptr())
                self.backward(dout, B)
                self._adam_launch(0.0)
            self._graphs[B] = (graph, xs, ts, lbuf)
            return loss.clone()
        graph, xs, ts, lbuf = g
        xs.copy_(x)
        ts.copy_(target)
        self.t += 1
        self._set_hyper(lr, 0.9, 0.999, 1e-8)
        graph.replay()
        return lbuf.clone()

    def loss(self, x: torch.Tensor, target: torch.Tensor, B: int) -> float:
        out = self.forward(x, B)
        loss = self._buf("loss", (1,))
        loss.zero_()
        _lib.call("amhd_nn_mse", ptr(out), ptr(target), out.numel(), None, ptr(loss), stream_ptr())
        self.check_gemm_status()
        return float(loss.item())

    # ------------------------------------------------- solver interaction
    def set_normalisation(self, in_mean, in_std, out_std):
        self.in_mean = torch.as_tensor(in_mean, dtype=F32, device=self.device)
        self.in_istd = 1.0 / torch.as_tensor(in_std, dtype=F32, device=self.device).clamp_min(1e-12)
        self.out_scale = torch.as_tensor(out_std, dtype=F32, device=self.device)

    def correct_state(self, state: torch.Tensor, grid: _lib.Grid) -> None:
        """Apply the corrector to one padded coarse state in place (interior; ghosts left stale)."""
        N = self.H * self.W
        x = self._buf("infer.x", (10, N))
        _lib.call("amhd_nn_pack", grid, ptr(state), ptr(self.in_mean), ptr(self.in_istd), ptr(x), N, 0, stream_ptr())
        y = self.forward(x, 1)
        self.check_gemm_status()  # an unwritten output must not reach the state
        _lib.call("amhd_nn_apply", grid, ptr(state), ptr(self.out_scale), ptr(y), N, 0, stream_ptr())

    def correct_solver(self, solver) -> None:
        self.correct_state(solver.U, solver._grid())
        solver.apply_bc(solver.U)


def pack_states(states: List[torch.Tensor], gamma: float, mean, istd, device="cuda") -> torch.Tensor:
    """[10][B*H*W] normalised network input from B padded solver states."""
    B = len(states)
    nx, ny = states[0].shape[1] - 4, states[0].shape[2] - 4
    N = nx * ny
    x = torch.empty((10, B * N), dtype=F32, device=device)
    for b, st in enumerate(states):
        g = make_grid(st, gamma)
        _lib.call("amhd_nn_pack", g, ptr(st), ptr(mean), ptr(istd), ptr(x), B * N, b, stream_ptr())
    return x
