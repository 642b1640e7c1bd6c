"""Tensor plumbing between PyTorch and the C ABI: dtype codes, grid
descriptors built from tensor strides, the current stream, padded states."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .config import NVAR, BC_PERIODIC

NG = 2


def as_cuda(a, dtype=None) -> torch.Tensor:
    """numpy array or tensor -> CUDA tensor (no copy when already suitable)."""
    if isinstance(a, np.ndarray):
        a = torch.from_numpy(np.ascontiguousarray(a))
    if not isinstance(a, torch.Tensor):
        raise TypeError(f"expected a torch.Tensor or numpy array, got {type(a)!r}")
    if dtype is not None and a.dtype != dtype:
        a = a.to(dtype)
    if a.device.type != "cuda":
        if not torch.cuda.is_available():
            raise RuntimeError("a CUDA device is required (the solver has no CPU path)")
        a = a.to("cuda")
    return a


def dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float64:
        return _lib.AMHD_F64
    if t.dtype == torch.float32:
        return _lib.AMHD_F32
    raise TypeError(f"state arrays must be float64 or float32, got {t.dtype}")


def torch_dtype(precision: str) -> torch.dtype:
    return torch.float64 if precision == "fp64" else torch.float32


def stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def make_grid(state: torch.Tensor, gamma: float, dx: float = 1.0, dy: float = 1.0, cfl: float = 0.3,
              glm_alpha: float = 1.5, bc_x: int = BC_PERIODIC, bc_y: int = BC_PERIODIC, powell: bool = False,
              limiter: int = 0) -> _lib.Grid:
    """Grid descriptor of a [10, nx+4, ny+4] tensor whose last axis is unit-stride."""
    if state.dim() != 3 or state.shape[0] != NVAR:
        raise ValueError(f"state must have shape [10, nx+4, ny+4], got {tuple(state.shape)}")
    if state.stride(2) != 1:
        raise ValueError("state's last axis must be contiguous")
    g = _lib.Grid()
    g.nx = state.shape[1] - 2 * NG
    g.ny = state.shape[2] - 2 * NG
    g.pitch = state.stride(1)
    g.var_stride = state.stride(0)
    g.dtype = dtype_code(state)
    g.dx, g.dy = float(dx), float(dy)
    g.gamma, g.cfl, g.glm_alpha = float(gamma), float(cfl), float(glm_alpha)
    g.bc_x, g.bc_y = int(bc_x), int(bc_y)
    g.powell = int(bool(powell))
    g.limiter = int(limiter)
    return g


def padded_state(nx: int, ny: int, dtype: torch.dtype, device="cuda"):
    """Zeroed storage in the padded layout of the fused kernels, and its
    [10, nx+4, ny+4] view."""
    code = _lib.AMHD_F64 if dtype == torch.float64 else _lib.AMHD_F32
    pitch, rows = _lib.padded_layout(nx, ny, code)
    storage = torch.zeros((NVAR, rows, pitch), dtype=dtype, device=device)
    view = storage[:, : nx + 2 * NG, : ny + 2 * NG]
    return storage, view


def is_padded(t: torch.Tensor) -> bool:
    nx, ny = t.shape[1] - 2 * NG, t.shape[2] - 2 * NG
    code = dtype_code(t)
    pitch, rows = _lib.padded_layout(nx, ny, code)
    es = t.element_size()
    return (t.stride(2) == 1 and t.stride(1) >= pitch and t.stride(0) >= rows * t.stride(1)
            and (t.stride(1) * es) % 16 == 0 and (t.stride(0) * es) % 16 == 0 and t.data_ptr() % 16 == 0)


def control_tensor(n: int = 1, device="cuda") -> torch.Tensor:
    size = ctypes.sizeof(_lib.Control)
    return torch.zeros((n, size), dtype=torch.uint8, device=device)


def write_controls(ctl: torch.Tensor, controls) -> None:
    """List of ctypes Control -> device control blocks (synchronous copy)."""
    size = ctypes.sizeof(_lib.Control)
    raw = bytearray(size * len(controls))
    for k, c in enumerate(controls):
        raw[k * size:(k + 1) * size] = bytes(c)
    ctl.copy_(torch.frombuffer(raw, dtype=torch.uint8).view(len(controls), size))


def read_controls(ctl: torch.Tensor):
    """Device control blocks -> list of ctypes Control (synchronises)."""
    raw = ctl.cpu().numpy()
    out = []
    for k in range(raw.shape[0]):
        c = _lib.Control()
        ctypes.memmove(ctypes.addressof(c), raw[k].ctypes.data, ctypes.sizeof(c))
        out.append(c)
    return out
