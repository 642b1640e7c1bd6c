"""Drop-in replacement of the reference's physics module (physics.py).

Same function names, arguments and return values; arrays are PyTorch CUDA
tensors (numpy arrays are accepted and moved to the GPU), and every function
runs a kernel of libaeromhd.so:

    cons_to_prim(U, gamma)        physics.py:284-301
    prim_to_cons(W, gamma)        physics.py:304-320
    muscl_x(W), muscl_y(W)        physics.py:323-350  -> (WL, WR)
    hlld_flux_x(WL, WR, gamma, ch)  physics.py:353-370 -> (F, max smax)
    hlld_flux_y(WL, WR, gamma, ch)  physics.py:373-379
    mhd_rankine_hugoniot(...)     physics.py:385-429 (host, once per set-up)

``xp`` plays the role ``xp = cp`` plays in the reference: torch, with the
array constructors defaulting to float64 on the current CUDA device (numpy's
and CuPy's default dtype), so set-up code written for the reference builds
float64 GPU arrays.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._tensors import as_cuda, make_grid, ptr, stream_ptr
from .config import FLOOR_PR, FLOOR_RHO, NVAR  # noqa: F401  (re-exported like the reference)


class _TorchXP:
    """torch namespace whose constructors default to float64 on the GPU (numpy/CuPy defaults)."""

    _F64 = torch.float64

    def __getattr__(self, name):
        return getattr(torch, name)

    @staticmethod
    def _dev(device):
        return device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")

    def zeros(self, *shape, dtype=None, device=None):
        return torch.zeros(*shape, dtype=dtype or self._F64, device=self._dev(device))

    def ones(self, *shape, dtype=None, device=None):
        return torch.ones(*shape, dtype=dtype or self._F64, device=self._dev(device))

    def empty(self, *shape, dtype=None, device=None):
        return torch.empty(*shape, dtype=dtype or self._F64, device=self._dev(device))

    def full(self, shape, value, dtype=None, device=None):
        return torch.full(shape, value, dtype=dtype or self._F64, device=self._dev(device))

    def asarray(self, a, dtype=None, device=None):
        if isinstance(a, torch.Tensor):
            return a.to(device=self._dev(device), dtype=dtype or a.dtype)
        arr = np.asarray(a)
        dt = dtype or (self._F64 if arr.dtype.kind == "f" else None)
        return torch.as_tensor(arr, dtype=dt, device=self._dev(device))

    def arange(self, *args, dtype=None, device=None):
        return torch.arange(*args, dtype=dtype, device=self._dev(device))

    def linspace(self, start, stop, num, dtype=None, device=None):
        return torch.linspace(start, stop, num, dtype=dtype or self._F64, device=self._dev(device))

    def where(self, cond, a, b):
        def t(v):
            return v if isinstance(v, torch.Tensor) else torch.tensor(v, dtype=self._F64, device=cond.device)
        return torch.where(cond, t(a), t(b))

    def maximum(self, a, b):
        def t(v, ref):
            return v if isinstance(v, torch.Tensor) else torch.tensor(v, dtype=ref.dtype, device=ref.device)
        ref = a if isinstance(a, torch.Tensor) else b
        return torch.maximum(t(a, ref), t(b, ref))


xp = _TorchXP()


def _state_like(t: torch.Tensor) -> torch.Tensor:
    return torch.empty_strided(t.size(), t.stride(), dtype=t.dtype, device=t.device)


def _as_state(a) -> torch.Tensor:
    t = as_cuda(a)
    if t.dtype not in (torch.float64, torch.float32):
        t = t.to(torch.float64)
    if t.stride(-1) != 1:
        t = t.contiguous()
    return t


def cons_to_prim(U, gamma, limiter: int = 0):
    """Conservative -> primitive on every cell (physics.py:284-301)."""
    U = _as_state(U)
    W = _state_like(U)
    g = make_grid(U, gamma, limiter=limiter)
    _lib.call("amhd_cons_to_prim", g, ptr(U), ptr(W), stream_ptr())
    return W


def prim_to_cons(W, gamma):
    """Primitive -> conservative on every cell (physics.py:304-320)."""
    W = _as_state(W)
    U = _state_like(W)
    g = make_grid(W, gamma)
    _lib.call("amhd_prim_to_cons", g, ptr(W), ptr(U), stream_ptr())
    return U


def _muscl(W, axis: int, limiter: str = "vanleer"):
    W = _as_state(W)
    nv, nxt, nyt = W.shape
    shape = (nv, nxt - 3, nyt) if axis == 0 else (nv, nxt, nyt - 3)
    WL = torch.empty(shape, dtype=W.dtype, device=W.device)
    WR = torch.empty_like(WL)
    g = make_grid(W, 1.4, limiter=_lib.LIMITER_CODES[limiter])
    _lib.call("amhd_muscl", g, axis, ptr(W), ptr(WL), ptr(WR), stream_ptr())
    return WL, WR


def muscl_x(W, limiter: str = "vanleer"):
    """Limited linear reconstruction in x (physics.py:323-335): WL, WR of shape [10, nx+1, ny+4]."""
    return _muscl(W, 0, limiter)


def muscl_y(W, limiter: str = "vanleer"):
    """Limited linear reconstruction in y (physics.py:338-350): WL, WR of shape [10, nx+4, ny+1]."""
    return _muscl(W, 1, limiter)


def _hlld(WL, WR, gamma, ch, axis, return_smax_array=False):
    WL = _as_state(WL)
    WR = as_cuda(WR, WL.dtype)
    shape = WL.shape
    WLc = WL.reshape(NVAR, -1).contiguous()
    WRc = WR.reshape(NVAR, -1).contiguous()
    n = WLc.shape[1]
    F = torch.empty_like(WLc)
    smax = torch.empty(n, dtype=WL.dtype, device=WL.device)
    code = _lib.AMHD_F64 if WL.dtype == torch.float64 else _lib.AMHD_F32
    _lib.call("amhd_hlld_flux", axis, code, ptr(WLc), ptr(WRc), ptr(F), ptr(smax), n, float(gamma), float(ch),
              stream_ptr())
    if return_smax_array:
        return F.reshape(shape), smax
    return F.reshape(shape), (float(smax.max()) if n else 0.0)


def hlld_flux_x(WL, WR, gamma, ch, return_smax_array: bool = False):
    """HLLD face fluxes for x faces (physics.py:353-370); returns (F, max signal speed)."""
    return _hlld(WL, WR, gamma, ch, 0, return_smax_array)


def hlld_flux_y(WL, WR, gamma, ch, return_smax_array: bool = False):
    """HLLD face fluxes for y faces (physics.py:373-379)."""
    return _hlld(WL, WR, gamma, ch, 1, return_smax_array)


def mhd_rankine_hugoniot(gamma, M, rho1, p1, By1):
    """Post-shock state of a Mach-M fast shock into (rho1, p1, By1 transverse).

    The reference's set-up helper (physics.py:385-429), evaluated on the host
    once per run: the hydrodynamic jump conditions when By1 = 0, otherwise a
    Newton iteration (central-difference derivative, at most 100 steps, the
    compression ratio kept in (1.001, (g+1)/(g-1) - 0.001)) on the energy
    jump condition with momentum and flux freezing eliminated.
    Returns (rho2, p2, vx2, By2, shock speed)."""
    g = float(gamma)
    m2 = M * M
    r_hydro = (g + 1) * m2 / ((g - 1) * m2 + 2)
    if abs(By1) < 1e-14:
        vs = M * np.sqrt(g * p1 / rho1)
        p2 = p1 * (2 * g * m2 - (g - 1)) / (g + 1)
        return rho1 * r_hydro, p2, vs * (1 - 1.0 / r_hydro), 0.0, vs

    vs = M * np.sqrt(g * p1 / rho1 + By1 ** 2 / rho1)
    r_max = (g + 1) / (g - 1)

    def p_behind(r):
        return p1 + rho1 * vs ** 2 * (1 - 1.0 / r) + 0.5 * By1 ** 2 * (1 - r ** 2)

    upstream = 0.5 * vs ** 2 + g / (g - 1) * p1 / rho1 + By1 ** 2 / rho1

    def residual(r):
        return upstream - (0.5 * vs ** 2 / r ** 2 + g / (g - 1) * p_behind(r) / (rho1 * r) + r * By1 ** 2 / rho1)

    r = min(r_hydro, r_max - 0.01)
    for _ in range(100):
        f = residual(r)
        h = 1e-6 * r
        fp = (residual(r + h) - residual(r - h)) / (2 * h)
        if abs(fp) < 1e-30:
            break
        r_next = min(max(r - f / fp, 1.001), r_max - 0.001)
        if abs(r_next - r) < 1e-12:
            r = r_next
            break
        r = r_next
    return rho1 * r, p_behind(r), vs * (1 - 1.0 / r), r * By1, vs


__all__ = ["xp", "cons_to_prim", "prim_to_cons", "muscl_x", "muscl_y", "hlld_flux_x", "hlld_flux_y",
           "mhd_rankine_hugoniot", "NVAR", "FLOOR_RHO", "FLOOR_PR"]
