"""TEST INFRASTRUCTURE ONLY: a CPU stand-in for decomp.GpuBackend built on the
float64 oracle, so that the row-split run loop (halo exchange, CFL max
reduction, finish) runs as gloo ranks on CPU.  Each piece follows the device
loop's semantics: a stage = the reference's SSP-RK3 stage on the local block
with its ghosts as given (oracle compute_rhs with x ghosts left alone), the
scalar clamp, psi damping on stage 3, then the local boundary fill; stage 3
and the loop start collect the CFL maxima (ordered float64 bits); finish
restates the device finalize (t, step, dt = min(cfl / max speed, t_end - t),
ch, damping, and the boundary energy of the block's physical x sides,
solver.py:225-240)."""
import ctypes
import math

import numpy as np
import torch

from oracle import oracle as O

NG = 2
BC_NONE = 3  # oracle code: x ghost rows left as they are


def _bits(x):
    return np.float64(x).view(np.int64)


def _val(b):
    return float(np.int64(b).view(np.float64))


class OracleBackend:
    def __init__(self, cfg, r0, r1):
        from aeromhd_cuda_b200.config import BC_PERIODIC, bc_x_code, bc_y_code
        from aeromhd_cuda_b200.decomp import cut_sides
        self.cfg = cfg
        self.n = r1 - r0
        self.cut_x = cut_sides(r0, r1, cfg.nx)
        self.periodic_x = bc_x_code(cfg) == BC_PERIODIC
        self.bc_x, self.bc_y = bc_x_code(cfg), bc_y_code(cfg)
        shape = (10, self.n + 2 * NG, cfg.ny + 2 * NG)
        self.bufs = tuple(torch.zeros(shape, dtype=torch.float64) for _ in range(3))
        self._red = torch.zeros(4, dtype=torch.int64)
        self.c = dict(t=0.0, t_end=0.0, dt=0.0, ch=0.0, decay=1.0, step=0, max_steps=0, active=0, e_bnd=0.0)

    def _boundary_flux(self, U):
        """solver.py:225-240 on the block's physical sides: the flux in through
        its first row minus the flux out through its last."""
        g, dy = self.cfg.gamma, self.cfg.dy
        W = O.cons_to_prim(U, g)

        def side(i):
            w, e = W[:, i, NG:-NG], U[7, i, NG:-NG]
            pt = w[7] + 0.5 * (w[4] ** 2 + w[5] ** 2 + w[6] ** 2)
            vb = w[1] * w[4] + w[2] * w[5] + w[3] * w[6]
            return float(np.sum(((e + pt) * w[1] - w[4] * vb) * dy))
        left = 0.0 if self.cut_x & 1 else side(NG)
        right = 0.0 if self.cut_x & 2 else side(self.n + NG - 1)
        return left - right

    def state(self, k):
        return self.bufs[k]

    def red(self):
        return self._red

    def _fill(self, A):
        O.lib().orc_apply_bc(A.numpy().ctypes.data_as(ctypes.c_void_p), A.shape[1], A.shape[2], self.bc_x, self.bc_y)

    def _maxima(self, A, interior):
        W = O.cons_to_prim(A.numpy(), self.cfg.gamma)
        if interior:
            W = W[:, NG:-NG, NG:-NG]
        b2 = W[4] ** 2 + W[5] ** 2 + W[6] ** 2
        q = (self.cfg.gamma * W[7] / W[0] + b2 / W[0], np.abs(W[1]) + np.abs(W[2]), np.abs(W[1]), np.abs(W[2]))
        m = torch.tensor([_bits(np.max(x)) for x in q], dtype=torch.int64)
        self._red.copy_(torch.maximum(self._red, m))

    def control_init_split(self, t, t_end, step, max_steps):
        self.c.update(t=t, t_end=t_end, step=step, max_steps=max_steps, active=1, decay=1.0, e_bnd=0.0)
        self._red.zero_()
        self._maxima(self.bufs[0], interior=False)
        self._fill(self.bufs[0])

    def stage(self, k):
        cfg = self.cfg
        U0, U1, U2 = (b.numpy() for b in self.bufs)
        Uin = (U0, U1, U2)[k - 1]
        out = (U1, U2, U0)[k - 1]
        R = np.zeros_like(Uin)
        W = np.empty_like(Uin)
        src = np.ascontiguousarray(Uin)
        O.lib().orc_compute_rhs(src.ctypes.data_as(ctypes.c_void_p), self.n, cfg.ny, float(cfg.gamma),
                                float(cfg.dx), float(cfg.dy), BC_NONE, self.bc_y, int(cfg.powell_enabled()),
                                float(self.c["ch"]), W.ctypes.data_as(ctypes.c_void_p),
                                R.ctypes.data_as(ctypes.c_void_p))
        dt = self.c["dt"]
        if k == 1:
            new = U0 + dt * R
        elif k == 2:
            new = 0.75 * U0 + 0.25 * (src + dt * R)
        else:
            new = (1.0 / 3.0) * U0 + (2.0 / 3.0) * (src + dt * R)
        rho = np.maximum(new[0], 1e-12)
        new[9] = rho * np.clip(new[9] / rho, 0.0, 1.0)
        if k == 3 and self.c["ch"] > 0:
            new[8] *= self.c["decay"]
        out[:] = new
        self._fill(self.bufs[k % 3])
        if k == 3:
            self._maxima(self.bufs[0], interior=True)

    def finish(self, advance):
        c, cfg = self.c, self.cfg
        if not (c["active"] or not advance):
            self._red.zero_()
            return
        if advance:
            c["t"] += c["dt"]
            c["step"] += 1
        if c["t"] < c["t_end"] and c["step"] < c["max_steps"]:
            r = [_val(x) for x in self._red.tolist()]
            ch = max(1.0, math.sqrt(r[0]) + r[1]) * 1.5
            sx, sy = (r[2] + ch) / cfg.dx, (r[3] + ch) / cfg.dy
            dtc = cfg.cfl / max(sx, sy)
            dt = min(c["t_end"] - c["t"], dtc)
            c.update(ch=ch, dt=dt, active=int(dt > 1e-16),
                     decay=math.exp(-cfg.glm_alpha * ch * dt / min(cfg.dx, cfg.dy)))
            if c["active"] and not self.periodic_x:
                c["e_bnd"] += self._boundary_flux(self.bufs[0].numpy()) * dt
        else:
            c["active"] = 0
        self._red.zero_()
