"""Device colour-field diagnostics (amhd_diagnostics_colour) against the
reference's numpy formulas (solver.py:358-383) evaluated on the host from the
same state: per-row colour variance and per-column interface positions,
including columns without an interface (NaN) and ties of |dC/dx|."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def host_reference(U, dx, x_arr):
    """solver.py:358-378 restated in numpy on the host (test oracle only)."""
    rho = np.maximum(U[0, 2:-2, 2:-2], 1e-12)
    C = np.clip(U[9, 2:-2, 2:-2] * (1.0 / rho), 0.0, 1.0)
    nx, ny = C.shape
    C_bar = C.sum(axis=1) / ny
    cp2 = np.mean((C - C_bar[:, None]) ** 2, axis=1)
    grad = np.abs(np.gradient(C, dx, axis=0))
    pos = np.full(ny, np.nan)
    peak = np.argmax(grad, axis=0)
    for j in np.nonzero(grad.max(axis=0) > 1e-6)[0]:
        ip = int(peak[j])
        hw = min(10, ip, nx - ip - 1)
        if hw > 0:
            wgt = grad[ip - hw:ip + hw + 1, j]
            ws = np.sum(wgt)
            if ws > 1e-12:
                pos[j] = np.sum(x_arr[ip - hw:ip + hw + 1] * wgt) / ws
    return cp2, pos


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_colour_rows_and_interface_positions(precision):
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import ptr, stream_ptr
    from aeromhd_cuda_b200.config import Config
    from aeromhd_cuda_b200.solver import MHDSolver
    s = MHDSolver(Config(nx=120, ny=48, B_transverse=0.2, t_end=1.0, precision=precision))
    s.initialize()
    s.advance(max_steps=60, chunk=30)
    U = s.U.detach().cpu().numpy().astype(np.float64)
    # columns 0-5: no interface (C uniform along x); columns 6-7: a step with a
    # tie of |dC/dx| between two rows; column 8: the step at the first row
    U[9, :, 2:8] = 0.5 * U[0, :, 2:8]
    U[9, :, 8:10] = 0.0
    U[9, 60:, 8:10] = U[0, 60:, 8:10]
    U[9, 70, 8:10] = 0.5 * U[0, 70, 8:10]
    U[9, 2:3, 10] = U[0, 2:3, 10]
    s.U = U
    g = s._grid()
    nx, ny = s.cfg.nx, s.cfg.ny
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    rows = torch.zeros(7 * nx, dtype=torch.float64, device="cuda")
    cp2 = torch.zeros(nx, dtype=torch.float64, device="cuda")
    pos = torch.zeros(ny, dtype=torch.float64, device="cuda")
    _lib.call("amhd_diagnostics", g, ptr(s.U), float(s.cfg.x_min), ptr(out), ptr(rows), stream_ptr())
    _lib.call("amhd_diagnostics_colour", g, ptr(s.U), float(s.cfg.x_min), ptr(rows), ptr(cp2), ptr(pos),
              stream_ptr())
    x_arr = s.cfg.x_min + (np.arange(nx) + 0.5) * s.cfg.dx
    ref_cp2, ref_pos = host_reference(np.asarray(s.U.cpu(), dtype=np.float64), s.cfg.dx, x_arr)
    d_cp2, d_pos = cp2.cpu().numpy() / ny, pos.cpu().numpy()
    np.testing.assert_allclose(d_cp2, ref_cp2, rtol=1e-12, atol=1e-15)
    assert np.array_equal(np.isnan(d_pos), np.isnan(ref_pos))
    assert np.isnan(d_pos[:6]).all() and not np.isnan(d_pos).all()
    ok = ~np.isnan(ref_pos)
    # same operations in the same order (numpy's pairwise sums): equal to the last bits
    np.testing.assert_allclose(d_pos[ok], ref_pos[ok], rtol=1e-14, atol=0)
