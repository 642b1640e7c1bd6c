"""The reference drivers' shocked-interface studies on the device loop.

run_convergence_study (main.py:294-396) at its first resolution (100 x 50,
the driver set-up of main.py:446-458 to t = 0.15, By = 0 and 1.5):
MHDSolver.run() -- device loop, diagnostics every diag_interval steps --
against the float64 CPU oracle advanced from the same initial state, with the
reference's integral mixing width (solver.py:350-355) evaluated in numpy on
the oracle's state at the same steps.  The device loop takes its psi damping
factor from the device's exp(), so the bar is 1e-12 relative (not bitwise)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def mixing_width_integral(O, U, gamma, x_int):
    W = O.cons_to_prim(U, gamma)
    C = np.clip(W[9, 2:-2, 2:-2], 0.0, 1.0)
    c_bar = np.mean(C, axis=1)
    return float(np.trapezoid(c_bar * (1.0 - c_bar), x_int))


@pytest.mark.parametrize("by", [0.0, 1.5])
def test_convergence_study_resolution_matches_oracle(oracle, by):
    from aeromhd_cuda_b200 import cases
    from aeromhd_cuda_b200.solver import MHDSolver, to_numpy
    O = oracle
    cfg = cases.convergence_config(100, 50, by, "fp64")
    s = MHDSolver(cfg)
    s.initialize()
    U0 = to_numpy(s.U).astype(np.float64)
    s.run()

    o = O.OracleSolver(cases.convergence_config(100, 50, by, "fp64"))
    o.U = U0.copy()
    x_int = o.x[2:-2]
    hist = [mixing_width_integral(O, o.U, cfg.gamma, x_int)]   # run() records the initial state first

    def on_step(sol):
        if sol.step % cfg.diag_interval == 0:
            hist.append(mixing_width_integral(O, sol.U, cfg.gamma, x_int))

    o.advance(on_step=on_step)
    hist.append(mixing_width_integral(O, o.U, cfg.gamma, x_int))   # run() ends with the final state's
    assert s.step == o.step and abs(s.t - o.t) <= 1e-15
    dev = list(s.diag_mixing_width_integral)
    assert len(dev) == len(hist), (len(dev), len(hist))
    np.testing.assert_allclose(dev, hist, rtol=1e-10, atol=1e-14)
    err = float(np.abs(to_numpy(s.U) - o.U).sum() / np.abs(o.U).sum())
    assert err < 1e-12, err
    peak = cases._peak_after(s, s.diag_mixing_width_integral)
    assert peak > 0.0
    print(f"By={by}: {s.step} steps, peak integral mixing width {peak:.6f}, state rel L1 vs oracle {err:.2e}")
