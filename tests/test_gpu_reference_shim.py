"""The reference's CuPy path on the GPU (the reference's modules, unchanged,
over the torch-backed CuPy stand-in of baseline/refshim.py, its HLLD kernel
string compiled by NVRTC) against this library's float64 solver from the same
initial state: the timed comparator of the benchmark computes what the
library computes.  NVRTC contracts multiply-adds by default (as CuPy's
RawKernel does), so the two differ in the last bits: the bar is 1e-12
relative L1 after three steps, and dt within 1e-13.  Skipped when the
reference modules are not available."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "baseline", "run_reference.py")

pytestmark = pytest.mark.gpu


def _have_reference():
    from conftest import reference_available
    return reference_available()


@pytest.mark.skipif(not _have_reference(), reason="reference modules not available")
def test_reference_cupy_path_on_gpu_matches_the_fp64_solver(tmp_path):
    from aeromhd_cuda_b200 import cases
    from aeromhd_cuda_b200.physics import cons_to_prim
    from aeromhd_cuda_b200.solver import MHDSolver
    n, steps = 64, 3
    out, init = tmp_path / "u.npy", tmp_path / "u0.npy"
    r = subprocess.run([sys.executable, RUNNER, "--backend", "torch", "--device", "cuda", "--n", str(n),
                        "--check-steps", str(steps), "--out", str(out), "--out-initial", str(init)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert "unavailable" not in info, info
    ref = np.load(out)
    s = MHDSolver(cases.orszag_tang_config(n, "fp64", t_end=1e30))
    s.U = np.load(init)
    for _ in range(steps):
        s.dt = s.compute_dt(cons_to_prim(s.U, s.cfg.gamma))
        s.step_ssprk3()
        s.t += s.dt
    got = s.U.cpu().numpy()
    assert abs(s.dt - info["dt"]) <= 1e-13 * info["dt"]
    err = np.abs(got - ref)[:, 2:-2, 2:-2].sum() / np.abs(ref)[:, 2:-2, 2:-2].sum()
    assert err < 1e-12, err


@pytest.mark.skipif(not _have_reference(), reason="reference modules not available")
def test_reference_cupy_path_timing_runs():
    r = subprocess.run([sys.executable, RUNNER, "--backend", "torch", "--device", "cuda", "--n", "256",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["finite"] and info["zone_updates_per_s"] > 0 and "torch-shim" in info["stand_in"], info
