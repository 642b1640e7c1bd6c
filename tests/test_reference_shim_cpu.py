"""The stand-ins that run the reference's own modules without CuPy
(baseline/refshim.py): the torch-backed one, on the CPU, reproduces the
numpy-backed one bit for bit over three steps of the reference's step loop on
the Orszag-Tang vortex, and the numpy-backed one reproduces this repository's
float64 oracle.  The torch-backed stand-in is the one the benchmark runs on
the GPU as the reference's CuPy path; this pins its array semantics (float64
defaults, scalar operands, slicing, the HLLD kernel call) on the CPU.  Each
run is a subprocess: a process imports the reference over one stand-in.
Skipped when the reference modules are not available (baseline/_ref or
AMHD_REFERENCE_DIR)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "baseline", "run_reference.py")


def _have_reference():
    from conftest import reference_available
    return reference_available()


pytestmark = pytest.mark.skipif(not _have_reference(), reason="reference modules not available")


def _run(tmp_path, backend, n=48, steps=3, device="cpu"):
    out, init = tmp_path / f"{backend}.npy", tmp_path / f"{backend}_0.npy"
    r = subprocess.run([sys.executable, RUNNER, "--backend", backend, "--device", device, "--n", str(n),
                        "--check-steps", str(steps), "--out", str(out), "--out-initial", str(init)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["steps"] == steps, info
    return np.load(init), np.load(out), info


def test_torch_stand_in_equals_numpy_stand_in_bitwise(tmp_path):
    i_np, u_np, a = _run(tmp_path, "numpy")
    i_t, u_t, b = _run(tmp_path, "torch")
    assert np.array_equal(i_np, i_t)
    assert a["dt"] == b["dt"] and a["glm_ch"] == b["glm_ch"]
    assert np.array_equal(u_np, u_t), float(np.abs(u_np - u_t).max())


def test_numpy_stand_in_equals_the_oracle(tmp_path, oracle):
    from aeromhd_cuda_b200 import cases
    init, ref, info = _run(tmp_path, "numpy", n=40, steps=3)
    o = oracle.OracleSolver(cases.orszag_tang_config(40, "fp64", t_end=1e30))
    o.U = init.copy()
    for _ in range(3):
        o.dt = o.compute_dt(oracle.cons_to_prim(o.U, o.cfg.gamma))
        o.step_ssprk3()
        o.t += o.dt
    assert o.dt == info["dt"]
    assert np.array_equal(o.U, ref)
