"""float32 state with float64 pressure recovery against float64 over the full
horizons of the benchmark configurations, where rounding error has the
longest time to accumulate:

* the single shocked interface, 2048 x 512 on [0, 4] x [0, 1], Mach 3,
  density ratio 3, Bx = 0.1, GLM + Powell, to t = 3 (about 40,000 steps),
  through ``MHDSolver.run()`` (diagnostics every 200 steps);
* the Orszag-Tang vortex, 512^2 to t = 0.5 (about 4,800 steps).

Both precisions start from the same state (the float64 initial state rounded
once).  Bar: relative L1 <= 1e-5 for every conserved variable of the final
state; psi, which starts at zero, as max |diff| <= 1e-5 of the mean |B|.  The
shocked interface also compares the float64 diagnostics of the two runs:
total mass and energy, the boundary energy and the mixing-width history."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BAR = 1e-5


def _pair(cfg64, cfg32, init):
    from aeromhd_cuda_b200 import cases
    from aeromhd_cuda_b200.solver import MHDSolver
    s64, s32 = MHDSolver(cfg64), MHDSolver(cfg32)
    init(s64)
    init(s32)
    cases.same_initial_state(s32, s64)
    return s32, s64


def test_shock_interface_2048x512_to_t3_fp32_within_1e5_of_fp64():
    from aeromhd_cuda_b200 import cases
    cfgs = [cases.shock_interface_config(2048, 512, p, t_end=3.0) for p in ("fp64", "fp32")]
    s32, s64 = _pair(cfgs[0], cfgs[1], lambda s: s.initialize())
    s64.run()
    s32.run()
    assert abs(s32.t - 3.0) < 1e-12 and abs(s64.t - 3.0) < 1e-12
    assert abs(s32.step - s64.step) <= 2, (s32.step, s64.step)
    err = cases.precision_errors(s32, s64)
    print("shocked interface t=3, fp32 vs fp64:", err, "steps", s32.step, s64.step)
    assert max(err.values()) <= BAR, err
    # float64 diagnostics of the two runs
    m32, m64 = np.array(s32.diag_mass_total), np.array(s64.diag_mass_total)
    e32, e64 = np.array(s32.diag_energy_total), np.array(s64.diag_energy_total)
    assert abs(m32[-1] - m64[-1]) <= BAR * abs(m64[-1])
    assert abs(e32[-1] - e64[-1]) <= BAR * abs(e64[-1])
    eb32, eb64 = s32._cumulative_boundary_energy, s64._cumulative_boundary_energy
    assert abs(eb32 - eb64) <= BAR * abs(e64[0]), (eb32, eb64)
    # mixing-width histories, sampled every 200 steps: compare at the float64 run's times
    t32, t64 = np.array(s32.diag_times), np.array(s64.diag_times)
    mw32 = np.interp(t64, t32, np.array(s32.diag_mixing_width_integral))
    mw64 = np.array(s64.diag_mixing_width_integral)
    dev = float(np.max(np.abs(mw32 - mw64)) / np.max(np.abs(mw64)))
    print("mixing-width history: max |diff| / peak", dev)
    assert dev <= 1e-3, dev


def test_orszag_tang_512_to_t05_fp32_within_1e5_of_fp64():
    from aeromhd_cuda_b200 import cases, initial_conditions as ic
    cfgs = [cases.orszag_tang_config(512, p, t_end=0.5) for p in ("fp64", "fp32")]
    s32, s64 = _pair(cfgs[0], cfgs[1], lambda s: s.set_primitive(ic.orszag_tang(s)))
    s64.advance(chunk=200)
    s32.advance(chunk=200)
    assert abs(s32.t - 0.5) < 1e-12 and abs(s64.t - 0.5) < 1e-12
    err = cases.precision_errors(s32, s64)
    print("Orszag-Tang 512^2 t=0.5, fp32 vs fp64:", err, "steps", s32.step, s64.step)
    assert max(err.values()) <= BAR, err
