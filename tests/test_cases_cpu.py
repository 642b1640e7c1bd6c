"""The runnable benchmark cases are configured as stated (no GPU needed)."""
import math

from aeromhd_cuda_b200 import cases
from aeromhd_cuda_b200.initial_conditions import cp_alfven_box


def test_shock_interface_case_parameters():
    c = cases.shock_interface_config()
    assert (c.nx, c.ny, c.x_min, c.x_max, c.y_min, c.y_max) == (2048, 512, 0.0, 4.0, 0.0, 1.0)
    assert c.mach == 3.0 and c.shock_x == 0.5 and c.interface_x == 1.0
    assert c.perturbation_amp == 0.05 and c.perturbation_mode == 2 and c.perturbation_shape == "cos"
    assert c.density_ratio == 3.0 and c.interface_cells == 2.0 and c.bx0 == 0.1 and c.noise_amp == 1e-3
    assert c.gamma == 5.0 / 3.0 and c.bc_y_type == "periodic" and c.get_bc_x() == "extrapolation"
    assert c.powell_enabled() and c.t_end == 3.0 and c.precision == "fp32"


def test_orszag_tang_case_parameters():
    c = cases.orszag_tang_config(512, "fp64")
    assert (c.nx, c.ny, c.x_max, c.y_max, c.t_end) == (512, 512, 1.0, 1.0, 0.5)
    assert c.get_bc_x() == "periodic" and c.bc_y_type == "periodic" and c.gamma == 5.0 / 3.0


def test_cp_alfven_box_holds_one_wavelength():
    lx, ly = cp_alfven_box(30.0)
    a = math.radians(30.0)
    assert abs(lx * math.cos(a) - 1.0) < 1e-15 and abs(ly * math.sin(a) - 1.0) < 1e-15


def test_reference_driver_cases_parameters():
    """The reference drivers' shocked-interface set-up (main.py:446-458) and the
    convergence study's resolutions and diagnostic cadence (main.py:306-312, :476-492)."""
    r = cases.REFERENCE_RMI
    assert (r["nx"], r["ny"], r["x_max"], r["y_max"], r["t_end"], r["mach"]) == (400, 200, 6.0, 2.0, 0.25, 10.0)
    assert r["bc_x_type"] == "characteristic" and r["powell_source"] and r["use_char_bc"]
    assert cases.REFERENCE_RMI_CASES == {"Hydro (B=0)": 0.0, "MHD (By=0.5)": 0.5, "MHD (By=1.5)": 1.5}
    for nx, ny, every in ((100, 50, 40), (200, 100, 20), (400, 200, 10)):
        c = cases.convergence_config(nx, ny, 1.5)
        assert (c.nx, c.ny, c.t_end, c.diag_interval, c.B_transverse) == (nx, ny, 0.15, every, 1.5)
        assert c.snapshot_times == [0.0, 0.15] and c.precision == "fp64"


def test_bench_launch_counts_and_committed_profile():
    """bench.py's launch counts (4 per run-loop step and one ghost fill per loop
    call with the marching kernel; stage + fill per stage in the row-split loop)
    and the figures it reads from the committed ncu summary."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.loop_launches(-24, 1000) == 4001 and bench.loop_launches(8, 10) == 40
    assert bench.split_launches(-24, 10) == 70 and bench.split_launches(8, 10) == 40
    tr = bench.profile_traffic(-24)
    assert tr["precision"] == "fp32" and int(tr["n"]) > 0 and float(tr["dram_bytes_per_step"]) > 0
    assert 0 < float(tr["issue_active_pct"]) <= 100
