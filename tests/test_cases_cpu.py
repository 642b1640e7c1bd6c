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
