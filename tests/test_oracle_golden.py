"""The CPU oracle against outputs of the reference itself (tests/golden).

The oracle keeps the reference's operation order and is built without FMA
contraction, so every comparison here is bit-exact (np.array_equal) except
the boundary-energy diagnostic, whose sum order differs (rtol 1e-12).
"""
import numpy as np
import pytest

from aeromhd_cuda_b200.config import Config
from conftest import golden

STEP_CASES = [(bx, by, B) for bx in ("periodic", "extrapolation", "characteristic")
              for by in ("periodic", "outflow") for B in (0.0, 0.5)]


def test_hlld_faces_bit_exact(oracle):
    g = golden("hlld_faces.npz")
    for k, ch in enumerate(g["chs"]):
        F, _ = oracle.hlld_flux_x(g["WL"], g["WR"], g["gamma"], ch)
        assert np.array_equal(F, g[f"Fx_{k}"])
        assert np.array_equal(oracle.hlld_face_smax(g["WL"], g["WR"], g["gamma"], ch), g[f"smaxx_{k}"])
        F, _ = oracle.hlld_flux_y(g["WL"], g["WR"], g["gamma"], ch)
        assert np.array_equal(F, g[f"Fy_{k}"])
        assert np.array_equal(oracle.hlld_face_smax(g["WL"], g["WR"], g["gamma"], ch, y=True), g[f"smaxy_{k}"])


def test_hlld_golden_covers_every_region():
    """The fixture must exercise all six flux regions of the kernel (physics.py:177-263)."""
    g = golden("hlld_faces.npz")
    WL, WR, gamma = g["WL"], g["WR"], float(g["gamma"])
    regions = set()
    for ch in g["chs"]:
        for i in range(WL.shape[1]):
            regions.add(_region(WL[:, i], WR[:, i], gamma, ch))
    assert regions == {"L", "R", "LS", "LDS", "RDS", "RS"}


def _region(wl, wr, gamma, ch):
    # a plain-python restatement of the wave-speed part, only to classify faces
    rl, rr = max(wl[0], 1e-12), max(wr[0], 1e-12)
    pl, pr = max(wl[7], 1e-12), max(wr[7], 1e-12)
    if ch > 0:
        bxf = 0.5 * (wl[4] + wr[4]) - 0.5 / ch * (wr[8] - wl[8])
    else:
        bxf = 0.5 * (wl[4] + wr[4])
    bx2 = bxf * bxf

    def cf(r, p, by, bz):
        bm2 = bx2 + by * by + bz * bz
        a2 = gamma * p / r
        tmp = a2 + bm2 / r
        disc = max(tmp * tmp - 4.0 * a2 * bx2 / r, 0.0)
        return np.sqrt(max(0.5 * (tmp + np.sqrt(disc)), 0.0))

    cl, cr = cf(rl, pl, wl[5], wl[6]), cf(rr, pr, wr[5], wr[6])
    SL = min(wl[1] - cl, wr[1] - cr)
    SR = max(wl[1] + cl, wr[1] + cr)
    if ch > 0:
        SL, SR = min(SL, -ch), max(SR, ch)
    if SL >= 0:
        return "L"
    if SR <= 0:
        return "R"
    ptl, ptr = pl + 0.5 * (bx2 + wl[5] ** 2 + wl[6] ** 2), pr + 0.5 * (bx2 + wr[5] ** 2 + wr[6] ** 2)
    dsl, dsr = SL - wl[1], SR - wr[1]
    den = dsr * rr - dsl * rl
    if abs(den) < 1e-14:
        den = 1e-14 if den >= 0 else -1e-14
    SM = (dsr * rr * wr[1] - dsl * rl * wl[1] - ptr + ptl) / den
    SM = min(max(SM, SL + 1e-14), SR - 1e-14)
    d1 = SL - SM if abs(SL - SM) >= 1e-14 else 1e-14
    d2 = SR - SM if abs(SR - SM) >= 1e-14 else 1e-14
    rls, rrs = max(rl * dsl / d1, 1e-12), max(rr * dsr / d2, 1e-12)
    SAL = min(max(SM - abs(bxf) / max(np.sqrt(rls), 1e-14), SL), SM)
    SAR = min(max(SM + abs(bxf) / max(np.sqrt(rrs), 1e-14), SM), SR)
    if SAL >= 0:
        return "LS"
    if SM >= 0:
        return "LDS"
    if SAR >= 0:
        return "RDS"
    return "RS"


def test_conversions_and_muscl_bit_exact(oracle):
    g = golden("conversions.npz")
    W = oracle.cons_to_prim(g["U"], g["gamma"])
    assert np.array_equal(W, g["W"])
    assert np.array_equal(oracle.prim_to_cons(g["W"], g["gamma"]), g["U2"])
    WL, WR = oracle.muscl_x(g["W"])
    assert np.array_equal(WL, g["WLx"]) and np.array_equal(WR, g["WRx"])
    WL, WR = oracle.muscl_y(g["W"])
    assert np.array_equal(WL, g["WLy"]) and np.array_equal(WR, g["WRy"])


def _step_cfg(bcx, bcy, By):
    return Config(nx=10, ny=8, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.8, cfl=0.3, gamma=5.0 / 3.0,
                  B_transverse=By, powell_source=True, bc_x_type=bcx, bc_y_type=bcy, glm_alpha=1.5)


@pytest.mark.parametrize("k", range(len(STEP_CASES)))
def test_three_steps_bit_exact(oracle, k):
    g = golden("steps.npz")
    cfg = _step_cfg(*STEP_CASES[k])
    s = oracle.OracleSolver(cfg)
    s.U = g[f"U0_{k}"].copy()
    for n in range(3):
        W = oracle.cons_to_prim(s.U, cfg.gamma)
        s.dt = s.compute_dt(W)
        assert s.dt == g[f"dt_{k}"][n]
        assert cfg.glm_ch == g[f"ch_{k}"][n]
        s.step_ssprk3()
    assert np.array_equal(s.U, g[f"U3_{k}"])
    np.testing.assert_allclose(s._cumulative_boundary_energy, g[f"ebnd_{k}"], rtol=1e-12, atol=1e-15)


def test_single_routines_bit_exact(oracle):
    g = golden("steps.npz")
    cfg = _step_cfg("periodic", "outflow", 0.5)
    cfg.glm_ch = 2.0
    s = oracle.OracleSolver(cfg)
    s._glm_ch_frozen = 2.0
    U = g["rhs_U"].copy()
    R = s.compute_rhs(U)
    assert np.array_equal(U, g["rhs_Ubc"])       # apply_bc mutates its argument (solver.py:276)
    assert np.array_equal(R, g["rhs_R"])
    S = s._compute_powell_source(U, oracle.cons_to_prim(U, cfg.gamma))
    assert np.array_equal(S, g["rhs_S"])
    Uc = g["bounds_in"].copy()
    assert np.array_equal(s.enforce_scalar_bounds(Uc), g["bounds_out"])


def brio_wu_cfg(nx):
    return Config(nx=nx, ny=4, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.05, t_end=0.1, cfl=0.30, gamma=2.0,
                  mach=1.0, B_transverse=0.0, interface_x=0.5, perturbation_amp=0.0, density_ratio=1.0,
                  powell_source=False, use_char_bc=False, bc_x_type="extrapolation", bc_y_type="periodic")


@pytest.mark.parametrize("nx", [200, 800])
def test_brio_wu_bit_exact(oracle, nx):
    g = golden("brio_wu.npz")
    cfg = brio_wu_cfg(nx)
    s = oracle.OracleSolver(cfg)
    s.U = np.repeat(g[f"U0_{nx}"][:, :, None], s.ny_tot, axis=2).copy()
    s.advance()
    assert s.step == int(g[f"steps_{nx}"])
    assert s.t == float(g[f"t_{nx}"])
    assert np.array_equal(s.U[:, :, 2], g[f"row_{nx}"])
    assert np.all(s.U == s.U[:, :, 2:3])


def test_brio_wu_reference_checks(oracle):
    """main.py:88-97 pass criteria on the oracle's own 800-cell run."""
    cfg = brio_wu_cfg(800)
    g = golden("brio_wu.npz")
    s = oracle.OracleSolver(cfg)
    s.U = np.repeat(g["U0_800"][:, :, None], s.ny_tot, axis=2).copy()
    s.advance_native()
    W = oracle.cons_to_prim(s.U, cfg.gamma)
    rho, By, vx = W[0, 2:-2, 2], W[5, 2:-2, 2], W[1, 2:-2, 2]
    assert 0.1 < rho.min() < 0.18 and 0.9 < rho.max() < 1.05
    assert len(np.unique(np.round(rho, 2))) > 10
    assert np.any(By[:-1] * By[1:] < 0)
    assert vx.max() - vx.min() > 0.5


def test_alfven_convergence(oracle):
    g = golden("alfven.npz")
    errs = []
    for k, nx in enumerate(g["resolutions"]):
        nx = int(nx)
        cfg = Config(nx=nx, ny=4, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.05, t_end=float(g["period"]), cfl=0.25,
                     gamma=5.0 / 3.0, B_transverse=0.0, powell_source=False, use_char_bc=False,
                     bc_x_type="periodic", bc_y_type="periodic")
        s = oracle.OracleSolver(cfg)
        s.U = np.repeat(g[f"U0_{nx}"][:, :, None], s.ny_tot, axis=2).copy()
        W0 = oracle.cons_to_prim(s.U, cfg.gamma)
        s.advance(max_steps=100000)
        assert s.step == int(g["steps"][k])
        assert np.array_equal(s.U[:, :, 2], g[f"row_{nx}"])
        W = oracle.cons_to_prim(s.U, cfg.gamma)
        errs.append(float(np.mean(np.abs(W[5, 2:-2, 2] - W0[5, 2:-2, 2]))))
    np.testing.assert_allclose(errs, g["L1"], rtol=1e-9)
    res = g["resolutions"]
    orders = [np.log(errs[i - 1] / errs[i]) / np.log(res[i] / res[i - 1]) for i in range(1, len(errs))]
    assert np.mean(orders) >= 1.9


def test_contact_bit_exact(oracle):
    g = golden("contact.npz")
    cfg = Config(nx=400, ny=4, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.01, t_end=0.2, cfl=0.30, gamma=5.0 / 3.0,
                 B_transverse=0.0, powell_source=False, use_char_bc=False, bc_x_type="extrapolation",
                 bc_y_type="periodic")
    s = oracle.OracleSolver(cfg)
    s.U = np.repeat(g["U0"][:, :, None], s.ny_tot, axis=2).copy()
    s.advance()
    assert s.step == int(g["steps"])
    assert np.array_equal(s.U[:, :, 2], g["row"])


def test_rmi_run_loop_bit_exact(oracle):
    g = golden("rmi.npz")
    cfg = Config(nx=48, ny=24, t_end=0.25, cfl=0.30, mach=10.0, B_transverse=0.5, powell_source=True,
                 use_char_bc=True, bc_x_type="characteristic", bc_y_type="periodic")
    s = oracle.OracleSolver(cfg)
    s.U = g["U_init"].copy()
    s.advance(max_steps=int(g["steps"]))
    assert s.t == float(g["t"]) and cfg.glm_ch == float(g["ch"])
    assert np.array_equal(s.U, g["U_final"])
    np.testing.assert_allclose(s._cumulative_boundary_energy, g["ebnd"], rtol=1e-12)


def test_orszag_tang_bit_exact(oracle):
    g = golden("orszag_tang.npz")
    cfg = Config(nx=32, ny=32, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, t_end=0.5, cfl=0.4, gamma=5.0 / 3.0,
                 B_transverse=0.0, powell_source=False, bc_x_type="periodic", bc_y_type="periodic")
    s = oracle.OracleSolver(cfg)
    s.U = g["U0"].copy()
    s.advance(max_steps=int(g["steps"]))
    assert s.t == float(g["t"])
    assert np.array_equal(s.U, g["U_final"])


def test_native_loop_matches_python_loop(oracle):
    """orc_advance (used for CPU timing) == the Python-driven loop (exp may differ by 1 ulp)."""
    g = golden("orszag_tang.npz")
    cfg = Config(nx=32, ny=32, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, cfl=0.4, gamma=5.0 / 3.0,
                 powell_source=False, bc_x_type="periodic", bc_y_type="periodic")
    a, b = oracle.OracleSolver(cfg), oracle.OracleSolver(Config(**{**cfg.__dict__}))
    a.U = g["U0"].copy()
    b.U = g["U0"].copy()
    a.advance(max_steps=10)
    b.advance_native(max_steps=10)
    assert a.step == b.step == 10
    np.testing.assert_allclose(a.U, b.U, rtol=1e-13, atol=1e-13)
