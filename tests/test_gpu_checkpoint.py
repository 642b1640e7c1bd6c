"""Checkpoint / resume on the GPU: a run saved part-way, reloaded into a new
solver (or ensemble) and continued reproduces the uninterrupted run bit for
bit (state, t, step); the boundary-energy sum agrees to 1e-12 (the resumed
run adds the two parts in another order)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def ot_cfg(n, precision):
    from aeromhd_cuda_b200.config import Config
    return Config(nx=n, ny=n, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, t_end=0.5, cfl=0.4, gamma=5.0 / 3.0,
                  powell_source=False, bc_x_type="periodic", bc_y_type="periodic", precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_solver_resume_is_bitwise(tmp_path, precision):
    from aeromhd_cuda_b200 import checkpoint as ck, initial_conditions as ic
    from aeromhd_cuda_b200.solver import MHDSolver
    a = MHDSolver(ot_cfg(72, precision))
    a.set_primitive(ic.orszag_tang(a))
    b = MHDSolver(ot_cfg(72, precision))
    b.U = a.U.clone()
    a.advance(max_steps=30, chunk=10)
    b.advance(max_steps=12, chunk=12)
    ck.save_checkpoint(b, str(tmp_path / "ot"))
    del b
    c = ck.load_checkpoint(str(tmp_path / "ot"))
    assert c.step == 12 and c.cfg.precision == precision
    c.advance(max_steps=30, chunk=9)
    assert c.step == a.step == 30
    assert c.t == a.t
    assert torch.equal(c.U, a.U)


def test_solver_resume_shock_interface_with_diagnostics(tmp_path):
    """Outflow/characteristic x boundaries, Powell source, the reference's run()
    diagnostics history: continued after reload."""
    from aeromhd_cuda_b200 import checkpoint as ck
    from aeromhd_cuda_b200.config import Config
    from aeromhd_cuda_b200.solver import MHDSolver
    cfg = dict(nx=96, ny=40, B_transverse=0.3, t_end=1.0)
    a = MHDSolver(Config(**cfg))
    a.initialize()
    b = MHDSolver(Config(**cfg))
    b.initialize()
    a.advance(max_steps=40, chunk=20)
    b.advance(max_steps=20, chunk=20)
    b.compute_diagnostics()
    ck.save_checkpoint(b, str(tmp_path / "si"))
    c = ck.load_checkpoint(str(tmp_path / "si"))
    assert len(c.diag_times) == 1 and c.diag_energy_total == b.diag_energy_total
    assert c._rh_results == pytest.approx(b._rh_results)
    c.advance(max_steps=40, chunk=20)
    assert c.step == a.step == 40 and c.t == a.t
    assert torch.equal(c.U, a.U)
    ea, ec = a._cumulative_boundary_energy, c._cumulative_boundary_energy
    assert abs(ec - ea) <= 1e-12 * max(abs(ea), 1e-30)


def test_ensemble_resume_is_bitwise(tmp_path):
    from aeromhd_cuda_b200 import checkpoint as ck
    from aeromhd_cuda_b200.ensemble import Ensemble, draw_configs
    cfgs = draw_configs(4, seed=5, t_end=3.0, precision="fp32", ny_choices=(32, 64))
    a = Ensemble(cfgs)
    a.initialize()
    a.start()
    a.advance(10, graph=False)
    ck.save_ensemble(a, str(tmp_path / "ens"))
    a.advance(10, graph=False)
    b, metas = ck.load_ensemble(str(tmp_path / "ens"))
    assert [m["step"] for m in metas] == [10] * 4
    b.advance(10, graph=False)
    ca, cb = a.controls(), b.controls()
    for k in range(4):
        assert ca[k].step == cb[k].step == 20 and ca[k].t == cb[k].t
        assert torch.equal(a.state(k), b.state(k)), k
