"""Row-split grid on the GPU.  (1) The split run loop with one rank equals the
device loop (amhd_advance) bit for bit.  (2) Two and three blocks of one grid
advanced in lockstep in one process -- the GPU stages of every block, then the
ghost-row exchange and the CFL max reduction done here by plain copies --
equal the unsplit grid bit for bit, so the multi-GPU run (the same stages,
with NCCL doing the copies and the reduction) does too; their boundary
energies add up to the unsplit grid's."""
import pytest
import torch

pytestmark = pytest.mark.gpu

NG = 2


def cfgs():
    from aeromhd_cuda_b200.config import Config
    ot = Config(nx=70, ny=48, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, t_end=0.5, cfl=0.4, gamma=5.0 / 3.0,
                powell_source=False, bc_x_type="periodic", bc_y_type="periodic")
    si = Config(nx=96, ny=40, B_transverse=0.3, t_end=1.0)
    return {"orszag_tang": ot, "shock_interface": si}


def initial(name, cfg):
    from aeromhd_cuda_b200 import initial_conditions as ic
    from aeromhd_cuda_b200.solver import MHDSolver
    s = MHDSolver(cfg)
    if name == "orszag_tang":
        s.set_primitive(ic.orszag_tang(s))
    else:
        s.initialize()
    return s


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["orszag_tang", "shock_interface"])
def test_one_rank_split_loop_equals_device_loop(name, precision):
    from dataclasses import replace
    from aeromhd_cuda_b200.decomp import DecomposedSolver
    cfg = replace(cfgs()[name], precision=precision)
    a = initial(name, cfg)
    U0 = a.U.clone()
    a.advance(max_steps=25, chunk=25, graph=False)
    d = DecomposedSolver(replace(cfg))
    d.set_global_state(U0)
    d.advance(25)
    assert d.step == a.step == 25 and d.t == a.t
    assert torch.equal(d.gather_state(), a.U)
    assert d.boundary_energy() == a._cumulative_boundary_energy


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", ["orszag_tang", "shock_interface"])
def test_blocks_in_lockstep_equal_unsplit_grid(name, world):
    from aeromhd_cuda_b200.config import BC_PERIODIC, bc_x_code
    from aeromhd_cuda_b200.decomp import GpuBackend, neighbours, split_rows
    cfg = cfgs()[name]
    a = initial(name, cfg)
    U0 = a.U.clone()
    steps = 20
    a.advance(max_steps=steps, chunk=steps, graph=False)
    rows = split_rows(cfg.nx, world)
    bs = [GpuBackend(cfg, r0, r1) for r0, r1 in rows]
    for b, (r0, r1) in zip(bs, rows):
        b.state(0).copy_(U0[:, r0:r1 + 2 * NG])
    periodic = bc_x_code(cfg) == BC_PERIODIC

    def exchange(k):
        sent = [(b.state(k)[:, NG:2 * NG].clone(), b.state(k)[:, b.n:b.n + NG].clone()) for b in bs]
        for r, b in enumerate(bs):
            left, right = neighbours(r, world, periodic)
            if left is not None:
                b.state(k)[:, 0:NG].copy_(sent[left][1])
            if right is not None:
                b.state(k)[:, b.n + NG:b.n + 2 * NG].copy_(sent[right][0])

    def reduce_max():
        m = torch.stack([b.red() for b in bs]).max(dim=0).values
        for b in bs:
            b.red().copy_(m)

    for b in bs:
        b.control_init_split(0.0, cfg.t_end, 0, steps)
    exchange(0)
    reduce_max()
    for b in bs:
        b.finish(0)
    for _ in range(steps):
        for s in (1, 2, 3):
            for b in bs:
                b.stage(s)
            exchange(s % 3)
        reduce_max()
        for b in bs:
            b.finish(1)
    for b, (r0, r1) in zip(bs, rows):
        c = b.control()
        assert c.step == steps and c.t == a.t
        assert torch.equal(b.state(0), a.U[:, r0:r1 + 2 * NG])
    # boundary energy: only the first and the last block hold physical x sides
    e_split = sum(float(b.control().e_bnd) for b in bs)
    e_ref = a._cumulative_boundary_energy
    if periodic:
        assert e_split == e_ref == 0.0
    else:
        assert e_ref != 0.0 and abs(e_split - e_ref) <= 1e-12 * abs(e_ref), (e_split, e_ref)
