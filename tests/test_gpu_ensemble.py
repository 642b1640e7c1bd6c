"""Batched ensemble on the GPU: instance i of a packed ensemble advances
exactly (bitwise) as the same grid run alone, for every tile shape and work
order; instances stop at their own end time; the autotuner runs."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def small_configs(precision, n=6, seed=11):
    from aeromhd_cuda_b200.ensemble import draw_configs
    return draw_configs(n, seed=seed, t_end=3.0, precision=precision, ny_choices=(32, 64))


@pytest.mark.parametrize("tile_x", [8, -16, -24])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_instances_equal_single_grid_runs(precision, tile_x):
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200.ensemble import Ensemble
    from aeromhd_cuda_b200.solver import MHDSolver
    cfgs = small_configs(precision)
    ens = Ensemble(cfgs, tile_x=tile_x)
    ens.initialize()
    ens.start(max_steps=12)
    ens.advance(12)
    ctl = ens.controls()
    _lib.call("amhd_set_tiling", tile_x, 0)
    for k, c in enumerate(cfgs):
        s = MHDSolver(c)
        s.initialize()
        s.advance(max_steps=12, chunk=12)
        assert s.step == ctl[k].step == 12
        assert s.t == ctl[k].t
        assert torch.equal(s.U, ens.state(k)), k


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_schedules_give_identical_results(precision):
    """Work order and grid size never change a result.  The tile shape does not
    either in float64 (built without contraction); in float32 each tile-shape
    instantiation may contract multiply-adds differently, so there the bar
    across tile shapes is 1e-6 relative."""
    from aeromhd_cuda_b200.ensemble import Ensemble
    cfgs = small_configs(precision, n=5, seed=12)
    ref = {}
    for tx, order, ctas in [(8, "instance", -1), (8, "interleave", 0), (8, "largest_first", 200),
                            (4, "instance", -1), (4, "interleave", 0), (16, "largest_first", 0)]:
        if precision == "fp64" and tx == 16:
            continue
        ens = Ensemble(cfgs, tile_x=tx, order=order, ctas=ctas)
        ens.initialize()
        ens.start(max_steps=6)
        ens.advance(6)
        if tx not in ref:
            ref[tx] = ens.U.clone()
        assert torch.equal(ens.U, ref[tx]), (tx, order, ctas)
        base = ref[8]
        if precision == "fp64":
            assert torch.equal(ens.U, base), (tx, order, ctas)
        else:
            rel = float((ens.U.double() - base.double()).abs().sum() / base.double().abs().sum())
            assert rel < 1e-6, (tx, rel)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_marching_work_queue_gives_identical_results(precision):
    """A persistent marching grid whose warps draw items from the device work
    queue, over several graph replays and eager calls in a row (each launch
    resets the queue for the next), equals one CTA per 4 items and the static
    split bit for bit, with the last strips' row chunks sharing warps or not;
    the queue is back at zero after every call."""
    from aeromhd_cuda_b200.ensemble import Ensemble
    cfgs = small_configs(precision, n=5, seed=16)
    out = []
    for order, ctas, dynamic, pack in [("instance", -1, True, True), ("instance", 0, True, True),
                                       ("largest_first", 0, True, True), ("interleave", 37, True, True),
                                       ("instance", 0, False, True), ("instance", 0, True, False),
                                       ("interleave", -1, True, False)]:
        # pack=False: one row chunk of the last column strip per warp instead of 2 or 4
        ens = Ensemble(cfgs, tile_x=-16, order=order, ctas=ctas, dynamic=dynamic, pack=pack)
        assert ens.uses_queue() == (ctas >= 0 and dynamic)
        ens.initialize()
        ens.start(max_steps=9)
        ens.advance(3)
        ens.advance(3)
        ens.advance(3, graph=False)
        torch.cuda.synchronize()
        assert ens.queue.tolist() == [0, 0], (order, ctas, dynamic, pack)
        assert all(c.step == 9 for c in ens.controls())
        out.append(ens.U.clone())
    for u in out[1:]:
        assert torch.equal(u, out[0])


def test_instances_stop_at_their_end_time():
    from aeromhd_cuda_b200.ensemble import Ensemble
    cfgs = small_configs("fp32", n=4, seed=13)
    ens = Ensemble(cfgs)
    ens.initialize()
    ens.start(t_end=0.01)
    steps = ens.run(chunk=8)
    ctl = ens.controls()
    assert all(abs(c.t - 0.01) < 1e-12 and not c.active for c in ctl)
    assert len(set(steps.tolist())) > 1            # different grids, different dt


def test_autotuner_picks_a_candidate_and_restores_state():
    from aeromhd_cuda_b200.autotune import Cache, candidates, tune_ensemble
    from aeromhd_cuda_b200.ensemble import Ensemble
    cfgs = small_configs("fp32", n=4, seed=14)
    ens = Ensemble(cfgs)
    ens.initialize()
    ens.start(max_steps=100)
    before = ens.U.clone()
    best, timings = tune_ensemble(ens, steps=2, cands=candidates(True, "fp32")[:6], cache=Cache())
    assert best in timings and all(t > 0 for t in timings.values())
    assert torch.equal(ens.U, before)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("tile_x", [8, -16])
def test_tma_staging_matches_plain_loads(tile_x, precision):
    """The tile + halo (tiled kernel) or the rows (marching kernel, per-instance
    tensor maps in device memory) staged by TMA (cp.async.bulk.tensor), or by
    128-bit loads / per-lane cp.async: identical results (float32 marching: the
    two instantiations may contract multiply-adds differently, bar 1e-6)."""
    from aeromhd_cuda_b200.ensemble import Ensemble
    cfgs = small_configs(precision, n=4, seed=15)
    out = []
    for tma in (True, False):
        ens = Ensemble(cfgs, tile_x=tile_x, use_tma=tma, ctas=0)
        assert ens.tma_staging() == tma
        ens.initialize()
        ens.start(max_steps=5)
        ens.advance(5)
        out.append(ens.U.clone())
    if precision == "fp64" or tile_x > 0:
        assert torch.equal(out[0], out[1])
    else:
        rel = float((out[0].double() - out[1].double()).abs().sum() / out[1].double().abs().sum())
        assert rel < 1e-6, rel
