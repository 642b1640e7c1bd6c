"""Host-side logic of the batched ensemble and the autotuner (no GPU)."""
import numpy as np
import pytest

from aeromhd_cuda_b200 import _lib
from aeromhd_cuda_b200.autotune import Cache, Candidate, candidates, choose, signature, tune
from aeromhd_cuda_b200.ensemble import draw_configs, pack_layout, shard, tile_counts, work_list


def test_draws_follow_the_ensemble_recipe():
    cfgs = draw_configs(256, seed=3)
    assert len(cfgs) == 256
    ny = np.array([c.ny for c in cfgs])
    assert set(ny) <= {32, 64, 128, 256} and len(set(ny)) == 4
    assert all(c.nx == 4 * c.ny for c in cfgs)
    assert all(2.0 <= c.mach <= 5.0 and 1.5 <= c.density_ratio <= 5.0 for c in cfgs)
    assert all(1 <= c.perturbation_mode <= 8 and 0.01 <= c.perturbation_amp <= 0.08 for c in cfgs)
    assert all(0 <= c.bx0 <= 0.3 and 0 <= c.b1 <= 0.3 and 1 <= c.b_mode <= 6 for c in cfgs)
    cells = sum(c.nx * c.ny for c in cfgs)
    assert 15e6 < cells < 30e6            # ~22 M cells expected
    again = draw_configs(256, seed=3)
    assert [c.mach for c in again] == [c.mach for c in cfgs]     # seeded
    assert [c.mach for c in draw_configs(256, seed=4)] != [c.mach for c in cfgs]


@pytest.mark.parametrize("code", [_lib.AMHD_F32, _lib.AMHD_F64])
def test_pack_layout_is_aligned_and_disjoint(code):
    cfgs = draw_configs(40, seed=1)
    layouts, total = pack_layout(cfgs, code)
    es = 4 if code == _lib.AMHD_F32 else 8
    end = 0
    for (off, pitch, rows), c in zip(layouts, cfgs):
        assert off >= end and (off * es) % 16 == 0
        assert pitch >= c.ny + 4 and rows >= c.nx + 4 and (pitch * es) % 16 == 0
        end = off + 10 * rows * pitch
    assert total >= end


@pytest.mark.parametrize("order", ["instance", "interleave", "largest_first"])
def test_work_list_is_a_permutation_grouped_by_instance(order):
    cfgs = draw_configs(30, seed=2)
    counts = tile_counts(cfgs, 8)
    tile_order, tile_inst, first = work_list(counts, order)
    n = int(counts.sum())
    assert sorted(tile_order.tolist()) == list(range(n))
    for k in range(len(cfgs)):
        ids = np.arange(first[k], first[k] + counts[k])
        assert np.all(tile_inst[ids] == k)
        # each instance's tiles are taken in increasing order (any schedule)
        pos = [p for p, t in enumerate(tile_order) if first[k] <= t < first[k] + counts[k]]
        assert list(tile_order[pos]) == list(ids)
    if order == "interleave":
        assert len(set(tile_inst[tile_order[: len(cfgs)]])) == len(cfgs)


def test_shard_balances_cells_and_covers_everything():
    cfgs = draw_configs(256, seed=5)
    cells = np.array([c.nx * c.ny for c in cfgs])
    for world in (1, 2, 4, 8):
        parts = [shard(cfgs, world, r) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(cfgs)))
        loads = np.array([cells[p].sum() for p in parts])
        assert loads.max() - loads.min() <= cells.max()


def test_candidates_and_choice():
    ens = candidates(True, "fp32")
    assert Candidate(8, "interleave", 0) in ens and len(ens) == 7 * 3 * 2
    assert Candidate(-32, "instance", 0) in ens  # warp-marching kernel, 32 rows per item
    assert all(c.tile_x != 16 for c in candidates(True, "fp64"))
    assert all(c.order == "instance" for c in candidates(False, "fp32"))
    t = {Candidate(8, "instance", -1): 1.0, Candidate(4, "instance", -1): 1.005, Candidate(16, "interleave", 0): 0.5}
    assert choose(t) == Candidate(16, "interleave", 0)
    t = {Candidate(8, "instance", -1): 1.0, Candidate(4, "instance", -1): 1.005, Candidate(16, "interleave", 0): 1.2}
    assert choose(t) == Candidate(4, "instance", -1)  # tie within 1%: simplest, then smaller tile
    t = {Candidate(8, "instance", -1): 1.0, Candidate(-32, "instance", -1): 1.004}
    assert choose(t) == Candidate(-32, "instance", -1)  # tie: the marching kernel (the library default)
    t = {Candidate(-24, "instance", -1): 1.0, Candidate(-24, "instance", 0): 1.006}
    assert choose(t) == Candidate(-24, "instance", 0)  # tie: the persistent grid (one launch per stage)
    t = {Candidate(8, "instance", -1): 1.0, Candidate(-32, "instance", -1): 0.7}
    assert choose(t) == Candidate(-32, "instance", -1)


def test_tune_uses_cache(tmp_path):
    path = str(tmp_path / "tune.json")
    calls = []

    def run(c):
        calls.append(c)
        return {4: 3.0, 8: 1.0, 16: 2.0}.get(c.tile_x, 4.0)

    key = signature("fp32", [(128, 32), (512, 128)], "B200")
    assert key == signature("fp32", [(512, 128), (128, 32)], "B200")
    assert key != signature("fp64", [(128, 32), (512, 128)], "B200")
    best, timings = tune(run, candidates(False), key, Cache(path))
    assert best.tile_x == 8 and len(calls) == len(timings) > 0
    n = len(calls)
    best2, t2 = tune(run, candidates(False), key, Cache(path))   # fresh cache object reads the file
    assert best2 == best and t2 == {} and len(calls) == n


def test_work_shapes_and_counts():
    from aeromhd_cuda_b200.config import Config
    from aeromhd_cuda_b200.ensemble import work_shape
    assert work_shape(8) == (8, 32) and work_shape(-32) == (32, 28)
    for bad in (0, 3, 5, -3, 32, -2000):
        with pytest.raises(ValueError):
            work_shape(bad)
    cfgs = [Config(nx=100, ny=60), Config(nx=64, ny=28)]
    assert list(tile_counts(cfgs, 8)) == [13 * 2, 8 * 1]
    assert list(tile_counts(cfgs, -32)) == [4 * 3, 2 * 1]


def test_ensemble_default_geometry():
    """An ensemble starts with 32-row marching items in float32 and the
    library default (16 rows) in float64."""
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200.ensemble import default_tile_x
    assert default_tile_x("fp32") == -32
    assert default_tile_x("fp64") == _lib.default_tile_x("fp64") == -16


def _packed_item_cells(nx, ny, rows, pack):
    """Cells (row, column) each marching work item updates, restating the
    kernel's item decode (march_walk, amhd_kernels.cuh): packed items first
    (segments of 32/P lanes, segment s on row chunk P m + s, the short last
    chunk alone), then the full-width strips' items chunk-major.  Also checks
    that every segment of an item walks as many rows and reads rows inside
    the padded grid."""
    from aeromhd_cuda_b200.ensemble import MARCH_COLS, march_items
    NG = 2
    chunks, strips = -(-nx // rows), -(-ny // MARCH_COLS)
    P = pack if pack > 1 else 1
    plain = strips - 1 if P > 1 else strips
    full = nx // rows
    n_packed = (-(-full // P) + (1 if full * rows < nx else 0)) if P > 1 else 0
    out = []
    for local in range(march_items(nx, ny, rows, pack)):
        cells, heights = [], set()
        for lane in range(32):
            seg_w, lane_c, live = 32, lane, True
            if local >= n_packed:
                strip, chunk = (local - n_packed) % plain, (local - n_packed) // plain
                n_rows = min(rows, nx - chunk * rows)
            else:
                seg = lane >> 3 if P == 4 else lane >> 4
                seg_w = 8 if P == 4 else 16
                lane_c, strip = lane - seg * seg_w, strips - 1
                if local < -(-full // P):
                    chunk = local * P + seg
                    live = chunk < full
                    chunk = chunk if live else local * P
                    n_rows = rows
                else:
                    chunk, live, n_rows = full, seg == 0, nx - full * rows
            heights.add(n_rows)
            j, ib = MARCH_COLS * strip + lane_c, NG + chunk * rows
            assert 0 <= ib - 2 and ib + n_rows + 1 <= nx + 2 * NG - 1
            if live and NG <= lane_c < seg_w - NG and j < NG + ny:
                cells += [(i, j) for i in range(ib, ib + n_rows)]
        assert len(heights) == 1 and heights.pop() >= 1
        out.append(cells)
    return out


@pytest.mark.parametrize("nx,rows", [(1, 4), (23, 24), (24, 24), (75, 8), (100, 32), (256, 16)])
def test_packed_items_update_every_cell_once(nx, rows):
    """With the last strip's row chunks packed (march_pack) or not, the work
    items of a grid update every interior cell exactly once."""
    from aeromhd_cuda_b200.ensemble import march_pack
    for ny in (1, 2, 3, 4, 5, 16, 28, 30, 32, 33, 40, 60, 64, 100, 128, 256):
        want = {(i, j) for i in range(2, nx + 2) for j in range(2, ny + 2)}
        for pack in (1, march_pack(ny)):
            seen = [c for item in _packed_item_cells(nx, ny, rows, pack) for c in item]
            assert len(seen) == len(set(seen)) and set(seen) == want, (nx, ny, rows, pack)
