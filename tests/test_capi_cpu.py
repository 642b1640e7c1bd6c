"""The C ABI library without a GPU: it builds, loads, exports every symbol
include/aeromhd.h declares, agrees on struct layouts, and rejects bad
arguments before touching the device."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "aeromhd.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char \*)\s*(amhd_\w+)\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def L():
    from aeromhd_cuda_b200 import build, _lib
    build.build()
    return _lib.lib()


def test_header_lists_entry_points():
    names = header_functions()
    assert "amhd_step_ssprk3" in names and "amhd_advance" in names and len(names) >= 25


def test_library_exports_every_declared_symbol(L):
    from aeromhd_cuda_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_lib.exported_names()) == header_functions()


def test_struct_layouts_match(L):
    from aeromhd_cuda_b200 import _lib
    assert L.amhd_control_size() == ctypes.sizeof(_lib.Control) == 160
    assert ctypes.sizeof(_lib.Grid) == 80
    assert ctypes.sizeof(_lib.Instance) == 112


def test_version_and_padded_layout(L):
    from aeromhd_cuda_b200 import _lib
    assert b"sm_100a" in L.amhd_version()
    assert _lib.padded_layout(2048, 512, _lib.AMHD_F32) == (516, 2052)
    assert _lib.padded_layout(800, 4, _lib.AMHD_F64) == (36, 804)
    assert _lib.padded_layout(100, 50, _lib.AMHD_F32) == (68, 116)


def test_argument_errors_are_codes_not_crashes(L):
    from aeromhd_cuda_b200 import _lib
    p, r = ctypes.c_int32(), ctypes.c_int32()
    assert L.amhd_padded_layout(1, 8, 0, ctypes.byref(p), ctypes.byref(r)) == _lib.AMHD_ERR_ARG
    assert b"2x2" in L.amhd_last_error()
    assert L.amhd_padded_layout(8, 8, 7, ctypes.byref(p), ctypes.byref(r)) == _lib.AMHD_ERR_ARG
    assert L.amhd_set_tiling(5, 0) == _lib.AMHD_ERR_ARG
    assert L.amhd_set_tiling(-3, 0) == _lib.AMHD_ERR_ARG      # marching items need at least 4 rows
    assert L.amhd_set_tiling(-2000, 0) == _lib.AMHD_ERR_ARG
    assert L.amhd_set_tiling(8, 0) == _lib.AMHD_OK
    assert L.amhd_set_tiling(-16, 0) == _lib.AMHD_OK
    assert L.amhd_set_tiling(_lib.DEFAULT_TILE_X, 0) == _lib.AMHD_OK  # 0: per-precision default
    assert (_lib.default_tile_x("fp32"), _lib.default_tile_x("fp64")) == (-24, -16)
    g = _lib.Grid(nx=8, ny=8, pitch=4, dtype=0, var_stride=1000, dx=0.1, dy=0.1, gamma=1.4, cfl=0.3,
                  glm_alpha=1.5)
    # pitch < ny+4 is refused before any device call
    assert L.amhd_apply_bc(ctypes.byref(g), None, None) == _lib.AMHD_ERR_ARG
    g.pitch = 12
    g.var_stride = 12 * 12
    assert L.amhd_cons_to_prim(ctypes.byref(g), None, None, None) == _lib.AMHD_ERR_ARG
    g.gamma = 1.0
    assert L.amhd_enforce_scalar_bounds(ctypes.byref(g), ctypes.c_void_p(16), None) == _lib.AMHD_ERR_ARG
    g.gamma = 1.4
    # the fused step needs the padded layout and aligned pointers
    assert L.amhd_step_ssprk3(ctypes.byref(g), ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), 0.1,
                              1.0, 1.0, None, None) == _lib.AMHD_ERR_ARG
    assert b"pitch" in L.amhd_last_error()
    assert L.amhd_hlld_flux(2, 0, None, None, None, None, 4, 1.4, 1.0, None) == _lib.AMHD_ERR_ARG
    assert L.amhd_hlld_flux(0, 0, None, None, None, None, 0, 1.4, 1.0, None) == _lib.AMHD_OK


def test_new_entry_points_reject_bad_arguments(L):
    """amhd_step_host_n, the GEMM operand relayouts and the persistent-GEMM
    switch refuse bad arguments with codes, before any device call."""
    from aeromhd_cuda_b200 import _lib
    p, r = ctypes.c_int32(), ctypes.c_int32()
    assert L.amhd_padded_layout(8, 8, 0, ctypes.byref(p), ctypes.byref(r)) == _lib.AMHD_OK
    g = _lib.Grid(nx=8, ny=8, pitch=p.value, dtype=0, var_stride=r.value * p.value, dx=0.1, dy=0.1, gamma=1.4,
                  cfl=0.3, glm_alpha=1.5)
    buf = ctypes.c_void_p(256)
    out = (ctypes.c_double * 4)()
    step_n = L.amhd_step_host_n
    assert step_n(ctypes.byref(g), None, buf, buf, buf, buf, 0.0, 1.0, 3, out, None) == _lib.AMHD_ERR_ARG
    assert step_n(ctypes.byref(g), buf, buf, buf, buf, buf, 0.0, 1.0, 0, out, None) == _lib.AMHD_ERR_ARG
    assert b"n_steps" in L.amhd_last_error()
    g.pitch = 4  # below ny + 4
    assert step_n(ctypes.byref(g), buf, buf, buf, buf, buf, 0.0, 1.0, 3, out, None) == _lib.AMHD_ERR_ARG
    assert L.amhd_nn_flip3(buf, 4, 3, 35, buf, None) == _lib.AMHD_ERR_ARG   # ldo < cout * 9
    assert L.amhd_nn_flip3(None, 4, 3, 40, buf, None) == _lib.AMHD_ERR_ARG
    assert L.amhd_nn_pad_cols(buf, 4, 90, 89, buf, None) == _lib.AMHD_ERR_ARG  # ldo < cols
    assert L.amhd_nn_pad_cols(buf, 0, 90, 96, buf, None) == _lib.AMHD_ERR_ARG
    assert L.amhd_nn_set_gemm_persistent(2) == _lib.AMHD_ERR_ARG
    assert L.amhd_nn_set_gemm_persistent(0) == _lib.AMHD_OK
    assert L.amhd_nn_set_gemm_persistent(1) == _lib.AMHD_OK


def test_march_item_counts_agree_with_the_library(L):
    """The ensemble's work-list arithmetic (ensemble.march_pack / march_items)
    equals the library's (amhd_march_pack / amhd_march_items), and the packed
    items cover every (chunk, strip) exactly once: the full-width strips' items
    plus one segment per full-height chunk of the last strip and one item for
    a short last chunk."""
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200.ensemble import MARCH_COLS, march_items, march_pack
    for ny in range(1, 300):
        P = march_pack(ny)
        assert L.amhd_march_pack(ny) == P
        rem = ny % MARCH_COLS
        if P > 1:
            assert rem + 4 <= 32 // P  # the leftover columns and their halo fit a segment
        else:
            assert rem == 0 or rem > 12
    assert [march_pack(n) for n in (32, 64, 128, 256, 2048)] == [4, 2, 1, 4, 4]
    for nx in (1, 2, 5, 23, 24, 25, 48, 100, 128, 256, 1024, 2048):
        for ny in (2, 4, 16, 28, 29, 32, 40, 56, 64, 128, 256, 2048):
            for rows in (4, 16, 24, 32):
                chunks, strips = -(-nx // rows), -(-ny // MARCH_COLS)
                for pack in (0, 1, march_pack(ny)):
                    n = march_items(nx, ny, rows, pack)
                    assert L.amhd_march_items(nx, ny, rows, pack) == n
                    if pack <= 1:
                        assert n == chunks * strips
                    else:
                        full = nx // rows
                        segs = (n - (strips - 1) * chunks) * pack
                        assert full <= segs - (pack if nx % rows else 0) < full + pack
    assert ensemble_counts_2048() == (73 * 86 + 22 + 1, 74 * 86)
    assert L.amhd_march_items(0, 8, 8, 1) == _lib.AMHD_ERR_ARG
    assert L.amhd_march_items(64, 64, 8, 4) == _lib.AMHD_ERR_ARG  # 64 leaves 8 columns: 2 chunks to a warp
    assert L.amhd_march_items(64, 128, 8, 2) == _lib.AMHD_ERR_ARG  # 128 leaves 16: none
    assert L.amhd_set_march_pack(2) == _lib.AMHD_ERR_ARG
    assert L.amhd_set_march_pack(0) == _lib.AMHD_OK
    assert L.amhd_set_march_pack(1) == _lib.AMHD_OK


def ensemble_counts_2048():
    from aeromhd_cuda_b200.ensemble import march_items, march_pack
    return march_items(2048, 2048, 24, march_pack(2048)), march_items(2048, 2048, 24, 1)


def test_corrector_padding_rows_zeroed_once_per_shape():
    """The corrector's zero-padded GEMM workspaces (K rounded up to a multiple of
    8 for the TMA path): the padding rows are zeroed when the buffer or its
    shape is new, and left alone on the next calls of the same shape (a captured
    training step must not contain the fill)."""
    import torch
    from aeromhd_cuda_b200.corrector import Corrector, _round8
    assert (_round8(90), _round8(96), _round8(1)) == (96, 96, 8)
    c = Corrector(16, 16, device="cpu")
    t = c._padded_rows("e1.col", 90, 96, 10)
    assert t.shape == (96, 10) and torch.all(t[90:] == 0)
    t.fill_(1.0)
    t = c._padded_rows("e1.col", 90, 96, 10)
    assert torch.all(t[90:] == 1)            # same shape: not refilled
    t = c._padded_rows("e1.col", 90, 96, 8)  # new shape: the padding rows of the new view are zeroed
    assert torch.all(t[90:] == 0)
    u = c._padded_rows("colg", 96, 96, 10)   # nothing to pad
    assert u.shape == (96, 10)


def test_config_keeps_reference_fields_and_defaults():
    from aeromhd_cuda_b200.config import Config
    c = Config()
    ref = dict(nx=400, ny=200, x_min=0.0, x_max=6.0, y_min=0.0, y_max=2.0, t_end=0.25, cfl=0.30, max_steps=200000,
               gamma=5.0 / 3.0, mach=10.0, interface_x=1.5, perturbation_amp=0.15, perturbation_mode=4,
               density_ratio=3.0, interface_width=2.0, B_transverse=0.0, glm_ch=0.0, glm_alpha=1.5,
               powell_source=True, use_char_bc=True, bc_x_type="auto", bc_y_type="periodic",
               enable_smoothing=False, diag_interval=20)
    for k, v in ref.items():
        assert getattr(c, k) == v, k
    assert c.snapshot_times == [0.0, 0.05, 0.10, 0.15, 0.20, 0.25]
    assert c.get_bc_x() == "characteristic"
    assert Config(use_char_bc=False).get_bc_x() == "extrapolation"
    assert c.dx == 6.0 / 400 and c.dy == 2.0 / 200
    assert c.powell_enabled() is False and Config(B_transverse=0.5).powell_enabled() is True
    assert Config(powell_mode="on").powell_enabled() is True
    with pytest.raises(ValueError):
        Config(nx=1).validate()
    with pytest.raises(ValueError):
        Config(precision="fp16").validate()


def test_config_matches_reference_dataclass_when_available():
    """Field names and defaults against the reference's own Config (imported in a
    child process so the stand-in modules it needs never reach this one)."""
    import subprocess
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import refshim
    if refshim.REFERENCE_DIR is None:
        pytest.skip("reference modules not available")
    code = (
        "import sys; sys.path[:0] = [%r, %r]\n"
        "import refshim\n"
        "from dataclasses import fields\n"
        "from aeromhd_cuda_b200.config import Config\n"
        "R = refshim.load_reference()\n"
        "ref = {f.name for f in fields(R.config.Config)}\n"
        "mine = {f.name for f in fields(Config)}\n"
        "assert ref <= mine, ref - mine\n"
        "a, b = R.config.Config(), Config()\n"
        "bad = [f for f in ref if getattr(a, f) != getattr(b, f)]\n"
        "assert not bad, bad\n"
        "assert int(R.config.ConsVar.RHOC) == 9 and int(R.config.PrimVar.CLR) == 9\n"
        "print('CONFIG-OK')\n") % (ROOT, os.path.join(ROOT, "tests", "golden"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert "CONFIG-OK" in out.stdout, out.stdout + out.stderr


def test_rankine_hugoniot_matches_reference_golden():
    import numpy as np
    from aeromhd_cuda_b200.physics import mhd_rankine_hugoniot
    from conftest import golden
    g = golden("rmi.npz")
    assert np.array_equal(np.array(mhd_rankine_hugoniot(5.0 / 3.0, 3.0, 1.0, 1.0, 0.0)), g["rh_hydro"])
    assert np.array_equal(np.array(mhd_rankine_hugoniot(5.0 / 3.0, 10.0, 1.0, 1.0, 1.5)), g["rh_mhd"])
    got = mhd_rankine_hugoniot(5.0 / 3.0, 10.0, 1.0, 1.0, 0.5)
    assert got == tuple(float(g[f"rh_{k}"]) for k in ("rho2", "p2", "vx2", "By2", "vs"))
