"""amhd_diagnostics_noalloc: the diagnostics entry point for callers that may
not allocate device memory (a host framework that owns all device memory and
only passes its plugins inputs and outputs, or a loop that must not risk an
allocation synchronising the device).  Its row scratch is a fixed array
inside the library instead of a caller buffer.

Checked through the C ABI against amhd_diagnostics (caller-provided scratch)
on two calls in a row on different states, so that the second call also
shows nothing is left over from the first.  This file is collected last so
that a run stopping at the first failure has run every other test already;
it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _state(n, precision, seed):
    from aeromhd_cuda_b200 import initial_conditions as ic
    from aeromhd_cuda_b200.config import Config
    from aeromhd_cuda_b200.solver import MHDSolver
    cfg = Config(nx=n, ny=n // 2, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.5, cfl=0.4, gamma=5.0 / 3.0,
                 powell_source=False, bc_x_type="periodic", bc_y_type="periodic", precision=precision)
    s = MHDSolver(cfg)
    s.set_primitive(ic.orszag_tang(s))
    s.advance(max_steps=seed, chunk=seed, graph=False)   # different states for the two calls
    return s


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_diagnostics_match_the_allocating_entry_point(precision):
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import ptr, stream_ptr
    for call, steps in enumerate((3, 8)):
        s = _state(96, precision, steps)
        g = s._grid()
        ref = torch.full((8,), float("nan"), dtype=torch.float64, device="cuda")
        rows = torch.zeros(7 * s.cfg.nx, dtype=torch.float64, device="cuda")
        _lib.call("amhd_diagnostics", g, ptr(s.U), float(s.cfg.x_min), ptr(ref), ptr(rows), stream_ptr())
        got = torch.full((8,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _lib.call("amhd_diagnostics_noalloc", g, ptr(s.U), float(s.cfg.x_min), ptr(got), stream_ptr())
        torch.cuda.synchronize()
        if call == 1:  # the first call may load the library's kernels; later calls take no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        r, o = ref.cpu().numpy()[:7], got.cpu().numpy()[:7]
        assert np.all(np.isfinite(r)), call
        np.testing.assert_allclose(o, r, rtol=1e-12, atol=0.0, err_msg=f"call {call}")


def test_noalloc_rejects_grids_beyond_its_fixed_scratch():
    from aeromhd_cuda_b200 import _lib
    g = _lib.Grid(nx=20000, ny=4, pitch=8, dtype=0, var_stride=20004 * 8, dx=0.1, dy=0.1, gamma=1.4, cfl=0.3,
                  glm_alpha=1.5)
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = _lib.lib().amhd_diagnostics_noalloc(ctypes.byref(g), ctypes.c_void_p(out.data_ptr()), 0.0,
                                             ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.AMHD_ERR_ARG
    assert b"16384" in _lib.lib().amhd_last_error()
