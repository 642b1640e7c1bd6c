"""Host-side status checks: the control flags after which a state must not be
used, and the tensor-core GEMM wait flag, raise instead of letting a run carry
on with stale or unwritten data.  No GPU: the flags are set on the host and the
library's status call is replaced by a stand-in that reports a failed wait."""
import ctypes

import pytest

from aeromhd_cuda_b200 import _lib


def _control(flags):
    c = _lib.Control()
    c.flags = flags
    c.step = 7
    return c


def test_clean_flags_pass():
    _lib.check_control(_control(0))
    _lib.check_control(_control(_lib.AMHD_FLAG_DT_TINY | _lib.AMHD_FLAG_PAUSED))


def test_timeout_flag_raises_timeout_error():
    with pytest.raises(_lib.AmhdError) as e:
        _lib.check_control(_control(_lib.AMHD_FLAG_TIMEOUT), "test")
    assert e.value.code == _lib.AMHD_ERR_TIMEOUT and "step 7" in str(e.value)


def test_nonfinite_flag_raises_floating_point_error():
    with pytest.raises(FloatingPointError):
        _lib.check_control(_control(_lib.AMHD_FLAG_NONFINITE))


@pytest.mark.parametrize("flag", [0, 1])
def test_gemm_status_raises_when_a_wait_gave_up(monkeypatch, flag):
    calls = []

    def fake_call(name, *args):
        calls.append(name)
        assert name == "amhd_nn_gemm_status"
        args[0]._obj.value = flag

    monkeypatch.setattr(_lib, "call", fake_call)
    if flag:
        with pytest.raises(_lib.AmhdError) as e:
            _lib.check_gemm_status("test")
        assert e.value.code == _lib.AMHD_ERR_TIMEOUT
    else:
        _lib.check_gemm_status("test")
    assert calls == ["amhd_nn_gemm_status"]


def test_corrector_checks_the_gemm_status(monkeypatch):
    """Corrector.check_gemm_status goes through the same check (no GPU needed to call it)."""
    from aeromhd_cuda_b200.corrector import Corrector
    seen = []
    monkeypatch.setattr(_lib, "check_gemm_status", lambda where="": seen.append(where))
    Corrector.check_gemm_status(None)
    assert seen == ["corrector"]


def test_timeout_flag_value_matches_the_header():
    import os
    hdr = open(os.path.join(os.path.dirname(_lib.HERE), "include", "aeromhd.h")).read()
    assert f"#define AMHD_FLAG_TIMEOUT {_lib.AMHD_FLAG_TIMEOUT}" in hdr
    assert ctypes.sizeof(_lib.Control) == 160
