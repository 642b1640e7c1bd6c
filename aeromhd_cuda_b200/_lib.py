"""ctypes binding of libaeromhd.so (C ABI in include/aeromhd.h).

There is no fallback: if the library is missing the import of the solver
fails with a message saying how to build it.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaeromhd.so")

AMHD_OK = 0
AMHD_ERR_ARG = -1
AMHD_ERR_CUDA = -2
AMHD_ERR_NONFINITE = -3
AMHD_ERR_TIMEOUT = -4
AMHD_ERR_UNSUPPORTED = -5

AMHD_F64 = 0
AMHD_F32 = 1
LIMITER_CODES = {"vanleer": 0, "minmod": 1}
# stage-kernel geometry the library starts with (amhd_set_tiling): 0 = per precision,
# the warp-marching kernel with default_tile_x(precision) rows per item
DEFAULT_TILE_X = 0


def default_tile_x(precision: str) -> int:
    """Rows per marching item of the library default: 24 in float32, 16 in float64
    (float64 runs 2 CTAs per SM, where 16-row items fill whole waves at 2048^2)."""
    return -24 if precision == "fp32" else -16

# amhd_set_tma mode the library starts with: bit 0 the tiled kernel's tile + halo,
# bit 1 the marching kernel's rows staged by TMA
DEFAULT_TMA = 1

AMHD_FLAG_NONFINITE = 1
AMHD_FLAG_DT_TINY = 2
AMHD_FLAG_PAUSED = 4
AMHD_FLAG_TIMEOUT = 8

_c = ctypes
_I32, _I64, _D, _P, _U32, _U64 = _c.c_int32, _c.c_int64, _c.c_double, _c.c_void_p, _c.c_uint32, _c.c_uint64


class Grid(_c.Structure):
    _fields_ = [("nx", _I32), ("ny", _I32), ("pitch", _I32), ("dtype", _I32), ("var_stride", _I64),
                ("dx", _D), ("dy", _D), ("gamma", _D), ("cfl", _D), ("glm_alpha", _D),
                ("bc_x", _I32), ("bc_y", _I32), ("powell", _I32), ("limiter", _I32)]


class Control(_c.Structure):
    _fields_ = [("t", _D), ("t_end", _D), ("dt", _D), ("dt_cfl", _D), ("ch", _D), ("decay", _D), ("e_bnd", _D),
                ("last_dt", _D), ("step", _I64), ("max_steps", _I64), ("active", _I32), ("flags", _I32),
                ("red", _U64 * 4), ("queue", _I32 * 2), ("snap_t", _D), ("scratch", _D),
                ("e_bnd_next", _D), ("reserved", _D)]


class Instance(_c.Structure):
    _fields_ = [("grid", Grid), ("offset", _I64), ("first_tile", _I32), ("tiles_x", _I32), ("tiles_y", _I32),
                ("cut_x", _I32), ("pack", _I32), ("reserved", _I32)]


class NNTensor(_c.Structure):
    _fields_ = [("w", _P), ("g", _P), ("m", _P), ("v", _P), ("w_bf16", _P), ("n", _I64), ("weight_decay", _c.c_float),
                ("pad_", _I32)]


class AmhdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libaeromhd error {code}: {msg}")
        self.code = code


_SIGS = {
    "amhd_version": ([], _c.c_char_p),
    "amhd_last_error": ([], _c.c_char_p),
    "amhd_init": ([], _c.c_int),
    "amhd_padded_layout": ([_I32, _I32, _I32, _c.POINTER(_I32), _c.POINTER(_I32)], _c.c_int),
    "amhd_control_size": ([], _c.c_size_t),
    "amhd_set_tiling": ([_I32, _I32], _c.c_int),
    "amhd_stage_info": ([_I32, _I32, _c.POINTER(_I32), _c.POINTER(_I32), _c.POINTER(_I32)], _c.c_int),
    "amhd_cons_to_prim": ([_c.POINTER(Grid), _P, _P, _P], _c.c_int),
    "amhd_prim_to_cons": ([_c.POINTER(Grid), _P, _P, _P], _c.c_int),
    "amhd_muscl": ([_c.POINTER(Grid), _I32, _P, _P, _P, _P], _c.c_int),
    "amhd_hlld_flux": ([_I32, _I32, _P, _P, _P, _P, _I64, _D, _D, _P], _c.c_int),
    "amhd_apply_bc": ([_c.POINTER(Grid), _P, _P], _c.c_int),
    "amhd_enforce_scalar_bounds": ([_c.POINTER(Grid), _P, _P], _c.c_int),
    "amhd_compute_dt": ([_c.POINTER(Grid), _P, _P, _c.POINTER(_D), _c.POINTER(_D), _P], _c.c_int),
    "amhd_compute_dt_cons": ([_c.POINTER(Grid), _P, _P, _c.POINTER(_D), _c.POINTER(_D), _P], _c.c_int),
    "amhd_boundary_energy_flux": ([_c.POINTER(Grid), _P, _P, _c.POINTER(_D), _P], _c.c_int),
    "amhd_powell_source": ([_c.POINTER(Grid), _P, _P, _P], _c.c_int),
    "amhd_compute_rhs": ([_c.POINTER(Grid), _P, _P, _D, _P], _c.c_int),
    "amhd_step_ssprk3": ([_c.POINTER(Grid), _P, _P, _P, _D, _D, _D, _P, _P], _c.c_int),
    "amhd_rk_stage": ([_c.POINTER(Grid), _I32, _P, _P, _P, _D, _D, _D, _P], _c.c_int),
    "amhd_control_init": ([_c.POINTER(Grid), _P, _P, _D, _D, _I64, _I64, _P], _c.c_int),
    "amhd_control_resume": ([_P, _I32, _D, _P], _c.c_int),
    "amhd_advance": ([_c.POINTER(Grid), _P, _P, _P, _P, _I32, _P], _c.c_int),
    "amhd_advance_compensated": ([_c.POINTER(Grid), _P, _P, _P, _P, _P, _I32, _P], _c.c_int),
    "amhd_advance_profile": ([_c.POINTER(Grid), _P, _P, _P, _P, _I32, _c.POINTER(_D), _P], _c.c_int),
    "amhd_step_host": ([_c.POINTER(Grid), _P, _P, _P, _P, _P, _D, _D, _c.POINTER(_D), _P], _c.c_int),
    "amhd_step_host_n": ([_c.POINTER(Grid), _P, _P, _P, _P, _P, _D, _D, _I32, _c.POINTER(_D), _P], _c.c_int),
    "amhd_diagnostics": ([_c.POINTER(Grid), _P, _D, _P, _P, _P], _c.c_int),
    "amhd_diagnostics_noalloc": ([_c.POINTER(Grid), _P, _D, _P, _P], _c.c_int),
    "amhd_diagnostics_colour": ([_c.POINTER(Grid), _P, _D, _P, _P, _P, _P], _c.c_int),
    "amhd_control_init_split": ([_c.POINTER(Grid), _P, _P, _D, _D, _I64, _I64, _P], _c.c_int),
    "amhd_advance_stage": ([_c.POINTER(Grid), _I32, _P, _P, _P, _P, _P], _c.c_int),
    "amhd_advance_finish": ([_c.POINTER(Grid), _P, _P, _I32, _I32, _P], _c.c_int),
    "amhd_ensemble_advance": ([_P, _I32, _P, _P, _I32, _I32, _I32, _P, _P, _P, _P, _I32, _I32, _P, _P, _P],
                              _c.c_int),
    "amhd_ensemble_tensormaps": ([_P, _I32, _I32, _I32, _P, _P, _P, _P], _c.c_int),
    "amhd_set_tma": ([_I32], _c.c_int),
    "amhd_march_pack": ([_I32], _c.c_int),
    "amhd_march_items": ([_I32, _I32, _I32, _I32], _c.c_int),
    "amhd_set_march_pack": ([_I32], _c.c_int),
    "amhd_selftest_wait": ([_I32, _I64, _P, _P], _c.c_int),
    "amhd_ensemble_continue": ([_P, _P, _I32, _I32, _P, _P, _D, _P], _c.c_int),
    "amhd_ensemble_init": ([_P, _P, _I32, _I32, _P, _P, _D, _I64, _P], _c.c_int),
    "amhd_nn_last_error": ([], _c.c_char_p),
    "amhd_nn_gemm": ([_I32, _I32, _I32, _I32, _I32, _P, _I32, _P, _I32, _P, _I32, _c.c_float, _c.c_float, _I32, _P],
                     _c.c_int),
    "amhd_nn_gemm_tc": ([_I32, _I32, _I32, _I32, _I32, _P, _I32, _P, _I32, _P, _I32, _c.c_float, _c.c_float, _I32,
                         _P], _c.c_int),
    "amhd_nn_gemm_status": ([_P], _c.c_int),
    "amhd_nn_gemm_tc_paths": ([_P, _P], _c.c_int),
    "amhd_nn_set_gemm_path": ([_I32], _c.c_int),
    "amhd_nn_set_gemm_persistent": ([_I32], _c.c_int),
    "amhd_nn_im2col3": ([_P, _I32, _I32, _I32, _I32, _P, _P], _c.c_int),
    "amhd_nn_col2im3": ([_P, _I32, _I32, _I32, _I32, _P, _P], _c.c_int),
    "amhd_nn_cast_bf16": ([_P, _P, _I64, _P], _c.c_int),
    "amhd_nn_flip3": ([_P, _I32, _I32, _I32, _P, _P], _c.c_int),
    "amhd_nn_pad_cols": ([_P, _I32, _I32, _I32, _P, _P], _c.c_int),
    "amhd_nn_bias_act": ([_P, _P, _I32, _I64, _I32, _P], _c.c_int),
    "amhd_nn_relu_bwd": ([_P, _P, _I64, _P], _c.c_int),
    "amhd_nn_bias_grad": ([_P, _I32, _I64, _P, _P], _c.c_int),
    "amhd_nn_pool2": ([_P, _I32, _I32, _I32, _P, _I32, _P], _c.c_int),
    "amhd_nn_up2": ([_P, _I32, _I32, _I32, _P, _I32, _P], _c.c_int),
    "amhd_nn_axpy": ([_P, _P, _c.c_float, _I64, _P], _c.c_int),
    "amhd_nn_mse": ([_P, _P, _I64, _P, _P, _P], _c.c_int),
    "amhd_nn_adam": ([_P, _P, _P, _P, _P, _I64, _c.c_float, _c.c_float, _c.c_float, _c.c_float, _I32, _c.c_float, _P],
                     _c.c_int),
    "amhd_nn_adam_multi": ([_P, _I32, _I64, _P, _P], _c.c_int),
    "amhd_nn_restrict": ([_c.POINTER(Grid), _P, _I32, _P, _I64, _I32, _I32, _P], _c.c_int),
    "amhd_nn_pack": ([_c.POINTER(Grid), _P, _P, _P, _P, _I64, _I32, _P], _c.c_int),
    "amhd_nn_apply": ([_c.POINTER(Grid), _P, _P, _P, _I64, _I32, _P], _c.c_int),
    "amhd_nn_apply_guarded": ([_c.POINTER(Grid), _P, _P, _P, _I64, _I32, _c.c_float, _c.c_float, _I32, _P, _P],
                              _c.c_int),
}

_lib = None


def exported_names():
    return list(_SIGS)


def lib():
    """Load libaeromhd.so (fails loudly if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m aeromhd_cuda_b200.build` "
                              "(nvcc, sm_100a); there is no CPU fallback")
        L = _c.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        if L.amhd_control_size() != _c.sizeof(Control):
            raise ImportError("amhd_control layout mismatch between include/aeromhd.h and _lib.py")
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != AMHD_OK:
        raise AmhdError(rc, lib().amhd_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    rc = getattr(lib(), name)(*args)
    if rc != AMHD_OK and name.startswith("amhd_nn_"):
        raise AmhdError(rc, lib().amhd_nn_last_error().decode(errors="replace"))
    check(rc)


def check_control(c, where: str = "run loop") -> None:
    """Raise on the control flags after which a state must not be used.

    AMHD_FLAG_NONFINITE (a step wrote a non-finite value) raises
    FloatingPointError; AMHD_FLAG_TIMEOUT (a bounded device wait gave up, so
    a tile of the state was not updated) raises AmhdError(AMHD_ERR_TIMEOUT).
    The run loop's finalize kernel stops an instance whose flags carry either."""
    if c.flags & AMHD_FLAG_TIMEOUT:
        raise AmhdError(AMHD_ERR_TIMEOUT, f"{where}: a bounded device wait expired at step {c.step}, t={c.t}; "
                                          "tiles of the state were not updated")
    if c.flags & AMHD_FLAG_NONFINITE:
        raise FloatingPointError(f"{where}: non-finite state at step {c.step}, t={c.t}")


def check_gemm_status(where: str = "corrector") -> None:
    """Read (and clear) the tensor-core GEMM wait flag; raise if a GEMM gave up.

    A tcgen05 GEMM whose bounded wait expired skips its epilogue, leaving its
    output unwritten; nothing else reports it.  The call synchronises."""
    flag = _I32(0)
    call("amhd_nn_gemm_status", _c.byref(flag))
    if flag.value:
        raise AmhdError(AMHD_ERR_TIMEOUT, f"{where}: a tensor-core GEMM wait expired; its output was not written")


def padded_layout(nx: int, ny: int, dtype_code: int):
    pitch, rows = _I32(), _I32()
    call("amhd_padded_layout", nx, ny, dtype_code, _c.byref(pitch), _c.byref(rows))
    return pitch.value, rows.value
