"""Import the reference's Python modules on a CPU-only machine, unchanged.

Golden-vector harness: used by ``make_golden.py`` (and by an optional
cross-check test that skips itself when the reference checkout is absent).
Nothing on the GPU path imports it.

The reference needs CuPy and matplotlib; neither is installed here.  Before
importing it this module injects stand-ins:

* ``cupy`` -> numpy for every array expression (``xp = cp`` in physics.py:29).
  ``cupy.RawKernel(code, name)`` compiles the reference's OWN kernel string
  (physics.py:43-276, read from the imported module at run time, never
  copied) as host C++ with g++ (``-ffp-contract=off``), runs the grid of
  blocks with OpenMP and is called through ctypes.
* ``matplotlib``, ``matplotlib.pyplot``, ``matplotlib.lines`` -> inert stubs
  (no figure is drawn by anything the goldens run).

solver.py creates ``rmi_output_gpu/`` in the current directory at import
(solver.py:40-42), so the import runs inside a temporary directory.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
import sys
import tempfile
import types

import numpy as np

REFERENCE_DIR = os.environ.get("AMHD_REFERENCE_DIR", "/root/reference")

_PRELUDE = r"""
#include <math.h>
struct amhd_shim_dim3 { unsigned x, y, z; };
static thread_local amhd_shim_dim3 blockIdx, blockDim, threadIdx;
#define __global__
#define __restrict__ __restrict
"""

_LAUNCHER = r"""
extern "C" void amhd_shim_launch(int grid, int block, const double* a0, const double* a1, double* a2,
                                 double* a3, int n, double g, double ch, double fr, double fp)
{
    #pragma omp parallel for schedule(static)
    for (int b = 0; b < grid; ++b) {
        blockIdx.x = b; blockIdx.y = 0; blockIdx.z = 0;
        blockDim.x = block; blockDim.y = 1; blockDim.z = 1;
        for (int t = 0; t < block; ++t) {
            threadIdx.x = t; threadIdx.y = 0; threadIdx.z = 0;
            %s(a0, a1, a2, a3, n, g, ch, fr, fp);
        }
    }
}
"""


class _HostRawKernel:
    """cupy.RawKernel stand-in: the kernel text compiled as host C++."""

    def __init__(self, code: str, name: str):
        if name != "hlld_flux_x_kernel":
            raise NotImplementedError(f"shim only knows the reference's HLLD kernel signature, not {name}")
        src = _PRELUDE + code + (_LAUNCHER % name)
        tag = hashlib.sha1(src.encode()).hexdigest()[:16]
        d = os.path.join(tempfile.gettempdir(), "amhd_refshim")
        os.makedirs(d, exist_ok=True)
        so = os.path.join(d, f"refkernel_{tag}.so")
        if not os.path.exists(so):
            cpp = os.path.join(d, f"refkernel_{tag}.cpp")
            with open(cpp, "w") as f:
                f.write(src)
            subprocess.check_call(["g++", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                                   "-shared", "-o", so, cpp])
        self._lib = ctypes.CDLL(so)
        P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        self._lib.amhd_shim_launch.argtypes = [I, I, P, P, P, P, I, D, D, D, D]

    def __call__(self, grid, block, args):
        WL, WR, F, smax, n, g, ch, fr, fp = args
        for a in (WL, WR, F, smax):
            assert isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
        self._lib.amhd_shim_launch(int(grid[0]), int(block[0]), WL.ctypes.data, WR.ctypes.data, F.ctypes.data,
                                   smax.ctypes.data, int(n), float(g), float(ch), float(fr), float(fp))


def _fake_cupy() -> types.ModuleType:
    class _Mod(types.ModuleType):
        def __getattr__(self, name):
            return getattr(np, name)

    cp = _Mod("cupy")
    cp.__version__ = "numpy-shim"
    cp.ndarray = np.ndarray
    cp.asnumpy = np.asarray
    cp.RawKernel = _HostRawKernel

    class _Device:
        def __init__(self, i=0):
            self.id = i

        def use(self):
            return None

    runtime = types.SimpleNamespace(getDeviceProperties=lambda i: {
        "name": b"host-cpu (refshim)", "major": 0, "minor": 0, "totalGlobalMem": 0})
    cp.cuda = types.SimpleNamespace(Device=_Device, runtime=runtime)
    return cp


def _fake_matplotlib():
    class _Anything:
        def __getattr__(self, name):
            if name.startswith("__"):
                raise AttributeError(name)
            return _Anything()

        def __call__(self, *a, **k):
            return _Anything()

        def __iter__(self):
            return iter([])

    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    mpl.rcParams = {}
    plt = types.ModuleType("matplotlib.pyplot")
    def _plt_attr(name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Anything()

    plt.__getattr__ = _plt_attr
    lines = types.ModuleType("matplotlib.lines")
    lines.Line2D = _Anything
    mpl.pyplot = plt
    mpl.lines = lines
    return mpl, plt, lines


_loaded = None


def load_reference():
    """Return the reference modules (config, physics, solver, main)."""
    global _loaded
    if _loaded is not None:
        return _loaded
    if not os.path.isdir(REFERENCE_DIR):
        raise FileNotFoundError(REFERENCE_DIR)
    sys.modules.setdefault("cupy", _fake_cupy())
    mpl, plt, lines = _fake_matplotlib()
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.modules.setdefault("matplotlib.lines", lines)
    cwd = os.getcwd()
    tmp = tempfile.mkdtemp(prefix="amhd_ref_cwd_")
    os.chdir(tmp)
    sys.path.insert(0, REFERENCE_DIR)
    try:
        import config as rconfig  # noqa: E402
        import physics as rphysics  # noqa: E402
        import solver as rsolver  # noqa: E402
        import main as rmain  # noqa: E402
    finally:
        sys.path.remove(REFERENCE_DIR)
        os.chdir(cwd)
    _loaded = types.SimpleNamespace(config=rconfig, physics=rphysics, solver=rsolver, main=rmain, cwd=tmp)
    return _loaded
