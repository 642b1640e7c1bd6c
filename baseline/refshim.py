"""Run the reference's own Python modules, unchanged, without CuPy.

The reference (config.py, physics.py, solver.py, main.py) does all array work
through ``xp = cupy`` (physics.py:29) and its HLLD face solver through
``cupy.RawKernel`` (physics.py:43-278).  CuPy is not installed on these
machines, so before importing the modules this file puts a stand-in module
named ``cupy`` into ``sys.modules``:

* ``backend="numpy"``: arrays are numpy arrays; ``RawKernel(code, name)``
  compiles the reference's OWN kernel text (read from the imported module,
  never copied) as host C++ with g++ (``-ffp-contract=off``) and runs the grid
  of blocks with OpenMP.  This is the reference evaluated on host cores.
* ``backend="torch"``: arrays are PyTorch tensors on ``device`` (a CUDA device,
  or the CPU); every array expression of the reference becomes the matching
  torch operation, eagerly, one kernel per operation as in CuPy.  On a CUDA
  device ``RawKernel`` compiles the reference's kernel text with NVRTC for the
  device's architecture (NVRTC defaults, as CuPy uses them) and launches it on
  torch's current stream through the CUDA driver API; on the CPU it is the
  host-C++ kernel of the numpy backend.  This is the reference's CuPy path
  run on the same GPU, with torch in CuPy's place.

matplotlib (used only for plots) is replaced by inert stubs.  solver.py makes
``rmi_output_gpu/`` in the working directory at import (solver.py:40-42), so
the import runs inside a temporary directory.

Where the reference comes from: ``ref_dir`` if given, else
``$AMHD_REFERENCE_DIR``, else ``baseline/_ref`` next to this file (made by
``install_reference.py``).  Nothing in the library imports this file; the
benchmark's comparator legs and the golden-vector generator do.
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

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_REF = os.path.join(HERE, "_ref")
MODULES = ("config", "physics", "solver", "main")


def reference_dir(ref_dir: str | None = None) -> str:
    """The reference checkout to import, or FileNotFoundError saying how to get one."""
    for cand in (ref_dir, os.environ.get("AMHD_REFERENCE_DIR"), DEFAULT_REF):
        if cand and all(os.path.isfile(os.path.join(cand, m + ".py")) for m in MODULES):
            return cand
    raise FileNotFoundError("reference modules not found: set AMHD_REFERENCE_DIR, or run "
                            "`python baseline/install_reference.py --source <checkout>` to fill baseline/_ref")


# ------------------------------------------------------------ host kernel
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

KERNEL_NAME = "hlld_flux_x_kernel"


def _kernel_args(args):
    WL, WR, F, smax, n, g, ch, fr, fp = args
    return (WL, WR, F, smax), (int(n), float(g), float(ch), float(fr), float(fp))


class HostRawKernel:
    """cupy.RawKernel stand-in: the kernel text compiled as host C++, grid x block looped with OpenMP."""

    def __init__(self, code: str, name: str):
        if name != KERNEL_NAME:
            raise NotImplementedError(f"the stand-in knows the reference's HLLD kernel signature, not {name}")
        src = _PRELUDE + code + (_LAUNCHER % name)
        tag = hashlib.sha1(src.encode()).hexdigest()[:16]
        d = os.path.join(tempfile.gettempdir(), "amhd_refshim")
        os.makedirs(d, exist_ok=True)
        so = os.path.join(d, f"refkernel_{tag}.so")
        if not os.path.exists(so):
            cpp = os.path.join(d, f"refkernel_{tag}_{os.getpid()}.cpp")
            with open(cpp, "w") as f:
                f.write(src)
            tmp = so + f".{os.getpid()}.tmp"
            subprocess.check_call(["g++", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                                   "-shared", "-o", tmp, cpp])
            os.replace(tmp, so)
        self._lib = ctypes.CDLL(so)
        P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        self._lib.amhd_shim_launch.argtypes = [I, I, P, P, P, P, I, D, D, D, D]

    def __call__(self, grid, block, args):
        arrays, (n, g, ch, fr, fp) = _kernel_args(args)
        ptrs = []
        for a in arrays:
            a = a.numpy() if hasattr(a, "numpy") and not isinstance(a, np.ndarray) else a
            assert a.dtype == np.float64 and a.flags.c_contiguous
            ptrs.append(a.ctypes.data)
        self._lib.amhd_shim_launch(int(grid[0]), int(block[0]), *ptrs, n, g, ch, fr, fp)


class NvrtcRawKernel:
    """cupy.RawKernel stand-in on a CUDA device: NVRTC compiles the kernel text for
    the current device (default NVRTC options, as CuPy's RawKernel), the driver
    API loads it, and a call launches it on torch's current stream."""

    def __init__(self, code: str, name: str):
        import torch
        from cuda.bindings import driver as cu, nvrtc
        if name != KERNEL_NAME:
            raise NotImplementedError(f"the stand-in knows the reference's HLLD kernel signature, not {name}")
        self._cu = cu
        torch.cuda.init()
        torch.zeros(1, device="cuda")  # make torch's primary context current in this thread
        major, minor = torch.cuda.get_device_capability()
        self.arch = f"sm_{major}{minor}"

        def ok(res, what):
            err, *rest = res if isinstance(res, tuple) else (res,)
            if int(err) != 0:
                raise RuntimeError(f"{what} failed: {err}")
            return rest[0] if len(rest) == 1 else rest

        prog = ok(nvrtc.nvrtcCreateProgram(code.encode(), b"reference_hlld.cu", 0, [], []), "nvrtcCreateProgram")
        opts = [f"--gpu-architecture={self.arch}".encode()]
        res = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
        if int(res[0]) != 0:
            size = ok(nvrtc.nvrtcGetProgramLogSize(prog), "log size")
            log = b" " * size
            nvrtc.nvrtcGetProgramLog(prog, log)
            raise RuntimeError("NVRTC: " + log.decode(errors="replace"))
        size = ok(nvrtc.nvrtcGetCUBINSize(prog), "nvrtcGetCUBINSize")
        cubin = b" " * size
        ok(nvrtc.nvrtcGetCUBIN(prog, cubin), "nvrtcGetCUBIN")
        self._module = ok(cu.cuModuleLoadData(cubin), "cuModuleLoadData")
        self._fn = ok(cu.cuModuleGetFunction(self._module, name.encode()), "cuModuleGetFunction")
        self._ok = ok

    def __call__(self, grid, block, args):
        import torch
        arrays, (n, g, ch, fr, fp) = _kernel_args(args)
        for a in arrays:
            assert isinstance(a, torch.Tensor) and a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()
        cu = self._cu
        vals = tuple(a.data_ptr() for a in arrays) + (n, g, ch, fr, fp)
        types_ = (ctypes.c_void_p,) * 4 + (ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double)
        stream = cu.CUstream(torch.cuda.current_stream().cuda_stream)
        self._ok(cu.cuLaunchKernel(self._fn, int(grid[0]), 1, 1, int(block[0]), 1, 1, 0, stream, (vals, types_), 0),
                 "cuLaunchKernel")


# ------------------------------------------------------------ cupy stand-ins
class _Device:
    def __init__(self, i=0):
        self.id = i

    def use(self):
        return None


def numpy_cupy() -> types.ModuleType:
    """cupy backed by numpy (host cores)."""
    class _Mod(types.ModuleType):
        def __getattr__(self, name):
            return getattr(np, name)

    cp = _Mod("cupy")
    cp.__version__ = "numpy-shim"
    cp.ndarray = np.ndarray
    cp.asnumpy = np.asarray
    cp.RawKernel = HostRawKernel
    runtime = types.SimpleNamespace(getDeviceProperties=lambda i: {
        "name": b"host-cpu (numpy stand-in)", "major": 0, "minor": 0, "totalGlobalMem": 0})
    cp.cuda = types.SimpleNamespace(Device=_Device, runtime=runtime)
    return cp


def torch_cupy(device: str = "cuda") -> types.ModuleType:
    """cupy backed by PyTorch tensors on `device`, with numpy's default float64."""
    import torch
    dev = torch.device(device)
    f64 = torch.float64

    def _dtype(dtype):
        if dtype is None:
            return f64
        return {np.float64: f64, np.float32: torch.float32, float: f64, np.int32: torch.int32,
                np.int64: torch.int64}.get(dtype, dtype)

    m = types.ModuleType("cupy")
    m.__version__ = f"torch-shim (torch {torch.__version__}, {dev})"
    m.ndarray = torch.Tensor
    m.float64, m.float32, m.int32, m.int64 = f64, torch.float32, torch.int32, torch.int64
    m.float_ = f64
    m.pi = np.pi
    m.asnumpy = lambda a: a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    m.zeros = lambda shape, dtype=None: torch.zeros(shape, dtype=_dtype(dtype), device=dev)
    m.ones = lambda shape, dtype=None: torch.ones(shape, dtype=_dtype(dtype), device=dev)
    m.empty = lambda shape, dtype=None: torch.empty(shape, dtype=_dtype(dtype), device=dev)
    m.zeros_like = lambda a, dtype=None: torch.zeros_like(a, dtype=None if dtype is None else _dtype(dtype))
    m.ones_like = lambda a, dtype=None: torch.ones_like(a, dtype=None if dtype is None else _dtype(dtype))
    m.empty_like = lambda a, dtype=None: torch.empty_like(a, dtype=None if dtype is None else _dtype(dtype))
    m.asarray = lambda a, dtype=None: (a if isinstance(a, torch.Tensor) and dtype is None
                                       else torch.as_tensor(np.asarray(a) if not isinstance(a, torch.Tensor) else a,
                                                            dtype=None if dtype is None else _dtype(dtype),
                                                            device=dev))
    m.array = lambda a, dtype=None: torch.tensor(np.asarray(a), dtype=None if dtype is None else _dtype(dtype),
                                                 device=dev)
    m.ascontiguousarray = lambda a: a.contiguous()
    # a Python scalar operand stays a kernel argument (no device copy), as in CuPy;
    # max/min with a scalar is exact and NaN-propagating either way
    def maximum(a, b):
        if not isinstance(b, torch.Tensor):
            return torch.clamp_min(a, float(b))
        if not isinstance(a, torch.Tensor):
            return torch.clamp_min(b, float(a))
        return torch.maximum(a, b)

    def minimum(a, b):
        if not isinstance(b, torch.Tensor):
            return torch.clamp_max(a, float(b))
        if not isinstance(a, torch.Tensor):
            return torch.clamp_max(b, float(a))
        return torch.minimum(a, b)

    def where(c, a, b):
        if isinstance(a, torch.Tensor):
            return torch.where(c, a, b if isinstance(b, torch.Tensor) else float(b))
        if isinstance(b, torch.Tensor):
            return torch.where(c, float(a), b)
        return torch.where(c, torch.tensor(float(a), dtype=f64, device=c.device), float(b))

    m.maximum, m.minimum = maximum, minimum

    m.where = where
    m.clip = lambda a, lo, hi: torch.clamp(a, lo, hi)
    m.max = lambda a, axis=None: torch.max(a) if axis is None else torch.amax(a, dim=axis)
    m.min = lambda a, axis=None: torch.min(a) if axis is None else torch.amin(a, dim=axis)
    m.sum = lambda a, axis=None: torch.sum(a) if axis is None else torch.sum(a, dim=axis)
    m.mean = lambda a, axis=None: torch.mean(a) if axis is None else torch.mean(a, dim=axis)
    for name in ("abs", "sqrt", "sin", "cos", "tanh", "exp", "log", "isfinite"):
        setattr(m, name, getattr(torch, name))
    m.meshgrid = lambda *a, indexing="xy": torch.meshgrid(*a, indexing=indexing)
    m.arange = lambda *a, dtype=None: torch.arange(*a, dtype=_dtype(dtype) if dtype else None, device=dev)
    m.RawKernel = NvrtcRawKernel if dev.type == "cuda" else HostRawKernel

    if dev.type == "cuda":
        def props(i):
            p = torch.cuda.get_device_properties(i)
            return {"name": p.name, "major": p.major, "minor": p.minor, "totalGlobalMem": p.total_memory}
    else:
        def props(i):
            return {"name": b"host-cpu (torch stand-in)", "major": 0, "minor": 0, "totalGlobalMem": 0}
    m.cuda = types.SimpleNamespace(Device=_Device, runtime=types.SimpleNamespace(getDeviceProperties=props))
    # the one ndarray method the reference calls that a tensor lacks: U.copy() (solver.py:314)
    if not hasattr(torch.Tensor, "copy"):
        torch.Tensor.copy = torch.Tensor.clone
    return m


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


def load_reference(backend: str = "numpy", device: str = "cuda", ref_dir: str | None = None, quiet: bool = False):
    """Import the reference modules over the chosen cupy stand-in (once per process).

    Returns a namespace with config, physics, solver, main, the directory
    they came from and the stand-in's label."""
    global _loaded
    if _loaded is not None:
        if _loaded.backend != (backend, device if backend == "torch" else None):
            raise RuntimeError(f"reference already loaded with the {_loaded.backend} stand-in in this process")
        return _loaded
    src = reference_dir(ref_dir)
    cp = numpy_cupy() if backend == "numpy" else torch_cupy(device)
    sys.modules["cupy"] = cp
    mpl, plt, lines = _fake_matplotlib()
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.modules.setdefault("matplotlib.lines", lines)
    cwd = os.getcwd()
    tmp = tempfile.mkdtemp(prefix="amhd_ref_cwd_")
    os.chdir(tmp)
    sys.path.insert(0, src)
    saved = sys.stdout
    try:
        if quiet:
            sys.stdout = open(os.devnull, "w")
        import config as rconfig  # noqa: E402
        import physics as rphysics  # noqa: E402
        import solver as rsolver  # noqa: E402
        import main as rmain  # noqa: E402
    finally:
        if quiet:
            sys.stdout.close()
            sys.stdout = saved
        sys.path.remove(src)
        os.chdir(cwd)
    _loaded = types.SimpleNamespace(config=rconfig, physics=rphysics, solver=rsolver, main=rmain, cwd=tmp,
                                    source=src, label=cp.__version__,
                                    backend=(backend, device if backend == "torch" else None))
    return _loaded
